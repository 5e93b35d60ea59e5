"""NumPy FP64 oracle of the warm-start U-Net (test infrastructure only; the product runs libnlf.so).

The network maps a density cell rho (B, n0, n1, n2) to the 6 corrector fields of the unit strains, as 18
channels (B, n0, n1, n2, 18) = u (6 cases x 3 components) / n0, channels-last everywhere. It has no counterpart
in the reference: the reference solves every corrector from u0 = 0 (nlfiber/linear.py:209-212, the `u0` hook of
`solve` and `C_full`), and the network only supplies that initial guess. Architecture (widths w0, w1, w2):

    L1  conv3 1 -> w0, relu            L7  conv3 (w2 + w1) -> w1, relu   on concat(up(a6), a4)
    L2  conv3 w0 -> w0, relu  = a2     L8  conv3 w1 -> w1, relu
        avg-pool 2                     L9  conv3 (w1 + w0) -> w0, relu   on concat(up(a8), a2)
    L3  conv3 w0 -> w1, relu           L10 conv3 w0 -> w0, relu
    L4  conv3 w1 -> w1, relu  = a4     L11 conv1 w0 -> 18 (linear)
        avg-pool 2
    L5  conv3 w1 -> w2, relu
    L6  conv3 w2 -> w2, relu

conv3 is a periodic 3x3x3 convolution: y[v] = b + sum_t W[t] x[v + off_t], tap t = 9 (di + 1) + 3 (dj + 1) +
(dk + 1) over the offsets (di, dj, dk) in {-1, 0, 1}^3, W[t] of shape (cout, cin). up is nearest-neighbour
upsampling by 2, avg-pool the mean of 2x2x2 blocks. The loss is sum_v w_v sum_c (y - t)^2 / 18 with per-voxel
weights w (the callers normalise them to sum 1 per batch). Parameters are one flat FP32 vector: per layer W
(ntaps, cout, cin) then b (cout).
"""
import numpy as np

OUT = 18


def layers(w0=16, w1=32, w2=64, cin=1, cout=OUT):
    """(cin, cout, ntaps, relu) of L1..L11."""
    return [(cin, w0, 27, 1), (w0, w0, 27, 1), (w0, w1, 27, 1), (w1, w1, 27, 1), (w1, w2, 27, 1),
            (w2, w2, 27, 1), (w2 + w1, w1, 27, 1), (w1, w1, 27, 1), (w1 + w0, w0, 27, 1), (w0, w0, 27, 1),
            (w0, cout, 1, 0)]


def param_count(widths=(16, 32, 64)):
    return sum(t * co * ci + co for ci, co, t, _ in layers(*widths))


def split(params, widths=(16, 32, 64)):
    out, o = [], 0
    for ci, co, t, _ in layers(*widths):
        W = params[o:o + t * co * ci].reshape(t, co, ci)
        o += t * co * ci
        b = params[o:o + co]
        o += co
        out.append((W, b))
    return out


def init_params(widths=(16, 32, 64), seed=0):
    """He-normal weights (std sqrt(2 / fan_in)), zero biases; the output layer starts small (std 1e-2 / fan)."""
    rng = np.random.default_rng(seed)
    ps = []
    for k, (ci, co, t, relu) in enumerate(layers(*widths)):
        std = np.sqrt(2.0 / (ci * t)) if relu else 1e-2 / np.sqrt(ci * t)
        ps.append(rng.standard_normal(t * co * ci) * std)
        ps.append(np.zeros(co))
    return np.concatenate(ps).astype(np.float32)


def _off(t):
    return t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def _shift(x, d, sign):
    """x[v + sign * d] with periodic wrap on the three spatial axes of (B, n0, n1, n2, C)."""
    return np.roll(x, shift=(-sign * d[0], -sign * d[1], -sign * d[2]), axis=(1, 2, 3))


def conv(x, W, b):
    y = np.zeros(x.shape[:4] + (W.shape[1],))
    for t in range(W.shape[0]):
        d = _off(t) if W.shape[0] == 27 else (0, 0, 0)
        y += _shift(x, d, 1) @ W[t].T
    return y + b


def conv_bwd(x, W, g):
    """Gradients of conv w.r.t. x, W, b for the output gradient g."""
    dx = np.zeros_like(x)
    dW = np.zeros_like(W)
    for t in range(W.shape[0]):
        d = _off(t) if W.shape[0] == 27 else (0, 0, 0)
        dx += _shift(g @ W[t], d, -1)
        dW[t] = np.einsum("bijkc,bijkd->cd", g, _shift(x, d, 1))
    return dx, dW, g.sum(axis=(0, 1, 2, 3))


def pool(x):
    B, a, b, c, C = x.shape
    return x.reshape(B, a // 2, 2, b // 2, 2, c // 2, 2, C).mean(axis=(2, 4, 6))


def pool_bwd(g):
    return up(g) / 8.0


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def up_bwd(g):
    B, a, b, c, C = g.shape
    return g.reshape(B, a // 2, 2, b // 2, 2, c // 2, 2, C).sum(axis=(2, 4, 6))


def forward(params, x, widths=(16, 32, 64)):
    """x (B, n0, n1, n2, 1) -> y (B, n0, n1, n2, 18) and the cache for backward."""
    P = split(np.asarray(params, np.float64), widths)
    relu = lambda z: np.maximum(z, 0.0)  # noqa: E731
    c = {"x": x}
    c["a1"] = relu(conv(x, *P[0]))
    c["a2"] = relu(conv(c["a1"], *P[1]))
    c["p1"] = pool(c["a2"])
    c["a3"] = relu(conv(c["p1"], *P[2]))
    c["a4"] = relu(conv(c["a3"], *P[3]))
    c["p2"] = pool(c["a4"])
    c["a5"] = relu(conv(c["p2"], *P[4]))
    c["a6"] = relu(conv(c["a5"], *P[5]))
    c["c1"] = np.concatenate([up(c["a6"]), c["a4"]], axis=-1)
    c["a7"] = relu(conv(c["c1"], *P[6]))
    c["a8"] = relu(conv(c["a7"], *P[7]))
    c["c2"] = np.concatenate([up(c["a8"]), c["a2"]], axis=-1)
    c["a9"] = relu(conv(c["c2"], *P[8]))
    c["a10"] = relu(conv(c["a9"], *P[9]))
    y = conv(c["a10"], *P[10])
    return y, c


def loss(y, t, w):
    return float(np.sum(w[..., None] * (y - t) ** 2) / y.shape[-1])


def backward(params, x, t, w, widths=(16, 32, 64)):
    """(loss, flat gradient) of loss(forward(x), t, w)."""
    P = split(np.asarray(params, np.float64), widths)
    y, c = forward(params, x, widths)
    L = loss(y, t, w)
    g = 2.0 * w[..., None] * (y - t) / y.shape[-1]
    grads = [None] * 11
    mask = lambda a, d: d * (a > 0)  # noqa: E731
    dx, dW, db = conv_bwd(c["a10"], P[10][0], g)
    grads[10] = (dW, db)
    g = mask(c["a10"], dx)
    dx, dW, db = conv_bwd(c["a9"], P[9][0], g)
    grads[9] = (dW, db)
    g = mask(c["a9"], dx)
    dc2, dW, db = conv_bwd(c["c2"], P[8][0], g)
    grads[8] = (dW, db)
    w1 = c["a8"].shape[-1]
    g = mask(c["a8"], up_bwd(dc2[..., :w1]))
    dx, dW, db = conv_bwd(c["a7"], P[7][0], g)
    grads[7] = (dW, db)
    g = mask(c["a7"], dx)
    dc1, dW, db = conv_bwd(c["c1"], P[6][0], g)
    grads[6] = (dW, db)
    w2 = c["a6"].shape[-1]
    g = mask(c["a6"], up_bwd(dc1[..., :w2]))
    dx, dW, db = conv_bwd(c["a5"], P[5][0], g)
    grads[5] = (dW, db)
    g = mask(c["a5"], dx)
    dp2, dW, db = conv_bwd(c["p2"], P[4][0], g)
    grads[4] = (dW, db)
    g = mask(c["a4"], pool_bwd(dp2) + dc1[..., w2:])
    dx, dW, db = conv_bwd(c["a3"], P[3][0], g)
    grads[3] = (dW, db)
    g = mask(c["a3"], dx)
    dp1, dW, db = conv_bwd(c["p1"], P[2][0], g)
    grads[2] = (dW, db)
    g = mask(c["a2"], pool_bwd(dp1) + dc2[..., w1:])
    dx, dW, db = conv_bwd(c["a1"], P[1][0], g)
    grads[1] = (dW, db)
    g = mask(c["a1"], dx)
    _, dW, db = conv_bwd(c["x"], P[0][0], g)
    grads[0] = (dW, db)
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return L, flat


def adam(params, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015) with bias correction; step counts from 1. Returns new (params, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
