"""The warm-start U-Net oracle (oracle/unet_ref.py) against finite differences and its own invariants (CPU)."""
import numpy as np

from oracle import unet_ref as U

W = (8, 8, 16)


def test_backward_matches_finite_differences():
    p = U.init_params(W, seed=1).astype(np.float64)
    rng = np.random.default_rng(0)
    x = rng.random((2, 4, 4, 4, 1))
    t = rng.standard_normal((2, 4, 4, 4, 18)) * 0.1
    w = rng.random((2, 4, 4, 4))
    w /= w.sum()
    _, g = U.backward(p, x, t, w, W)
    worst = 0.0
    for i in rng.choice(len(p), 40, replace=False):
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        fd = (U.loss(U.forward(pp, x, W)[0], t, w) - U.loss(U.forward(pm, x, W)[0], t, w)) / (2 * e)
        worst = max(worst, abs(fd - g[i]) / (abs(fd) + abs(g[i]) + 1e-12))
    assert worst < 1e-4, worst


def test_layout_periodicity_and_adam():
    assert U.param_count((16, 32, 64)) == len(U.init_params((16, 32, 64)))
    p = U.init_params(W, seed=2).astype(np.float64)
    rng = np.random.default_rng(3)
    x = rng.random((1, 8, 8, 8, 1))
    y, _ = U.forward(p, x, W)
    # a periodic shift of the cell by one coarse voxel (4 fine voxels) shifts the prediction
    ys, _ = U.forward(p, np.roll(x, 4, axis=1), W)
    assert np.allclose(np.roll(y, 4, axis=1), ys, atol=1e-12)
    g = rng.standard_normal(p.size)
    p1, m, v = U.adam(p, g, np.zeros_like(p), np.zeros_like(p), 1, 1e-3)
    assert np.allclose(p - p1, 1e-3 * np.sign(g), rtol=1e-3)  # the first bias-corrected step is ~ lr * sign(g)
