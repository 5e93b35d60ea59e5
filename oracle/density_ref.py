"""NumPy FP64 restatement of the reference's input generators. TEST ORACLE / INPUT GENERATOR ONLY.

symmetry   nlfiber/symmetry.py:26-102   octant <-> full cell, permutation projection, exact orbit copies
density    nlfiber/density.py:23-122    periodic hat filter, unit-std scaling, exact-volume threshold, binary
topology   nlfiber/topology.py:8-63     periodic labelling and floating-piece removal (for binary cells)
fiber      nlfiber/fiber.py:103-121     random_start
helpers    tests/helpers.py:8-24        schwarz_p_phi, binary_cell, grey_cell
"""
import itertools
from math import comb

import numpy as np
from scipy import ndimage


# --- symmetry (nlfiber/symmetry.py) -------------------------------------------------------------
def n_free(n_o, d=3):
    """nlfiber/symmetry.py:20-22."""
    return comb(n_o + d - 1, d)


def sym_perm(x, batch=0):
    """nlfiber/symmetry.py:25-33: average over all permutations of the last d axes."""
    x = np.asarray(x, dtype=np.float64)
    d = x.ndim - batch
    lead = tuple(range(batch))
    perms = list(itertools.permutations(range(d)))
    out = 0
    for p in perms:
        out = out + np.transpose(x, lead + tuple(batch + q for q in p))
    return out / len(perms)


def mirror(oct_, batch=0):
    """nlfiber/symmetry.py:36-41: octant -> full cell."""
    x = np.asarray(oct_)
    for ax in range(batch, x.ndim):
        x = np.concatenate([x, np.flip(x, ax)], axis=ax)
    return x


def fold(full, batch=0):
    """nlfiber/symmetry.py:44-52."""
    x = np.asarray(full)
    for ax in range(batch, x.ndim):
        n = x.shape[ax] // 2
        a = np.take(x, np.arange(n), axis=ax)
        b = np.flip(np.take(x, np.arange(n, 2 * n), axis=ax), ax)
        x = 0.5 * (a + b)
    return x


def project_full(full, batch=0):
    """nlfiber/symmetry.py:55-57."""
    return mirror(sym_perm(fold(full, batch), batch), batch)


def free_index(n_o, d=3):
    """nlfiber/symmetry.py:74-76."""
    return np.array(list(itertools.combinations_with_replacement(range(n_o), d)))


def to_free(oct_):
    """nlfiber/symmetry.py:79-82."""
    idx = free_index(oct_.shape[0], oct_.ndim)
    return oct_[tuple(idx.T)]


_REP = {}


def representative_index(n_o, d=3):
    """nlfiber/symmetry.py:88-96: for every octant index tuple, the position of its sorted tuple."""
    key = (n_o, d)
    if key not in _REP:
        idx = free_index(n_o, d)
        pos = {tuple(t): k for k, t in enumerate(idx)}
        grid = np.stack(np.meshgrid(*[np.arange(n_o)] * d, indexing="ij"), axis=-1).reshape(-1, d)
        _REP[key] = np.array([pos[tuple(sorted(g))] for g in grid]).reshape((n_o,) * d)
    return _REP[key]


def from_free(v, n_o, d=3):
    """nlfiber/symmetry.py:99-101."""
    return np.asarray(v)[representative_index(n_o, d)]


def exact_symmetrize(full):
    """nlfiber/symmetry.py:60-65: symmetric projection with one value copied exactly per orbit."""
    oct_ = sym_perm(fold(full))
    n_o, d = oct_.shape[0], oct_.ndim
    return mirror(from_free(to_free(oct_), n_o, d))


def sym_residual(full):
    """nlfiber/symmetry.py:68-71."""
    full = np.asarray(full, dtype=np.float64)
    return float(np.linalg.norm(full - project_full(full)) / (np.linalg.norm(full) + 1e-300))


# --- density (nlfiber/density.py) ---------------------------------------------------------------
def hat_kernel_fft(shape, r):
    """nlfiber/density.py:23-31."""
    grids = np.meshgrid(*[np.minimum(np.arange(n), n - np.arange(n)) for n in shape], indexing="ij")
    dist = np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))
    k = np.maximum(0.0, r - dist)
    if k.sum() == 0:
        k[(0,) * len(shape)] = 1.0
    k /= k.sum()
    return np.fft.rfftn(k)


def filt(x, kfft):
    """nlfiber/density.py:34-36."""
    return np.fft.irfftn(np.fft.rfftn(x) * kfft, s=x.shape, axes=tuple(range(x.ndim)))


def _sigmoid(t):
    return 0.5 * (1.0 + np.tanh(0.5 * t))


def solve_eta(u, v, beta):
    """nlfiber/density.py:43-63: bisection (200 halvings) then 3 Newton steps."""
    lo = np.min(u) - 40.0 / beta
    hi = np.max(u) + 40.0 / beta
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        big = np.mean(_sigmoid(beta * (u - mid))) > v
        lo, hi = (mid, hi) if big else (lo, mid)
    eta = 0.5 * (lo + hi)
    for _ in range(3):
        s = _sigmoid(beta * (u - eta))
        dv = -np.mean(beta * s * (1 - s))
        eta = eta - (np.mean(s) - v) / (-1.0 if dv == 0 else dv)
    return eta


def threshold(u, v, beta):
    """nlfiber/density.py:66-72 (value only)."""
    return _sigmoid(beta * (u - solve_eta(u, v, beta)))


class DensityMap:
    """nlfiber/density.py:75-122: phi (symmetric octant) -> rho (full cell) with volume v at sharpness beta."""

    def __init__(self, n_o, d=3, r=1.5, v=0.3):
        self.n_o, self.d, self.r, self.v = n_o, d, r, v
        self.n = 2 * n_o
        self.shape = (self.n,) * d
        self.kfft = hat_kernel_fft(self.shape, r)

    def smooth(self, phi):
        u = filt(mirror(sym_perm(phi)), self.kfft)
        u = u / (np.std(u) + 1e-12)
        return exact_symmetrize(u)

    def rho(self, phi, beta):
        return threshold(self.smooth(phi), self.v, beta)

    def binary(self, phi, up=1, v=None, remove_floating=True):
        """nlfiber/density.py:96-122: smooth, upsample by `up` (periodic multilinear, then exact_symmetrize),
        threshold at the volume fraction, remove floating pieces and grow back."""
        v = self.v if v is None else v
        u = np.asarray(self.smooth(phi), dtype=np.float64)
        if up > 1:
            u = exact_symmetrize(upsample_periodic(u, up))
        return binary_from_u(u, v, remove_floating)


def binary_from_u(u, v, remove_floating=True):
    """nlfiber/density.py:105-122, the steps of DensityMap.binary after the smoothing (and upsampling)."""
    u = np.asarray(u, dtype=np.float64)
    b = u > np.quantile(u, 1.0 - v)
    if remove_floating:
        for _ in range(500):
            b = remove_floating_pieces(b)
            missing = v - b.mean()
            if missing * b.size < 1 or not b.any():
                break
            front = _dilate_periodic(b) & ~b
            cand = np.sort(u[front])[::-1]
            if cand.size == 0:
                break
            k = min(max(int(round(missing * b.size)), 1), cand.size)
            b = b | (front & (u >= cand[k - 1]))
        b = remove_floating_pieces(b)
    return b


def upsample_periodic(c, f):
    """nlfiber/density.py:133-149: periodic multilinear resampling of a cell-centred field by a factor f, axis by
    axis (output index X samples x = (X + 0.5) n / m - 0.5 between floor(x) and floor(x) + 1, periodic)."""
    out = np.asarray(c, dtype=np.float64)
    for ax in range(out.ndim):
        n = out.shape[ax]
        m = int(round(n * f))
        x = (np.arange(m) + 0.5) * n / m - 0.5
        i0 = np.floor(x).astype(int)
        w = x - i0
        a = np.take(out, i0 % n, axis=ax)
        b = np.take(out, (i0 + 1) % n, axis=ax)
        shp = [1] * out.ndim
        shp[ax] = m
        w = w.reshape(shp)
        out = (1 - w) * a + w * b
    return out


def rho_vjp(dm, phi, beta, gbar):
    """Cotangent of phi for the cotangent gbar of rho = dm.rho(phi, beta): the linear map that JAX's reverse mode
    gives for nlfiber/density.py:66-72 (threshold, with the implicit d eta = d.du / 1.d, d = s (1 - s)) composed
    with DensityMap.smooth (density.py:84-88) and the symmetry maps (symmetry.py:25-65).

    Transposes used: exact_symmetrize^T averages a field over each symmetry orbit of the full cell (mirror^T sums
    the 8 mirror images, from_free^T sums an orbit's octant points, to_free^T puts the sum at the sorted triple,
    sym_perm^T = sym_perm spreads it back with 1/6 per permutation, fold^T = mirror / 8); the cone filter is
    symmetric (k(g) = k(-g)), so filt^T = filt; sym_perm^T = sym_perm; u / (std(u) + 1e-12) has
    d(std)/du_j = (u_j - mean u) / (N std)."""
    phi = np.asarray(phi, dtype=np.float64)
    gbar = np.asarray(gbar, dtype=np.float64)
    x = mirror(sym_perm(phi))
    u_raw = filt(x, dm.kfft)
    sd = np.std(u_raw)
    D = sd + 1e-12
    u_sym = exact_symmetrize(u_raw / D)
    eta = solve_eta(u_sym, dm.v, beta)
    s = _sigmoid(beta * (u_sym - eta))
    d = s * (1.0 - s)
    w = gbar * beta * d
    ubar = w - d * (w.sum() / d.sum())                      # threshold
    ubar = _orbit_mean(ubar)                                # exact_symmetrize^T
    N = ubar.size
    ubar = ubar / D - (np.sum(ubar * u_raw) / D ** 2) * (u_raw - u_raw.mean()) / (N * sd)   # unit-std scaling
    ubar = filt(ubar, dm.kfft)                              # filter (symmetric kernel)
    return sym_perm(_mirror_T(ubar))                        # mirror^T, sym_perm^T


def _mirror_T(full):
    """Transpose of mirror: the octant sum of the 8 mirror images."""
    x = np.asarray(full)
    for ax in range(x.ndim):
        n = x.shape[ax] // 2
        x = np.take(x, np.arange(n), axis=ax) + np.flip(np.take(x, np.arange(n, 2 * n), axis=ax), ax)
    return x


def _orbit_mean(full):
    """Mean of a full-cell field over each orbit of the 48 mirror / permutation symmetries (= exact_symmetrize^T,
    and the orthogonal projection onto symmetric fields)."""
    oct_sum = _mirror_T(full)
    n_o, d = oct_sum.shape[0], oct_sum.ndim
    rep = representative_index(n_o, d)
    tot = np.bincount(rep.ravel(), weights=oct_sum.ravel())
    cnt = np.bincount(rep.ravel()) * 2 ** d
    return mirror((tot / cnt)[rep])


def _dilate_periodic(b):
    """nlfiber/density.py:125-130."""
    out = b.copy()
    for ax in range(b.ndim):
        out = out | np.roll(out, 1, axis=ax) | np.roll(out, -1, axis=ax)
    return out


# --- topology (nlfiber/topology.py:8-63) ---------------------------------------------------------
def periodic_label(b, faces=False):
    """Connected components of a periodic binary array (26-connectivity in 3D, 8 in 2D; with `faces`, the
    face connectivity ndimage.generate_binary_structure(d, 1) that topology.py:90,116 uses for the void)."""
    b = np.asarray(b, dtype=bool)
    d = b.ndim
    p = np.pad(b, 1, mode="wrap")
    st = ndimage.generate_binary_structure(d, 1) if faces else np.ones((3,) * d, dtype=bool)
    lab, n = ndimage.label(p, structure=st)
    parent = np.arange(n + 1)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    core = lab[tuple(slice(1, -1) for _ in range(d))]
    for ax in range(d):
        for side, src in ((0, -2), (-1, 1)):
            sl_p = [slice(None)] * d
            sl_p[ax] = side
            sl_c = [slice(None)] * d
            sl_c[ax] = src
            a = lab[tuple(sl_p)].ravel()
            c = lab[tuple(sl_c)].ravel()
            for x, y in zip(a[(a > 0) & (c > 0)], c[(a > 0) & (c > 0)]):
                rx, ry = find(x), find(y)
                if rx != ry:
                    parent[max(rx, ry)] = min(rx, ry)
    roots = np.array([find(i) for i in range(n + 1)])
    core = roots[core]
    uniq = np.unique(core[core > 0])
    remap = np.zeros(n + 1, dtype=np.int64)
    remap[uniq] = np.arange(1, len(uniq) + 1)
    return remap[core], len(uniq)


def _spanning(labels, k):
    m = labels == k
    for ax in range(m.ndim):
        other = tuple(a for a in range(m.ndim) if a != ax)
        if not np.all(m.any(axis=other)):
            return False
    return True


def remove_floating_pieces(b):
    """nlfiber/topology.py:57-63: keep only the spanning solid components."""
    lab, n = periodic_label(b)
    keep = np.zeros(n + 1, dtype=bool)
    for k in range(1, n + 1):
        keep[k] = _spanning(lab, k)
    return keep[lab]


# --- generators (nlfiber/fiber.py:103-121, tests/helpers.py:8-24, README.md:62-66) ------------------
def random_start(n_o, d=3, seed=0, kmax=3, nterms=40):
    """nlfiber/fiber.py:103-121: random smooth symmetric pre-density, standardized."""
    rng = np.random.default_rng(seed)
    n = 2 * n_o
    x = (np.arange(n_o) + 0.5) / n
    f = np.zeros((n_o,) * d)
    for _ in range(nterms):
        k = rng.integers(0, kmax + 1, size=d)
        if not k.any():
            continue
        a = rng.standard_normal() / np.linalg.norm(k)
        term = np.ones(())
        for ax in range(d):
            shp = [1] * d
            shp[ax] = n_o
            term = term * np.cos(2 * np.pi * k[ax] * x).reshape(shp)
        f = f + a * term
    f = sym_perm(f)
    return (f - f.mean()) / (f.std() + 1e-12)


def schwarz_p_phi(n_o, d=3):
    """tests/helpers.py:8-11 (the README Schwarz-P pre-density)."""
    x = 2 * np.pi * (np.arange(n_o) + 0.5) / (2 * n_o)
    G = np.meshgrid(*[x] * d, indexing="ij")
    return -sum(np.cos(g) for g in G)


def grey_cell(n_o=4, d=3, v=0.35, beta=3.0, seed=0):
    """tests/helpers.py:21-24."""
    phi = random_start(n_o, d, seed=seed, kmax=1) + 0.5 * schwarz_p_phi(n_o, d)
    return DensityMap(n_o, d, r=1.0, v=v).rho(sym_perm(phi), beta)


def binary_cell(n_o=4, d=3, v=0.35, seed=None):
    """tests/helpers.py:14-18."""
    phi = schwarz_p_phi(n_o, d) if seed is None else random_start(n_o, d, seed=seed, kmax=1)
    return DensityMap(n_o, d, r=1.0, v=v).binary(np.asarray(phi))


# --- benchmark workloads (seeded synthetic cells; no dataset is involved) ---------------------------
def schwarz_p_cell(n_o=16, v=0.3, r=1.5, beta=16.0):
    """Single Schwarz-P cell of side 2 n_o at volume v (README.md:62-66 with DensityMap(16, r=1.5, v=0.3))."""
    return DensityMap(n_o, 3, r=r, v=v).rho(schwarz_p_phi(n_o), beta)


def random_cell(i, n_o=16, r=1.5, beta=16.0, kmax=2, vol_seed_base=10_000, v=None):
    """Cell i of the batched workload: phi = random_start(n_o, seed=i, kmax=2), v ~ U[0.2, 0.5] drawn from
    default_rng(vol_seed_base + i), filter r = 1.5, sharpness beta."""
    if v is None:
        v = float(np.random.default_rng(vol_seed_base + i).uniform(0.2, 0.5))
    phi = random_start(n_o, 3, seed=i, kmax=kmax)
    return DensityMap(n_o, 3, r=r, v=v).rho(phi, beta), v
