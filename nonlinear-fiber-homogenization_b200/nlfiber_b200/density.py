"""Pre-density phi -> physical density rho with exact volume (host side, NumPy).

Mirror of nlfiber/density.py and nlfiber/symmetry.py (and nlfiber/fiber.py:103-121 `random_start`): the input
side of the homogenization solve. It produces rho on the host; the solve itself runs on the GPU.

    u   = F mirror(sym_perm(phi)) / std    periodic hat filter on the full cell, unit standard deviation
    rho = sigmoid(beta (u - eta)),         eta such that mean(rho) = v (bisection, then Newton)

`exact_symmetrize` copies one value per symmetry orbit, so symmetric voxels are bit-identical and a threshold
never splits an orbit (nlfiber/symmetry.py:60-65).
"""
import itertools

import numpy as np


def sym_perm(x):
    """nlfiber/symmetry.py:25-33: average over all permutations of the axes."""
    x = np.asarray(x, dtype=np.float64)
    perms = list(itertools.permutations(range(x.ndim)))
    out = 0
    for p in perms:
        out = out + np.transpose(x, p)
    return out / len(perms)


def mirror(oct_):
    """nlfiber/symmetry.py:36-41: octant (n_o)^d -> full cell (2 n_o)^d."""
    x = np.asarray(oct_)
    for ax in range(x.ndim):
        x = np.concatenate([x, np.flip(x, ax)], axis=ax)
    return x


def fold(full):
    """nlfiber/symmetry.py:44-52: full cell -> octant, averaging the mirror images."""
    x = np.asarray(full)
    for ax in range(x.ndim):
        n = x.shape[ax] // 2
        x = 0.5 * (np.take(x, np.arange(n), axis=ax) + np.flip(np.take(x, np.arange(n, 2 * n), axis=ax), ax))
    return x


_REP = {}


def representative_index(n_o, d=3):
    """nlfiber/symmetry.py:88-96: for every octant index, the position of its sorted index tuple among the free
    entries (i <= j <= k), in lexicographic order of the sorted tuples."""
    key = (n_o, d)
    if key not in _REP:
        grid = np.stack(np.meshgrid(*[np.arange(n_o)] * d, indexing="ij"), axis=-1).reshape(-1, d)
        srt = np.sort(grid, axis=1)
        free = np.array(list(itertools.combinations_with_replacement(range(n_o), d)))
        code = lambda t: np.ravel_multi_index(tuple(t.T), (n_o,) * d)  # noqa: E731
        pos = np.full(n_o ** d, -1, dtype=np.int64)
        pos[code(free)] = np.arange(len(free))
        _REP[key] = pos[code(srt)].reshape((n_o,) * d)
    return _REP[key]


def exact_symmetrize(full):
    """nlfiber/symmetry.py:60-65: symmetric projection, one value copied exactly per orbit."""
    oct_ = sym_perm(fold(full))
    n_o, d = oct_.shape[0], oct_.ndim
    idx = np.array(list(itertools.combinations_with_replacement(range(n_o), d)))
    free_vals = oct_[tuple(idx.T)]  # nlfiber/symmetry.py:79-82 to_free
    return mirror(free_vals[representative_index(n_o, d)])


def hat_kernel_fft(shape, r):
    """nlfiber/density.py:23-31."""
    grids = np.meshgrid(*[np.minimum(np.arange(n), n - np.arange(n)) for n in shape], indexing="ij")
    dist = np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))
    k = np.maximum(0.0, r - dist)
    if k.sum() == 0:
        k[(0,) * len(shape)] = 1.0
    k /= k.sum()
    return np.fft.rfftn(k)


def _sigmoid(t):
    return 0.5 * (1.0 + np.tanh(0.5 * t))


def solve_eta(u, v, beta):
    """nlfiber/density.py:43-63: bisection (200 halvings), then 3 Newton steps."""
    u = np.asarray(u, dtype=np.float64)
    lo, hi = np.min(u) - 40.0 / beta, np.max(u) + 40.0 / beta
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if np.mean(_sigmoid(beta * (u - mid))) > v:
            lo = mid
        else:
            hi = mid
    eta = 0.5 * (lo + hi)
    for _ in range(3):
        s = _sigmoid(beta * (u - eta))
        dv = -np.mean(beta * s * (1 - s))
        eta = eta - (np.mean(s) - v) / (-1.0 if dv == 0 else dv)
    return eta


class DensityMap:
    """nlfiber/density.py:75-94: phi (symmetric octant (n_o)^d) -> rho (full cell (2 n_o)^d), volume v."""

    def __init__(self, n_o, d=3, r=1.5, v=0.3):
        self.n_o, self.d, self.r, self.v = n_o, d, r, v
        self.n = 2 * n_o
        self.shape = (self.n,) * d
        self.kfft = hat_kernel_fft(self.shape, r)

    def smooth(self, phi):
        x = mirror(sym_perm(phi))
        u = np.fft.irfftn(np.fft.rfftn(x) * self.kfft, s=x.shape, axes=tuple(range(x.ndim)))
        u = u / (np.std(u) + 1e-12)
        return exact_symmetrize(u)

    def rho(self, phi, beta):
        u = self.smooth(phi)
        return _sigmoid(beta * (u - solve_eta(u, self.v, beta)))

    def eta(self, phi, beta):
        return float(solve_eta(self.smooth(phi), self.v, beta))


def random_start(n_o, d=3, seed=0, kmax=3, nterms=40):
    """nlfiber/fiber.py:103-121: random smooth symmetric pre-density (low-frequency cosine series)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n_o) + 0.5) / (2 * n_o)
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
    """The Schwarz-P pre-density of the reference's README (README.md:62-66): -(cos X + cos Y + cos Z)."""
    x = 2 * np.pi * (np.arange(n_o) + 0.5) / (2 * n_o)
    return -sum(np.cos(g) for g in np.meshgrid(*[x] * d, indexing="ij"))


def random_cell(i, n_o=16, r=1.5, beta=16.0, kmax=2, vol_seed_base=10_000, v=None):
    """Seeded synthetic cell i: phi = random_start(n_o, seed=i, kmax=2), v ~ U[0.2, 0.5] from
    default_rng(vol_seed_base + i), hat filter r, sharpness beta. Returns (rho, v)."""
    if v is None:
        v = float(np.random.default_rng(vol_seed_base + i).uniform(0.2, 0.5))
    return DensityMap(n_o, 3, r=r, v=v).rho(random_start(n_o, 3, seed=i, kmax=kmax), beta), v
