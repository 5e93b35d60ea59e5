"""Pre-density phi -> physical density rho with exact volume.

Mirror of nlfiber/density.py and nlfiber/symmetry.py (and nlfiber/fiber.py:103-121 `random_start`): the input
side of the homogenization solve. `DensityMap` runs on the host (NumPy, bit-identical to the test oracle);
`GpuDensityMap` is the same map for batches of cubic cells in libnlf.so (nlf_density_*), on CUDA tensors.

    u   = F mirror(sym_perm(phi)) / std    periodic hat filter on the full cell, unit standard deviation
    rho = sigmoid(beta (u - eta)),         eta such that mean(rho) = v (bisection, then Newton)

`exact_symmetrize` copies one value per symmetry orbit, so symmetric voxels are bit-identical and a threshold
never splits an orbit (nlfiber/symmetry.py:60-65).
"""
import ctypes
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


class GpuDensityMap:
    """DensityMap on the GPU (nlfiber/density.py:75-94 smooth / rho / eta) for cubic cells, batched.

    phi is an octant (n_o)^3 pre-density (or a batch (ncell, n_o, n_o, n_o)); NumPy arrays are copied in, CUDA
    float64 tensors are used in place. Results are CUDA float64 tensors. The filter runs as a direct periodic sum
    over its taps and the volume bisection over the symmetry orbits, so values agree with `DensityMap` to
    rounding (not bitwise); symmetric voxels are bit-identical and mean(rho) = v to rounding."""

    def __init__(self, n_o, d=3, r=1.5, v=0.3):
        if d != 3:
            raise ValueError("GpuDensityMap takes cubic cells (d = 3)")
        from ._lib import check, lib
        self.n_o, self.d, self.r, self.v = int(n_o), d, float(r), float(v)
        self.n = 2 * self.n_o
        self.shape = (self.n,) * 3
        h = ctypes.c_void_p()
        check(lib.nlf_density_create(ctypes.byref(h), self.n_o, self.r))
        self._h = h
        self._lib = lib  # kept for __del__, which may run while the interpreter shuts down
        self.orbits = int(lib.nlf_density_orbits(h))
        self.stream = None

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(self, "_lib", None)
        if h is not None and h.value and lib is not None:
            lib.nlf_density_destroy(h)
            self._h = None

    def _phi(self, phi):
        import torch
        if torch.is_tensor(phi):
            phi = phi.to(device="cuda", dtype=torch.float64).contiguous()
        else:
            phi = torch.as_tensor(np.ascontiguousarray(np.asarray(phi, dtype=np.float64)), device="cuda")
        if phi.dim() == 3:
            phi = phi.unsqueeze(0)
        if tuple(phi.shape[1:]) != (self.n_o,) * 3:
            raise ValueError(f"phi must be (ncell, {self.n_o}, {self.n_o}, {self.n_o}), got {tuple(phi.shape)}")
        return phi

    def run(self, phi, beta, v=None, rho=True, smooth=False, eta=True):
        """The map for a batch: {"rho": (ncell, n, n, n), "u": smoothed field or None, "eta": (ncell,)};
        v is a scalar or one volume fraction per cell (default: the map's v)."""
        import torch
        from ._lib import check, lib, ptr
        phi = self._phi(phi)
        nc = phi.shape[0]
        vv = torch.as_tensor(np.broadcast_to(np.asarray(self.v if v is None else v, dtype=np.float64), (nc,)).copy(),
                             device="cuda")
        out = {k: (torch.empty((nc,) + self.shape, dtype=torch.float64, device="cuda") if want else None)
               for k, want in (("rho", rho), ("u", smooth))}
        out["eta"] = torch.empty(nc, dtype=torch.float64, device="cuda") if eta else None
        check(lib.nlf_density_rho(self._h, nc, ptr(phi), ptr(vv), float(beta), ptr(out["rho"]), ptr(out["u"]),
                                  ptr(out["eta"]), self.stream))
        return out

    def vjp(self, phi, beta, rho_bar, v=None):
        """Cotangents of phi for cotangents of rho (the reverse mode of `rho`, with the implicit d eta of
        nlfiber/density.py:66-72). phi (n_o,)*3 with rho_bar (nrow, n, n, n), or a batch (ncell, n_o, n_o, n_o)
        with rho_bar (ncell, nrow, n, n, n). Returns (nrow, n_o, n_o, n_o) or (ncell, nrow, n_o, n_o, n_o)."""
        import torch
        from ._lib import check, lib, ptr
        single = np.ndim(phi) == 3
        phi = self._phi(phi)
        nc = phi.shape[0]
        if torch.is_tensor(rho_bar):
            g = rho_bar.to(device="cuda", dtype=torch.float64).contiguous()
        else:
            g = torch.as_tensor(np.ascontiguousarray(np.asarray(rho_bar, dtype=np.float64)), device="cuda")
        if single:
            g = g.reshape((1, -1) + self.shape)
        if g.dim() != 5 or g.shape[0] != nc or tuple(g.shape[2:]) != self.shape:
            raise ValueError(f"rho_bar must be (ncell, nrow) + {self.shape}, got {tuple(g.shape)}")
        nrow = g.shape[1]
        vv = torch.as_tensor(np.broadcast_to(np.asarray(self.v if v is None else v, dtype=np.float64), (nc,)).copy(),
                             device="cuda")
        out = torch.empty((nc, nrow) + (self.n_o,) * 3, dtype=torch.float64, device="cuda")
        check(lib.nlf_density_vjp(self._h, nc, nrow, ptr(phi), ptr(vv), float(beta), ptr(g), ptr(out), self.stream))
        return out[0] if single else out

    def smooth(self, phi):
        return self.run(phi, 1.0, rho=False, smooth=True, eta=False)["u"][0]

    def rho(self, phi, beta):
        return self.run(phi, beta, eta=False)["rho"][0]

    def eta(self, phi, beta):
        return float(self.run(phi, beta, rho=False)["eta"][0])


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
