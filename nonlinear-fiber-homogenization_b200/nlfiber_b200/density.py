"""Pre-density phi -> physical density rho with exact volume, on the GPU (nlfiber/density.py and
nlfiber/symmetry.py for cubic and square cells, batched, in libnlf.so: nlf_density_*).

    u   = F mirror(sym_perm(phi)) / std    periodic cone filter on the full cell, unit standard deviation
    rho = sigmoid(beta (u - eta)),         eta such that mean(rho) = v (bisection, then Newton)

The symmetric projection copies one value per symmetry orbit, so symmetric voxels are bit-identical and a threshold
never splits an orbit (nlfiber/symmetry.py:60-65). Inputs are NumPy arrays or CUDA float64 tensors; results are
CUDA float64 tensors, ready for `LinearHomogenization.C_full_batched`.
"""
import ctypes

import numpy as np


class GpuDensityMap:
    """DensityMap on the GPU (nlfiber/density.py:75-94 smooth / rho / eta) for cubic (d = 3) and square (d = 2)
    cells, batched.

    phi is an octant (n_o)^d pre-density (or a batch (ncell,) + (n_o,)*d); NumPy arrays are copied in, CUDA
    float64 tensors are used in place. Results are CUDA float64 tensors. The filter runs as a direct periodic sum
    over its taps and the volume bisection over the symmetry orbits, so values agree with `DensityMap` to
    rounding (not bitwise); symmetric voxels are bit-identical and mean(rho) = v to rounding."""

    def __init__(self, n_o, d=3, r=1.5, v=0.3):
        if d not in (2, 3):
            raise ValueError("GpuDensityMap takes cubic (d = 3) or square (d = 2) cells")
        from ._lib import check, lib
        self.n_o, self.d, self.r, self.v = int(n_o), int(d), float(r), float(v)
        self.n = 2 * self.n_o
        self.shape = (self.n,) * self.d
        h = ctypes.c_void_p()
        check(lib.nlf_density_create_d(ctypes.byref(h), self.n_o, self.d, self.r))
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
        if phi.dim() == self.d:
            phi = phi.unsqueeze(0)
        if tuple(phi.shape[1:]) != (self.n_o,) * self.d:
            raise ValueError(f"phi must be (ncell,) + {(self.n_o,) * self.d}, got {tuple(phi.shape)}")
        return phi

    def run(self, phi, beta, v=None, rho=True, smooth=False, eta=True):
        """The map for a batch: {"rho": (ncell,) + shape, "u": smoothed field or None, "eta": (ncell,)};
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
        nlfiber/density.py:66-72). phi (n_o,)*d with rho_bar (nrow,) + shape, or a batch (ncell,) + (n_o,)*d with
        rho_bar (ncell, nrow) + shape. Returns (nrow,) + (n_o,)*d or (ncell, nrow) + (n_o,)*d."""
        import torch
        from ._lib import check, lib, ptr
        single = (phi.dim() if torch.is_tensor(phi) else np.ndim(phi)) == self.d
        phi = self._phi(phi)
        nc = phi.shape[0]
        if torch.is_tensor(rho_bar):
            g = rho_bar.to(device="cuda", dtype=torch.float64).contiguous()
        else:
            g = torch.as_tensor(np.ascontiguousarray(np.asarray(rho_bar, dtype=np.float64)), device="cuda")
        if single:
            g = g.reshape((1, -1) + self.shape)
        if g.dim() != 2 + self.d or g.shape[0] != nc or tuple(g.shape[2:]) != self.shape:
            raise ValueError(f"rho_bar must be (ncell, nrow) + {self.shape}, got {tuple(g.shape)}")
        nrow = g.shape[1]
        vv = torch.as_tensor(np.broadcast_to(np.asarray(self.v if v is None else v, dtype=np.float64), (nc,)).copy(),
                             device="cuda")
        out = torch.empty((nc, nrow) + (self.n_o,) * self.d, dtype=torch.float64, device="cuda")
        check(lib.nlf_density_vjp(self._h, nc, nrow, ptr(phi), ptr(vv), float(beta), ptr(g), ptr(out), self.stream))
        return out[0] if single else out

    def smooth(self, phi):
        return self.run(phi, 1.0, rho=False, smooth=True, eta=False)["u"][0]

    def rho(self, phi, beta):
        return self.run(phi, beta, eta=False)["rho"][0]

    def eta(self, phi, beta):
        return float(self.run(phi, beta, rho=False)["eta"][0])

    def binary(self, phi, up=1, v=None, remove_floating=True):
        """nlfiber/density.py:96-122: the binary cell of phi, a NumPy bool array of side 2 n_o (2 (m / 2) with
        m = round(2 n_o up) when up > 1). The smoothed field u (nlf_density_rho), its periodic multilinear
        upsampling by `up` with exact symmetrization (nlf_upsample_sym), the threshold at the volume fraction v and
        the removal of floating pieces with regrowth towards v (nlf_topo_binary) all run on the device."""
        from .topology import cells, upsample_sym
        v = self.v if v is None else v
        u = self.run(phi, 1.0, rho=False, smooth=True, eta=False)["u"][0]
        if up > 1:
            u = upsample_sym(u, up)
        return cells(self.d, u.shape[0]).binary(u, v, remove_floating)
