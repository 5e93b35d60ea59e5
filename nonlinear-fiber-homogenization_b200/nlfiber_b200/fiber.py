"""The constraint map of the fiber on the GPU: phi (symmetric octant) -> normalized stiffness invariants
c(phi) = (C11, C12, C44) / E in 3D, (C11, C12, C66) / E in 2D (plane strain), and its Jacobian
(nlfiber/fiber.py:17-60).

Value: the density map (libnlf.so nlf_density_rho), the cubic two-case corrector solve and C assembly
(nlf_linear_solve, nlf_bilinear). Jacobian rows: dc_k/drho with the correctors held fixed (nlf_dC_drho, exact
because the correctors are stationary), pulled back through the density map (nlf_density_vjp) -- the three
VJPs of the reference's `value_and_jac` (fiber.py:34-39), without JAX. Cubic (d = 3) and square (d = 2) cells.
Binary check (fiber.py:62-81): the binary cell of the density map on the GPU (GpuDensityMap.binary, floating
pieces removed), re-solved.
"""
import numpy as np

from .density import GpuDensityMap
from .linear import LinearHomogenization, cubic_invariants, cubic_leakage, unit_strain


class Fiber:
    """nlfiber/fiber.py:17-60 Fiber(n_o, d=3, v, r, E, nu, emin, p, tol): value, value_jac and rho, with the
    correctors of the last solve kept as the next warm start (`self.u`). Extra keyword arguments go to the
    solver (e.g. precond="scaled", energy_tol)."""

    def __init__(self, n_o, d=3, v=0.3, r=1.5, E=1.0, nu=0.3, emin=1e-3, p=3.0, tol=1e-9, **solver):
        self.n_o, self.d, self.v = n_o, d, v
        self.dm = GpuDensityMap(n_o, d, r, v)
        self._mat = dict(E=E, nu=nu, emin=emin, p=p, tol=tol, **solver)
        self.lh = LinearHomogenization(self.dm.shape, **self._mat)
        self._lh_bin = {}
        self.u = None  # warm start of the correctors
        self.solves = 0

    def _u0(self, warm):
        if self.u is None or not warm:
            return np.zeros((2,) + self.lh.shape + (3,))
        return self.u

    def _solve(self, phi, beta, warm):
        rho = self.dm.rho(phi, float(beta))
        c, u2, _ = self.lh.invariants(rho, self._u0(warm))
        self.u = u2
        self.solves += 1
        return rho, np.asarray(c), u2

    def value(self, phi, beta, warm=True):
        """nlfiber/fiber.py:47-51."""
        return self._solve(phi, beta, warm)[1]

    def value_jac(self, phi, beta, warm=True):
        """nlfiber/fiber.py:53-57: (c (3,), J (3,) + (n_o,)*d), J[k] = dc_k / dphi."""
        rho, c, u2 = self._solve(phi, beta, warm)
        lh = self.lh
        u3 = np.ascontiguousarray(np.stack([u2[0], lh.swap_xy(u2[0]), u2[1]]))
        Es = np.stack([unit_strain(0), unit_strain(1), unit_strain(lh._shear())])
        dC = lh.dC_drho(rho, Es, u3)
        rows = np.ascontiguousarray((np.stack([dC[0, 0], dC[1, 0], dC[2, 2]]) / lh.E).reshape((3,) + self.dm.shape))
        J = self.dm.vjp(phi, float(beta), rows)
        return c, J.cpu().numpy()

    def rho(self, phi, beta):
        """nlfiber/fiber.py:59-60 (a CUDA tensor)."""
        return self.dm.rho(phi, float(beta))

    # --- binary check (nlfiber/fiber.py:62-81) ----------------------------------------------------------------
    def lh_for(self, shape):
        """The solver for binary cells of this shape (kept per shape)."""
        shape = tuple(shape)
        if shape not in self._lh_bin:
            self._lh_bin[shape] = LinearHomogenization(shape, **self._mat)
        return self._lh_bin[shape]

    def binary_check(self, phi, up=1, full=False):
        """nlfiber/fiber.py:67-81: binarize (upsampled by `up`), drop floating pieces, re-solve. Returns
        dict(c, vol, cell[, C, leak])."""
        b = self.dm.binary(phi, up=up)
        lh = self.lh_for(b.shape)
        rho = b.astype(np.float64)
        out = dict(vol=float(b.mean()), cell=b)
        if full:
            C, _, _ = lh.C_full(rho)
            C = np.asarray(C)
            out.update(C=C, c=cubic_invariants(C) / lh.E, leak=cubic_leakage(C))
        else:
            c, _, _ = lh.invariants(rho)
            out["c"] = np.asarray(c)
        self.solves += 1
        return out
