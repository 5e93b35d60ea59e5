"""Periodic finite-strain homogenization on voxel grids, computed on the GPU by libnlf.so.

Drop-in for the hot path of nlfiber/mech.py: `Cell` (energy, residual, mean stress, displacement gradient,
preconditioner) and `Mixed` (mixed macroscopic control, Newton-CG with Eisenstat-Walker forcing and the Armijo
line search). The energy, residual, matrix-free tangent matvec and the preconditioned CG run on the device in
FP64; the Newton loop stays on the host, as in the reference (mech.py:302-346). The tangent is never stored:
`Mixed.tangent(z, Fb)` returns the linearization point and `hvp_A` applies the closed-form second derivative.

Not here (they are callers of this path): `grad_rho`, `lowest_eigs`, `effective_tangent`, `rank_one_min`, `toec`.
"""
import ctypes

import numpy as np

from ._lib import lib, check, ptr, as_f64
from .linear import NODES, dN_ref, lame, VOIGT, unit_strain  # noqa: F401  (mech.py:26)

DN = dN_ref()
I3 = np.eye(3)
STALL_RTOL = 1e-6  # mech.py:53
MATERIALS = ("linear", "neohooke")  # mech.py:52


def voigt_tensor(I):
    """mech.py:56-64."""
    H = np.zeros((3, 3))
    i, j = VOIGT[I]
    if i == j:
        H[i, i] = 1.0
    else:
        H[i, j] = H[j, i] = 0.5
    return H


def to_voigt(M):
    """mech.py:67-70."""
    S = 0.5 * (M + M.T)
    return np.array([S[0, 0], S[1, 1], S[2, 2], 2 * S[1, 2], 2 * S[0, 2], 2 * S[0, 1]])


def _is_dev(a):
    return hasattr(a, "is_cuda") and a.is_cuda


def _empty_like_kind(ref, shape):
    """An output buffer on the device of `ref` (a CUDA torch tensor) or on the host."""
    if _is_dev(ref):
        import torch
        return torch.empty(shape, dtype=torch.float64, device=ref.device)
    return np.empty(shape)


def _norm(v):
    if _is_dev(v):
        import torch
        return float(torch.linalg.vector_norm(v))
    return float(np.linalg.norm(v))


def _dot(a, b):
    if _is_dev(a):
        import torch
        return float(torch.dot(a, b))
    return float(a @ b)


def _linesearch(E, gnorm, x, dx, E0, slope, gn):
    """mech.py:73-85: halve from t = 1 until Armijo (1e-4) holds, or the energy is flat to rounding and the
    gradient norm drops; None below t = 1e-6."""
    tol = 64 * np.finfo(np.float64).eps * max(abs(E0), 1e-300)
    t = 1.0
    while t > 1e-6:
        Et = E(x + t * dx)
        if np.isfinite(Et):
            if Et <= E0 + 1e-4 * t * slope:
                return t
            if Et <= E0 + tol and gnorm(x + t * dx) < gn:
                return t
        t *= 0.5
    return None


class Cell:
    """mech.py:88-192: a periodic voxel cell; rho (nx, ny, nz) or (n, n) in [0, 1]."""

    def __init__(self, rho, E=1.0, nu=0.3, material="neohooke", wls=(500.0, 0.01), emin=1e-3, p=3.0):
        rho = np.ascontiguousarray(np.asarray(rho, dtype=np.float64))
        if rho.ndim == 2:
            rho = rho[..., None]
        if material not in MATERIALS:
            raise KeyError(material)
        self.rho, self.shape = rho, tuple(rho.shape)
        self.N = int(np.prod(self.shape))
        self.E, self.nu, self.material, self.wls, self.emin, self.p = E, nu, material, wls, emin, p
        self.lam, self.mu = lame(E, nu)
        self.wq = 1.0 / (8.0 * self.N)
        h = ctypes.c_void_p()
        b, r0 = (0.0, 0.0) if wls is None else (float(wls[0]), float(wls[1]))
        check(lib.nlf_mech_create(ctypes.byref(h), *self.shape, float(E), float(nu), MATERIALS.index(material), b,
                                  r0, float(emin), float(p)))
        self._h = h
        self.stream = None
        self.s = np.empty(self.shape)
        gam = np.empty(self.shape) if wls is not None else None
        sws = ctypes.c_double()
        check(lib.nlf_mech_set_rho(h, ptr(rho), ptr(self.s), ptr(gam), ctypes.byref(sws), None))
        self.gamma = gam if wls is not None else None
        self.sws = sws.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.nlf_mech_destroy(h)
            self._h = None

    def scale_of(self, rho):
        """mech.py:105-106."""
        return self.emin + (1.0 - self.emin) * np.clip(np.asarray(rho, dtype=np.float64), 0.0, 1.0) ** self.p

    def with_rho(self, rho):
        """mech.py:115-116."""
        return Cell(rho, self.E, self.nu, self.material, self.wls, self.emin, self.p)

    def tiled(self, k):
        """mech.py:118-121: k x k x k supercell (2D: k x k x 1)."""
        reps = (k, k, 1) if self.shape[2] == 1 else (k, k, k)
        return Cell(np.tile(self.rho, reps), self.E, self.nu, self.material, self.wls, self.emin, self.p)

    # --- discretization ------------------------------------------------------------------------------------
    def grad_w(self, w):
        """mech.py:127-129: (8, nx, ny, nz, 3, 3), H[..., i, j] = d w_i / d x_j at each Gauss point."""
        w = as_f64(w)
        out = np.empty((8,) + self.shape + (3, 3))
        check(lib.nlf_mech_grad_w(self._h, ptr(w), ptr(out), self.stream))
        return out

    def energy(self, w, Fbar, rho=None):
        """mech.py:141-152 (rho: evaluate with another density, as the reference's adjoint uses it)."""
        if rho is not None:
            return self.with_rho(rho).energy(w, Fbar)
        W = ctypes.c_double()
        check(lib.nlf_mech_energy(self._h, ptr(as_f64(w)), ptr(as_f64(Fbar)), ctypes.byref(W), None, None,
                                  self.stream))
        return W.value

    def grad(self, w, Fbar):
        """(dW/dw (nx, ny, nz, 3), dW/dFbar (3, 3)): the reference's jax.grad of `energy` (mech.py:168-169).
        dW/dw is a CUDA tensor when w is one."""
        W = ctypes.c_double()
        gw = _empty_like_kind(w, self.shape + (3,))
        P = np.empty((3, 3))
        check(lib.nlf_mech_energy(self._h, ptr(as_f64(w)), ptr(as_f64(Fbar)), ctypes.byref(W), ptr(gw), ptr(P),
                                  self.stream))
        return gw, P

    def mean_stress(self, w, Fbar):
        """mech.py:191-192: Pbar = dW / dFbar."""
        return self.grad(w, Fbar)[1]

    def hvp(self, w, Fbar, v, dFbar):
        """Second derivative of W at (w, Fbar) applied to (v, dFbar): (dw part, dFbar part)."""
        hv = _empty_like_kind(v, self.shape + (3,))
        hP = np.empty((3, 3))
        check(lib.nlf_mech_hvp(self._h, ptr(as_f64(w)), ptr(as_f64(Fbar)), ptr(as_f64(v)), ptr(as_f64(dFbar)),
                               ptr(hv), ptr(hP), self.stream))
        return hv, hP

    def precond_w(self, r):
        """mech.py:187-189."""
        z = _empty_like_kind(r, self.shape + (3,))
        check(lib.nlf_mech_precond_w(self._h, ptr(as_f64(r)), ptr(z), self.stream))
        return z


class Tangent:
    """The linearization point (z, Fb) standing in for the reference's stored tangent (mech.py:239-240)."""

    def __init__(self, w, F):
        self.w, self.F = w, F


class Mixed:
    """mech.py:195-346: Fbar components in `free` are unknowns with zero conjugate stress, the rest prescribed.
    Unknown z = (w, Fbar_free); minimizes W(z) by Newton-CG."""

    def __init__(self, cell, free=((1, 1), (2, 2)), forcing="ew", precond="fft", device=None):
        """precond "fft" is the reference's preconditioner (homogeneous inverse / sws); "scaled" wraps the same
        inverse in the node stiffness scaling (same solution, fewer CG iterations at high contrast). The choice
        is kept by the cell's device handle. device="cuda" keeps the Newton state z and every Newton vector in
        CUDA tensors that the library reads and writes in place (only scalars and the macro values go to the
        host); None keeps them in NumPy, as the reference's host loop does."""
        self.device = device
        self.c = cell
        self.free = [tuple(f) for f in free]
        self.forcing = forcing
        if precond not in ("fft", "scaled"):
            raise ValueError(f"precond must be 'fft' or 'scaled', got {precond!r}")
        self.precond_kind = precond
        check(lib.nlf_mech_set_precond(cell._h, 1 if precond == "scaled" else 0))
        self.shape = cell.shape
        self.nw = 3 * cell.N
        self.k = len(self.free)
        self.idx = tuple(np.array(self.free).T) if self.k else None
        self._free_idx = np.ascontiguousarray(np.array(self.free, dtype=np.int32).ravel() if self.k else
                                              np.zeros(2, np.int32))

    def unpack(self, z, Fb):
        """mech.py:209-211."""
        if not _is_dev(z):
            z = np.asarray(z)
        w = z[: self.nw].reshape(self.shape + (3,))
        F = np.array(Fb, dtype=np.float64)
        if self.k:
            F[self.idx] = z[self.nw:].cpu().numpy() if _is_dev(z) else z[self.nw:]
        return w, F

    def _as_state(self, v):
        """v in the state's kind: a CUDA float64 tensor with device="cuda", else a NumPy array."""
        if self.device is None:
            return v.cpu().numpy() if _is_dev(v) else np.asarray(v, dtype=np.float64)
        import torch
        return torch.as_tensor(v, dtype=torch.float64, device=self.device)

    def _cat(self, w, tail):
        """(w part, macro tail) -> one vector of the state's kind."""
        if _is_dev(w):
            import torch
            return torch.cat([w.reshape(-1), torch.as_tensor(np.asarray(tail, dtype=np.float64), device=w.device)])
        return np.concatenate([np.asarray(w).ravel(), np.asarray(tail, dtype=np.float64)])

    def z0(self, Fb):
        """mech.py:243-245."""
        Fb = np.asarray(Fb, dtype=np.float64)
        return self._as_state(np.concatenate([np.zeros(self.nw), Fb[self.idx] if self.k else np.zeros(0)]))

    def proj(self, v):
        """mech.py:247-250."""
        w = v[: self.nw].reshape(self.shape + (3,))
        if _is_dev(v):
            import torch
            w = w - w.mean(dim=(0, 1, 2))
            return torch.cat([w.reshape(-1), v[self.nw:]])
        w = w - w.mean(axis=(0, 1, 2))
        return np.concatenate([w.ravel(), v[self.nw:]])

    def Ez(self, z, Fb):
        """mech.py:215-217."""
        return self.c.energy(*self.unpack(z, Fb))

    def _E(self, z, Fb):
        return self.Ez(z, Fb)

    def _g(self, z, Fb):
        """Gradient of Ez in z (mech.py:221)."""
        gw, P = self.c.grad(*self.unpack(z, Fb))
        return self._cat(gw, P[self.idx] if self.k else np.zeros(0))

    def tangent(self, z, Fb):
        return Tangent(*self.unpack(z, Fb))

    def hvp_A(self, A, v):
        """mech.py:233-236 with the tangent applied matrix-free at A's linearization point."""
        v = self._as_state(v)
        dF = np.zeros((3, 3))
        if self.k:
            dF[self.idx] = v[self.nw:].cpu().numpy() if _is_dev(v) else v[self.nw:]
        vw = v[: self.nw].reshape(self.shape + (3,))
        hv, hP = self.c.hvp(A.w, A.F, vw.contiguous() if _is_dev(vw) else np.ascontiguousarray(vw), dF)
        return self._cat(hv, hP[self.idx] if self.k else np.zeros(0))

    def macro_diag(self, A, Fb=None):
        """mech.py:252-258."""
        d = []
        for j in range(self.k):
            if self.device is None:
                e = np.zeros(self.nw + self.k)
            else:
                import torch
                e = torch.zeros(self.nw + self.k, dtype=torch.float64, device=self.device)
            e[self.nw + j] = 1.0
            d.append(float(self.hvp_A(A, e)[self.nw + j]))
        return np.abs(np.array(d)) + 1e-12

    def precond(self, r, dmac, swscale):
        """mech.py:260-262."""
        rw = r[: self.nw].reshape(self.shape + (3,))
        w = self.c.precond_w(rw.contiguous() if _is_dev(rw) else np.ascontiguousarray(rw)) / swscale
        tail = (r[self.nw:].cpu().numpy() if _is_dev(r) else r[self.nw:]) / dmac
        return self._cat(w, tail)

    def _sws(self):
        """mech.py:292-294 (1 for the scaled preconditioner, which carries the stiffness itself)."""
        return 1.0 if self.precond_kind == "scaled" else self.c.sws

    def _cgA(self, A, b, dmac, sws, tol, maxit):
        """mech.py:264-290 on the device: (x, iterations, converged, negative curvature)."""
        x = _empty_like_kind(b, self.nw + self.k)
        it, conv, neg = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        dm = np.ascontiguousarray(np.asarray(dmac, dtype=np.float64) if self.k else np.ones(1))
        check(lib.nlf_mech_cg(self.c._h, ptr(as_f64(A.w)), ptr(as_f64(A.F)), self.k, ptr(self._free_idx),
                              ptr(as_f64(b)), ptr(dm), float(sws), float(tol), int(maxit), ptr(x),
                              ctypes.byref(it), ctypes.byref(conv), ctypes.byref(neg), 8, self.c.stream))
        return x, it.value, bool(conv.value), bool(neg.value)

    def solve_linear(self, A, b, tol=1e-10, maxit=20000):
        """mech.py:296-300."""
        dmac = self.macro_diag(A, None) if self.k else np.zeros(0)
        x, it, conv, neg = self._cgA(A, b, dmac, self._sws(), tol, int(maxit))
        return x, it, conv

    def solve(self, Fbar, z0=None, rtol=1e-9, maxnewton=30, cg_tol=1e-6, cg_maxit=20000, g_ref=None):
        """mech.py:302-346: Newton-CG. Returns (w, Fbar_full, log) with log['z'] the state."""
        Fb = np.asarray(Fbar, dtype=np.float64)
        z = self.z0(Fb) if z0 is None else self._as_state(z0)
        g0, log = g_ref, dict(newton=0, cg=0, converged=False, gnorm=[], negative_curvature=False)
        eta, gprev = None, None
        sws = self._sws()
        for k in range(maxnewton):
            g = self.proj(self._g(z, Fb))
            gn = _norm(g)
            g0 = gn if g0 is None else g0
            log["gnorm"].append(gn)
            if gn <= rtol * max(g0, 1e-300) or gn < 1e-14:
                log["converged"] = True
                break
            tol = cg_tol
            if self.forcing == "ew":
                e_new = 0.1 if gprev is None else 0.9 * (gn / gprev) ** 2
                if eta is not None and 0.9 * eta ** 2 > 0.1:
                    e_new = max(e_new, 0.9 * eta ** 2)
                eta = min(e_new, 0.1)
                tol = max(eta, cg_tol, 0.5 * rtol * g0 / gn) if gprev is not None else max(eta, cg_tol)
            gprev = gn
            A = self.tangent(z, Fb)
            dmac = self.macro_diag(A, Fb) if self.k else np.zeros(0)
            dz, its, ok, neg = self._cgA(A, -g, dmac, sws, tol, int(cg_maxit))
            log["cg"] += int(its)
            log["negative_curvature"] |= bool(neg)
            E0, slope = float(self._E(z, Fb)), _dot(g, dz)
            if slope >= 0:
                dz = -self.proj(self.precond(g, dmac, sws))
                slope = _dot(g, dz)
            t = _linesearch(lambda x: self._E(x, Fb), lambda x: _norm(self.proj(self._g(x, Fb))),
                            z, dz, E0, slope, gn)
            log["newton"] = k + 1
            if t is None:
                log["linesearch_failed"] = True
                if gn <= STALL_RTOL * g0:
                    log["converged"] = log["roundoff_floor"] = True
                break
            z = z + t * dz
        w, F = self.unpack(z, Fb)
        log["z"], log["g0"] = z, g0
        return w, F, log


# --- third-order elastic constants (mech.py:458-515) --------------------------------------------------------------
def toec(cell, chi):
    """mech.py:458-493: C (6x6) and the Lagrangian-strain third-order constants T (6x6x6) of `cell` from the linear
    correctors chi (6, nx, ny, nz, 3) of the unit Voigt strains (nlf_mech_toec; f'' and f''' in closed form)."""
    C = np.empty((6, 6))
    T = np.empty((6, 6, 6))
    check(lib.nlf_mech_toec(cell._h, ptr(as_f64(chi)), ptr(C), ptr(T), cell.stream))
    return C, T


CUBIC_TOEC = {  # mech.py:496-503: index triples averaged into each cubic constant
    "C111": [(0, 0, 0), (1, 1, 1), (2, 2, 2)],
    "C112": [(0, 0, 1), (0, 0, 2), (1, 1, 0), (1, 1, 2), (2, 2, 0), (2, 2, 1)],
    "C123": [(0, 1, 2)],
    "C144": [(0, 3, 3), (1, 4, 4), (2, 5, 5)],
    "C155": [(0, 4, 4), (0, 5, 5), (1, 3, 3), (1, 5, 5), (2, 3, 3), (2, 4, 4)],
    "C456": [(3, 4, 5)],
}


def cubic_toec(T):
    """mech.py:511-515: the six cubic TOECs as means over their index triples."""
    return {k: float(np.mean([T[i] for i in v])) for k, v in CUBIC_TOEC.items()}
