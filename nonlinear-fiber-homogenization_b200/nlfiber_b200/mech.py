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


def _backtrack(energy_at, gnorm_at, E0, slope, gn, c1=1e-4, t_min=1e-6):
    """Step length along a descent direction (the rule of nlfiber/mech.py:73-85). Trial steps t = 1, 1/2, 1/4, ...
    while t > t_min; a trial is accepted when its energy is finite and either meets the sufficient-decrease
    (Armijo) condition E(t) <= E0 + c1 t slope, or lies within 64 ulps of E0 (the energy is flat to rounding)
    while the gradient norm at t is below gn. Returns the accepted t, or None."""
    flat = E0 + 64 * np.finfo(np.float64).eps * max(abs(E0), 1e-300)
    trials = 1.0 / 2.0 ** np.arange(64)
    for t in trials[trials > t_min]:
        e = energy_at(float(t))
        if not np.isfinite(e):
            continue
        if e <= E0 + c1 * t * slope or (e <= flat and gnorm_at(float(t)) < gn):
            return float(t)
    return None


class _Forcing:
    """CG tolerance per Newton step (the rule of nlfiber/mech.py:310-322). With Eisenstat-Walker forcing
    (Eisenstat & Walker 1996, choice 2 with gamma 0.9 and exponent 2): eta = 0.1 at the first step, then
    0.9 (||g|| / ||g_prev||)^2, kept at least 0.9 eta_prev^2 when that exceeds 0.1, and capped at 0.1; the
    tolerance is max(eta, cg_tol), and from the second step on also at least 1/2 rtol g0 / ||g|| (no tighter than
    the outer test needs). Without it, the fixed cg_tol."""

    def __init__(self, ew):
        self.ew = ew
        self.g_last = None
        self.eta = None

    def tolerance(self, gn, g0, rtol, cg_tol):
        first = self.g_last is None
        tol = cg_tol
        if self.ew:
            eta = 0.1 if first else 0.9 * (gn / self.g_last) ** 2
            floor = 0.9 * self.eta ** 2 if self.eta is not None else 0.0
            self.eta = min(max(eta, floor) if floor > 0.1 else eta, 0.1)
            tol = max(self.eta, cg_tol) if first else max(self.eta, cg_tol, 0.5 * rtol * g0 / gn)
        self.g_last = gn
        return tol


class Cell:
    """mech.py:88-192: a periodic voxel cell; rho (nx, ny, nz) or (n, n) in [0, 1]."""

    def __init__(self, rho, E=1.0, nu=0.3, material="neohooke", wls=(500.0, 0.01), emin=1e-3, p=3.0, stream=None):
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
        self._lib = lib
        self.stream = stream  # CUDA stream (cudaStream_t as an int) of every call of this cell; None: the default
        self.s = np.empty(self.shape)
        gam = np.empty(self.shape) if wls is not None else None
        sws = ctypes.c_double()
        check(lib.nlf_mech_set_rho(h, ptr(rho), ptr(self.s), ptr(gam), ctypes.byref(sws), self.stream))
        self.gamma = gam if wls is not None else None
        self.sws = sws.value

    def __del__(self):
        h = getattr(self, "_h", None)
        lb = getattr(self, "_lib", None)  # the module global may be gone while the interpreter shuts down
        if h is not None and h.value and lb is not None:
            lb.nlf_mech_destroy(h)
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

    # --- stability (mech.py:363-416): the Hessian applied on the GPU (nlf_mech_hvp), LOBPCG on the host --------
    def _diag_scale(self):
        """mech.py:395-416: 1 / sqrt(|D| + 1e-30), D the Hessian diagonal at the undeformed state, probed per
        component with the 8 node colours of the 2x2x2 colouring (24 tangent matvecs) and per macro unknown."""
        if getattr(self, "_dsc", None) is None:
            A = self.tangent(self.z0(np.eye(3)), np.eye(3))
            d = np.zeros(self.nw + self.k)
            par = np.indices(self.shape) % 2
            col = par[0] + 2 * par[1] + 4 * par[2]
            dw = d[: self.nw].reshape(self.shape + (3,))
            for cc in range(8):
                for comp in range(3):
                    e = np.zeros(self.shape + (3,))
                    e[..., comp] = col == cc
                    hv = self.hvp_A(A, np.concatenate([e.ravel(), np.zeros(self.k)]))
                    hv = (hv.cpu().numpy() if _is_dev(hv) else np.asarray(hv))[: self.nw].reshape(self.shape + (3,))
                    dw[..., comp][col == cc] = hv[..., comp][col == cc]
            for j in range(self.k):
                e = np.zeros(self.nw + self.k)
                e[self.nw + j] = 1.0
                hv = self.hvp_A(A, e)
                d[self.nw + j] = float(hv[self.nw + j])
            self._dsc = 1.0 / np.sqrt(np.abs(d) + 1e-30)
        return self._dsc

    def lowest_eigs(self, z, Fb, k=4, X=None, tol=1e-5, maxiter=2000):
        """mech.py:363-393: lowest eigenvalues of D^-1/2 H D^-1/2 (rigid translations excluded). With
        device="cuda" the LOBPCG iteration runs on the device (`lobpcg_device`); otherwise scipy's LOBPCG as in the
        reference, each block applied column by column as tangent matvecs on the GPU. Returns (values, vectors
        in z coordinates, iterations)."""
        if self.device is not None:
            return self._lowest_eigs_device(z, Fb, k, X, tol, maxiter)
        from scipy.sparse.linalg import LinearOperator, lobpcg
        A = self.tangent(z, np.asarray(Fb, dtype=np.float64))
        dsc = self._diag_scale()
        nz = self.nw + self.k
        T = np.zeros((nz, 3))
        for i in range(3):
            T[i:self.nw:3, i] = 1.0
        Y, _ = np.linalg.qr(T / dsc[:, None])

        def mm(v):
            V = np.asarray(v, dtype=np.float64).reshape(nz, -1) * dsc[:, None]
            cols = []
            for j in range(V.shape[1]):
                h = self.hvp_A(A, np.ascontiguousarray(V[:, j]))
                cols.append(h.cpu().numpy() if _is_dev(h) else np.asarray(h))
            return (np.stack(cols, axis=1) * dsc[:, None]).reshape(np.shape(v))

        op = LinearOperator((nz, nz), matvec=mm, matmat=mm, dtype=np.float64)
        if X is None:
            X = np.random.default_rng(0).standard_normal((nz, k))
        vals, vecs, hist = lobpcg(op, X, Y=Y, largest=False, tol=tol, maxiter=maxiter, retLambdaHistory=True)
        o = np.argsort(vals)
        return vals[o], vecs[:, o] * dsc[:, None], len(hist)

    def _lowest_eigs_device(self, z, Fb, k, X, tol, maxiter):
        import torch
        dev = self.device
        A = self.tangent(self._as_state(z), np.asarray(Fb, dtype=np.float64))
        dsc = torch.as_tensor(self._diag_scale(), device=dev)
        nz = self.nw + self.k
        T = torch.zeros((nz, 3), dtype=torch.float64, device=dev)
        for i in range(3):
            T[i:self.nw:3, i] = 1.0
        Y, _ = torch.linalg.qr(T / dsc[:, None])

        def op(V):
            out = torch.empty_like(V)
            Vs = V * dsc[:, None]
            for j in range(V.shape[1]):
                out[:, j] = self.hvp_A(A, Vs[:, j].contiguous())
            return out * dsc[:, None]

        if X is None:
            X = np.random.default_rng(0).standard_normal((nz, k))
        vals, vecs, its = lobpcg_device(op, torch.as_tensor(np.asarray(X), dtype=torch.float64, device=dev), Y, tol,
                                        maxiter)
        return vals, (vecs * dsc[:, None]).cpu().numpy(), its

    def _direction(self, z, Fb, g, tol, cg_maxit, sws, log):
        """Newton direction at z: CG on the tangent for H dz = -g (counted in the log); when it is not a descent
        direction (g . dz >= 0, e.g. after negative curvature), the preconditioned steepest descent
        -proj(M g) instead (nlfiber/mech.py:323-331). Returns (dz, g . dz)."""
        A = self.tangent(z, Fb)
        dmac = self.macro_diag(A, Fb) if self.k else np.zeros(0)
        dz, its, _ok, neg = self._cgA(A, -g, dmac, sws, tol, int(cg_maxit))
        log["cg"] += int(its)
        log["negative_curvature"] |= bool(neg)
        slope = _dot(g, dz)
        if slope >= 0:
            dz = -self.proj(self.precond(g, dmac, sws))
            slope = _dot(g, dz)
        return dz, slope

    def solve(self, Fbar, z0=None, rtol=1e-9, maxnewton=30, cg_tol=1e-6, cg_maxit=20000, g_ref=None):
        """mech.py:302-346: Newton-CG on the energy in z = (w, free Fbar entries). Each step: the projected
        gradient g and its norm (logged); stop when ||g|| <= rtol max(g0, 1e-300) or ||g|| < 1e-14, with g0 =
        g_ref or the first norm; else a CG direction to the forcing tolerance, a backtracking step, and the
        update. A failed line search ends the solve, as converged at the round-off floor when ||g|| <=
        STALL_RTOL g0. Returns (w, Fbar_full, log) with the reference's log keys and log['z'] the state."""
        Fb = np.asarray(Fbar, dtype=np.float64)
        z = self.z0(Fb) if z0 is None else self._as_state(z0)
        log = {"newton": 0, "cg": 0, "converged": False, "gnorm": [], "negative_curvature": False}
        forcing = _Forcing(self.forcing == "ew")
        sws = self._sws()
        g0 = g_ref
        for step in range(maxnewton):
            g = self.proj(self._g(z, Fb))
            gn = _norm(g)
            log["gnorm"].append(gn)
            g0 = gn if g0 is None else g0
            if gn <= rtol * max(g0, 1e-300) or gn < 1e-14:
                log["converged"] = True
                break
            dz, slope = self._direction(z, Fb, g, forcing.tolerance(gn, g0, rtol, cg_tol), cg_maxit, sws, log)
            t = _backtrack(lambda t: self._E(z + t * dz, Fb), lambda t: _norm(self.proj(self._g(z + t * dz, Fb))),
                           float(self._E(z, Fb)), slope, gn)
            log["newton"] = step + 1
            if t is None:
                log["linesearch_failed"] = True
                if gn <= STALL_RTOL * g0:
                    log["converged"] = log["roundoff_floor"] = True
                break
            z = z + t * dz
        w, F = self.unpack(z, Fb)
        log["z"], log["g0"] = z, g0
        return w, F, log


def effective_tangent(cell, w, Fbar, cg_tol=1e-10, precond="scaled"):
    """mech.py:419-436: A_abcd = d Pbar_ab / d Fbar_cd at the equilibrium (w, Fbar) under full control. For each
    unit E_cd: the tangent matvec at (0, E) gives (d grad_w/dF) E and dP/dF E; one CG solve H dz = -(d grad_w/dF)
    E; then A = dP/dF E + dP/dw dz (all on the GPU). precond "scaled" (node-scaled FFT inverse) or "fft" (the
    reference's) only changes the CG iteration count; it is left set on the cell afterwards."""
    full = Mixed(cell, free=[], precond=precond)
    Fb = np.asarray(Fbar, dtype=np.float64)
    z = w.reshape(-1) if _is_dev(w) else np.asarray(w, dtype=np.float64).ravel()
    At = full.tangent(z, Fb)
    wz = At.w
    zero = _empty_like_kind(wz, cell.shape + (3,))
    zero[...] = 0.0
    A = np.zeros((3, 3, 3, 3))
    for c in range(3):
        for d in range(3):
            E = np.zeros((3, 3))
            E[c, d] = 1.0
            hw, dPF = cell.hvp(wz, Fb, zero, E)
            dz, _, _ = full.solve_linear(At, -hw.reshape(-1), cg_tol)
            dzw = dz.reshape(cell.shape + (3,))
            _, dPz = cell.hvp(wz, Fb, dzw.contiguous() if _is_dev(dzw) else np.ascontiguousarray(dzw), np.zeros((3, 3)))
            A[:, :, c, d] = dPF + dPz
    return A


def lobpcg_device(op, X, Y=None, tol=1e-5, maxiter=2000):
    """The smallest eigenpairs of a symmetric operator by LOBPCG (Knyazev, SIAM J. Sci. Comput. 23 (2001)), with
    every block on the device: op maps an (n, m) CUDA tensor to A times it; X (n, m) starts the iteration; Y
    (n, c), orthonormal, spans a constraint space the iterates stay orthogonal to. Each iteration forms
    W = A X - X diag(theta) (columns of converged pairs are dropped), orthonormalises [X, W, P] by QR (columns
    scaled to unit norm first; P is dropped for the step if the block is numerically rank deficient), and solves
    the projected 3m x 3m eigenproblem; A applied to the new basis is recombined from A X, A W and A P, so one
    block application (of W) per iteration; the operator is applied as P A P, P the projector onto the complement
    of Y (as scipy's constrained LOBPCG). Stops when every residual norm is at most tol. Returns (eigenvalues
    ascending as a NumPy array, eigenvectors (n, m), iterations)."""
    import torch

    def cons(V):
        return V if Y is None else V - Y @ (Y.T @ V)

    def opc(V):  # the operator restricted to the complement of Y (P A P)
        return cons(op(cons(V))) if Y is not None else op(V)

    m = X.shape[1]
    X = cons(X)
    X, _ = torch.linalg.qr(X)
    AX = opc(X)
    G = X.T @ AX
    th, C = torch.linalg.eigh(0.5 * (G + G.T))
    X, AX = X @ C, AX @ C
    P = AP = None
    it = 0
    for it in range(1, maxiter + 1):
        R = AX - X * th[None, :]
        rn = torch.linalg.vector_norm(R, dim=0)
        active = rn > tol
        if not bool(active.any()):
            break
        W = cons(R[:, active])
        W = W / torch.linalg.vector_norm(W, dim=0).clamp_min(1e-300)[None, :]
        AW = opc(W)
        blocks, ablocks = [X, W], [AX, AW]
        if P is not None:
            pn = torch.linalg.vector_norm(P, dim=0).clamp_min(1e-300)[None, :]
            blocks.append(P / pn)
            ablocks.append(AP / pn)
        S, AS = torch.cat(blocks, dim=1), torch.cat(ablocks, dim=1)
        Q, Rq = torch.linalg.qr(S)
        d = torch.abs(torch.diagonal(Rq))
        if P is not None and bool((d < 1e-10 * d.max()).any()):
            S, AS = torch.cat(blocks[:2], dim=1), torch.cat(ablocks[:2], dim=1)
            Q, Rq = torch.linalg.qr(S)
        AQ = torch.linalg.solve_triangular(Rq, AS, upper=True, left=False)
        G = Q.T @ AQ
        w, V = torch.linalg.eigh(0.5 * (G + G.T))
        th, C = w[:m], V[:, :m]
        Xn, AXn = Q @ C, AQ @ C
        P, AP = Q[:, m:] @ C[m:, :], AQ[:, m:] @ C[m:, :]
        X, AX = Xn, AXn
    o = torch.argsort(th)
    return th[o].cpu().numpy(), X[:, o], it


def fibonacci_sphere(m):
    """mech.py:439-443."""
    i = np.arange(m) + 0.5
    polar = np.arccos(1.0 - 2.0 * i / m)
    az = np.pi * (1.0 + 5.0 ** 0.5) * i
    return np.stack([np.cos(az) * np.sin(polar), np.sin(az) * np.sin(polar), np.cos(polar)], axis=1)


def rank_one_min(A, m=1000, plane=False):
    """mech.py:446-455: min over unit n of the smallest eigenvalue of Q_ik = A_ijkl n_j n_l (host, 3x3 work)."""
    if plane:
        th = np.linspace(0.0, np.pi, m, endpoint=False)
        ns = np.stack([np.cos(th), np.sin(th), np.zeros_like(th)], axis=1)
    else:
        ns = fibonacci_sphere(m)
    Q = np.einsum("ijkl,nj,nl->nik", A, ns, ns)
    Q = 0.5 * (Q + np.swapaxes(Q, 1, 2))
    if plane:
        Q = Q[:, :2, :2]
    ev = np.linalg.eigvalsh(Q)[:, 0]
    i = int(np.argmin(ev))
    return float(ev[i]), ns[i]


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
