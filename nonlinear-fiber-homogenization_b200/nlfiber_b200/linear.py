"""Small-strain periodic homogenization on voxel grids, computed on the GPU by libnlf.so.

Drop-in for nlfiber/linear.py (redcican/nonlinear-fiber-homogenization): same constructor, methods,
attributes and module functions; values are NumPy float64 arrays instead of JAX arrays. Inputs may also be CUDA
float64 torch tensors, which the library reads in place.

Unit cell of nx x ny x nz trilinear hexahedra (Q1, 2x2x2 Gauss points) of unit size, periodic; 2D cells (n, n)
are solved as (n, n, 1). Element stiffness s_e E with s = emin + (1 - emin) rho^p. Voigt order xx yy zz yz xz
xy, engineering shear. For a macroscopic strain E_I the periodic corrector u_I solves K u_I = -f_I and
C_IJ = (1/N_e) sum_e s_e b_e(E_I + u_I, E_J + u_J) (nlfiber/linear.py:1-13).

Beyond the reference: `precision="mixed"` (FP32 operator and PCG inside FP64 iterative refinement),
`precond="scaled"` (the FFT inverse of a Poisson-ratio-0 reference medium wrapped in the node stiffness
scaling S^-0.47, same converged solution), batched calls over many cells of one shape, and `dC_drho`, the sensitivity of C that the reference
gets by autodiff with the correctors held fixed.
"""
import ctypes
import itertools

import numpy as np

from . import _lib
from ._lib import lib, check, ptr, as_f64

# nlfiber/linear.py:21-24
VOIGT = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
NODES = np.array([[a, b, c] for c in (0, 1) for b in (0, 1) for a in (0, 1)])
_GP1 = 0.5 + np.array([-1.0, 1.0]) / (2 * np.sqrt(3.0))
GPTS = np.array([[x, y, z] for z in _GP1 for y in _GP1 for x in _GP1])

_PREC = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}
_PC = {"fft": _lib.PC_FFT, "scaled": _lib.PC_FFT_SCALED}


def clip01(x):
    """nlfiber/linear.py:27-30."""
    x = np.asarray(x, dtype=np.float64)
    return np.where(x > 1.0, 1.0, np.where(x < 0.0, 0.0, x))


def dN_ref():
    """nlfiber/linear.py:33-41: shape-function gradients of the unit Q1 element [gauss, node, dim]."""
    d = np.zeros((8, 8, 3))
    for gi, (x, y, z) in enumerate(GPTS):
        for a, (i, j, k) in enumerate(NODES):
            fx, fy, fz = (x if i else 1 - x), (y if j else 1 - y), (z if k else 1 - z)
            sx, sy, sz = (1 if i else -1), (1 if j else -1), (1 if k else -1)
            d[gi, a] = [sx * fy * fz, fx * sy * fz, fx * fy * sz]
    return d


def lame(E, nu):
    """nlfiber/linear.py:44-45."""
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def iso_D(E, nu):
    """nlfiber/linear.py:48-54."""
    lam, mu = lame(E, nu)
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    D[[3, 4, 5], [3, 4, 5]] = mu
    return D


def B_matrices():
    """nlfiber/linear.py:57-71: strain-displacement matrices (8 Gauss points, 6, 24), engineering shear."""
    dN = dN_ref()
    B = np.zeros((8, 6, 24))
    for g, a in itertools.product(range(8), range(8)):
        dx, dy, dz = dN[g, a]
        c = 3 * a
        B[g, 0, c], B[g, 1, c + 1], B[g, 2, c + 2] = dx, dy, dz
        B[g, 3, c + 1], B[g, 3, c + 2] = dz, dy
        B[g, 4, c + 0], B[g, 4, c + 2] = dz, dx
        B[g, 5, c + 0], B[g, 5, c + 1] = dy, dx
    return B


def unit_strain(I):
    """nlfiber/linear.py:74-77."""
    e = np.zeros(6)
    e[I] = 1.0
    return e


def _proj(u):
    """nlfiber/linear.py:95-96."""
    u = np.asarray(u)
    return u - np.mean(u, axis=(-4, -3, -2), keepdims=True)


class LinearHomogenization:
    """Linear homogenization on a fixed grid (nlfiber/linear.py:99-264). `shape` is (nx, ny, nz) or (n, n) for
    plane strain. Extra keyword arguments select the solver variant; the defaults are the reference's FP64
    algorithm."""

    def __init__(self, shape, E=1.0, nu=0.3, emin=1e-3, p=3.0, dtype=np.float64, tol=1e-9, maxit=4000,
                 precision="fp64", precond="fft", inner_tol=1e-3, inner_maxit=200, max_sweeps=20, check_every=8,
                 slots=0, use_graphs=False, scale_x0=False, energy_tol=0.0, per_case=0, autotune=False):
        shape = tuple(int(n) for n in shape)
        self.plane = len(shape) == 2
        self.shape = shape + (1,) if self.plane else shape
        self.E, self.nu, self.emin, self.p = float(E), float(nu), float(emin), float(p)
        self.dtype, self.tol, self.maxit = dtype, float(tol), int(maxit)
        self.precision, self.precond_kind = precision, precond
        self.inner_tol, self.inner_maxit, self.max_sweeps = inner_tol, inner_maxit, max_sweeps
        self.check_every = check_every
        self.slots, self.use_graphs, self.scale_x0 = int(slots), bool(use_graphs), bool(scale_x0)
        self.energy_tol = float(energy_tol)
        self.per_case = int(per_case)
        B = B_matrices()
        D = iso_D(E, nu)
        self.Dm = D
        self.Ke = sum(B[g].T @ D @ B[g] for g in range(8)) / 8.0
        self.G = sum(D @ B[g] for g in range(8)) / 8.0
        self.N = int(np.prod(self.shape))
        h = ctypes.c_void_p()
        check(lib.nlf_linear_create(ctypes.byref(h), *self.shape, self.E, self.nu, self.emin, self.p, self.tol,
                                    self.maxit))
        self._h = h
        self._lib = lib
        self._Kinv = None
        self.stream = None  # cudaStream_t handle (int) used by every call; None = the legacy default stream
        if autotune:
            self.autotune()

    def autotune(self, nvec=24, reps=3, force=False, report=False):
        """Pick the fastest tile of the stiffness apply for this grid (nlf_linear_autotune) in the solver's
        precision(s): FP64, and FP32 too for precision="mixed"; on FP64 cubes of 32 or 64 also the Kinv mode of the
        preconditioner (table or closed form). The choice is cached per grid for the process. With report=True
        every variant is timed and {precision: [ms per launch of each apply variant, then for FP64 cubes the
        preconditioner, entry Kinv mode + nk x twiddle mode with nk = 3 Kinv modes at 64^3 (2 at 32^3; zeros
        elsewhere)]} is returned."""
        out = {}
        precs = ["fp64"] + (["mixed"] if self.precision == "mixed" else [])
        for pr in precs:
            code = _PREC[pr]
            ms = np.zeros(lib.nlf_apply_variants(code) + (12 if pr == "fp64" else 0)) if report else None
            check(lib.nlf_linear_autotune(self._h, code, int(nvec), int(reps), int(force), ptr(ms), self.stream))
            if report:
                out[pr] = ms.tolist()
        return out

    def apply_tile(self, precision="fp64"):
        """(variant, TY, TZ, min CTAs per SM) of the apply tile this handle uses."""
        v, ty, tz, mb = (ctypes.c_int() for _ in range(4))
        check(lib.nlf_linear_get_apply_variant(self._h, _PREC[precision], ctypes.byref(v), ctypes.byref(ty),
                                               ctypes.byref(tz), ctypes.byref(mb)))
        return v.value, ty.value, tz.value, mb.value

    @property
    def kinv_mode(self):
        """0: the FP64 cube preconditioner reads its Kinv table; 1: it computes the entries in closed form; 2 (64^3):
        closed form with pass B's slabs staged through shared memory."""
        return int(lib.nlf_linear_get_kinv_mode(self._h))

    @kinv_mode.setter
    def kinv_mode(self, mode):
        check(lib.nlf_linear_set_kinv_mode(self._h, int(mode)))

    @property
    def fft_twiddles(self):
        """0: passes A and C of the FP64 cube preconditioner keep their twiddles in registers; 1: in shared
        memory (fewer registers, 3 CTAs per SM); 2: as 1, with pass C's spectrum rows and x/p update moved in
        whole rows through shared memory (4 CTAs per SM at 64^3); 3: as 2, with pass A's row inputs coalesced
        too."""
        return int(lib.nlf_linear_get_fft_twiddles(self._h))

    @fft_twiddles.setter
    def fft_twiddles(self, shared):
        check(lib.nlf_linear_set_fft_twiddles(self._h, int(shared)))

    def set_apply_tile(self, variant, precision="fp64"):
        """Use apply tile variant `variant` (0 = default) for this handle."""
        check(lib.nlf_linear_set_apply_variant(self._h, _PREC[precision], int(variant)))

    def __del__(self):
        h = getattr(self, "_h", None)
        lb = getattr(self, "_lib", None)  # the module global may be gone while the interpreter shuts down
        if h is not None and h.value and lb is not None:
            lb.nlf_linear_destroy(h)
            self._h = None

    # --- options ---------------------------------------------------------------------------------------------
    def opts(self, precision=None, precond=None, tol=None, maxit=None):
        return _lib.default_opts(
            precision=_PREC[precision or self.precision], precond=_PC[precond or self.precond_kind],
            tol=self.tol if tol is None else float(tol), maxit=self.maxit if maxit is None else int(maxit),
            inner_tol=float(self.inner_tol), inner_maxit=int(self.inner_maxit), max_sweeps=int(self.max_sweeps),
            check_every=int(self.check_every), slots=self.slots, use_graphs=int(self.use_graphs),
            scale_x0=int(self.scale_x0), energy_tol=self.energy_tol, per_case=self.per_case)

    def _cell(self, a, extra=()):
        """Coerce a per-cell field to (nx, ny, nz) + extra, adding the plane-strain axis where needed."""
        a = as_f64(a)
        if self.plane and tuple(a.shape) == self.shape[:2] + tuple(extra):
            a = a.reshape(self.shape + tuple(extra))
        return a

    # --- operators ----------------------------------------------------------------------------------------------
    @property
    def Kinv(self):
        """(nx, ny, nz//2+1, 3, 3) inverse symbol of the unit-stiffness operator (nlfiber/linear.py:154-165).
        It is real symmetric: the imaginary part of the reference's complex array is rounding."""
        if self._Kinv is None:
            n0, n1, n2 = self.shape
            k6 = np.empty((n0, n1, n2 // 2 + 1, 6))
            check(lib.nlf_precond_symbol(self._h, ptr(k6)))
            K = np.empty(k6.shape[:3] + (3, 3))
            for q, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]):
                K[..., a, b] = k6[..., q]
                K[..., b, a] = k6[..., q]
            self._Kinv = K.astype(np.complex128)
        return self._Kinv

    def stiffness_scale(self, rho):
        """nlfiber/linear.py:137-141."""
        rho = self._cell(rho)
        out = np.empty(rho.shape)
        ncell = int(np.prod(rho.shape)) // self.N
        check(lib.nlf_stiffness_scale(self._h, ncell, ptr(rho), ptr(out), self.stream))
        return out

    def apply_K(self, s, u, precision="fp64"):
        """nlfiber/linear.py:143-144: K(s) u for u (..., nx, ny, nz, 3). precision="mixed" runs the FP32
        operator of the mixed-precision solver."""
        s = self._cell(s)
        u = as_f64(u)
        nvec = int(np.prod(u.shape)) // (3 * self.N)
        out = np.empty(u.shape)
        check(lib.nlf_apply_K_ex(self._h, ptr(s), nvec, ptr(u), ptr(out), _PREC[precision], self.stream))
        return out

    def load(self, s, Es):
        """nlfiber/linear.py:146-149: assembled a(E_I, .) for Es (m, 6): (m, nx, ny, nz, 3)."""
        s = self._cell(s)
        Es = as_f64(np.atleast_2d(Es))
        out = np.empty((Es.shape[0],) + self.shape + (3,))
        check(lib.nlf_load(self._h, ptr(s), ptr(Es), Es.shape[0], ptr(out), self.stream))
        return out

    def residual(self, s, Es, u):
        """nlfiber/linear.py:151-152."""
        return _proj(self.apply_K(s, u) + self.load(s, Es))

    def precond(self, r, precision="fp64", precond="fft", s=None):
        """nlfiber/linear.py:167-170: irfftn(Kinv rfftn(r)) for r (..., nx, ny, nz, 3). precond="scaled" (needs
        the stiffness scale s) wraps the inverse of a Poisson-ratio-0 reference medium in the node scaling
        w = (root mean square of s around the node)^-0.47;
        precision="mixed" runs it in FP32."""
        r = as_f64(r)
        nvec = int(np.prod(r.shape)) // (3 * self.N)
        out = np.empty(r.shape)
        s = None if s is None else self._cell(s)
        check(lib.nlf_precond_ex(self._h, nvec, ptr(r), ptr(out), _PREC[precision], _PC[precond], ptr(s), self.stream))
        return out

    # --- solver ---------------------------------------------------------------------------------------------
    def solve_batched(self, s, Es, u0=None, **opt):
        """Corrector solve for ncell cells of this shape: s (ncell, nx, ny, nz), Es (m, 6),
        u0 (ncell, m, nx, ny, nz, 3) or None. Returns (u, iterations per cell, status)."""
        s = as_f64(s)
        ncell = int(np.prod(s.shape)) // self.N
        Es = as_f64(np.atleast_2d(Es))
        m = Es.shape[0]
        u0 = None if u0 is None else as_f64(u0)
        u = np.empty((ncell, m) + self.shape + (3,))
        it = np.zeros(ncell, dtype=np.int32)
        o = self.opts(**opt)
        st = check(lib.nlf_linear_solve(self._h, ncell, ptr(s), ptr(Es), m, ptr(u0), ptr(u), ptr(it),
                                        ctypes.byref(o), self.stream))
        return u, it, st

    def solve(self, s, Es, u0=None, **opt):
        """nlfiber/linear.py:212-217: (u (m, nx, ny, nz, 3), iterations)."""
        s = self._cell(s)
        u0 = None if u0 is None else as_f64(u0)[None]
        u, it, _ = self.solve_batched(s[None], Es, u0, **opt)
        return u[0], int(it[0])

    def _solve_rhs(self, s, b, **opt):
        """nlfiber/linear.py:208-210: PCG from zero for right-hand sides b (m, nx, ny, nz, 3)."""
        s = self._cell(s)
        b = as_f64(b)
        m = b.shape[0]
        u = np.empty(b.shape)
        it = np.zeros(1, dtype=np.int32)
        o = self.opts(**opt)
        check(lib.nlf_linear_solve_rhs(self._h, 1, ptr(s), m, ptr(b), ptr(u), ptr(it), ctypes.byref(o), self.stream))
        return u, int(it[0])

    def correctors(self, s, Es, u0):
        """nlfiber/linear.py:118-121 (the value; its custom VJP's backward is `correctors_vjp`)."""
        return self.solve(s, Es, u0)[0]

    def correctors_vjp(self, s, Es, u, ubar, rho=None, **opt):
        """nlfiber/linear.py:124-131, the backward of `correctors`: lam solves K(s) lam = -proj(ubar) and
        sbar = d<lam, residual(s, Es, u)>/ds. With rho (s=None), s = stiffness_scale(rho) and the result is the
        cotangent of rho. Returns (sbar (nx, ny, nz), lam (m, nx, ny, nz, 3), iterations)."""
        Es = as_f64(np.atleast_2d(Es))
        m = Es.shape[0]
        u = as_f64(u)
        ubar = as_f64(ubar)
        sv = None if s is None else self._cell(s)
        rv = None if rho is None else self._cell(rho)
        sbar = np.empty(self.shape)
        lam = np.empty((m,) + self.shape + (3,))
        it = np.zeros(1, dtype=np.int32)
        o = self.opts(**opt)
        check(lib.nlf_correctors_vjp(self._h, 1, ptr(sv), ptr(rv), ptr(Es), m, ptr(u), ptr(ubar), ptr(sbar),
                                     ptr(lam), ptr(it), ctypes.byref(o), self.stream))
        return sbar, lam, int(it[0])

    # --- homogenized stiffness -----------------------------------------------------------------------------
    def bilinear(self, s, Es, u):
        """nlfiber/linear.py:220-229: C_IJ = mean_e s_e b_e(E_I + u_I, E_J + u_J), Es (m, 6), u (m, ..., 3)."""
        s = self._cell(s)
        Es = as_f64(np.atleast_2d(Es))
        u = as_f64(u)
        m = Es.shape[0]
        C = np.empty((m, m))
        check(lib.nlf_bilinear(self._h, 1, ptr(s), ptr(Es), m, ptr(u), ptr(C), self.stream))
        return C

    def dC_drho(self, rho, Es, u):
        """dC_IJ / drho_e with u held fixed (the reference's VJP of `bilinear` through `stiffness_scale`,
        nlfiber/linear.py:10-12,259-264): (m, m, nx, ny, nz)."""
        rho = self._cell(rho)
        Es = as_f64(np.atleast_2d(Es))
        u = as_f64(u)
        m = Es.shape[0]
        out = np.empty((m, m) + self.shape)
        check(lib.nlf_dC_drho(self._h, 1, ptr(rho), ptr(Es), m, ptr(u), ptr(out), self.stream))
        return out

    def C_full_batched(self, rho, u0=None, want_u=False, want_dC=False, out_C=None, out_u=None, **opt):
        """C (ncell, 6, 6) of ncell cells of this shape in one batched solve. Returns a dict with C, it, status
        and, when asked, u (ncell, 6, nx, ny, nz, 3) and dC (ncell, 6, 6, nx, ny, nz). rho, out_C and out_u (the
        correctors' buffer, implies want_u) may be CUDA float64 torch tensors (device resident) or pinned host
        tensors."""
        rho = as_f64(rho)
        ncell = int(np.prod(rho.shape)) // self.N
        C = np.empty((ncell, 6, 6)) if out_C is None else out_C
        u = out_u if out_u is not None else (np.empty((ncell, 6) + self.shape + (3,)) if want_u else None)
        dC = np.empty((ncell, 6, 6) + self.shape) if want_dC else None
        it = np.zeros(ncell, dtype=np.int32)
        u0 = None if u0 is None else as_f64(u0)
        o = self.opts(**opt)
        st = check(lib.nlf_C_full(self._h, ncell, ptr(rho), ptr(u0), ptr(C), ptr(u), ptr(dC), ptr(it),
                                  ctypes.byref(o), self.stream))
        return dict(C=C, u=u, dC=dC, it=it, status=st)

    def C_full(self, rho, u0=None, **opt):
        """nlfiber/linear.py:231-236: 6x6 C^H (all six unit strains). Returns (C, u, cg iterations)."""
        rho = self._cell(rho)
        u0 = None if u0 is None else as_f64(u0)[None]
        r = self.C_full_batched(rho[None], u0, want_u=True, **opt)
        return r["C"][0], r["u"][0], int(r["it"][0])

    # cubic (3D) or square (2D) symmetric cells: solve xx and the shear, get yy by the x<->y swap
    def _shear(self):
        return 5 if self.plane else 3

    def sym_cases(self):
        """nlfiber/linear.py:242-243."""
        return np.stack([unit_strain(0), unit_strain(self._shear())])

    @staticmethod
    def swap_xy(u):
        """nlfiber/linear.py:245-248."""
        return np.swapaxes(np.asarray(u), -4, -3)[..., [1, 0, 2]]

    def invariants_from(self, s, u2):
        """nlfiber/linear.py:250-257: (C11, C12, C44) / E (C66 in 2D)."""
        u2 = np.asarray(u2)
        u3 = np.ascontiguousarray(np.stack([u2[0], self.swap_xy(u2[0]), u2[1]]))
        Es = np.stack([unit_strain(0), unit_strain(1), unit_strain(self._shear())])
        C = self.bilinear(s, Es, u3)
        return np.array([C[0, 0], C[1, 0], C[2, 2]]) / self.E

    def invariants(self, rho, u0=None, **opt):
        """nlfiber/linear.py:259-264: (c, u2, cg iterations)."""
        s = self.stiffness_scale(rho)
        u2, it = self.solve(s, self.sym_cases(), u0, **opt)
        return self.invariants_from(s, u2), u2, it


def C_full_uneven(cells, handles=None, concurrent=False, **kw):
    """C (6x6), iterations and status of cells of different grid sizes: one handle (and one batched, slot-refilled
    solve) per grid shape, results in the input order. `cells` is a sequence of rho arrays (NumPy or CUDA float64
    torch tensors); `kw` are LinearHomogenization keywords (E, nu, emin, p, tol, maxit, precond, slots, ...).
    With concurrent=True (CUDA torch available) the shapes run at once on their own streams from host threads (the
    library is reentrant per handle). `handles` (dict shape -> LinearHomogenization) reuses handles across calls.
    Returns dict(C=(ncell, 6, 6), it=(ncell,), status=worst status, groups={shape: indices})."""
    groups = {}
    for i, r in enumerate(cells):
        groups.setdefault(tuple(int(n) for n in r.shape), []).append(i)
    handles = {} if handles is None else handles
    C = np.empty((len(cells), 6, 6))
    it = np.zeros(len(cells), dtype=np.int32)
    status = [0]

    def run(shape, idx):
        lh = handles.get(shape)
        if lh is None:
            lh = handles[shape] = LinearHomogenization(shape, **kw)
        if concurrent:
            import torch
            st = torch.cuda.Stream()
            lh.stream = st.cuda_stream
        rho = cells[idx[0]]
        if hasattr(rho, "data_ptr") and not isinstance(rho, np.ndarray):
            import torch
            batch = torch.stack([cells[i] for i in idx])
        else:
            batch = np.stack([np.asarray(cells[i], dtype=np.float64) for i in idx])
        r = lh.C_full_batched(batch)
        C[idx] = r["C"]
        it[idx] = r["it"]
        status[0] = max(status[0], r["status"])

    if concurrent and len(groups) > 1:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(len(groups)) as ex:
            for f in [ex.submit(run, sh, ix) for sh, ix in groups.items()]:
                f.result()
    else:
        for sh, ix in groups.items():
            run(sh, ix)
    return dict(C=C, it=it, status=status[0], groups=groups)


# nlfiber/linear.py:267-291
def cubic_invariants(C):
    C = np.asarray(C)
    return np.array([np.mean([C[0, 0], C[1, 1], C[2, 2]]), np.mean([C[0, 1], C[0, 2], C[1, 2]]),
                     np.mean([C[3, 3], C[4, 4], C[5, 5]])])


def cubic_leakage(C):
    C = np.asarray(C)
    c11, c12, c44 = cubic_invariants(C)
    Cc = np.zeros((6, 6))
    Cc[:3, :3] = c12
    Cc[[0, 1, 2], [0, 1, 2]] = c11
    Cc[[3, 4, 5], [3, 4, 5]] = c44
    return float(np.linalg.norm(C - Cc) / np.linalg.norm(C))


def hashin_shtrikman(v, E=1.0, nu=0.3):
    lam, mu = lame(E, nu)
    K = lam + 2 * mu / 3
    K_hs = K + (1 - v) / (-1 / K + 3 * v / (3 * K + 4 * mu)) if v < 1 else K
    G_hs = mu + (1 - v) / (-1 / mu + 6 * v * (K + 2 * mu) / (5 * mu * (3 * K + 4 * mu))) if v < 1 else mu
    return K_hs, G_hs
