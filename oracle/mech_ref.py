"""NumPy FP64 restatement of nlfiber/mech.py (finite-strain periodic homogenization). TEST ORACLE ONLY.

The reference obtains the residual and the tangent by JAX autodiff of the energy (mech.py:154-169,227-238);
here they are the closed forms of the same functions (first Piola stress and its derivative, applied to a
direction without forming the 81-entry tangent). tests/test_mech_oracle.py checks both against finite
differences of the energy and the small-strain limit against the linear oracle.
"""
import numpy as np

from .linear_ref import NODES, dN_ref, lame

DN = dN_ref()  # [gauss, node, dim]
I3 = np.eye(3)
STALL_RTOL = 1e-6  # nlfiber/mech.py:53


def clip01(x):
    return np.where(x > 1.0, 1.0, np.where(x < 0.0, 0.0, x))


# --- materials (nlfiber/mech.py:38-52) --------------------------------------------------------------------------
def psi_linear(F, lam, mu):
    H = F - I3
    eps = 0.5 * (H + np.swapaxes(H, -1, -2))
    tr = np.trace(eps, axis1=-2, axis2=-1)
    return 0.5 * lam * tr ** 2 + mu * np.sum(eps * eps, axis=(-2, -1))


def psi_neohooke(F, lam, mu):
    J = np.linalg.det(F)
    I1 = np.sum(F * F, axis=(-2, -1))
    with np.errstate(invalid="ignore", divide="ignore"):
        lnJ = np.log(J)
    return 0.5 * mu * (I1 - 3.0) - mu * lnJ + 0.5 * lam * lnJ ** 2


def sig_linear(F, lam, mu):
    """d psi_linear / dF = lam tr(eps) I + 2 mu eps."""
    H = F - I3
    eps = 0.5 * (H + np.swapaxes(H, -1, -2))
    return lam * np.trace(eps, axis1=-2, axis2=-1)[..., None, None] * I3 + 2 * mu * eps


def P_neohooke(F, lam, mu):
    """d psi_neohooke / dF = mu (F - F^-T) + lam ln J F^-T."""
    Fit = np.swapaxes(np.linalg.inv(F), -1, -2)
    lnJ = np.log(np.linalg.det(F))
    return mu * (F - Fit) + lam * lnJ[..., None, None] * Fit


def dP_neohooke(F, dF, lam, mu):
    """Directional derivative of P_neohooke: mu dF + (mu - lam lnJ) F^-T dF^T F^-T + lam (F^-T : dF) F^-T."""
    Fit = np.swapaxes(np.linalg.inv(F), -1, -2)
    lnJ = np.log(np.linalg.det(F))
    t = Fit @ np.swapaxes(dF, -1, -2) @ Fit
    return mu * dF + (mu - lam * lnJ)[..., None, None] * t + lam * np.sum(Fit * dF, axis=(-2, -1))[..., None, None] * Fit


def dsig_linear(dF, lam, mu):
    e = 0.5 * (dF + np.swapaxes(dF, -1, -2))
    return lam * np.trace(e, axis1=-2, axis2=-1)[..., None, None] * I3 + 2 * mu * e


class Cell:
    """nlfiber/mech.py:88-192 (energy, residual, mean stress; tangent as a matvec)."""

    def __init__(self, rho, E=1.0, nu=0.3, material="neohooke", wls=(500.0, 0.01), emin=1e-3, p=3.0):
        rho = np.asarray(rho, dtype=np.float64)
        if rho.ndim == 2:
            rho = rho[..., None]
        self.rho, self.shape = rho, tuple(rho.shape)
        self.N = int(np.prod(self.shape))
        self.E, self.nu, self.material, self.wls, self.emin, self.p = E, nu, material, wls, emin, p
        self.lam, self.mu = lame(E, nu)
        self.wq = 1.0 / (8.0 * self.N)
        self.s = self.emin + (1.0 - self.emin) * clip01(rho) ** self.p  # mech.py:105-106
        self.gamma = self.gamma_of(rho)

    def gamma_of(self, rho):
        """mech.py:108-113."""
        if self.wls is None:
            return None
        b, r0 = self.wls
        v = clip01(rho) ** self.p
        return (np.tanh(b * r0) + np.tanh(b * (v - r0))) / (np.tanh(b * r0) + np.tanh(b * (1 - r0)))

    # mech.py:124-132
    def nodal(self, w):
        return np.stack([np.roll(w, shift=tuple(-o for o in off), axis=(0, 1, 2)) for off in NODES])

    def grad_w(self, w):
        return np.einsum("aijkc,gad->gijkcd", self.nodal(w), DN)

    def _gam(self):
        return np.ones(self.shape) if self.gamma is None else self.gamma

    # mech.py:134-139
    def psi_eff(self, F, gamma):
        psi = psi_neohooke if self.material == "neohooke" else psi_linear
        if gamma is None:
            return psi(F, self.lam, self.mu)
        g = gamma[..., None, None]
        Fg = I3 + g * (F - I3)
        return psi(Fg, self.lam, self.mu) - psi_linear(Fg, self.lam, self.mu) + psi_linear(F, self.lam, self.mu)

    def P_eff(self, F, gamma):
        """d psi_eff / dF."""
        Pm = P_neohooke if self.material == "neohooke" else sig_linear
        if gamma is None:
            return Pm(F, self.lam, self.mu)
        g = gamma[..., None, None]
        Fg = I3 + g * (F - I3)
        return g * (Pm(Fg, self.lam, self.mu) - sig_linear(Fg, self.lam, self.mu)) + sig_linear(F, self.lam, self.mu)

    def dP_eff(self, F, dF, gamma):
        """d^2 psi_eff / dF dF : dF."""
        if self.material == "neohooke":
            dPm = lambda Fx, d: dP_neohooke(Fx, d, self.lam, self.mu)  # noqa: E731
        else:
            dPm = lambda Fx, d: dsig_linear(d, self.lam, self.mu)  # noqa: E731
        if gamma is None:
            return dPm(F, dF)
        g = gamma[..., None, None]
        Fg = I3 + g * (F - I3)
        return g * g * (dPm(Fg, dF) - dsig_linear(dF, self.lam, self.mu)) + dsig_linear(dF, self.lam, self.mu)

    # mech.py:141-152
    def energy(self, w, Fbar):
        F = np.asarray(Fbar)[None, None, None, None] + self.grad_w(w)
        return self.wq * float(np.sum(self.s[None] * self.psi_eff(F, None if self.gamma is None else self.gamma[None])))

    def _scatter(self, Pg):
        """Nodal gradient of sum_g wq s P_g : grad(v): (nx, ny, nz, 3)."""
        out = np.zeros(self.shape + (3,))
        for a, off in enumerate(NODES):
            fa = np.einsum("gijkcd,gd->ijkc", Pg, DN[:, a])
            out = out + np.roll(fa, shift=tuple(off), axis=(0, 1, 2))
        return out

    def grad(self, w, Fbar):
        """(d W / d w, d W / d Fbar) = (residual (nx, ny, nz, 3), mean stress Pbar (3, 3)) (mech.py:166-169,191)."""
        F = np.asarray(Fbar)[None, None, None, None] + self.grad_w(w)
        gam = None if self.gamma is None else self.gamma[None]
        Pg = self.wq * self.s[None, ..., None, None] * self.P_eff(F, gam)
        return self._scatter(Pg), Pg.sum(axis=(0, 1, 2, 3))

    def mean_stress(self, w, Fbar):
        return self.grad(w, Fbar)[1]

    def hvp(self, w, Fbar, v, dFmac):
        """Tangent (second derivative of W at (w, Fbar)) applied to (v, dFmac): (dw part, dFbar part (3, 3))."""
        F = np.asarray(Fbar)[None, None, None, None] + self.grad_w(w)
        dF = np.asarray(dFmac)[None, None, None, None] + self.grad_w(v)
        gam = None if self.gamma is None else self.gamma[None]
        dP = self.wq * self.s[None, ..., None, None] * self.dP_eff(F, dF, gam)
        return self._scatter(dP), dP.sum(axis=(0, 1, 2, 3))

    def precond_symbol(self):
        """mech.py:172-185: Kinv of the homogeneous linear operator with unit stiffness and weight wq."""
        from .linear_ref import LinearHomogenization
        lh = LinearHomogenization(self.shape, E=self.E, nu=self.nu)
        return lh.Kinv * self.N  # the mech operator is the linear one divided by N (wq = 1 / (8 N))

    def precond_w(self, r):
        """mech.py:187-189."""
        Kinv = self.precond_symbol() if not hasattr(self, "_Kinv") else self._Kinv
        self._Kinv = Kinv
        rh = np.fft.rfftn(r, axes=(0, 1, 2))
        return np.fft.irfftn(np.einsum("...ac,...c->...a", Kinv, rh), s=self.shape, axes=(0, 1, 2))


# --- third-order elastic constants (nlfiber/mech.py:56-70,458-493) ----------------------------------------------
VOIGT_PAIRS = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))
PERMS3 = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def voigt_tensor(I):
    """nlfiber/mech.py:56-64: symmetric 3x3 tensor of the Voigt unit strain I (engineering shear)."""
    H = np.zeros((3, 3))
    i, j = VOIGT_PAIRS[I]
    if i == j:
        H[i, i] = 1.0
    else:
        H[i, j] = H[j, i] = 0.5
    return H


def to_voigt(M):
    """nlfiber/mech.py:67-70."""
    S = 0.5 * (M + M.T)
    return np.array([S[0, 0], S[1, 1], S[2, 2], 2 * S[1, 2], 2 * S[0, 2], 2 * S[0, 1]])


def toec_geometric(C):
    """The geometric correction 3 Sym_IJK C(e_I, voigt(e_J e_K)) of nlfiber/mech.py:482-492."""
    X = np.zeros((6, 6, 6))
    for J in range(6):
        for K in range(6):
            X[:, J, K] = to_voigt(voigt_tensor(J) @ voigt_tensor(K))
    CX = np.einsum("ia,ajk->ijk", C, X)
    return 3.0 * sum(np.transpose(CX, p) for p in PERMS3) / 6.0


def toec(cell, chi):
    """nlfiber/mech.py:458-493: C (6x6) and the Lagrangian-strain third-order constants T (6x6x6) from the linear
    correctors chi (6, nx, ny, nz, 3): f(s) = wq sum_{g,e} s_e psi_eff(I + sum_I s_I H_I), H_I = voigt(I) +
    grad chi_I, C = f''(0), T = f'''(0) - 3 Sym(C X). The reference takes f'' and f''' by autodiff; here they are
    the closed forms at F = I. psi_eff''(I) = psi_lin'' for either material: the WLS factor gamma cancels and the
    neo-Hookean energy linearises to psi_lin. psi_eff'''(I)[A, B, C] = gamma^3 psi_NH'''(I)[A, B, C], where
    psi_NH'''(I)[A, B, C] = -mu (tr ABC + tr ACB) - lam (trA tr BC + trB tr CA + trC tr AB); it is zero for the
    linear material."""
    lam, mu = cell.lam, cell.mu
    H = np.stack([voigt_tensor(I) + cell.grad_w(np.asarray(chi[I])) for I in range(6)])  # (6, 8, nx, ny, nz, 3, 3)
    w = cell.wq * cell.s[None]
    tr = np.trace(H, axis1=-2, axis2=-1)
    Ht = np.swapaxes(H, -1, -2)
    C = np.zeros((6, 6))
    for I in range(6):
        for J in range(6):
            dd = np.sum(H[I] * H[J], axis=(-2, -1)) + np.sum(H[I] * Ht[J], axis=(-2, -1))
            C[I, J] = np.sum(w * (lam * tr[I] * tr[J] + mu * dd))
    T3 = np.zeros((6, 6, 6))
    if cell.material == "neohooke":
        g3 = w * cell._gam()[None] ** 3
        mm = lambda A, B: np.einsum("...ab,...bc->...ac", A, B)  # noqa: E731
        trm = lambda A: np.trace(A, axis1=-2, axis2=-1)  # noqa: E731
        for I in range(6):
            for J in range(6):
                for K in range(6):
                    t1 = trm(mm(mm(H[I], H[J]), H[K])) + trm(mm(mm(H[I], H[K]), H[J]))
                    t2 = tr[I] * trm(mm(H[J], H[K])) + tr[J] * trm(mm(H[K], H[I])) + tr[K] * trm(mm(H[I], H[J]))
                    T3[I, J, K] = np.sum(g3 * (-mu * t1 - lam * t2))
    return C, T3 - toec_geometric(C)


class Mixed:
    """nlfiber/mech.py:195-346: mixed macroscopic control, Newton-CG on z = (w, Fbar_free)."""

    def __init__(self, cell, free=((1, 1), (2, 2)), forcing="ew"):
        self.c = cell
        self.free = [tuple(f) for f in free]
        self.forcing = forcing
        self.shape = cell.shape
        self.nw = 3 * cell.N
        self.k = len(self.free)

    def unpack(self, z, Fb):
        w = z[: self.nw].reshape(self.shape + (3,))
        F = np.array(Fb, dtype=np.float64)
        for j, (a, b) in enumerate(self.free):
            F[a, b] = z[self.nw + j]
        return w, F

    def z0(self, Fb):
        Fb = np.asarray(Fb, dtype=np.float64)
        return np.concatenate([np.zeros(self.nw), np.array([Fb[a, b] for a, b in self.free])])

    def proj(self, v):
        w = v[: self.nw].reshape(self.shape + (3,))
        w = w - w.mean(axis=(0, 1, 2))
        return np.concatenate([w.ravel(), v[self.nw:]])

    def E(self, z, Fb):
        return self.c.energy(*self.unpack(z, Fb))

    def g(self, z, Fb):
        gw, P = self.c.grad(*self.unpack(z, Fb))
        return np.concatenate([gw.ravel(), np.array([P[a, b] for a, b in self.free])])

    def hvp(self, z, Fb, v):
        w, F = self.unpack(z, Fb)
        dFm = np.zeros((3, 3))
        for j, (a, b) in enumerate(self.free):
            dFm[a, b] = v[self.nw + j]
        hw, hP = self.c.hvp(w, F, v[: self.nw].reshape(self.shape + (3,)), dFm)
        return np.concatenate([hw.ravel(), np.array([hP[a, b] for a, b in self.free])])

    def macro_diag(self, z, Fb):
        """mech.py:252-258."""
        d = []
        for j in range(self.k):
            e = np.zeros(self.nw + self.k)
            e[self.nw + j] = 1.0
            d.append(self.hvp(z, Fb, e)[self.nw + j])
        return np.abs(np.array(d)) + 1e-12

    def _sws(self):
        """mech.py:292-294."""
        return float(np.exp(np.mean(np.log(self.c.s))))

    def precond(self, r, dmac, sws):
        """mech.py:260-262."""
        w = self.c.precond_w(r[: self.nw].reshape(self.shape + (3,))) / sws
        return np.concatenate([w.ravel(), r[self.nw:] / dmac])

    def cg(self, z, Fb, b, dmac, sws, tol, maxit):
        """mech.py:264-290 (the same guards and exits). Returns (x, it, conv, neg)."""
        M = lambda r: self.proj(self.precond(r, dmac, sws))  # noqa: E731
        b = self.proj(b)
        bn = np.linalg.norm(b) + 1e-300
        z0 = M(b)
        x, r, p, rz, it, done, conv = np.zeros_like(b), b, z0, float(b @ z0), 0, False, False
        while not done and it < maxit:
            Ap = self.proj(self.hvp(z, Fb, p))
            pAp = float(p @ Ap)
            neg = pAp <= 0
            a = 0.0 if neg else rz / pAp
            x1, r1 = x + a * p, r - a * Ap
            conv1 = np.linalg.norm(r1) <= tol * bn
            z1 = M(r1)
            rz1 = float(r1 @ z1)
            p1 = z1 + (rz1 / (1.0 if rz == 0 else rz)) * p
            x1 = z0 if (neg and it == 0) else (x if neg else x1)
            x, r, p, rz, it, done, conv = x1, r1, p1, rz1, it + 1, neg or conv1, conv1 and not neg
        return x, it, conv, done and not conv

    def solve(self, Fbar, z0=None, rtol=1e-9, maxnewton=30, cg_tol=1e-6, cg_maxit=20000, g_ref=None):
        """mech.py:302-346."""
        Fb = np.asarray(Fbar, dtype=np.float64)
        z = self.z0(Fb) if z0 is None else np.asarray(z0, dtype=np.float64)
        g0, log = g_ref, dict(newton=0, cg=0, converged=False, gnorm=[], negative_curvature=False)
        eta, gprev = None, None
        sws = self._sws()
        for k in range(maxnewton):
            g = self.proj(self.g(z, Fb))
            gn = float(np.linalg.norm(g))
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
            dmac = self.macro_diag(z, Fb) if self.k else np.zeros(0)
            dz, its, ok, neg = self.cg(z, Fb, -g, dmac, sws, tol, cg_maxit)
            log["cg"] += its
            log["negative_curvature"] |= bool(neg)
            E0, slope = self.E(z, Fb), float(g @ dz)
            if slope >= 0:
                dz = -self.proj(self.precond(g, dmac, sws))
                slope = float(g @ dz)
            t = linesearch(lambda x: self.E(x, Fb), lambda x: float(np.linalg.norm(self.proj(self.g(x, Fb)))),
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


# --- stability (nlfiber/mech.py:363-455) ---------------------------------------------------------------------------
def diag_scale(mix):
    """nlfiber/mech.py:395-416: 1 / sqrt(|D| + 1e-30), D the Hessian diagonal at the undeformed state (Fbar = I,
    z = z0), probed per component with the 8 node colours of the 2x2x2 colouring (nodes of one colour do not
    share an element on an even grid) and per macro unknown with its unit vector."""
    Fb = I3
    z = mix.z0(Fb)
    d = np.zeros(mix.nw + mix.k)
    par = np.indices(mix.shape) % 2
    col = par[0] + 2 * par[1] + 4 * par[2]
    dw = d[: mix.nw].reshape(mix.shape + (3,))
    for cc in range(8):
        for comp in range(3):
            e = np.zeros(mix.shape + (3,))
            e[..., comp] = col == cc
            hv = mix.hvp(z, Fb, np.concatenate([e.ravel(), np.zeros(mix.k)]))[: mix.nw].reshape(mix.shape + (3,))
            dw[..., comp][col == cc] = hv[..., comp][col == cc]
    for j in range(mix.k):
        e = np.zeros(mix.nw + mix.k)
        e[mix.nw + j] = 1.0
        d[mix.nw + j] = mix.hvp(z, Fb, e)[mix.nw + j]
    return 1.0 / np.sqrt(np.abs(d) + 1e-30)


def lowest_eigs(mix, z, Fb, k=4, X=None, tol=1e-5, maxiter=2000):
    """nlfiber/mech.py:363-393: the lowest eigenvalues of D^-1/2 H D^-1/2 by LOBPCG (scipy), the 3 rigid
    translations excluded as constraints. Returns (values, vectors in z coordinates, iterations)."""
    from scipy.sparse.linalg import LinearOperator, lobpcg
    dsc = diag_scale(mix)
    nz = mix.nw + mix.k
    T = np.zeros((nz, 3))
    for i in range(3):
        T[i:mix.nw:3, i] = 1.0
    Y, _ = np.linalg.qr(T / dsc[:, None])

    def mm(v):
        V = np.asarray(v, dtype=np.float64).reshape(nz, -1) * dsc[:, None]
        out = np.stack([mix.hvp(z, Fb, V[:, j]) for j in range(V.shape[1])], axis=1) * dsc[:, None]
        return out.reshape(np.shape(v))

    op = LinearOperator((nz, nz), matvec=mm, matmat=mm, dtype=np.float64)
    if X is None:
        X = np.random.default_rng(0).standard_normal((nz, k))
    vals, vecs, hist = lobpcg(op, X, Y=Y, largest=False, tol=tol, maxiter=maxiter, retLambdaHistory=True)
    o = np.argsort(vals)
    return vals[o], vecs[:, o] * dsc[:, None], len(hist)


def effective_tangent(cell, w, Fbar, cg_tol=1e-10, cg_maxit=20000):
    """nlfiber/mech.py:419-436: A_abcd = d Pbar_ab / d Fbar_cd at the equilibrium (w, Fbar) under full control:
    for each unit E_cd, H dz = -(d grad_w / dF) E (one CG solve), A = dP/dF E + dP/dw dz."""
    full = Mixed(cell, free=[])
    Fb = np.asarray(Fbar, dtype=np.float64)
    z = np.asarray(w, dtype=np.float64).ravel()
    zero = np.zeros(cell.shape + (3,))
    A = np.zeros((3, 3, 3, 3))
    for c in range(3):
        for d in range(3):
            E = np.zeros((3, 3))
            E[c, d] = 1.0
            hw, dPF = cell.hvp(w, Fb, zero, E)
            dz, _, _, _ = full.cg(z, Fb, -hw.ravel(), np.zeros(0), full._sws(), cg_tol, cg_maxit)
            _, dPz = cell.hvp(w, Fb, dz.reshape(cell.shape + (3,)), np.zeros((3, 3)))
            A[:, :, c, d] = dPF + dPz
    return A


def fibonacci_sphere(m):
    """nlfiber/mech.py:439-443: m nearly uniform unit vectors."""
    i = np.arange(m) + 0.5
    polar = np.arccos(1.0 - 2.0 * i / m)
    az = np.pi * (1.0 + 5.0 ** 0.5) * i
    return np.stack([np.cos(az) * np.sin(polar), np.sin(az) * np.sin(polar), np.cos(polar)], axis=1)


def rank_one_min(A, m=1000, plane=False):
    """nlfiber/mech.py:446-455: min over unit n of the smallest eigenvalue of the acoustic tensor
    Q_ik = A_ijkl n_j n_l (n in the x-y plane for 2D cells). Returns (value, n)."""
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


def linesearch(E, gnorm, x, dx, E0, slope, gn):
    """mech.py:73-85."""
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
