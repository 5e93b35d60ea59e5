"""NumPy FP64 restatement of nlfiber/linear.py (small-strain periodic homogenization). TEST ORACLE ONLY.

Arrays follow the reference layout: a nodal field is (..., nx, ny, nz, 3) with z fastest, element e = (i, j, k)
owns the nodes e + NODES[a] (periodic), node order a = x + 2y + 4z, Voigt order xx yy zz yz xz xy with
engineering shear.
"""
import numpy as np

# nlfiber/linear.py:21-24
VOIGT = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
NODES = np.array([[a, b, c] for c in (0, 1) for b in (0, 1) for a in (0, 1)])
_GP1 = 0.5 + np.array([-1.0, 1.0]) / (2 * np.sqrt(3.0))
GPTS = np.array([[x, y, z] for z in _GP1 for y in _GP1 for x in _GP1])


def clip01(x):
    """nlfiber/linear.py:27-30 (value; its derivative is 1 on [0, 1] including both bounds)."""
    return np.where(x > 1.0, 1.0, np.where(x < 0.0, 0.0, x))


def dclip01(x):
    """Derivative of clip01 as the reference's jnp.where gives it: 1 for 0 <= x <= 1, else 0."""
    return np.where((x > 1.0) | (x < 0.0), 0.0, 1.0)


def dN_ref():
    """nlfiber/linear.py:33-41: shape-function gradients [gauss, node, dim]."""
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
    """nlfiber/linear.py:57-71: (8, 6, 24) strain-displacement matrices, engineering shear."""
    dN = dN_ref()
    B = np.zeros((8, 6, 24))
    for g in range(8):
        for a in range(8):
            dx, dy, dz = dN[g, a]
            c = 3 * a
            B[g, 0, c] = dx
            B[g, 1, c + 1] = dy
            B[g, 2, c + 2] = dz
            B[g, 3, c + 1], B[g, 3, c + 2] = dz, dy
            B[g, 4, c + 0], B[g, 4, c + 2] = dz, dx
            B[g, 5, c + 0], B[g, 5, c + 1] = dy, dx
    return B


def unit_strain(I):
    """nlfiber/linear.py:74-77."""
    e = np.zeros(6)
    e[I] = 1.0
    return e


def element_matrices(E, nu):
    """nlfiber/linear.py:108-112: (D, Ke (24x24), G (6x24))."""
    B = B_matrices()
    D = iso_D(E, nu)
    Ke = sum(B[g].T @ D @ B[g] for g in range(8)) / 8.0
    G = sum(D @ B[g] for g in range(8)) / 8.0
    return D, Ke, G


_AX = (-4, -3, -2)


def gather(u):
    """nlfiber/linear.py:80-83: nodal (..., nx, ny, nz, 3) -> element vectors (..., nx, ny, nz, 24)."""
    return np.concatenate([np.roll(u, shift=tuple(-o for o in off), axis=_AX) for off in NODES], axis=-1)


def scatter(fe):
    """nlfiber/linear.py:86-92: element vectors (..., 24) -> assembled nodal field (..., 3)."""
    out = 0
    for a, off in enumerate(NODES):
        out = out + np.roll(fe[..., 3 * a:3 * a + 3], shift=tuple(off), axis=_AX)
    return out


def proj(u):
    """nlfiber/linear.py:95-96: remove the mean of each component."""
    return u - np.mean(u, axis=(-4, -3, -2), keepdims=True)


class LinearHomogenization:
    """nlfiber/linear.py:99-264 restated in NumPy FP64 (no autodiff; dC/drho is the closed form of the
    reference's stop-gradient VJP through `bilinear`, nlfiber/linear.py:10-12,259-264)."""

    def __init__(self, shape, E=1.0, nu=0.3, emin=1e-3, p=3.0, tol=1e-9, maxit=4000):
        shape = tuple(int(s) for s in shape)
        self.plane = len(shape) == 2
        self.shape = shape + (1,) if self.plane else shape
        self.E, self.nu, self.emin, self.p = E, nu, emin, p
        self.tol, self.maxit = tol, maxit
        self.Dm, self.Ke, self.G = element_matrices(E, nu)
        self._precond_symbol()

    # nlfiber/linear.py:137-141
    def stiffness_scale(self, rho):
        rho = np.asarray(rho, dtype=np.float64)
        if self.plane and rho.ndim == 2:
            rho = rho[..., None]
        return self.emin + (1.0 - self.emin) * clip01(rho) ** self.p

    def dscale_drho(self, rho):
        rho = np.asarray(rho, dtype=np.float64)
        if self.plane and rho.ndim == 2:
            rho = rho[..., None]
        return (1.0 - self.emin) * self.p * clip01(rho) ** (self.p - 1.0) * dclip01(rho)

    # nlfiber/linear.py:143-144
    def apply_K(self, s, u):
        return scatter(s[..., None] * (gather(u) @ self.Ke))

    # nlfiber/linear.py:146-149
    def load(self, s, Es):
        fe = np.einsum("mi,ij->mj", Es, self.G)
        return scatter(s[None, ..., None] * fe[:, None, None, None, :])

    # nlfiber/linear.py:151-152
    def residual(self, s, Es, u):
        return proj(np.stack([self.apply_K(s, x) for x in u]) + self.load(s, Es))

    # nlfiber/linear.py:154-165
    def _precond_symbol(self):
        s1 = np.ones(self.shape)
        cols = []
        for c in range(3):
            e = np.zeros(self.shape + (3,))
            e[0, 0, 0, c] = 1.0
            cols.append(np.fft.rfftn(self.apply_K(s1, e), axes=(0, 1, 2)))
        Kh = np.stack(cols, axis=-1)
        Kh[0, 0, 0] = np.eye(3)
        tr = np.abs(np.trace(Kh, axis1=-2, axis2=-1))
        Kinv = np.linalg.inv(Kh + 1e-12 * tr[..., None, None] * np.eye(3))
        Kinv[0, 0, 0] = 0.0
        self.Kh = Kh
        self.Kinv = Kinv

    # nlfiber/linear.py:167-170
    def precond(self, r):
        rh = np.fft.rfftn(r, axes=(-4, -3, -2))
        zh = np.einsum("...ac,...c->...a", self.Kinv, rh)
        return np.fft.irfftn(zh, s=self.shape, axes=(-4, -3, -2))

    def _A(self, s, x):
        return np.stack([self.apply_K(s, xi) for xi in x])

    # nlfiber/linear.py:173-203 (lock-step batched PCG, same guards and stopping rule). M: the preconditioner
    # r -> z (default: the reference's `precond`; `ScaledPrecond` checks the library's node-scaled variant).
    def _cg(self, s, b, x0, maxit=None, history=None, M=None):
        maxit = self.maxit if maxit is None else maxit
        st = PCGState(self, s, b, x0, M)
        while st.it < maxit and st.active():
            st.step()
            if history is not None:
                history(st.it, st.x, st.r)
        return st.x, st.it

    # nlfiber/linear.py:205-217
    def solve(self, s, Es, u0=None, maxit=None, history=None, M=None):
        Es = np.asarray(Es, dtype=np.float64)
        s = np.asarray(s, dtype=np.float64)
        if u0 is None:
            u0 = np.zeros((Es.shape[0],) + self.shape + (3,))
        return self._cg(s, -self.load(s, Es), np.asarray(u0, dtype=np.float64), maxit, history, M)

    def _solve_rhs(self, s, b, maxit=None):
        """nlfiber/linear.py:208-210."""
        return self._cg(s, b, np.zeros_like(b), maxit)

    def element_bracket(self, Es, u):
        """The per-element bracket of nlfiber/linear.py:220-229: b_IJ(e) = E_I D E_J + E_I.G u_J + E_J.G u_I +
        u_I^T Ke u_J, shape (m, m, nx, ny, nz)."""
        ue = gather(u)
        KU = ue @ self.Ke
        GU = ue @ self.G.T
        EDE = Es @ self.Dm @ Es.T
        t1 = np.einsum("ie,jxyze->ijxyz", Es, GU)
        t2 = np.einsum("ixyze,jxyze->ijxyz", ue, KU)
        return EDE[:, :, None, None, None] + t1 + np.swapaxes(t1, 0, 1) + t2

    # nlfiber/linear.py:220-229
    def bilinear(self, s, Es, u):
        Es = np.asarray(Es, dtype=np.float64)
        return np.mean(s[None, None] * self.element_bracket(Es, u), axis=(2, 3, 4))

    def dC_drho(self, rho, Es, u):
        """dC_IJ/drho_e with the correctors held fixed (the value of the reference's VJP through bilinear and
        stiffness_scale, nlfiber/linear.py:10-12,137-141,220-229): (m, m, nx, ny, nz)."""
        b = self.element_bracket(np.asarray(Es, dtype=np.float64), u)
        return b * self.dscale_drho(rho)[None, None] / float(np.prod(self.shape))

    def correctors_vjp(self, s, Es, u, ubar, maxit=None):
        """nlfiber/linear.py:124-131 (the backward of `correctors`' custom VJP): lam = _solve_rhs(s, -proj(ubar)),
        sbar_e = sum_I lam_I,e . (Ke u_I,e + G^T E_I), the VJP of residual(s, Es, u) in s. Returns (sbar, lam)."""
        lam, _ = self._solve_rhs(s, -proj(np.asarray(ubar, dtype=np.float64)), maxit)
        le, ue = gather(lam), gather(u)
        Es = np.asarray(Es, dtype=np.float64)
        sbar = np.einsum("ixyze,ixyze->xyz", le, ue @ self.Ke) + np.einsum("ie,ixyze->xyz", Es, le @ self.G.T)
        return sbar, lam

    # nlfiber/linear.py:231-236
    def C_full(self, rho, u0=None, maxit=None, history=None, precond="fft"):
        """precond "scaled" runs the library's node-scaled preconditioner (`ScaledPrecond`) instead of the
        reference's: the same C at convergence, in far fewer iterations at high contrast."""
        s = self.stiffness_scale(rho)
        Es = np.eye(6)
        M = ScaledPrecond(self, s) if precond == "scaled" else None
        u, it = self.solve(s, Es, u0, maxit, history, M)
        return self.bilinear(s, Es, u), u, it

    # nlfiber/linear.py:239-264
    def _shear(self):
        return 5 if self.plane else 3

    def sym_cases(self):
        return np.stack([unit_strain(0), unit_strain(self._shear())])

    @staticmethod
    def swap_xy(u):
        return np.swapaxes(u, -4, -3)[..., [1, 0, 2]]

    def invariants_from(self, s, u2):
        uyy = self.swap_xy(u2[0])
        u3 = np.stack([u2[0], uyy, u2[1]])
        Es = np.stack([unit_strain(0), unit_strain(1), unit_strain(self._shear())])
        C = self.bilinear(s, Es, u3)
        return np.array([C[0, 0], C[1, 0], C[2, 2]]) / self.E

    def invariants(self, rho, u0=None, maxit=None):
        s = self.stiffness_scale(rho)
        u2, it = self.solve(s, self.sym_cases(), u0, maxit)
        return self.invariants_from(s, u2), u2, it


class PCGState:
    """The state of the lock-step PCG of nlfiber/linear.py:173-203, advanced one iteration per `step` (the loop
    of `LinearHomogenization._cg`; also lets a caller time single iterations). Same guards as the reference:
    pAp == 0 -> 1, rz == 0 -> 1; x, r and z stay projected onto the mean-free subspace."""

    def __init__(self, lh, s, b, x0, M=None):
        self.lh, self.s = lh, s
        self.M = lh.precond if M is None else M
        b = proj(b)
        self.bn = np.sqrt(np.sum(b * b, axis=(1, 2, 3, 4))) + 1e-300
        self.x = proj(x0)
        self.r = b - proj(lh._A(s, self.x))
        z = proj(self.M(self.r))
        self.p = z
        self.rz = np.sum(self.r * z, axis=(1, 2, 3, 4))
        self.it = 0

    def rnorm(self):
        return np.sqrt(np.sum(self.r * self.r, axis=(1, 2, 3, 4)))

    def active(self):
        """The reference's loop condition: some case has ||r|| > tol ||b||."""
        return bool(np.any(self.rnorm() > self.lh.tol * self.bn))

    def step(self):
        col = (slice(None), None, None, None, None)
        Ap = proj(self.lh._A(self.s, self.p))
        pAp = np.sum(self.p * Ap, axis=(1, 2, 3, 4))
        a = self.rz / np.where(pAp == 0, 1.0, pAp)
        self.x = self.x + a[col] * self.p
        self.r = self.r - a[col] * Ap
        z = proj(self.M(self.r))
        rz1 = np.sum(self.r * z, axis=(1, 2, 3, 4))
        self.p = z + (rz1 / np.where(self.rz == 0, 1.0, self.rz))[col] * self.p
        self.rz = rz1
        self.it += 1


def node_scaling(s, expo=0.47):
    """Node scaling of the library's scaled preconditioner (NLF_PC_FFT_SCALED; no counterpart in the reference):
    w_n = S_n^-expo with S_n the root mean square of the stiffness scales of the 8 elements around node n (element
    e owns the nodes e + NODES[a], so they are the elements n - NODES[a])."""
    s = np.asarray(s, dtype=np.float64)
    acc = sum(np.roll(s * s, shift=tuple(int(o) for o in off), axis=(0, 1, 2)) for off in NODES)
    return (acc / 8.0) ** (-0.5 * expo)


class ScaledPrecond:
    """The library's node-scaled FFT preconditioner restated for the tests (no counterpart in the reference):
    z = w irfftn(Kinv0 rfftn(w r)), with w = node_scaling(s) and Kinv0 the reference's symbol inverse
    (nlfiber/linear.py:154-165) of the same element with Poisson ratio nu0 = 0. The converged solution is the
    reference's; only the iterates differ."""

    def __init__(self, lh, s, nu0=0.0, expo=0.47):
        self.ref = LinearHomogenization(lh.shape, E=lh.E, nu=nu0, emin=lh.emin, p=lh.p)
        self.w = node_scaling(s, expo)[..., None]

    def __call__(self, r):
        return self.w * self.ref.precond(self.w * r)


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


def rel_C_error(C, Cref):
    """max_IJ |C_IJ - C*_IJ| / max |C*| (the error measure of the throughput metric)."""
    C, Cref = np.asarray(C), np.asarray(Cref)
    return float(np.abs(C - Cref).max() / np.abs(Cref).max())
