"""CPU studies behind four design decisions of the solvers, on the oracle's PCG and Newton-CG. TEST
INFRASTRUCTURE ONLY: nothing in the library imports this file; it restates variants of the oracle's node-scaled
PCG and of its finite-strain tangent to measure them.

1. Mixed precision (the solver stays FP64). Three variants of the FP64 PCG with the node-scaled preconditioner on
   cells of the benchmark generator at a 1e-9 void floor, each run to the residual rule 1e-9:
     - "pc32": the preconditioner's FFTs and symbol product in FP32 (scipy.fft keeps float32), everything
       else FP64;
     - "spec32": FP64 FFT arithmetic, the half spectrum rounded to complex64 where it would be stored between
       the preconditioner's passes;
     - "apply32": the stiffness apply in FP32 inside FP64 PCG, with the FP64 residual replaced every k
       iterations (reliable updates).
   Measured (32^3, seed 0, three floating solid islands): FP64 192 iterations; pc32 470; spec32 393; apply32
   diverges (true residual 1e5 after 1500 iterations). Clean cells (seeds 1-3): pc32 costs 5-15 % more
   iterations. C stays exact wherever the iteration converges: the loss is in iterations, which no bandwidth
   saving of FP32 recovers.

2. Sensitivity of the iterates to rounding. A relative perturbation of 1e-15 of every preconditioned residual
   changes the 64^3 island cell's (seed 0) iterate by 4e-10 in the energy norm after 8 iterations and by 3e-2
   after 20 (emin 1e-9; 1e-4 after 20 at emin 1e-3). Two correct FP64 implementations therefore agree in their
   early iterates only; their converged C agree to rounding.

3. An FP32 tangent inside the FP64 Newton-CG of the finite-strain step (nlfiber/mech.py:199-346). The oracle's
   Newton (FP64 gradient, energy and line search) with the node-scaled CG preconditioner, its tangent matvec
   either FP64 or FP32 (element tangent, element forces and nodal sums in float32), one compression step of 1 %
   (Fbar_xx = 0.99, lateral stresses free) at emin 1e-6 (the finite-strain configuration's floor).
   Measured (32^3): seed 1 (one solid piece) FP64 4 Newton / 105 CG, FP32 4 / 113, the same lateral F to 1e-10;
   seed 5 (13 pieces) FP64 15 / 1043 and FP32 14 / 766, both stopping by the gradient rule but at lateral strains
   0.0021061 and 0.0021020: the floating pieces settle differently.

4. Block PCG over the 6 load cases of a cell (they share the operator), breakdown-free (Ji & Li 2017), with the
   node-scaled preconditioner and the lock-step rule (every case residual 1e-9), at a 1e-9 void floor.
   Measured (32^3): clean cells: seed 1, 84 lock-step iterations against 79 block iterations; seed 2, 77 against
   71; C unchanged. Island cells: seed 0, 192 against no convergence in 4000; seed 5, 303 against no
   convergence in 4000. The islands' near-null modes leave P^T A P and the Gram-based orthonormalization
   ill-conditioned. The island cells are the ones that bound a batch.

    python -m oracle.precision_studies block 16 0,5,1,2
    python -m oracle.precision_studies mixed 16 0,1,2,3     # octant size and seeds
    python -m oracle.precision_studies sensitivity 32 0 8 1e-9
    python -m oracle.precision_studies tangent32 16 1,5
"""
import sys

import numpy as np

from . import density_ref as OD
from . import linear_ref as OL

MAT = dict(E=1.0, nu=0.3, p=3.0)
_COL = (slice(None), None, None, None, None)


class ScaledPrecondF32:
    """The node-scaled preconditioner with its FFTs and symbol product in FP32 (mode "pc32") or in FP64 with the
    half spectrum rounded to complex64 after the forward transform and after the symbol (mode "spec32")."""

    def __init__(self, lh, s, mode):
        import scipy.fft as sf
        self.sf, self.mode, self.shape = sf, mode, lh.shape
        self.ref = OL.LinearHomogenization(lh.shape, E=lh.E, nu=0.0, emin=lh.emin, p=lh.p)
        self.w = OL.node_scaling(s)[..., None]

    def __call__(self, r):
        ax = (-4, -3, -2)
        if self.mode == "pc32":
            K = self.ref.Kinv.real.astype(np.float32)
            rh = self.sf.rfftn((self.w * r).astype(np.float32), axes=ax)
            z = self.sf.irfftn(np.einsum("...ac,...c->...a", K, rh), s=self.shape, axes=ax)
            return (z * self.w.astype(np.float32)).astype(np.float64)
        rh = np.fft.rfftn(self.w * r, axes=ax).astype(np.complex64).astype(np.complex128)
        zh = np.einsum("...ac,...c->...a", self.ref.Kinv, rh).astype(np.complex64).astype(np.complex128)
        return self.w * np.fft.irfftn(zh, s=self.shape, axes=ax)


def apply_f32(lh, s, p):
    """K(s) p with FP32 operands and arithmetic (gather, element matrix product, scatter)."""
    s32, Ke32 = s.astype(np.float32), lh.Ke.astype(np.float32)
    return np.stack([OL.scatter(s32[..., None] * (OL.gather(x.astype(np.float32)) @ Ke32)) for x in p]
                    ).astype(np.float64)


def pcg_apply32(lh, s, b, M, tol, maxit, every):
    """FP64 PCG with the apply in FP32 and the FP64 residual b - K x replaced every `every` iterations. Returns
    (x, iterations, the true relative residual at the end)."""
    P = OL.proj
    b = P(b)
    bn = np.sqrt((b * b).sum(axis=(1, 2, 3, 4)))
    x = np.zeros_like(b)
    r = b.copy()
    z = P(M(r))
    p = z.copy()
    rz = (r * z).sum(axis=(1, 2, 3, 4))
    it = 0
    while it < maxit:
        if it and it % every == 0:
            r = b - P(lh._A(s, x))
        if not np.any(np.sqrt((r * r).sum(axis=(1, 2, 3, 4))) > tol * bn):
            break
        Ap = P(apply_f32(lh, s, p))
        a = rz / (p * Ap).sum(axis=(1, 2, 3, 4))
        x = x + a[_COL] * p
        r = r - a[_COL] * Ap
        z = P(M(r))
        rz1 = (r * z).sum(axis=(1, 2, 3, 4))
        p = z + (rz1 / rz)[_COL] * p
        rz = rz1
        it += 1
    rt = b - P(lh._A(s, x))
    return x, it, float((np.sqrt((rt * rt).sum(axis=(1, 2, 3, 4))) / bn).max())


def mixed_study(n_o, seeds, emin=1e-9):
    out = []
    for sd in seeds:
        rho = OD.random_cell(sd, n_o=n_o, r=1.5, beta=16.0, kmax=2)[0]
        lh = OL.LinearHomogenization(rho.shape, **MAT, emin=emin, tol=1e-12, maxit=3000)
        s = lh.stiffness_scale(rho)
        us, _ = lh.solve(s, np.eye(6), M=OL.ScaledPrecond(lh, s))
        Cs = lh.bilinear(s, np.eye(6), us)
        lh.tol = 1e-9
        row = {"seed": sd}
        for name, M in (("fp64", OL.ScaledPrecond(lh, s)), ("pc32", ScaledPrecondF32(lh, s, "pc32")),
                        ("spec32", ScaledPrecondF32(lh, s, "spec32"))):
            u, it = lh.solve(s, np.eye(6), M=M)
            row[name] = (it, OL.rel_C_error(lh.bilinear(s, np.eye(6), u), Cs))
        _, it, rr = pcg_apply32(lh, s, -lh.load(s, np.eye(6)), OL.ScaledPrecond(lh, s), 1e-9, 1500, 25)
        row["apply32"] = (it, rr)
        out.append(row)
    return out


def sensitivity_study(n_o, seed, iters, emin, noise=1e-15):
    """Energy-norm and C distance between the oracle's scaled PCG iterate after `iters` iterations and the same
    run with every preconditioned residual perturbed by a relative `noise`."""
    rho = OD.random_cell(seed, n_o=n_o, r=1.5, beta=16.0, kmax=2)[0]
    oh = OL.LinearHomogenization(rho.shape, **MAT, emin=emin, tol=0.0)
    s = oh.stiffness_scale(rho)
    M = OL.ScaledPrecond(oh, s)
    rng = np.random.default_rng(0)
    u1, _ = oh.solve(s, np.eye(6), maxit=iters, M=M)
    u2, _ = oh.solve(s, np.eye(6), maxit=iters, M=lambda r: (lambda z: z * (1 + noise * rng.standard_normal(z.shape)))(M(r)))
    d = u2 - u1

    def en(v):
        return sum(np.sum(x * oh.apply_K(s, x)) for x in v)

    return {"energy_rel": float(np.sqrt(en(d) / en(u1))),
            "C_rel": OL.rel_C_error(oh.bilinear(s, np.eye(6), u2), oh.bilinear(s, np.eye(6), u1))}


def hvp_f32(cell):
    """The tangent matvec of mech_ref.Cell.hvp in float32: F and dF from the float32 state and direction, the
    neo-Hookean dP with the WLS void interpolation, the element forces and their nodal sums all in float32."""
    from . import mech_ref as OM
    f = np.float32
    DN = OM.DN.astype(f)
    s32, g32 = cell.s.astype(f), cell.gamma.astype(f)
    I3 = np.eye(3, dtype=f)
    lam, mu, wq = f(cell.lam), f(cell.mu), f(cell.wq)

    def gw(w):
        nod = np.stack([np.roll(w, shift=tuple(-o for o in off), axis=(0, 1, 2)) for off in OM.NODES])
        return np.einsum("aijkc,gad->gijkcd", nod, DN)

    def dP_nh(F, dF):
        Fit = np.swapaxes(np.linalg.inv(F), -1, -2)
        lnJ = np.log(np.linalg.det(F))
        t = Fit @ np.swapaxes(dF, -1, -2) @ Fit
        return mu * dF + (mu - lam * lnJ)[..., None, None] * t + lam * np.sum(Fit * dF, axis=(-2, -1))[..., None, None] * Fit

    def dsig(dF):
        e = f(0.5) * (dF + np.swapaxes(dF, -1, -2))
        return lam * np.trace(e, axis1=-2, axis2=-1)[..., None, None] * I3 + f(2) * mu * e

    def hvp(w, Fbar, v, dFmac):
        F = np.asarray(Fbar, f)[None, None, None, None] + gw(w.astype(f))
        dF = np.asarray(dFmac, f)[None, None, None, None] + gw(v.astype(f))
        g = g32[None][..., None, None]
        Fg = I3 + g * (F - I3)
        dP = wq * s32[None, ..., None, None] * (g * g * (dP_nh(Fg, dF) - dsig(dF)) + dsig(dF))
        out = np.zeros(cell.shape + (3,), f)
        for a, off in enumerate(OM.NODES):
            out = out + np.roll(np.einsum("gijkcd,gd->ijkc", dP, DN[:, a]), shift=tuple(off), axis=(0, 1, 2))
        return out.astype(np.float64), dP.sum(axis=(0, 1, 2, 3)).astype(np.float64)

    return hvp


def tangent32_study(n_o, seeds, e=0.01):
    """One compression step per cell, FP64 and FP32 tangent: Newton and CG iterations, convergence, lateral F."""
    from . import mech_ref as OM
    out = []
    for seed in seeds:
        rho = OD.random_cell(seed, n_o=n_o, r=1.5, beta=16.0, kmax=2)[0]
        for fp32 in (False, True):
            cell = OM.Cell(rho, E=1.0, nu=0.3, emin=1e-6)
            if fp32:
                cell.hvp = hvp_f32(cell)
            mx = OM.Mixed(cell)
            wn = OL.node_scaling(cell.s)[..., None]

            def precond(r, dmac, sws, mx=mx, cell=cell, wn=wn):
                z = wn * cell.precond_w(wn * r[: mx.nw].reshape(cell.shape + (3,)))
                return np.concatenate([z.ravel(), r[mx.nw:] / dmac])

            mx.precond = precond
            _, F, log = mx.solve(np.diag([1.0 - e, 1.0, 1.0]), rtol=1e-9, cg_tol=1e-6)
            out.append({"seed": seed, "fp32": fp32, "newton": log["newton"], "cg": log["cg"],
                        "converged": log["converged"], "F_lateral": [float(F[1, 1]), float(F[2, 2])]})
    return out


def _norms(v):
    return np.sqrt((v * v).sum(axis=(1, 2, 3, 4)))


def _orth(V, drop=1e-14):
    """Orthonormal basis of the vectors V[k] (a Gram eigen-decomposition; directions whose squared singular value is
    below `drop` times the largest are dropped: the rank-revealing step of breakdown-free block CG)."""
    k = V.shape[0]
    Vf = V.reshape(k, -1)
    w, Q = np.linalg.eigh(Vf @ Vf.T)
    keep = w > drop * w.max()
    T = Q[:, keep] / np.sqrt(w[keep])
    return (T.T @ Vf).reshape((int(keep.sum()),) + V.shape[1:])


def block_pcg(lh, s, b, M, tol, maxit):
    """Breakdown-free block PCG (Ji & Li 2017, after O'Leary 1980) over the m load cases of one cell, which share
    the operator: one block Krylov space for all cases, the search block orthonormalized (rank-revealing) every
    iteration. Mean-free projection, preconditioner and stopping rule (every case ||r|| <= tol ||b||) as the
    lock-step PCG. Returns (x, iterations, matvecs)."""
    P = OL.proj
    b = P(b)
    m = b.shape[0]
    bn = _norms(b)
    x = np.zeros_like(b)
    r = b.copy()
    p = _orth(P(M(r)))
    it = mv = 0
    while it < maxit and np.any(_norms(r) > tol * bn):
        q = P(lh._A(s, p))
        mv += p.shape[0]
        k = p.shape[0]
        Pf, Qf, Rf = p.reshape(k, -1), q.reshape(k, -1), r.reshape(m, -1)
        PQ = Pf @ Qf.T
        alpha = np.linalg.solve(PQ, Pf @ Rf.T)  # k x m
        x = x + (alpha.T @ Pf).reshape(x.shape)
        r = r - (alpha.T @ Qf).reshape(r.shape)
        it += 1
        if not np.any(_norms(r) > tol * bn):
            break
        z = P(M(r))
        beta = -np.linalg.solve(PQ, Qf @ z.reshape(m, -1).T)  # k x m
        p = _orth(z + (beta.T @ Pf).reshape(z.shape))
    return x, it, mv


def block_study(n_o, seeds, emin=1e-9, tol=1e-9):
    """Iterations of the lock-step PCG (the reference's algorithm with the library's node-scaled preconditioner)
    against block PCG over the 6 unit strains, to the same rule; C of each against a tight lock-step solve."""
    out = []
    for sd in seeds:
        rho = OD.random_cell(sd, n_o=n_o, r=1.5, beta=16.0, kmax=2)[0]
        lh = OL.LinearHomogenization(rho.shape, **MAT, emin=emin, tol=1e-12, maxit=4000)
        s = lh.stiffness_scale(rho)
        E = np.eye(6)
        us, its = lh.solve(s, E, M=OL.ScaledPrecond(lh, s))
        Cs = lh.bilinear(s, E, us)
        lh.tol = tol
        u, it = lh.solve(s, E, M=OL.ScaledPrecond(lh, s))
        ub, itb, mv = block_pcg(lh, s, -lh.load(s, E), OL.ScaledPrecond(lh, s), tol, 4000)
        out.append({"seed": sd, "lockstep": (it, OL.rel_C_error(lh.bilinear(s, E, u), Cs)),
                    "block": (itb, mv, OL.rel_C_error(lh.bilinear(s, E, ub), Cs)), "tight_iterations": its})
    return out


if __name__ == "__main__":
    if sys.argv[1] == "block":
        for row in block_study(int(sys.argv[2]), [int(v) for v in sys.argv[3].split(",")]):
            print(row, flush=True)
    elif sys.argv[1] == "tangent32":
        for row in tangent32_study(int(sys.argv[2]), [int(v) for v in sys.argv[3].split(",")]):
            print(row, flush=True)
    elif sys.argv[1] == "mixed":
        for row in mixed_study(int(sys.argv[2]), [int(v) for v in sys.argv[3].split(",")]):
            print(row, flush=True)
    else:
        print(sensitivity_study(int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]), float(sys.argv[5])))
