"""CPU studies behind two design decisions of the solver, on the oracle's PCG. TEST INFRASTRUCTURE ONLY: nothing
in the library imports this file; it restates variants of the oracle's node-scaled PCG to measure them.

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

    python -m oracle.precision_studies mixed 16 0,1,2,3     # octant size and seeds
    python -m oracle.precision_studies sensitivity 32 0 8 1e-9
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


if __name__ == "__main__":
    if sys.argv[1] == "mixed":
        for row in mixed_study(int(sys.argv[2]), [int(v) for v in sys.argv[3].split(",")]):
            print(row, flush=True)
    else:
        print(sensitivity_study(int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]), float(sys.argv[5])))
