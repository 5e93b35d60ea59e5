"""Generate tests/golden/bench_golden.npz: oracle C of cells of the benchmark workloads, solved tightly on the host.

The NumPy oracle (oracle/linear_ref.py, the restatement of nlfiber/linear.py) solves each cell's six unit-strain
correctors with its PCG to a relative residual of 1e-12 and assembles C. At a 1e-9 void floor the reference's own
preconditioner needs tens of thousands of iterations per 64^3 cell (days of NumPy time for a handful of cells), so
these solves use the oracle's restatement of the library's node-scaled preconditioner (`ScaledPrecond`): the
converged C is the reference's, only the iterates differ. The GPU tests and bench.py compare the library's C on
the same cells with these values.

Cells (seeded synthetic, the reference generator `random_start` through the oracle's density map):
  - "b64": 64^3 cells of the throughput workload (octant 32, kmax 2, v ~ U[0.2, 0.5] from default_rng(10000 + i),
    r 1.5, beta 16), seeds 0 (three floating solid islands), 5 (the slowest, many floating pieces), 12 (clean),
    27 (a long PCG plateau on its shear cases);
  - "b32": 32^3 cells of the batched workload (octant 16, same generator), seeds 0-7;
  - "schwarz": the Schwarz-P cell of 32^3 (octant 16, v 0.3, r 1.5, beta 16).
Material: E 1, nu 0.3, p 3, emin 1e-9.

    python tests/golden/make_bench_golden.py [--procs 8]      (about half an hour on 8 cores)
"""
import argparse
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "bench_golden.npz")
MAT = dict(E=1.0, nu=0.3, emin=1e-9, p=3.0)
TOL = 1e-12
B64 = (0, 5, 12, 27)
B32 = tuple(range(8))


def _solve(kind, seed):
    sys.path.insert(0, ROOT)
    from threadpoolctl import threadpool_limits

    from oracle import density_ref as OD
    from oracle import linear_ref as OL
    with threadpool_limits(1):
        if kind == "schwarz":
            rho = OD.schwarz_p_cell(16, v=0.3, r=1.5, beta=16.0)
        else:
            rho = OD.random_cell(seed, n_o=32 if kind == "b64" else 16, r=1.5, beta=16.0, kmax=2)[0]
        lh = OL.LinearHomogenization(rho.shape, **MAT, tol=TOL, maxit=4000)
        t0 = time.perf_counter()
        C, u, it = lh.C_full(rho, precond="scaled")
        s = lh.stiffness_scale(rho)
        res = lh.residual(s, np.eye(6), u)
        b = lh.load(s, np.eye(6))
        rrel = np.sqrt((res ** 2).sum(axis=(1, 2, 3, 4))) / np.sqrt((OL.proj(b) ** 2).sum(axis=(1, 2, 3, 4)))
        return dict(kind=kind, seed=seed, C=C, it=it, rrel=rrel, rho_sum=float(rho.sum()),
                    rho_max=float(rho.max()), seconds=time.perf_counter() - t0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=8)
    args = ap.parse_args()
    jobs = [("b64", s) for s in B64] + [("schwarz", 0)] + [("b32", s) for s in B32]
    with mp.get_context("spawn").Pool(args.procs) as pool:
        res = pool.starmap(_solve, jobs)
    out = {}
    for kind in ("b64", "b32", "schwarz"):
        rows = [r for r in res if r["kind"] == kind]
        out[f"{kind}_seeds"] = np.array([r["seed"] for r in rows])
        out[f"{kind}_C"] = np.stack([r["C"] for r in rows])
        out[f"{kind}_it"] = np.array([r["it"] for r in rows])
        out[f"{kind}_rrel"] = np.stack([r["rrel"] for r in rows])
        out[f"{kind}_rho_sum"] = np.array([r["rho_sum"] for r in rows])
        out[f"{kind}_rho_max"] = np.array([r["rho_max"] for r in rows])
        for r in rows:
            print(f"{kind} seed {r['seed']}: {r['it']} iterations, max rel residual {r['rrel'].max():.2e}, "
                  f"{r['seconds']:.0f} s", flush=True)
    out["tol"] = np.array(TOL)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
