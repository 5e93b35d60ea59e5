"""Generates tests/golden/linear_golden.npz from the NumPy oracle (a restatement of nlfiber/linear.py).

The reference itself cannot run here (it needs JAX), so these fixtures are oracle outputs on seeded inputs.
tests/test_oracle.py regenerates them and checks they are reproduced; the GPU tests compare against them.
Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import density_ref as OD  # noqa: E402
from oracle import linear_ref as OL  # noqa: E402


def make():
    out = {}
    rho = OD.grey_cell(4)
    C, u, it = OL.LinearHomogenization(rho.shape).C_full(rho)
    out.update(grey8_rho=rho, grey8_C=C, grey8_it=np.int64(it))
    rho2 = OD.grey_cell(4, d=2)
    c2, _, _ = OL.LinearHomogenization(rho2.shape).invariants(rho2)
    out.update(plane8_rho=rho2, plane8_c=c2)
    return out


if __name__ == "__main__":
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "linear_golden.npz")
    np.savez(path, **make())
    print("wrote", path)
