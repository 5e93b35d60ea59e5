"""CPU oracle for the voxel homogenization hot path. TEST INFRASTRUCTURE ONLY.

This package is a NumPy FP64 restatement of the reference's algorithm (nlfiber/linear.py, nlfiber/mech.py and
the input generators nlfiber/density.py, nlfiber/symmetry.py, nlfiber/fiber.py). Every function cites the
reference file:line it follows.

It exists to check the CUDA path: only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
its `--impl reference` arm) may import it. The product path (the C-ABI library and the nlfiber_b200 package)
never imports, links or runs anything from here, and fails loudly when its CUDA library is missing.

Pinning. The reference cannot be imported here (it needs JAX, which is absent) and ships no golden vectors, so
this restatement is pinned by the known-answer and consistency tests the reference itself holds for the path
(tests/test_core.py:78-99,101-122,135-142 and tests/test_mech.py:36-47,115-134 of the reference), restated in
tests/test_oracle.py, plus finite-difference checks of every closed-form derivative.
"""
