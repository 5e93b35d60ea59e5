"""CPU: the package's host-side input generator (nlfiber_b200.density, the mirror of nlfiber/density.py,
symmetry.py and fiber.random_start) reproduces the oracle's restatement bit for bit, and keeps the reference's
invariants: exact volume and exact orbit symmetry (tests/test_core.py:43-77 of the reference)."""
import numpy as np

from oracle import density_ref as OD


def test_generator_matches_oracle_bitwise():
    from nlfiber_b200 import density as D
    for n_o in (3, 4, 8):
        np.testing.assert_array_equal(D.representative_index(n_o), OD.representative_index(n_o))
    for i in range(3):
        r1, v1 = D.random_cell(i, n_o=6)
        r2, v2 = OD.random_cell(i, n_o=6)
        assert v1 == v2
        np.testing.assert_array_equal(r1, r2)
    np.testing.assert_array_equal(D.DensityMap(8, r=1.5, v=0.3).rho(D.schwarz_p_phi(8), 16.0),
                                  OD.schwarz_p_cell(8))


def test_exact_volume_and_symmetry():
    from nlfiber_b200 import density as D
    rho, v = D.random_cell(5, n_o=8, beta=16.0)
    assert abs(rho.mean() - v) < 1e-12
    np.testing.assert_array_equal(rho, rho[::-1])
    np.testing.assert_array_equal(rho, np.transpose(rho, (2, 0, 1)))
    np.testing.assert_array_equal(rho, np.transpose(rho, (1, 0, 2)))
