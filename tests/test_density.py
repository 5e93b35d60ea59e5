"""CPU: the oracle's restatement of the input side (nlfiber/density.py, symmetry.py, fiber.random_start) keeps the
reference's invariants: exact volume and exact orbit symmetry (tests/test_core.py:43-77 of the reference), and its
reverse mode is pinned by central differences."""
import numpy as np

from oracle import density_ref as OD


def test_exact_volume_and_symmetry():
    """The oracle's generator keeps the reference's invariants: mean(rho) = v and exact orbit symmetry."""
    rho, v = OD.random_cell(5, n_o=8, beta=16.0)
    assert abs(rho.mean() - v) < 1e-12
    np.testing.assert_array_equal(rho, rho[::-1])
    np.testing.assert_array_equal(rho, np.transpose(rho, (2, 0, 1)))
    np.testing.assert_array_equal(rho, np.transpose(rho, (1, 0, 2)))


def test_oracle_rho_vjp_matches_finite_differences():
    """The oracle's reverse mode of DensityMap.rho (threshold with the implicit d eta, the symmetry maps, the
    unit-std scaling and the cone filter), pinned by central differences of the oracle's forward map; the last
    case is the reference's own check (tests/test_core.py:43-53: d/dphi sum(rho(phi, 4)^3), DensityMap(4, r=1.5,
    v=0.27), a sym_perm'd direction)."""
    rng = np.random.default_rng(0)
    for n_o, r, v, beta in ((4, 1.5, 0.27, 4.0), (4, 1.0, 0.35, 8.0), (3, 2.5, 0.3, 16.0), (5, 1.5, 0.4, 2.0)):
        dm = OD.DensityMap(n_o, 3, r=r, v=v)
        phi = rng.standard_normal((n_o,) * 3)
        g = rng.standard_normal((2 * n_o,) * 3)
        d = rng.standard_normal((n_o,) * 3)
        h = 1e-6
        fd = (np.sum(g * dm.rho(phi + h * d, beta)) - np.sum(g * dm.rho(phi - h * d, beta))) / (2 * h)
        assert abs(np.sum(OD.rho_vjp(dm, phi, beta, g) * d) - fd) <= 1e-8 * abs(fd)
    dm = OD.DensityMap(4, r=1.5, v=0.27)
    phi = OD.sym_perm(np.random.default_rng(2).standard_normal((4, 4, 4)))
    d = OD.sym_perm(np.random.default_rng(3).standard_normal((4, 4, 4)))
    grad = OD.rho_vjp(dm, phi, 4.0, 3.0 * dm.rho(phi, 4.0) ** 2)
    h = 1e-6
    fd = (np.sum(dm.rho(phi + h * d, 4.0) ** 3) - np.sum(dm.rho(phi - h * d, 4.0) ** 3)) / (2 * h)
    assert abs(np.vdot(grad, d) - fd) <= 1e-7 * abs(fd) + 1e-10
