"""CPU: the finite-strain oracle (a restatement of nlfiber/mech.py with closed-form stress and tangent) against
finite differences of its energy, the small-strain limit of the linear oracle (the tangent at F = I is the
linear stiffness K(s) / N, mech.py:1-17), and a small Newton solve against the linear C (the reference's
tests/test_mech.py:36-47,138-146 pin the same limits)."""
import numpy as np
import pytest

from oracle import density_ref as OD
from oracle import linear_ref as OL
from oracle import mech_ref as OM


@pytest.fixture(scope="module")
def cell():
    return OM.Cell(OD.grey_cell(3, beta=3.0))  # 6^3, wls on


@pytest.mark.parametrize("material,wls", [("neohooke", (500.0, 0.01)), ("neohooke", None), ("linear", None)])
def test_gradient_and_tangent_match_finite_differences(material, wls):
    rho = OD.grey_cell(3, beta=3.0)
    c = OM.Cell(rho, material=material, wls=wls)
    rng = np.random.default_rng(0)
    w = 0.05 * rng.standard_normal(c.shape + (3,))
    Fb = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
    gw, P = c.grad(w, Fb)
    v = rng.standard_normal(c.shape + (3,))
    dF = rng.standard_normal((3, 3))
    h = 1e-6
    fd = (c.energy(w + h * v, Fb + h * dF) - c.energy(w - h * v, Fb - h * dF)) / (2 * h)
    an = np.sum(gw * v) + np.sum(P * dF)
    assert abs(fd - an) < 1e-7 * abs(an) + 1e-12
    hw, hP = c.hvp(w, Fb, v, dF)
    g1, P1 = c.grad(w + h * v, Fb + h * dF)
    g2, P2 = c.grad(w - h * v, Fb - h * dF)
    fdw, fdP = (g1 - g2) / (2 * h), (P1 - P2) / (2 * h)
    assert np.abs(hw - fdw).max() < 1e-6 * np.abs(fdw).max()
    assert np.abs(hP - fdP).max() < 1e-6 * np.abs(fdP).max()


def test_tangent_at_identity_is_linear_stiffness(cell):
    rng = np.random.default_rng(1)
    v = rng.standard_normal(cell.shape + (3,))
    hw, _ = cell.hvp(np.zeros(cell.shape + (3,)), np.eye(3), v, np.zeros((3, 3)))
    lh = OL.LinearHomogenization(cell.shape, emin=cell.emin)
    Kv = lh.apply_K(cell.s, v) / cell.N
    assert np.abs(hw - Kv).max() < 1e-12 * np.abs(Kv).max()


def test_small_strain_solve_matches_linear_C(cell):
    """Uniaxial strain e = 1e-4 under full control: Pbar = C eps to O(e); lateral control: nu = nu0(C)."""
    C, _, _ = OL.LinearHomogenization(cell.shape, emin=cell.emin).C_full(cell.rho)
    e = 1e-4
    full = OM.Mixed(cell, free=[])
    w, F, log = full.solve(np.diag([1 + e, 1.0, 1.0]), rtol=1e-10, cg_tol=1e-10)
    assert log["converged"]
    P = cell.mean_stress(w, F)
    np.testing.assert_allclose([P[0, 0], P[1, 1], P[2, 2]], C[:3, 0] * e, rtol=2e-3)
    mix = OM.Mixed(cell, [(1, 1), (2, 2)])
    w, F, log = mix.solve(np.diag([1 + e, 1.0, 1.0]), rtol=1e-10, cg_tol=1e-10)
    assert log["converged"]
    S = np.linalg.inv(C)
    nu0 = -S[1, 0] / S[0, 0]
    assert abs(-(F[1, 1] - 1) / e - nu0) < 1e-3


@pytest.mark.parametrize("material,wls", [("neohooke", (500.0, 0.01)), ("neohooke", None), ("linear", None)])
def test_toec_closed_forms_match_finite_differences(material, wls):
    """nlfiber/mech.py:458-493 takes C = f''(0) and f'''(0) of f(s) = wq sum s psi_eff(I + sum_I s_I H_I) by
    autodiff; the oracle's closed forms are checked by central differences of that f (built from the oracle's
    psi_eff), whose truncation error is O(h^2)."""
    rng = np.random.default_rng(0)
    rho = OD.random_cell(1, n_o=2)[0]
    cell = OM.Cell(rho, material=material, wls=wls, emin=1e-3)
    chi = 0.05 * rng.standard_normal((6,) + rho.shape + (3,))
    C, T = OM.toec(cell, chi)
    T3 = T + OM.toec_geometric(C)
    H = np.stack([OM.voigt_tensor(I) + cell.grad_w(chi[I]) for I in range(6)])

    def f(sv):
        F = np.eye(3) + np.tensordot(sv, H, axes=1)
        return cell.wq * np.sum(cell.s[None] * cell.psi_eff(F, None if cell.gamma is None else cell.gamma[None]))

    e, h = np.eye(6), 1e-3
    for I in range(6):
        for J in range(6):
            fd = (f(h * (e[I] + e[J])) - f(h * (e[I] - e[J])) - f(h * (e[J] - e[I])) + f(-h * (e[I] + e[J]))) / (4 * h * h)
            assert abs(fd - C[I, J]) <= 1e-5 * np.abs(C).max()
    h = 2e-3
    for I, J, K in [(0, 0, 0), (0, 1, 2), (3, 3, 0), (1, 4, 4), (2, 5, 3), (3, 4, 5), (5, 5, 5)]:
        a, b, c = e[I] * h, e[J] * h, e[K] * h
        fd = (f(a + b + c) - f(a + b - c) - f(a - b + c) + f(a - b - c) - f(-a + b + c) + f(-a + b - c)
              + f(-a - b + c) - f(-a - b - c)) / (8 * h ** 3)
        assert abs(fd - T3[I, J, K]) <= 1e-4 * max(np.abs(T3).max(), 1.0)
