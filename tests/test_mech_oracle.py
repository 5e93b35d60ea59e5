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


def _stab_cell():
    return OM.Cell(OD.random_cell(4, n_o=2)[0], emin=1e-3)


def test_effective_tangent_matches_finite_differences():
    """nlfiber/mech.py:419-436: A = dPbar/dFbar of the re-equilibrated cell (full control), against central
    differences of the mean stress of Newton solves at Fbar +- h E (h = 1e-4: the error is O(h^2), 2.6e-9 here;
    at h = 1e-5 the perturbed Newton solve stalls on its relative tolerance)."""
    cell = _stab_cell()
    full = OM.Mixed(cell, free=[])
    w, F, log = full.solve(np.diag([1.03, 1.0, 1.0]), rtol=1e-12, cg_tol=1e-12)
    assert log["converged"]
    A = OM.effective_tangent(cell, w, F, cg_tol=1e-13)
    h = 1e-4
    for c, d in ((0, 0), (1, 2), (2, 1), (0, 1)):
        E = np.zeros((3, 3))
        E[c, d] = 1.0
        wp, Fp, _ = full.solve(F + h * E, z0=w.ravel(), rtol=1e-13, cg_tol=1e-13)
        wm, Fm, _ = full.solve(F - h * E, z0=w.ravel(), rtol=1e-13, cg_tol=1e-13)
        fd = (cell.mean_stress(wp, Fp) - cell.mean_stress(wm, Fm)) / (2 * h)
        assert np.abs(fd - A[:, :, c, d]).max() <= 2e-8


def test_lowest_eigs_match_dense_spectrum():
    """nlfiber/mech.py:363-416: the probed diagonal is the Hessian's diagonal, and LOBPCG's lowest eigenvalues of
    D^-1/2 H D^-1/2 (translations excluded) are those of the dense operator restricted to the complement."""
    cell = _stab_cell()
    mix = OM.Mixed(cell)
    z, Fb = mix.z0(np.eye(3)), np.eye(3)
    # residual tolerance 1e-7: the residuals' rounding floor here is near 1e-8, where scipy stops with a warning;
    # the eigenvalues' error is second order in the residual
    vals, _, _ = OM.lowest_eigs(mix, z, Fb, k=4, tol=1e-7, maxiter=2000)
    dsc = OM.diag_scale(mix)
    nz = mix.nw + mix.k
    Hd = np.stack([mix.hvp(z, Fb, np.eye(nz)[:, j]) for j in range(nz)], axis=1)
    assert np.abs(1.0 / np.sqrt(np.abs(np.diag(Hd)) + 1e-30) - dsc).max() <= 1e-14 * dsc.max()
    S = dsc[:, None] * Hd * dsc[None, :]
    T = np.zeros((nz, 3))
    for i in range(3):
        T[i:mix.nw:3, i] = 1.0
    Y, _ = np.linalg.qr(T / dsc[:, None])
    Qf, _ = np.linalg.qr(np.concatenate([Y, np.random.default_rng(1).standard_normal((nz, nz - 3))], axis=1))
    ev = np.linalg.eigvalsh(Qf[:, 3:].T @ (0.5 * (S + S.T)) @ Qf[:, 3:])[:4]
    np.testing.assert_allclose(vals, ev, rtol=1e-7)


def test_rank_one_min_isotropic():
    """The acoustic tensor of isotropic linear elasticity has smallest eigenvalue mu for every direction."""
    lam, mu = OL.lame(1.0, 0.3)
    d = np.eye(3)
    A = (lam * np.einsum("ij,kl->ijkl", d, d) + mu * (np.einsum("ik,jl->ijkl", d, d) + np.einsum("il,jk->ijkl", d, d)))
    v, n = OM.rank_one_min(A, m=200)
    assert abs(v - mu) < 1e-12 and abs(np.linalg.norm(n) - 1.0) < 1e-12
