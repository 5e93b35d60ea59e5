"""CPU tests: the oracle against the reference's own known answers (tests/test_core.py:78-142 of the
reference, restated), the golden fixtures, finite differences of every closed-form derivative, and the mode form
of the element operator that the CUDA kernels use, against the reference's dense Ke."""
import os
import sys

import numpy as np

from oracle import density_ref as OD
from oracle import linear_ref as OL

HERE = os.path.dirname(os.path.abspath(__file__))


def test_uniform_solid_is_isotropic_material():
    C, _, _ = OL.LinearHomogenization((4, 4, 4), E=2.0, nu=0.25).C_full(np.ones((4, 4, 4)))
    np.testing.assert_allclose(C, OL.iso_D(2.0, 0.25), atol=1e-10)


def test_full_vs_cubic_path_and_symmetry():
    rho = OD.grey_cell(4)
    lh = OL.LinearHomogenization(rho.shape)
    C, _, _ = lh.C_full(rho)
    np.testing.assert_allclose(C, C.T, atol=1e-12)
    assert OL.cubic_leakage(C) < 1e-8
    c, _, _ = lh.invariants(rho)
    np.testing.assert_allclose(c, OL.cubic_invariants(C), rtol=1e-8)


def test_plane_strain_equals_extruded_3d():
    rho2 = OD.grey_cell(4, d=2)
    c2, _, _ = OL.LinearHomogenization(rho2.shape).invariants(rho2)
    rho3 = np.repeat(rho2[..., None], 3, axis=2)
    C3, _, _ = OL.LinearHomogenization(rho3.shape).C_full(rho3)
    np.testing.assert_allclose(c2, [C3[0, 0], C3[1, 0], C3[5, 5]], rtol=1e-8)


def test_hashin_shtrikman_bounds_cell():
    rho = OD.binary_cell(6, v=0.3).astype(float)
    C, _, _ = OL.LinearHomogenization(rho.shape).C_full(rho)
    c11, c12, c44 = OL.cubic_invariants(C)
    Khs, Ghs = OL.hashin_shtrikman(rho.mean())
    assert (c11 + 2 * c12) / 3 < Khs and c44 < Ghs


def test_precond_symbol_is_real_symmetric():
    lh = OL.LinearHomogenization((6, 8, 4))
    assert np.abs(lh.Kh.imag).max() < 1e-12
    np.testing.assert_allclose(lh.Kinv, np.swapaxes(lh.Kinv, -1, -2), atol=1e-14)


def test_dC_drho_matches_finite_differences():
    rho = OD.grey_cell(4)
    lh = OL.LinearHomogenization(rho.shape)
    C, u, _ = lh.C_full(rho)
    dC = lh.dC_drho(rho, np.eye(6), u)
    d = np.random.default_rng(0).standard_normal(rho.shape)
    h = 1e-6
    fd = (lh.bilinear(lh.stiffness_scale(rho + h * d), np.eye(6), u)
          - lh.bilinear(lh.stiffness_scale(rho - h * d), np.eye(6), u)) / (2 * h)
    an = np.tensordot(dC, d, 3)
    assert np.abs(fd - an).max() < 1e-8 * np.abs(an).max()


def test_golden_fixtures_reproduce():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden
    g = np.load(os.path.join(HERE, "golden", "linear_golden.npz"))
    fresh = make_golden.make()
    for k, v in fresh.items():
        np.testing.assert_allclose(g[k], v, rtol=1e-12, atol=1e-15, err_msg=k)


def _elem_force_modes(ue, lam, mu):
    """The mode form of s Ke u_e used by csrc/nlf_element.cuh, in NumPy (s = 1)."""
    u = ue.reshape(2, 2, 2, 3)  # [z][y][x][comp], node a = x + 2y + 4z

    def bf(a, ax):
        a0, a1 = np.take(a, 0, axis=ax), np.take(a, 1, axis=ax)
        return np.stack([a0 + a1, a1 - a0], axis=ax)

    c = bf(bf(bf(u, 2), 1), 0).reshape(8, 3)
    l1, m1, l2, m2, k7 = lam / 16, mu / 16, lam / 48, mu / 48, (lam + 4 * mu) / 144
    f = np.zeros((8, 3))
    H = np.array([[c[1][k], c[2][k], c[4][k]] for k in range(3)])
    S = l1 * np.trace(H) * np.eye(3) + m1 * (H + H.T)
    f[1], f[2], f[4] = S[:, 0], S[:, 1], S[:, 2]
    a, b, g = c[3], c[5], c[6]
    trx, tre, trz = a[1] + b[2], a[0] + g[2], b[0] + g[1]
    f[3] = [m2 * a[0] + l2 * tre + 2 * m2 * a[0], l2 * trx + 3 * m2 * a[1], m2 * (b[1] + a[2]) + m2 * (a[2] + g[0])]
    f[5] = [m2 * b[0] + l2 * trz + 2 * m2 * b[0], m2 * (b[1] + a[2]) + m2 * (b[1] + g[0]), l2 * trx + 3 * m2 * b[2]]
    f[6] = [m2 * (g[0] + a[2]) + m2 * (g[0] + b[1]), l2 * trz + 3 * m2 * g[1], l2 * tre + 3 * m2 * g[2]]
    f[7] = k7 * c[7]
    F = f.reshape(2, 2, 2, 3)

    def bft(a, ax):
        s, d = np.take(a, 0, axis=ax), np.take(a, 1, axis=ax)
        return np.stack([s - d, s + d], axis=ax)

    return bft(bft(bft(F, 0), 1), 2).reshape(8, 3)


def test_element_mode_form_equals_dense_Ke():
    for E, nu in ((1.0, 0.3), (2.0, 0.25), (0.7, 0.45)):
        lam, mu = OL.lame(E, nu)
        _, Ke, _ = OL.element_matrices(E, nu)
        rng = np.random.default_rng(0)
        for _ in range(10):
            ue = rng.standard_normal((8, 3))
            ref = (ue.reshape(24) @ Ke).reshape(8, 3)
            np.testing.assert_allclose(_elem_force_modes(ue, lam, mu), ref, atol=1e-14 * np.abs(Ke).max() * 10)


def test_oracle_correctors_vjp_matches_finite_differences():
    """The backward of `correctors`' custom VJP (nlfiber/linear.py:118-134): <sbar, ds> equals the directional
    derivative of <ubar, u(s)> with u(s) the converged correctors, by central differences of the oracle's solve."""
    rng = np.random.default_rng(3)
    shape = (4, 4, 4)
    lh = OL.LinearHomogenization(shape, emin=1e-3, tol=1e-14, maxit=5000)
    s = 0.1 + 0.9 * rng.random(shape)
    Es = np.stack([OL.unit_strain(0), OL.unit_strain(3)])
    ubar = rng.standard_normal((2,) + shape + (3,))
    ds = rng.standard_normal(shape)
    u, _ = lh.solve(s, Es)
    sbar, lam = lh.correctors_vjp(s, Es, u, ubar)
    h = 1e-6
    fp = np.sum(ubar * lh.solve(s + h * ds, Es)[0])
    fm = np.sum(ubar * lh.solve(s - h * ds, Es)[0])
    fd = (fp - fm) / (2 * h)
    assert abs(np.sum(sbar * ds) - fd) <= 1e-7 * abs(fd)
