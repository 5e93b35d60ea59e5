"""GPU: the density map of libnlf.so (nlf_density_*, nlfiber_b200.density.GpuDensityMap) against the oracle's
restatement of nlfiber/density.py and nlfiber/symmetry.py (oracle/density_ref.py), and the reference's own
invariants of that map (tests/test_core.py:43-77: exact volume, exact orbit symmetry).

Tolerances: the GPU filters by a direct periodic sum over the cone's taps where the reference multiplies FFTs,
and reduces in another order, so values agree to rounding: 1e-12 absolute on rho (in [0, 1]) and eta, 1e-12 on
the unit-variance smoothed field. Symmetry is exact (bitwise): one value is computed per orbit and copied."""
import numpy as np
import pytest

from oracle import density_ref as OD

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _gpu(n_o, r, v):
    from nlfiber_b200.density import GpuDensityMap
    return GpuDensityMap(n_o, 3, r=r, v=v)


@pytest.mark.parametrize("n_o,r,v,beta,seed", [
    (4, 1.5, 0.27, 2.0, 2), (4, 1.5, 0.27, 8.0, 2), (4, 1.5, 0.27, 32.0, 2),
    (4, 1.0, 0.35, 3.0, 0), (6, 1.5, 0.3, 16.0, 5), (4, 3.0, 0.3, 4.0, 1), (8, 2.5, 0.25, 32.0, 3),
    (5, 1.5, 0.4, 16.0, 7), (16, 1.5, 0.3, 16.0, 11),
])
def test_rho_smooth_eta_match_oracle(n_o, r, v, beta, seed):
    phi = np.random.default_rng(seed).standard_normal((n_o,) * 3)
    dm = OD.DensityMap(n_o, 3, r=r, v=v)
    u_o = dm.smooth(phi)
    eta_o = OD.solve_eta(u_o, v, beta)
    rho_o = dm.rho(phi, beta)
    out = _gpu(n_o, r, v).run(phi, beta, smooth=True)
    rho, u, eta = (out[k].cpu().numpy() for k in ("rho", "u", "eta"))
    assert np.abs(u[0] - u_o).max() < TOL
    assert abs(eta[0] - eta_o) < TOL
    assert np.abs(rho[0] - rho_o).max() < TOL
    assert abs(rho[0].mean() - v) < 1e-12


def test_exact_orbit_symmetry_and_volume():
    """tests/test_core.py:35-41,43-48 of the reference: the full cell has all 48 symmetries exactly, and the
    volume is exact for every sharpness."""
    n_o = 6
    phi = np.random.default_rng(2).standard_normal((n_o,) * 3)
    g = _gpu(n_o, 1.5, 0.27)
    for beta in (2.0, 8.0, 32.0):
        out = g.run(phi, beta, smooth=True)
        for f in (out["rho"][0].cpu().numpy(), out["u"][0].cpu().numpy()):
            np.testing.assert_array_equal(f, f[::-1])
            np.testing.assert_array_equal(f, f[:, ::-1])
            np.testing.assert_array_equal(f, f[:, :, ::-1])
            np.testing.assert_array_equal(f, np.transpose(f, (2, 0, 1)))
            np.testing.assert_array_equal(f, np.transpose(f, (1, 0, 2)))
        assert abs(float(out["rho"][0].mean()) - 0.27) < 1e-12


def test_orbit_count_is_n_free():
    """nlfiber/symmetry.py:20-22: C(n_o + 2, 3) free entries."""
    for n_o in (1, 2, 5, 32):
        assert _gpu(n_o, 1.5, 0.3).orbits == OD.n_free(n_o)


def test_batch_with_per_cell_volumes_is_cellwise():
    """A batch with one volume per cell gives, bit for bit, the single-cell results."""
    n_o, beta = 8, 16.0
    phis = np.stack([OD.random_start(n_o, 3, seed=s, kmax=2) for s in range(5)])
    vols = np.array([0.2, 0.3, 0.45, 0.27, 0.5])
    g = _gpu(n_o, 1.5, 0.3)
    out = g.run(phis, beta, v=vols, smooth=True)
    for i in range(5):
        one = g.run(phis[i], beta, v=vols[i], smooth=True)
        for k in ("rho", "u", "eta"):
            np.testing.assert_array_equal(out[k][i].cpu().numpy(), one[k][0].cpu().numpy())
        rho_o = OD.DensityMap(n_o, 3, r=1.5, v=float(vols[i])).rho(phis[i], beta)
        assert np.abs(out["rho"][i].cpu().numpy() - rho_o).max() < TOL


def test_host_and_device_pointers_agree():
    """The C ABI takes host or device arrays; both give the same bits."""
    import ctypes

    import torch

    from nlfiber_b200._lib import check, lib
    n_o, beta, nc = 4, 8.0, 3
    phi = np.random.default_rng(9).standard_normal((nc, n_o, n_o, n_o))
    v = np.array([0.3, 0.35, 0.4])
    g = _gpu(n_o, 1.5, 0.3)
    n = 2 * n_o
    rho_h = np.empty((nc, n, n, n))
    eta_h = np.empty(nc)
    check(lib.nlf_density_rho(g._h, nc, phi.ctypes.data, v.ctypes.data, ctypes.c_double(beta), rho_h.ctypes.data,
                              None, eta_h.ctypes.data, None))
    out = g.run(torch.as_tensor(phi, device="cuda"), beta, v=v)
    np.testing.assert_array_equal(rho_h, out["rho"].cpu().numpy())
    np.testing.assert_array_equal(eta_h, out["eta"].cpu().numpy())


def test_benchmark_cells_match_oracle_generator():
    """The 64^3 cells of the benchmark (bench.gpu_cells: bench.synth_phi(seed, 32) on the host, v ~ U[0.2, 0.5]
    from default_rng(10000 + i), then the GPU map with r = 1.5, beta = 16) agree with the oracle's generator."""
    import bench
    seeds = [0, 1]
    rho_d = bench.gpu_cells(seeds, 32)
    for k, i in enumerate(seeds):
        rho_h, v = OD.random_cell(i, n_o=32, r=1.5, beta=16.0, kmax=2)
        rho = rho_d[k].cpu().numpy()
        assert np.abs(rho - rho_h).max() < TOL
        assert abs(rho.mean() - v) < 1e-12


def test_bad_arguments_raise():
    from nlfiber_b200._lib import NlfError
    from nlfiber_b200.density import GpuDensityMap
    with pytest.raises(NlfError):
        GpuDensityMap(0, 3, r=1.5)
    with pytest.raises(NlfError):
        GpuDensityMap(4, 3, r=float("nan"))
    g = GpuDensityMap(4, 3, r=1.5)
    with pytest.raises(NlfError):
        g.run(np.zeros((4, 4, 4)), -1.0)
    with pytest.raises(ValueError):
        g.run(np.zeros((5, 5, 5)), 8.0)


def test_gather_filter_path_agrees(tmp_path):
    """The direct-gather filter (used when a tile's staged region would not fit in shared memory; forced here by
    NLF_DENSITY_GATHER=1 in a child process) gives the tiled filter's values: the per-voxel sums are the same, only
    the grouping of the standard deviation's partial sums differs."""
    import os
    import subprocess
    import sys
    n_o, r, v, beta = 6, 2.5, 0.3, 16.0
    phi = np.random.default_rng(4).standard_normal((n_o,) * 3)
    np.save(tmp_path / "phi.npy", phi)
    code = ("import numpy as np; from nlfiber_b200.density import GpuDensityMap; "
            f"g = GpuDensityMap({n_o}, 3, r={r}, v={v}); "
            f"o = g.run(np.load(r'{tmp_path / 'phi.npy'}'), {beta}, smooth=True); "
            f"np.save(r'{tmp_path / 'rho.npy'}', o['rho'][0].cpu().numpy()); "
            f"np.save(r'{tmp_path / 'u.npy'}', o['u'][0].cpu().numpy())")
    from conftest import PKG_DIR, ROOT
    env = dict(os.environ, NLF_DENSITY_GATHER="1",
               PYTHONPATH=os.pathsep.join([PKG_DIR, ROOT, os.environ.get("PYTHONPATH", "")]))
    subprocess.run([sys.executable, "-c", code], check=True, env=env, timeout=300)
    out = _gpu(n_o, r, v).run(phi, beta, smooth=True)
    assert np.abs(np.load(tmp_path / "u.npy") - out["u"][0].cpu().numpy()).max() < 1e-14
    assert np.abs(np.load(tmp_path / "rho.npy") - out["rho"][0].cpu().numpy()).max() < 1e-13


@pytest.mark.parametrize("n_o,r,v,beta", [(4, 1.5, 0.27, 4.0), (3, 2.5, 0.3, 16.0), (5, 1.0, 0.4, 8.0),
                                          (8, 1.5, 0.3, 16.0), (16, 1.5, 0.25, 32.0)])
def test_vjp_matches_oracle(n_o, r, v, beta):
    """nlf_density_vjp against the oracle's reverse mode (pinned by finite differences on the CPU), for a batch of
    2 cells with per-cell volumes and 3 cotangent rows each. Tolerance 1e-10 of the largest entry: the filter and
    the reductions round differently."""
    rng = np.random.default_rng(n_o)
    phis = rng.standard_normal((2,) + (n_o,) * 3)
    vols = np.array([v, v + 0.05])
    g = rng.standard_normal((2, 3) + (2 * n_o,) * 3)
    out = _gpu(n_o, r, v).vjp(phis, beta, g, v=vols).cpu().numpy()
    for i in range(2):
        dm = OD.DensityMap(n_o, 3, r=r, v=float(vols[i]))
        for k in range(3):
            ref = OD.rho_vjp(dm, phis[i], beta, g[i, k])
            assert np.abs(out[i, k] - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())


def test_fiber_value_jac_matches_oracle_chain_and_finite_differences():
    """nlfiber/fiber.py:34-39,53-57 on the GPU: c = (C11, C12, C44) / E of the two-case solve and its Jacobian
    rows dc_k/dphi (dC/drho with the correctors held fixed, pulled back through the density map). Checked against
    the oracle's chain (oracle solve, dC_drho, rho_vjp) and against central differences of the GPU value."""
    from nlfiber_b200.fiber import Fiber
    from oracle import linear_ref as OL
    n_o, beta, v = 4, 8.0, 0.35
    phi = OD.sym_perm(np.random.default_rng(5).standard_normal((n_o,) * 3))
    fib = Fiber(n_o, v=v, r=1.5, emin=1e-3, tol=1e-13, maxit=20000)
    c, J = fib.value_jac(phi, beta, warm=False)
    dm = OD.DensityMap(n_o, 3, r=1.5, v=v)
    rho = dm.rho(phi, beta)
    lh = OL.LinearHomogenization(rho.shape, emin=1e-3, tol=1e-13, maxit=20000)
    c_o, u2, _ = lh.invariants(rho)
    np.testing.assert_allclose(c, c_o, rtol=1e-10)
    u3 = np.stack([u2[0], lh.swap_xy(u2[0]), u2[1]])
    Es = np.stack([OL.unit_strain(0), OL.unit_strain(1), OL.unit_strain(3)])
    dC = lh.dC_drho(rho, Es, u3)
    for k, (I, Jx) in enumerate(((0, 0), (1, 0), (2, 2))):
        ref = OD.rho_vjp(dm, phi, beta, dC[I, Jx] / lh.E)
        assert np.abs(J[k] - ref).max() <= 1e-8 * np.abs(ref).max()
    d = OD.sym_perm(np.random.default_rng(6).standard_normal((n_o,) * 3))
    h = 1e-5
    fd = (fib.value(phi + h * d, beta, warm=False) - fib.value(phi - h * d, beta, warm=False)) / (2 * h)
    jd = np.tensordot(J, d, axes=3)
    np.testing.assert_allclose(jd, fd, rtol=1e-6, atol=1e-9)


# ---- square cells (d = 2): the same map on a quadrant (n_o)^2 and a full cell (2 n_o)^2 ----------------------

def _gpu2(n_o, r, v):
    from nlfiber_b200.density import GpuDensityMap
    return GpuDensityMap(n_o, 2, r=r, v=v)


@pytest.mark.parametrize("n_o,r,v,beta,seed", [(4, 1.5, 0.27, 8.0, 2), (6, 1.5, 0.3, 16.0, 5), (8, 2.5, 0.25, 32.0, 3),
                                               (5, 1.0, 0.4, 4.0, 7), (32, 1.5, 0.3, 16.0, 11)])
def test_square_rho_smooth_eta_match_oracle(n_o, r, v, beta, seed):
    """DensityMap(n_o, d=2) (nlfiber/density.py:75-94, symmetry.py for d = 2) on the GPU against the oracle."""
    phi = np.random.default_rng(seed).standard_normal((n_o,) * 2)
    dm = OD.DensityMap(n_o, 2, r=r, v=v)
    u_o = dm.smooth(phi)
    eta_o = OD.solve_eta(u_o, v, beta)
    rho_o = dm.rho(phi, beta)
    g = _gpu2(n_o, r, v)
    assert g.orbits == n_o * (n_o + 1) // 2
    out = g.run(phi, beta, smooth=True)
    rho, u, eta = (out[k].cpu().numpy() for k in ("rho", "u", "eta"))
    assert np.abs(u[0] - u_o).max() < TOL
    assert abs(eta[0] - eta_o) < TOL
    assert np.abs(rho[0] - rho_o).max() < TOL
    assert abs(rho[0].mean() - v) < 1e-12
    for f in (rho[0], u[0]):  # the 8 symmetries of the square, exactly
        np.testing.assert_array_equal(f, f[::-1])
        np.testing.assert_array_equal(f, f[:, ::-1])
        np.testing.assert_array_equal(f, f.T)


@pytest.mark.parametrize("n_o,r,v,beta", [(4, 1.5, 0.27, 4.0), (5, 1.0, 0.4, 8.0), (16, 1.5, 0.25, 32.0)])
def test_square_vjp_matches_oracle(n_o, r, v, beta):
    """nlf_density_vjp on squares against the oracle's reverse mode (pinned by finite differences on the CPU), for
    2 cells with per-cell volumes and 3 cotangent rows each."""
    rng = np.random.default_rng(n_o)
    phis = rng.standard_normal((2,) + (n_o,) * 2)
    vols = np.array([v, v + 0.05])
    g = rng.standard_normal((2, 3) + (2 * n_o,) * 2)
    out = _gpu2(n_o, r, v).vjp(phis, beta, g, v=vols).cpu().numpy()
    for i in range(2):
        dm = OD.DensityMap(n_o, 2, r=r, v=float(vols[i]))
        for k in range(3):
            ref = OD.rho_vjp(dm, phis[i], beta, g[i, k])
            assert np.abs(out[i, k] - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())


def test_square_fiber_value_jac_matches_oracle_chain_and_finite_differences():
    """nlfiber/fiber.py:17-60 with d = 2: c = (C11, C12, C66) / E of the plane-strain two-case solve and its
    Jacobian rows, against the oracle's chain and central differences of the GPU value."""
    from nlfiber_b200.fiber import Fiber
    from oracle import linear_ref as OL
    n_o, beta, v = 6, 8.0, 0.35
    phi = OD.sym_perm(np.random.default_rng(5).standard_normal((n_o,) * 2))
    fib = Fiber(n_o, d=2, v=v, r=1.5, emin=1e-3, tol=1e-13, maxit=20000)
    c, J = fib.value_jac(phi, beta, warm=False)
    assert J.shape == (3, n_o, n_o)
    dm = OD.DensityMap(n_o, 2, r=1.5, v=v)
    rho = dm.rho(phi, beta)
    lh = OL.LinearHomogenization(rho.shape, emin=1e-3, tol=1e-13, maxit=20000)
    c_o, u2, _ = lh.invariants(rho)
    np.testing.assert_allclose(c, c_o, rtol=1e-10)
    u3 = np.stack([u2[0], lh.swap_xy(u2[0]), u2[1]])
    Es = np.stack([OL.unit_strain(0), OL.unit_strain(1), OL.unit_strain(lh._shear())])
    dC = lh.dC_drho(rho, Es, u3)
    for k, (I, Jx) in enumerate(((0, 0), (1, 0), (2, 2))):
        ref = OD.rho_vjp(dm, phi, beta, dC[I, Jx].reshape(rho.shape) / lh.E)
        assert np.abs(J[k] - ref).max() <= 1e-8 * np.abs(ref).max()
    d = OD.sym_perm(np.random.default_rng(6).standard_normal((n_o,) * 2))
    h = 1e-5
    fd = (fib.value(phi + h * d, beta, warm=False) - fib.value(phi - h * d, beta, warm=False)) / (2 * h)
    jd = np.tensordot(J, d, axes=2)
    np.testing.assert_allclose(jd, fd, rtol=1e-6, atol=1e-9)
