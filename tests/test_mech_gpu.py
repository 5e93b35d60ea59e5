"""Parity of the CUDA finite-strain path (libnlf.so through nlfiber_b200.mech) with the NumPy oracle (a
restatement of nlfiber/mech.py whose closed forms are checked by finite differences in test_mech_oracle.py):
energy, residual, mean stress, tangent matvec, preconditioner, the CG iterates and a Newton-CG solve."""
import os

os.environ.setdefault("NLF_POISON_WORKSPACE", "1")

import numpy as np  # noqa: E402
import pytest  # noqa: E402

from oracle import density_ref as OD  # noqa: E402
from oracle import mech_ref as OM  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    from nlfiber_b200 import mech
    return mech


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("material,wls", [("neohooke", (500.0, 0.01)), ("neohooke", None), ("linear", None)])
@pytest.mark.parametrize("shape_n", [3, 4])
def test_energy_residual_tangent(M, material, wls, shape_n):
    rho = OD.grey_cell(shape_n, beta=3.0)
    c, o = M.Cell(rho, material=material, wls=wls), OM.Cell(rho, material=material, wls=wls)
    np.testing.assert_allclose(c.s, o.s, rtol=1e-14)
    if wls is not None:
        np.testing.assert_allclose(c.gamma, o.gamma, rtol=1e-13, atol=1e-15)
    rng = np.random.default_rng(3)
    w = 0.05 * rng.standard_normal(c.shape + (3,))
    Fb = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
    assert rel(c.energy(w, Fb), o.energy(w, Fb)) < 1e-12
    gw, P = c.grad(w, Fb)
    gwo, Po = o.grad(w, Fb)
    assert rel(gw, gwo) < 1e-12 and rel(P, Po) < 1e-12
    v = rng.standard_normal(c.shape + (3,))
    dF = rng.standard_normal((3, 3))
    hv, hP = c.hvp(w, Fb, v, dF)
    hvo, hPo = o.hvp(w, Fb, v, dF)
    assert rel(hv, hvo) < 1e-12 and rel(hP, hPo) < 1e-12
    assert rel(c.grad_w(w), o.grad_w(w)) < 1e-13
    assert rel(c.precond_w(v), o.precond_w(v)) < 1e-11


def test_cg_iterates_match_oracle(M):
    rho = OD.grey_cell(3, beta=3.0)
    c, o = M.Cell(rho), OM.Cell(rho)
    mix, omix = M.Mixed(c, [(1, 1), (2, 2)]), OM.Mixed(o, [(1, 1), (2, 2)])
    Fb = np.diag([1.03, 1.0, 1.0])
    rng = np.random.default_rng(4)
    z = omix.z0(Fb) + np.concatenate([0.01 * rng.standard_normal(omix.nw), np.zeros(2)])
    g = omix.proj(omix.g(z, Fb))
    dmac = omix.macro_diag(z, Fb)
    sws = omix._sws()
    x, it, conv, neg = mix._cgA(mix.tangent(z, Fb), -g, dmac, sws, 0.0, 25)
    xo, ito, convo, nego = omix.cg(z, Fb, -g, dmac, sws, 0.0, 25)
    assert it == ito == 25 and conv == convo and neg == nego
    assert rel(x, xo) < 1e-8
    np.testing.assert_allclose(mix.macro_diag(mix.tangent(z, Fb)), dmac, rtol=1e-12)


def test_newton_solve_matches_oracle(M):
    """Uniaxial stretch 3% with free lateral stretches (qoi.LATERAL[0]): same Newton history and state."""
    rho = OD.grey_cell(3, beta=3.0)
    c, o = M.Cell(rho), OM.Cell(rho)
    Fb = np.diag([1.03, 1.0, 1.0])
    w, F, log = M.Mixed(c, [(1, 1), (2, 2)]).solve(Fb, rtol=1e-10, cg_tol=1e-10)
    wo, Fo, logo = OM.Mixed(o, [(1, 1), (2, 2)]).solve(Fb, rtol=1e-10, cg_tol=1e-10)
    assert log["converged"] and logo["converged"]
    assert log["newton"] == logo["newton"]
    np.testing.assert_allclose(F, Fo, atol=1e-9)
    assert rel(c.mean_stress(w, F), o.mean_stress(wo, Fo)) < 1e-8


def test_scaled_mech_preconditioner_same_solution_fewer_cg(M):
    """The node-scaled mech preconditioner (nlf_mech_set_precond) reaches the reference preconditioner's Newton
    solution, with fewer CG iterations on a high-contrast cell."""
    rho = OD.random_cell(3, n_o=8, beta=16.0)[0]
    Fb = np.diag([0.98, 1.0, 1.0])
    res = {}
    for pc in ("fft", "scaled"):
        c = M.Cell(rho, emin=1e-6)
        w, F, log = M.Mixed(c, [(1, 1), (2, 2)], precond=pc).solve(Fb, rtol=1e-10, cg_tol=1e-10)
        assert log["converged"], (pc, log["gnorm"])
        res[pc] = (F, c.mean_stress(w, F), log["cg"])
    np.testing.assert_allclose(res["scaled"][0], res["fft"][0], atol=1e-8)
    assert rel(res["scaled"][1], res["fft"][1]) < 1e-6
    assert res["scaled"][2] < res["fft"][2], (res["scaled"][2], res["fft"][2])


def test_device_resident_newton_matches_host_loop(M):
    """Mixed(device="cuda") keeps z and the Newton vectors on the GPU: the same converged state as the host loop,
    to the rounding of the mean removals (done by the device instead of NumPy) within the Newton tolerance."""
    rho = OD.random_cell(5, n_o=8, beta=8.0)[0]
    Fb = np.diag([0.98, 1.0, 1.0])
    out = {}
    for dev in (None, "cuda"):
        c = M.Cell(rho, emin=1e-3)
        w, F, log = M.Mixed(c, [(1, 1), (2, 2)], precond="scaled", device=dev).solve(Fb, rtol=1e-10, cg_tol=1e-8)
        assert log["converged"]
        w = w.cpu().numpy() if hasattr(w, "cpu") else w
        out[dev] = (w, F, log["newton"], c.mean_stress(w, F))
    # the stop at rtol 1e-10 sits near the rounding floor, so the two may stop one Newton step apart
    assert abs(out[None][2] - out["cuda"][2]) <= 1
    np.testing.assert_allclose(out["cuda"][1], out[None][1], atol=1e-10)
    assert rel(out["cuda"][3], out[None][3]) < 1e-6
    assert rel(out["cuda"][0], out[None][0]) < 1e-4


def test_concurrent_cells_match_sequential(M):
    """Cells solved from several host threads, each on its own CUDA stream (handles made beforehand), give the same
    Newton states, iteration counts and stresses as the same cells solved one after the other: the graph captures
    of their CG solves do not interfere."""
    import threading
    import torch
    rhos = [OD.random_cell(i, n_o=8, beta=8.0)[0] for i in (0, 1, 5)]
    Fb = np.diag([0.98, 1.0, 1.0])

    def solve(c):
        w, F, log = M.Mixed(c, [(1, 1), (2, 2)], precond="scaled", device="cuda").solve(Fb, rtol=1e-9, cg_tol=1e-8)
        torch.cuda.current_stream().synchronize()
        return w.cpu().numpy(), F, log["newton"], log["cg"]

    seq = [solve(M.Cell(r, emin=1e-6)) for r in rhos]
    cells = [M.Cell(r, emin=1e-6) for r in rhos]
    par = [None] * len(cells)

    def run(i):
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            cells[i].stream = s.cuda_stream
            par[i] = solve(cells[i])

    th = [threading.Thread(target=run, args=(i,)) for i in range(len(cells))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for a, b in zip(seq, par):
        assert b is not None
        assert a[2] == b[2] and a[3] == b[3]
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


def test_small_strain_limit_is_linear_C(M):
    from nlfiber_b200 import linear as L
    rho = OD.grey_cell(3, beta=3.0)
    c = M.Cell(rho)
    C, _, _ = L.LinearHomogenization(rho.shape, emin=c.emin, tol=1e-12).C_full(rho)
    e = 1e-4
    w, F, log = M.Mixed(c, free=[]).solve(np.diag([1 + e, 1.0, 1.0]), rtol=1e-10, cg_tol=1e-10)
    assert log["converged"]
    P = c.mean_stress(w, F)
    np.testing.assert_allclose([P[0, 0], P[1, 1], P[2, 2]], C[:3, 0] * e, rtol=2e-3)


@pytest.mark.parametrize("material,wls", [("neohooke", (500.0, 0.01)), ("neohooke", None), ("linear", None)])
def test_toec_matches_oracle(M, material, wls):
    """nlf_mech_toec (nlfiber/mech.py:458-493) against the oracle's closed forms (pinned by finite differences in
    test_mech_oracle.py), with the linear correctors of the cell; C from the TOEC path equals the linear C^H of the
    same cell (the small-strain limit the reference builds in). Tolerance 1e-11: summation order only."""
    from oracle import linear_ref as OL
    rho = OD.random_cell(3, n_o=4)[0]
    cell, ocell = M.Cell(rho, material=material, wls=wls, emin=1e-3), OM.Cell(rho, material=material, wls=wls,
                                                                              emin=1e-3)
    lh = OL.LinearHomogenization(rho.shape, emin=1e-3, tol=1e-12, maxit=20000)
    Clin, u, _ = lh.C_full(rho)
    C, T = M.toec(cell, u)
    Co, To = OM.toec(ocell, u)
    assert rel(C, Co) < 1e-11
    assert rel(T, To) < 1e-11
    assert rel(C, Clin) < 1e-9
    chi = 0.05 * np.random.default_rng(1).standard_normal(u.shape)
    C2, T2 = M.toec(cell, chi)
    C2o, T2o = OM.toec(ocell, chi)
    assert rel(C2, C2o) < 1e-11 and rel(T2, T2o) < 1e-11
    cub = M.cubic_toec(T)
    assert set(cub) == {"C111", "C112", "C123", "C144", "C155", "C456"}


@pytest.mark.parametrize("n_o", [2, 4])
def test_stability_matches_oracle(M, n_o):
    """nlfiber/mech.py:363-455 on the GPU matvec: the probed Hessian diagonal, LOBPCG's lowest eigenvalues of the
    scaled Hessian at a deformed equilibrium, the effective tangent (9 CG solves) and its rank-one minimum,
    against the oracle's restatements (pinned in test_mech_oracle.py) at the same state."""
    import warnings
    rho = OD.random_cell(4, n_o=n_o)[0]
    cell, ocell = M.Cell(rho, emin=1e-3), OM.Cell(rho, emin=1e-3)
    ofull = OM.Mixed(ocell, free=[])
    w, F, log = ofull.solve(np.diag([1.03, 1.0, 1.0]), rtol=1e-12, cg_tol=1e-12)
    assert log["converged"]
    A = M.effective_tangent(cell, w, F, cg_tol=1e-13)
    Ao = OM.effective_tangent(ocell, w, F, cg_tol=1e-13)
    assert rel(A, Ao) < 1e-9
    v, n = M.rank_one_min(A)
    vo, no = OM.rank_one_min(Ao)
    assert abs(v - vo) <= 1e-9 * abs(vo)
    mix, omix = M.Mixed(cell), OM.Mixed(ocell)
    assert rel(mix._diag_scale(), OM.diag_scale(omix)) < 1e-12
    z = omix.z0(F)
    z[: omix.nw] = w.ravel()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        vals, vecs, it = mix.lowest_eigs(z, F, k=4, tol=1e-8)
        ovals, _, _ = OM.lowest_eigs(omix, z, F, k=4, tol=1e-8)
    np.testing.assert_allclose(vals, ovals, rtol=1e-6)
    assert vecs.shape == (omix.nw + omix.k, 4)
    # the device-resident LOBPCG (state, blocks and matvecs on the GPU)
    import torch
    dmix = M.Mixed(cell, device="cuda")
    # (a residual of 1e-8 is below this operator's rounding floor, where scipy's LOBPCG stops at maxiter too; at
    # 1e-6 the triply degenerate lowest cluster of these cubic cells is pinned to ~1e-6 relative)
    dvals, dvecs, dit = dmix.lowest_eigs(torch.as_tensor(z, device="cuda"), F, k=4, tol=1e-6)
    np.testing.assert_allclose(dvals, ovals, rtol=1e-5)
    assert dit < 2000 and dvecs.shape == (omix.nw + omix.k, 4)
