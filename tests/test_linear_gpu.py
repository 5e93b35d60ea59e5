"""Parity of the CUDA small-strain path (libnlf.so through nlfiber_b200.linear) with the NumPy FP64 oracle
(a restatement of nlfiber/linear.py) and the reference's own known-answer tests (tests/test_core.py:78-142 of
the reference). Tolerances are written per test; FP64 operators agree with the oracle to rounding."""
import os

# every solve starts from a NaN-filled workspace, so reads of unwritten values fail the tests
os.environ.setdefault("NLF_POISON_WORKSPACE", "1")

import numpy as np  # noqa: E402
import pytest  # noqa: E402

from oracle import density_ref as OD
from oracle import linear_ref as OL

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "linear_golden.npz")


@pytest.fixture(scope="module")
def L():
    from nlfiber_b200 import linear
    return linear


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


SHAPES = [(8, 8, 8), (6, 6, 6), (4, 8, 16), (12, 10, 6), (16, 16, 16), (32, 32, 32), (8, 8, 1), (5, 7, 3)]


@pytest.mark.parametrize("shape", SHAPES)
def test_apply_load_precond_symbol(L, shape):
    rng = np.random.default_rng(1)
    s = 1e-3 + rng.random(shape)
    u = rng.standard_normal((3,) + shape + (3,))
    lh, oh = L.LinearHomogenization(shape), OL.LinearHomogenization(shape)
    assert rel(lh.apply_K(s, u), np.stack([oh.apply_K(s, x) for x in u])) < 1e-13
    Es = rng.standard_normal((4, 6))
    assert rel(lh.load(s, Es), oh.load(s, Es)) < 1e-13
    assert rel(lh.Kinv, oh.Kinv) < 1e-12
    assert rel(lh.precond(u), oh.precond(u)) < 1e-12


# the scaled preconditioner wraps the FFT inverse of a reference medium with Poisson ratio 0 (E does not matter)
SCALED_REF_NU = 0.0


def _scaled_oracle(oh, s, r):
    sn = np.sqrt(sum(np.roll(s, shift=tuple(off), axis=(0, 1, 2)) ** 2 for off in OL.NODES) / 8.0)
    w = (sn ** -0.47)[..., None]
    ref = OL.LinearHomogenization(oh.shape, E=oh.E, nu=SCALED_REF_NU)
    return w * ref.precond(w * r)


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 16, 16), (32, 32, 32), (64, 64, 64), (6, 6, 6), (8, 8, 1)])
def test_fp32_and_scaled_operators(L, shape):
    """The FP32 operators of the mixed-precision solver agree with the FP64 oracle to FP32 rounding
    (rel 2e-6); the FP64 scaled preconditioner to FP64 rounding."""
    rng = np.random.default_rng(2)
    s = 1e-3 + rng.random(shape)
    u = rng.standard_normal((2,) + shape + (3,))
    lh, oh = L.LinearHomogenization(shape), OL.LinearHomogenization(shape)
    Ku = np.stack([oh.apply_K(s, x) for x in u])
    assert rel(lh.apply_K(s, u, precision="mixed"), Ku) < 2e-6
    assert rel(lh.precond(u, precision="mixed"), oh.precond(u)) < 2e-6
    zs = _scaled_oracle(oh, s, u)
    assert rel(lh.precond(u, precond="scaled", s=s), zs) < 1e-12
    assert rel(lh.precond(u, precision="mixed", precond="scaled", s=s), zs) < 2e-6


def test_mixed_low_contrast_matches_fp64(L):
    rho = OD.grey_cell(4)
    lh = L.LinearHomogenization(rho.shape, tol=1e-10)
    C, _, it = lh.C_full(rho)
    Cm, _, itm = lh.C_full(rho, precision="mixed")
    assert rel(Cm, C) < 1e-9, (rel(Cm, C), itm)


def test_fp64_pcg_trajectory_matches_oracle(L):
    """Same algorithm, same iterates: 25 iterations with tol = 0 agree to rounding."""
    rho = OD.grey_cell(4)
    lh = L.LinearHomogenization(rho.shape, tol=0.0, maxit=25)
    oh = OL.LinearHomogenization(rho.shape, tol=0.0, maxit=25)
    s = oh.stiffness_scale(rho)
    Es = np.eye(6)[[0, 3]]
    u, it = lh.solve(s, Es)
    uo, ito = oh.solve(s, Es)
    assert it == ito == 25
    assert rel(u, uo) < 1e-9


def test_C_full_and_dC_match_oracle(L):
    rho = OD.grey_cell(4)
    lh, oh = L.LinearHomogenization(rho.shape), OL.LinearHomogenization(rho.shape)
    C, u, it = lh.C_full(rho)
    Co, uo, ito = oh.C_full(rho)
    assert abs(it - ito) <= 1
    assert rel(C, Co) < 1e-10
    assert rel(u, uo) < 1e-6
    dC = lh.dC_drho(rho, np.eye(6), u)
    dCo = oh.dC_drho(rho, np.eye(6), u)
    assert rel(dC, dCo) < 1e-12
    assert rel(lh.bilinear(oh.stiffness_scale(rho), np.eye(6), u), oh.bilinear(oh.stiffness_scale(rho), np.eye(6), u)) < 1e-13


def test_golden_fixtures(L):
    g = np.load(GOLDEN)
    rho = g["grey8_rho"]
    C, _, it = L.LinearHomogenization(rho.shape).C_full(rho)
    assert rel(C, g["grey8_C"]) < 1e-10
    assert abs(it - int(g["grey8_it"])) <= 1
    rho2 = g["plane8_rho"]
    c2, _, _ = L.LinearHomogenization(rho2.shape).invariants(rho2)
    assert rel(c2, g["plane8_c"]) < 1e-9


def test_uniform_solid_is_isotropic_material(L):
    """tests/test_core.py:88-91 of the reference."""
    C, _, _ = L.LinearHomogenization((4, 4, 4), E=2.0, nu=0.25).C_full(np.ones((4, 4, 4)))
    np.testing.assert_allclose(C, L.iso_D(2.0, 0.25), atol=1e-10)


def test_full_vs_cubic_path_and_symmetry(L):
    """tests/test_core.py:78-86 of the reference."""
    rho = OD.grey_cell(4)
    lh = L.LinearHomogenization(rho.shape)
    C, _, _ = lh.C_full(rho)
    np.testing.assert_allclose(C, C.T, atol=1e-12)
    assert L.cubic_leakage(C) < 1e-8
    c, _, _ = lh.invariants(rho)
    np.testing.assert_allclose(c, L.cubic_invariants(C), rtol=1e-8)


def test_plane_strain_equals_extruded_3d(L):
    """tests/test_core.py:93-99 of the reference."""
    rho2 = OD.grey_cell(4, d=2)
    c2, _, _ = L.LinearHomogenization(rho2.shape).invariants(rho2)
    rho3 = np.repeat(rho2[..., None], 3, axis=2)
    C3, _, _ = L.LinearHomogenization(rho3.shape).C_full(rho3)
    np.testing.assert_allclose(c2, [C3[0, 0], C3[1, 0], C3[5, 5]], rtol=1e-8)


def test_hashin_shtrikman_bounds_cell(L):
    """tests/test_core.py:135-142 of the reference."""
    rho = OD.binary_cell(6, v=0.3).astype(float)
    C, _, _ = L.LinearHomogenization(rho.shape).C_full(rho)
    c11, c12, c44 = L.cubic_invariants(C)
    K = (c11 + 2 * c12) / 3
    Khs, Ghs = L.hashin_shtrikman(rho.mean())
    assert K < Khs and c44 < Ghs


def test_batched_equals_single_and_deterministic(L):
    cells = np.stack([OD.random_cell(i, n_o=4, beta=8.0)[0] for i in range(3)])
    lh = L.LinearHomogenization(cells.shape[1:])
    r = lh.C_full_batched(cells, want_u=True)
    r2 = lh.C_full_batched(cells, want_u=True)
    assert np.array_equal(r["C"], r2["C"]) and np.array_equal(r["u"], r2["u"])
    for i in range(3):
        C, u, it = lh.C_full(cells[i])
        assert np.array_equal(C, r["C"][i]) and it == r["it"][i]


def test_slot_refill_and_graphs_equal_lock_step(L):
    """Five 32^3 cells through two slots (a converged cell hands its slot to the next one), with the iterations
    replayed from a CUDA graph, give bit for bit the lock-step batch's u, C and iteration counts; the status
    says converged, and a cap below the needed iterations says not converged (status 1)."""
    cells = np.stack([OD.random_cell(i, n_o=16, beta=8.0)[0] for i in range(5)])
    lock = L.LinearHomogenization(cells.shape[1:], precond="scaled", tol=1e-8, maxit=2000, check_every=4)
    slot = L.LinearHomogenization(cells.shape[1:], precond="scaled", tol=1e-8, maxit=2000, check_every=4,
                                  slots=2, use_graphs=True)
    a = lock.C_full_batched(cells, want_u=True)
    b = slot.C_full_batched(cells, want_u=True)
    assert a["status"] == 0 and b["status"] == 0
    assert np.array_equal(a["it"], b["it"]), (a["it"], b["it"])
    assert np.array_equal(a["u"], b["u"]) and np.array_equal(a["C"], b["C"])
    assert len(set(a["it"].tolist())) > 1  # the cells really stop at different iterations
    short = slot.C_full_batched(cells, maxit=int(a["it"].min()) - 1)
    assert short["status"] == 1 and np.all(short["it"] == a["it"].min() - 1)


def test_energy_guard_and_warm_start_plumbing(L):
    """The energy guard never stops a cell earlier than the residual rule and keeps C within 1e-8 of a long run;
    a warm start from the converged correctors needs (almost) no iteration, and the energy-optimal scaling
    recovers an exact multiple of them at once."""
    cells = np.stack([OD.random_cell(i, n_o=8, beta=16.0)[0] for i in range(6)])
    kw = dict(emin=1e-9, precond="scaled", maxit=4000, check_every=4)
    star = L.LinearHomogenization(cells.shape[1:], tol=1e-14, **kw).C_full_batched(cells)["C"]
    res = L.LinearHomogenization(cells.shape[1:], tol=1e-9, **kw).C_full_batched(cells, want_u=True)
    grd = L.LinearHomogenization(cells.shape[1:], tol=1e-9, energy_tol=1e-10, **kw).C_full_batched(cells)
    assert res["status"] == 0 and grd["status"] == 0
    assert np.all(grd["it"] >= res["it"]), (grd["it"], res["it"])
    assert max(rel(grd["C"][i], star[i]) for i in range(len(cells))) < 1e-8
    ws = L.LinearHomogenization(cells.shape[1:], tol=1e-9, **kw)
    assert np.all(ws.C_full_batched(cells, u0=res["u"])["it"] <= 4)
    sc = L.LinearHomogenization(cells.shape[1:], tol=1e-9, scale_x0=True, **kw)
    half = sc.C_full_batched(cells, u0=0.5 * res["u"])
    assert np.all(half["it"] <= 4), half["it"]


def test_uneven_batch_equals_per_size_batches(L):
    """Cells of two grid sizes in one call (one handle per size, run concurrently on their own streams) give the
    per-size batches' C and iterations bit for bit, in the input order."""
    import torch
    a = [OD.random_cell(i, n_o=4, beta=8.0)[0] for i in range(3)]
    b = [OD.random_cell(10 + i, n_o=8, beta=8.0)[0] for i in range(2)]
    cells = [torch.tensor(c, device="cuda") for c in (a[0], b[0], a[1], b[1], a[2])]
    kw = dict(precond="scaled", tol=1e-9, maxit=2000, check_every=4)
    r = L.C_full_uneven(cells, concurrent=True, **kw)
    ra = L.LinearHomogenization(a[0].shape, **kw).C_full_batched(np.stack(a))
    rb = L.LinearHomogenization(b[0].shape, **kw).C_full_batched(np.stack(b))
    assert r["status"] == 0
    assert np.array_equal(r["C"][[0, 2, 4]], ra["C"]) and np.array_equal(r["C"][[1, 3]], rb["C"])
    assert np.array_equal(r["it"][[0, 2, 4]], ra["it"]) and np.array_equal(r["it"][[1, 3]], rb["it"])


def test_high_contrast_variants_reach_the_fp64_C(L):
    """emin = 1e-9 Schwarz-P 16^3: the scaled preconditioner (FP64 and FP32-in-FP64 refinement) and the
    reference preconditioner (long run) reach the same C; every entry within 1e-8 of max |C|."""
    rho = OD.schwarz_p_cell(8)
    lh = L.LinearHomogenization(rho.shape, emin=1e-9, tol=1e-11, maxit=4000)
    Cs, _, its = lh.C_full(rho, precond="scaled")
    Cm, _, itm = lh.C_full(rho, precond="scaled", precision="mixed")
    Cr, _, itr = lh.C_full(rho, tol=0.0, maxit=4000)
    assert rel(Cm, Cs) < 1e-8, (rel(Cm, Cs), itm)
    assert rel(Cr, Cs) < 1e-8, (rel(Cr, Cs), itr)
    assert its < 200 and itm < 400


def test_not_converged_is_silent_and_bad_args_raise(L):
    rho = OD.grey_cell(4)
    lh = L.LinearHomogenization(rho.shape, maxit=3)
    _, _, it = lh.C_full(rho)
    assert it == 3
    from nlfiber_b200 import _lib
    with pytest.raises(_lib.NlfError):
        L.LinearHomogenization((0, 4, 4))


@pytest.mark.parametrize("shape", [(6, 6, 6), (32, 32, 32)])
def test_correctors_vjp_matches_oracle(L, shape):
    """nlf_correctors_vjp (the backward of nlfiber/linear.py:118-134's custom VJP: K lam = -proj(ubar), then the VJP
    of the residual in s) against the oracle's restatement (pinned by finite differences in test_oracle.py), on a
    grid with the generic FFT passes and one with the register-resident ones; with s, and with rho (cotangent of
    rho through the stiffness scale). Both solves to a 1e-12 relative residual; tolerance 1e-8 of the largest
    entry."""
    rng = np.random.default_rng(shape[0])
    n = shape[0]
    rho = OD.random_cell(2, n_o=n // 2)[0]
    lh = L.LinearHomogenization(shape, emin=1e-3, tol=1e-12, maxit=20000)
    oh = OL.LinearHomogenization(shape, emin=1e-3, tol=1e-12, maxit=20000)
    s = oh.stiffness_scale(rho)
    Es = np.stack([OL.unit_strain(0), OL.unit_strain(3), OL.unit_strain(5)])
    u, _ = oh.solve(s, Es)
    ubar = rng.standard_normal(u.shape)
    sb_o, lam_o = oh.correctors_vjp(s, Es, u, ubar)
    sb, lam, it = lh.correctors_vjp(s, Es, u, ubar)
    assert it > 0
    assert np.abs(sb - sb_o).max() <= 1e-8 * np.abs(sb_o).max()
    assert np.abs(lam - lam_o).max() <= 1e-8 * np.abs(lam_o).max()
    rb, _, _ = lh.correctors_vjp(None, Es, u, ubar, rho=rho)
    rb_o = sb_o * oh.dscale_drho(rho)
    assert np.abs(rb - rb_o).max() <= 1e-8 * np.abs(rb_o).max()


def test_apply_tile_variants_and_autotune(L):
    """Every tile variant of the stiffness apply gives the oracle's K(s) u to rounding (FP64 1e-13, FP32 2e-6),
    on a grid that is not a multiple of the tiles; the autotuner keeps one of them and reports a time for each."""
    from nlfiber_b200 import _lib
    shape = (20, 24, 36)
    rng = np.random.default_rng(5)
    s = 1e-9 + rng.random(shape) ** 3
    u = rng.standard_normal((2,) + shape + (3,))
    lh, oh = L.LinearHomogenization(shape), OL.LinearHomogenization(shape)
    Ku = np.stack([oh.apply_K(s, x) for x in u])
    for prec, tol in (("fp64", 1e-13), ("mixed", 2e-6)):
        for v in range(_lib.lib.nlf_apply_variants(_lib.PREC_FP64 if prec == "fp64" else _lib.PREC_MIXED)):
            lh.set_apply_tile(v, prec)
            assert lh.apply_tile(prec)[0] == v
            assert rel(lh.apply_K(s, u, precision=prec), Ku) < tol, (prec, lh.apply_tile(prec))
    times = lh.autotune(nvec=4, reps=2, report=True)
    v = lh.apply_tile("fp64")[0]
    nv = _lib.lib.nlf_apply_variants(_lib.PREC_FP64)
    ta = times["fp64"][:nv]  # then the preconditioner's two Kinv modes, timed on cubes of 32 and 64 only
    assert len(times["fp64"]) == nv + 12 and min(ta) > 0 and times["fp64"][nv:] == [0.0] * 12
    assert ta[v] == min(ta)


@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 64, 64)])
def test_preconditioner_kinv_closed_form(L, shape):
    """The register-resident preconditioner with its Kinv entries in closed form (kinv_mode 1) equals the oracle's
    table-based inverse symbol (nlfiber/linear.py:154-170) to FP64 rounding, unscaled and scaled."""
    rng = np.random.default_rng(3)
    s = 1e-9 + rng.random(shape) ** 3
    u = rng.standard_normal((2,) + shape + (3,))
    lh, oh = L.LinearHomogenization(shape), OL.LinearHomogenization(shape)
    for mode in ((1, 2) if shape[0] == 64 else (1,)):
        lh.kinv_mode = mode
        assert lh.kinv_mode == mode
        assert rel(lh.precond(u), oh.precond(u)) < 1e-12
        assert rel(lh.precond(u, precond="scaled", s=s), _scaled_oracle(oh, s, u)) < 1e-12
    lh.kinv_mode = 0
    assert rel(lh.precond(u, precond="scaled", s=s), _scaled_oracle(oh, s, u)) < 1e-12
    for mode in (1, 2, 3):  # passes A and C with shared-memory twiddles, and with staged spectrum rows
        lh.fft_twiddles = mode
        assert lh.fft_twiddles == mode
        assert rel(lh.precond(u), oh.precond(u)) < 1e-12
        assert rel(lh.precond(u, precond="scaled", s=s), _scaled_oracle(oh, s, u)) < 1e-12
