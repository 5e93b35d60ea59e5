"""CPU tests of the package's device-agnostic host logic (no GPU, no compute call into libnlf.so): the LOBPCG of
`Mixed.lowest_eigs` on the device (`lobpcg_device`, torch code that runs on any device), the rank-one
ellipticity minimum and the cubic TOEC map, each against an independent computation; and the bench's host-side
pieces: the per-entry C errors and the CPU arm (the oracle on all host cores)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def M():
    from nlfiber_b200 import mech
    return mech


def _dense_spd(n, seed):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n))
    return B @ B.T / n + np.diag(np.linspace(0.01, 5.0, n))


@pytest.mark.parametrize("constrained", [False, True])
def test_lobpcg_device_matches_dense_eigensolve(M, constrained):
    """Knyazev's LOBPCG restated in torch: the lowest 4 eigenvalues of a dense SPD operator (on CPU tensors), with
    and without a 3-column constraint space, against numpy's eigh of the operator restricted to the complement."""
    import torch
    n = 240
    A = _dense_spd(n, 0)
    At = torch.as_tensor(A)
    rng = np.random.default_rng(1)
    Y = None
    Q = np.eye(n)
    if constrained:
        Yn, _ = np.linalg.qr(rng.standard_normal((n, 3)))
        Y = torch.as_tensor(Yn)
        Qf, _ = np.linalg.qr(np.concatenate([Yn, rng.standard_normal((n, n - 3))], axis=1))
        Q = Qf[:, 3:]
    vals, vecs, it = M.lobpcg_device(lambda V: At @ V, torch.as_tensor(rng.standard_normal((n, 4))), Y, 1e-9, 1000)
    ref = np.linalg.eigvalsh(Q.T @ A @ Q)[:4]
    np.testing.assert_allclose(vals, ref, rtol=1e-10)
    assert it < 1000
    V = vecs.numpy()
    AV = A @ V
    if constrained:  # eigenpairs of the operator restricted to the complement of Y: P A V = V diag(vals)
        Yn = Y.numpy()
        AV = AV - Yn @ (Yn.T @ AV)
        assert np.abs(Yn.T @ V).max() < 1e-12
    np.testing.assert_allclose(AV, V * vals[None, :], atol=1e-8)


def test_rank_one_min_isotropic_and_plane(M):
    """For isotropic linear elasticity every direction's acoustic tensor has smallest eigenvalue mu; the 2D
    variant searches the x-y plane only."""
    from nlfiber_b200.linear import lame
    lam, mu = lame(1.0, 0.3)
    d = np.eye(3)
    A = lam * np.einsum("ij,kl->ijkl", d, d) + mu * (np.einsum("ik,jl->ijkl", d, d) + np.einsum("il,jk->ijkl", d, d))
    for plane in (False, True):
        v, n = M.rank_one_min(A, m=300, plane=plane)
        assert abs(v - mu) < 1e-12 and abs(np.linalg.norm(n) - 1.0) < 1e-12
        if plane:
            assert n[2] == 0.0
    pts = M.fibonacci_sphere(500)
    np.testing.assert_allclose(np.linalg.norm(pts, axis=1), 1.0, atol=1e-14)
    assert np.abs(pts.mean(axis=0)).max() < 1e-2


def test_cubic_toec_means_over_equivalent_entries(M):
    """cubic_toec averages each cubic constant over its equivalent Voigt index triples (nlfiber/mech.py:496-515);
    a T built from known cubic values returns them."""
    vals = {"C111": -3.0, "C112": -1.0, "C123": 0.2, "C144": -0.1, "C155": -0.5, "C456": 0.05}
    T = np.zeros((6, 6, 6))
    for k, idx in M.CUBIC_TOEC.items():
        for t in idx:
            T[t] = vals[k]
    out = M.cubic_toec(T)
    assert out == pytest.approx(vals, abs=1e-15)


def test_bench_entry_errors_are_per_cell_normalised_maxima():
    """bench.entry_errors: each (I, J) error is the max over cells of |dC_IJ| / max |C*| of the cell, so its max
    over entries is the metric's C error (bench.rel_err)."""
    import bench
    rng = np.random.default_rng(0)
    Cs = rng.standard_normal((5, 6, 6)) * np.array([1.0, 10.0, 0.1, 2.0, 5.0])[:, None, None]
    C = Cs + 1e-9 * rng.standard_normal(Cs.shape)
    ent = np.array(bench.entry_errors(C, Cs))
    assert ent.shape == (6, 6)
    ref = np.max(np.abs(C - Cs) / np.abs(Cs).reshape(5, -1).max(1)[:, None, None], axis=0)
    np.testing.assert_allclose(ent, ref, rtol=0, atol=0)
    assert ent.max() == pytest.approx(bench.rel_err(C, Cs).max(), rel=1e-15)


def test_bench_reference_arm_line_on_all_cores():
    """`bench.py --impl reference` (a 16^3 grid here, to keep it short): one JSON line in the driver's contract,
    its CPU sample run as one single-threaded process per host core, `cores` the process count; the solver
    description sits outside `config` (so both arms carry the same config), and the iteration extrapolation and
    the same-algorithm figure are stated."""
    import json
    import subprocess
    import sys

    import bench
    out = subprocess.run([sys.executable, bench.__file__, "--impl", "reference", "--steps", "2", "--warmup", "1",
                          "--n", "16"], capture_output=True, text=True, timeout=600, check=True)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "cells/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"] == bench.workload_config(16, 64, 1) and "solver" in line
    assert line["extrapolation"]["iterations_timed_per_process"] == 2
    assert line["cpu_same_algorithm"]["value"] > line["value"]
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["value"] == line["value"]
    assert cpu["cores"] == min(bench.cpu_processes(16), 64)  # one per core, at most one per cell
    assert cpu["sample"].startswith(f"{cpu['cores']} cells of 16^3 x 6 cases, one per single-threaded process")


def test_bench_reference_arm_loads_no_library():
    """The reference arm runs the oracle only: generating its cells and timing them loads no libnlf.so."""
    import subprocess
    import sys

    import bench
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', "
            "'--n', '16']; runpy.run_path(%r, run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); print('LIBNLF' if 'libnlf' in maps else 'CLEAN')" % bench.__file__)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, check=True)
    assert out.stdout.strip().splitlines()[-1] == "CLEAN"


def test_cpu_reference_parallel_rounds():
    """Two processes, one 16^3 cell each, two rounds (the first also running the node-scaled preconditioner):
    per round one row per process with positive setup and per-iteration times."""
    import bench
    res = bench.cpu_reference_parallel(8, [(1, True), (1, False)], procs=2)
    assert len(res) == 2 and all(len(r) == 2 for r in res)
    for k, rows in enumerate(res):
        for setup, t_ref, t_sc in rows:
            assert setup > 0 and t_ref > 0
            assert (t_sc is not None and t_sc > 0) if k == 0 else t_sc is None
    assert bench.cpu_rate(res[1], 100) > 0


def test_bench_generator_matches_the_oracle_generator():
    """bench.synth_phi / synth_volume draw the seeded pre-densities the oracle's restatement of the reference
    generator draws (nlfiber/fiber.py:103-121): equal to rounding, same volumes."""
    import bench
    from oracle import density_ref as OD
    for seed, n_o in ((0, 8), (5, 16), (12, 32)):
        a, b = bench.synth_phi(seed, n_o), OD.random_start(n_o, 3, seed=seed, kmax=2)
        assert np.abs(a - b).max() < 1e-13
        assert bench.synth_volume(seed) == float(np.random.default_rng(10_000 + seed).uniform(0.2, 0.5))


def _q1_gradients():
    """Shape-function gradients of the unit-cube Q1 element at the 2x2x2 Gauss points, dN[g][a][d] (node
    a = ax + 2 ay + 4 az, Gauss point g likewise; nlfiber/linear.py:22-41), as libnlf.so's finite-strain kernels
    load them."""
    h = 1.0 / (2.0 * np.sqrt(3.0))
    g1 = (0.5 - h, 0.5 + h)
    dN = np.zeros((8, 8, 3))
    for g in range(8):
        x, y, z = g1[g & 1], g1[(g >> 1) & 1], g1[(g >> 2) & 1]
        for a in range(8):
            i, j, k = a & 1, (a >> 1) & 1, (a >> 2) & 1
            fx, fy, fz = (x if i else 1 - x), (y if j else 1 - y), (z if k else 1 - z)
            dN[g, a] = [(1 if i else -1) * fy * fz, fx * (1 if j else -1) * fz, fx * fy * (1 if k else -1)]
    return dN, h


def _butterfly(v, transpose=False):
    """The element's sum/difference butterfly over x, y, z (nlf_element.cuh butterfly8 / butterfly8_t)."""
    v = np.array(v, dtype=np.float64)
    pairs = [[(a, a + 1) for a in range(0, 8, 2)], [((q & 1) + ((q >> 1) << 2), (q & 1) + ((q >> 1) << 2) + 2)
                                                    for q in range(4)], [(a, a + 4) for a in range(4)]]
    for lev in (reversed(pairs) if transpose else pairs):
        for a, b in lev:
            if transpose:
                v[a], v[b] = v[a] - v[b], v[a] + v[b]
            else:
                v[a], v[b] = v[a] + v[b], v[b] - v[a]
    return v


def test_mode_form_gradients_and_forces_of_the_cached_tangent_matvec():
    """The algebra of the finite-strain CG matvec (k_mech_hvp_tc): the direction's gradient at each Gauss point
    from the 7 scaled modes of the butterfly, with the macro direction added to the constant-strain modes, and the
    element forces as signed mode sums then the transposed butterfly, equal the shape-function forms
    dF_g = dFm + sum_a v_a (x) dN[g][a] and f_a = sum_g P_g dN[g][a] to rounding."""
    dN, h = _q1_gradients()
    rng = np.random.default_rng(3)
    vn, dFm, P = rng.standard_normal((3, 8)), rng.standard_normal((3, 3)), rng.standard_normal((8, 3, 3))
    km = np.array([_butterfly(vn[c]) for c in range(3)])
    km[:, 1] = 0.25 * km[:, 1] + dFm[:, 0]
    km[:, 2] = 0.25 * km[:, 2] + dFm[:, 1]
    km[:, 4] = 0.25 * km[:, 4] + dFm[:, 2]
    km[:, [3, 5, 6]] *= 0.5 * h
    km[:, 7] *= h * h
    nm = np.zeros((3, 8))
    for g in range(8):
        sx, sy, sz = (1 if g & 1 else -1), (1 if (g >> 1) & 1 else -1), (1 if g >> 2 else -1)
        dF = np.stack([km[:, 1] + sy * km[:, 3] + sz * km[:, 5] + sy * sz * km[:, 7],
                       km[:, 2] + sx * km[:, 3] + sz * km[:, 6] + sx * sz * km[:, 7],
                       km[:, 4] + sx * km[:, 5] + sy * km[:, 6] + sx * sy * km[:, 7]], axis=1)
        np.testing.assert_allclose(dF, dFm + vn @ dN[g], atol=1e-14)
        px, py, pz = P[g][:, 0], P[g][:, 1], P[g][:, 2]
        nm[:, 1] += px
        nm[:, 2] += py
        nm[:, 4] += pz
        nm[:, 3] += sy * px + sx * py
        nm[:, 5] += sz * px + sx * pz
        nm[:, 6] += sz * py + sy * pz
        nm[:, 7] += sy * sz * px + sx * sz * py + sx * sy * pz
    nm[:, [1, 2, 4]] *= 0.25
    nm[:, [3, 5, 6]] *= 0.5 * h
    nm[:, 7] *= h * h
    f = np.array([_butterfly(nm[c], transpose=True) for c in range(3)])
    np.testing.assert_allclose(f, np.einsum("gcd,gad->ca", P, dN), atol=1e-14)
