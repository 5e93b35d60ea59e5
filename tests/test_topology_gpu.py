"""GPU: binary cells (libnlf.so nlf_topo_*, nlf_upsample_sym; nlfiber_b200.topology, GpuDensityMap.binary,
Fiber.binary_check) against the oracle's restatement of nlfiber/topology.py:8-63 and nlfiber/density.py:96-149
(oracle/density_ref.py), and the reference's own invariants of the binary map (tests/test_core.py:55-75,
145-157: volume to one symmetry orbit, no floating pieces, exact symmetry; the rod / cross / isolated-voxel
components).

Everything here is integer or order work on the same inputs, so the bar is bitwise: the same components (up to
their numbering), the same kept voxels, the same order statistics, the same upsampled field (numpy's operation
order, no contraction). Where the GPU also computes the smoothed field itself (GpuDensityMap.binary), its u agrees
with the oracle's to ~1e-15, and the binary cells are still equal as long as no two orbits' values are that close
at a threshold; the test asserts equality on these seeds."""
import numpy as np
import pytest

from oracle import density_ref as OD

pytestmark = pytest.mark.gpu


def _cells(d, n):
    from nlfiber_b200.topology import PeriodicCells
    return PeriodicCells(d, n)


def _same_partition(la, lb):
    """True when two labelings (0 = background) group the voxels the same way."""
    if not np.array_equal(la > 0, lb > 0):
        return False
    a, b = la[la > 0], lb[lb > 0]
    pairs = np.unique(np.stack([a, b]), axis=1)
    return len(np.unique(pairs[0])) == pairs.shape[1] == len(np.unique(pairs[1]))


@pytest.mark.parametrize("d,n,p,faces,seed", [
    (3, 6, 0.3, False, 0), (3, 7, 0.25, False, 1), (3, 16, 0.12, False, 2), (3, 16, 0.35, True, 3),
    (3, 33, 0.2, False, 4), (3, 2, 0.5, False, 5), (3, 1, 1.0, False, 6), (2, 9, 0.4, False, 7),
    (2, 32, 0.45, True, 8), (2, 64, 0.3, False, 9), (3, 24, 0.0, False, 10), (3, 12, 1.0, True, 11),
])
def test_periodic_label_matches_oracle(d, n, p, faces, seed):
    b = np.random.default_rng(seed).random((n,) * d) < p
    lab, nc = _cells(d, n).label(b, faces=faces)
    lab_o, nc_o = OD.periodic_label(b, faces=faces)
    assert nc == nc_o
    assert _same_partition(lab, lab_o)
    if nc:
        # numbered 1..n in the order of each component's first voxel
        first = [np.flatnonzero(lab.ravel() == k)[0] for k in range(1, nc + 1)]
        assert first == sorted(first)


def test_reference_components_case():
    """tests/test_core.py:145-157: a rod along x through the periodic boundary is one component that does not
    span; a cross spans all axes and is kept whole; an isolated voxel floats."""
    from nlfiber_b200 import topology as T
    b = np.zeros((6, 6, 6), bool)
    b[:, 2, 2] = True
    lab, n = T.periodic_label(b)
    assert n == 1
    assert T.remove_floating(b).sum() == 0
    b[2, :, 2] = b[2, 2, :] = True
    assert T.remove_floating(b).sum() == b.sum()
    b2 = b.copy()
    b2[5, 5, 5] = True
    kept, nc, ns = _cells(3, 6).remove_floating(b2, counts=True)
    assert (nc, ns) == (2, 1)
    assert np.array_equal(kept, b)


@pytest.mark.parametrize("d,n,p,seed", [
    (3, 8, 0.35, 0), (3, 16, 0.3, 1), (3, 16, 0.18, 2), (3, 31, 0.25, 3), (2, 40, 0.45, 4), (2, 17, 0.55, 5),
])
def test_remove_floating_matches_oracle(d, n, p, seed):
    b = np.random.default_rng(seed).random((n,) * d) < p
    assert np.array_equal(_cells(d, n).remove_floating(b), OD.remove_floating_pieces(b))


def test_remove_floating_in_place_on_device():
    import torch
    b = np.random.default_rng(3).random((20, 20, 20)) < 0.3
    t = torch.as_tensor(b, device="cuda")
    out = _cells(3, 20).remove_floating(t)
    assert out.data_ptr() == t.data_ptr()
    assert np.array_equal(t.cpu().numpy(), OD.remove_floating_pieces(b))


@pytest.mark.parametrize("seed", range(4))
def test_select_order_statistics(seed):
    rng = np.random.default_rng(seed)
    n = 18
    u = rng.standard_normal((n,) * 3)
    if seed % 2:
        u = np.round(u, 1)  # ties
    u.ravel()[:5] = [0.0, -0.0, 1e-300, -1e-300, 0.0]
    mask = rng.random(u.shape) < 0.2 if seed > 1 else None
    vals = np.sort(u.ravel() if mask is None else u[mask])
    c = _cells(3, n)
    for r in sorted({0, 1, len(vals) // 3, len(vals) // 2, len(vals) - 2, len(vals) - 1}):
        assert c.select(u, r, mask) == vals[r]


@pytest.mark.parametrize("d,n_o,f", [(3, 6, 2), (3, 4, 1.5), (3, 6, 1.25), (2, 8, 3), (2, 10, 1.3), (3, 5, 3)])
def test_upsample_sym_bitwise(d, n_o, f):
    """nlfiber/density.py:104,133-149: exact_symmetrize(upsample_periodic(u, f)) of the oracle's smoothed field,
    bit for bit (an odd m = round(n f) loses its last layer in the fold, as the reference's does)."""
    from nlfiber_b200.topology import upsample_sym
    u = OD.DensityMap(n_o, d, r=1.5, v=0.3).smooth(OD.random_start(n_o, d, seed=n_o, kmax=3))
    ref = OD.exact_symmetrize(OD.upsample_periodic(u, f))
    out = upsample_sym(u, f).cpu().numpy()
    assert out.shape == ref.shape
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("d,n_o,r,v,seed,up", [
    (3, 8, 2.5, 0.25, s, 1) for s in range(8)] + [
    (3, 6, 1.5, 0.3, 0, 2), (3, 8, 1.5, 0.35, 3, 1.5), (2, 16, 2.0, 0.3, 1, 1), (2, 12, 1.5, 0.4, 2, 2),
    (3, 16, 1.5, 0.3, 4, 1),
])
def test_binary_from_oracle_field_bitwise(d, n_o, r, v, seed, up):
    """The steps after the smoothing on the oracle's own u: quantile threshold, floating-piece removal and
    regrowth (nlfiber/density.py:105-122) give the oracle's cell exactly."""
    u = OD.DensityMap(n_o, d, r=r, v=v).smooth(OD.random_start(n_o, d, seed=seed, kmax=3))
    if up > 1:
        u = OD.exact_symmetrize(OD.upsample_periodic(u, up))
    ref = OD.binary_from_u(u, v)
    c = _cells(d, u.shape[0])
    assert np.array_equal(c.binary(u, v), ref)
    assert np.array_equal(c.binary(u, v, remove_floating=False), u > np.quantile(u, 1.0 - v))


def test_density_binary_matches_oracle_and_reference_invariants():
    """GpuDensityMap.binary end to end (smoothing on the GPU too) against DensityMap.binary, with the reference's
    own checks (tests/test_core.py:55-75): volume to one orbit of 48 voxels, no floating pieces, symmetric."""
    from nlfiber_b200.density import GpuDensityMap
    from nlfiber_b200 import topology as T
    dm = GpuDensityMap(8, 3, r=2.5, v=0.25)
    dmo = OD.DensityMap(8, 3, r=2.5, v=0.25)
    kept = 0
    for seed in range(8):
        phi = OD.random_start(8, seed=seed, kmax=3)
        b = dm.binary(phi, up=1)
        assert np.array_equal(b, dmo.binary(phi, up=1))
        if not b.any():
            continue
        kept += 1
        assert abs(b.mean() - 0.25) * b.size <= 48
        _, nc, ns = T.cells(3, 16).remove_floating(b, counts=True)
        assert nc == ns
    assert kept >= 2
    phi = OD.schwarz_p_phi(6)
    b = GpuDensityMap(6, 3, r=1.5, v=0.3).binary(phi, up=2)
    assert b.shape == (24,) * 3
    assert abs(b.mean() - 0.3) < 48.0 / b.size
    assert OD.sym_residual(b.astype(float)) == 0.0
    assert np.array_equal(b, OD.DensityMap(6, 3, r=1.5, v=0.3).binary(phi, up=2))
    b2 = GpuDensityMap(12, 2, r=1.5, v=0.35).binary(OD.random_start(12, 2, seed=4, kmax=3), up=1.5)
    assert np.array_equal(b2, OD.DensityMap(12, 2, r=1.5, v=0.35).binary(OD.random_start(12, 2, seed=4, kmax=3),
                                                                       up=1.5))


@pytest.mark.parametrize("full", [False, True])
def test_binary_check_matches_oracle(full):
    """nlfiber/fiber.py:67-81 Fiber.binary_check: the binary cell re-solved; c (and with full, the 6x6 C and its
    cubic leakage) against the oracle's solve of the oracle's binary cell."""
    from nlfiber_b200.fiber import Fiber
    from oracle import linear_ref as OL
    n_o, v = 6, 0.3
    phi = OD.schwarz_p_phi(n_o)
    fib = Fiber(n_o, v=v, r=1.5, emin=1e-3, tol=1e-12, maxit=20000)
    out = fib.binary_check(phi, up=1, full=full)
    b = OD.DensityMap(n_o, 3, r=1.5, v=v).binary(phi)
    assert np.array_equal(out["cell"], b)
    assert out["vol"] == b.mean()
    lh = OL.LinearHomogenization(b.shape, emin=1e-3, tol=1e-12, maxit=20000)
    if full:
        C, _, _ = lh.C_full(b.astype(float))
        np.testing.assert_allclose(out["C"], C, rtol=1e-8, atol=1e-10 * np.abs(C).max())
        from nlfiber_b200.linear import cubic_invariants, cubic_leakage
        np.testing.assert_allclose(out["c"], cubic_invariants(C) / lh.E, rtol=1e-8)
        assert abs(out["leak"] - cubic_leakage(C)) < 1e-7
    else:
        c_o, _, _ = lh.invariants(b.astype(float))
        np.testing.assert_allclose(out["c"], c_o, rtol=1e-8)
    assert fib.solves == 1
