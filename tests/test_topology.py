"""CPU: the oracle's restatement of the binary map (nlfiber/density.py:96-149, nlfiber/topology.py:8-63) pinned to
the reference's own tests of it (tests/test_core.py:55-75,145-157), and the host half of the GPU binarization:
libnlf.so's numpy-"linear" quantile interpolation (nlf_quantile_linear, a host function) against np.quantile,
the entry points' argument checks (before any CUDA call) and the connectivity structures periodic_label takes."""
import ctypes

import numpy as np

from oracle import density_ref as OD


def test_oracle_binary_volume_after_floating_removal():
    """tests/test_core.py:55-67: the kept solid grows back to v (to one orbit of 48 voxels), nothing floats."""
    kept = 0
    for seed in range(8):
        b = OD.DensityMap(8, 3, r=2.5, v=0.25).binary(OD.random_start(8, seed=seed, kmax=3), up=1)
        if not b.any():
            continue
        kept += 1
        assert abs(b.mean() - 0.25) * b.size <= 48
        lab, n = OD.periodic_label(b)
        assert all(OD._spanning(lab, k) for k in range(1, n + 1))
    assert kept >= 2


def test_oracle_binary_upsampled_volume_and_symmetry():
    """tests/test_core.py:69-74: up = 2 doubles the side, keeps the volume to one orbit and the symmetry exact."""
    b = OD.DensityMap(6, 3, r=1.5, v=0.3).binary(OD.schwarz_p_phi(6), up=2)
    assert b.shape == (24,) * 3
    assert abs(b.mean() - 0.3) < 48.0 / b.size
    assert OD.sym_residual(b.astype(float)) < 1e-14


def test_oracle_components():
    """tests/test_core.py:145-157."""
    b = np.zeros((6, 6, 6), bool)
    b[:, 2, 2] = True
    lab, n = OD.periodic_label(b)
    assert n == 1 and not OD._spanning(lab, 1)
    b[2, :, 2] = b[2, 2, :] = True
    assert OD.remove_floating_pieces(b).sum() == b.sum()
    b2 = b.copy()
    b2[5, 5, 5] = True
    assert OD.remove_floating_pieces(b2).sum() == b.sum()
    # face connectivity splits diagonal neighbours
    c = np.zeros((4, 4), bool)
    c[0, 0] = c[1, 1] = True
    assert OD.periodic_label(c)[1] == 1 and OD.periodic_label(c, faces=True)[1] == 2


def test_oracle_upsample_keeps_linear_fields_periodic_mean():
    """upsample_periodic is an interpolation: a constant stays constant, the mean of a cosine is kept."""
    u = np.full((6, 6, 6), 0.7)
    assert np.allclose(OD.upsample_periodic(u, 2), 0.7)
    x = (np.arange(8) + 0.5) / 8
    f = np.cos(2 * np.pi * x)[:, None] * np.ones((8, 8))
    g = OD.upsample_periodic(f, 3)
    assert g.shape == (24, 24) and abs(g.mean()) < 1e-12


def test_quantile_linear_matches_numpy_bitwise():
    from nlfiber_b200._lib import lib
    rng = np.random.default_rng(0)
    out = ctypes.c_double()
    for t in range(600):
        n = int(rng.integers(1, 400))
        a = rng.standard_normal(n) * 10.0 ** rng.integers(-3, 4)
        if t % 3 == 0:
            a = np.round(a, 1)  # ties
        a = np.sort(a)
        for q in (0.0, 1.0, 0.5, 0.7, 0.75, float(rng.random()), 1.0 - float(rng.random()) * 1e-3):
            assert lib.nlf_quantile_linear(n, q, a.ctypes.data, ctypes.byref(out)) == 0
            assert out.value == np.quantile(a, q), (n, q)


def test_binary_entry_points_reject_bad_arguments_without_a_device():
    """The binary-cell entry points check their arguments before any CUDA call (status -1, message set)."""
    from nlfiber_b200._lib import NLF_EBADARG, lib
    h = ctypes.c_void_p()
    assert lib.nlf_topo_create(ctypes.byref(h), 4, 8) == NLF_EBADARG
    assert lib.nlf_topo_create(ctypes.byref(h), 3, 0) == NLF_EBADARG
    assert lib.nlf_topo_create(ctypes.byref(h), 3, 2048) == NLF_EBADARG  # 2^33 voxels
    assert lib.nlf_topo_create(None, 3, 8) == NLF_EBADARG
    assert b"nlf_topo_create" in lib.nlf_last_error()
    out = ctypes.c_double()
    assert lib.nlf_topo_binary(None, None, 0.3, 1, None, None, None) == NLF_EBADARG
    assert lib.nlf_topo_select(None, None, None, 0, ctypes.byref(out), None) == NLF_EBADARG
    assert lib.nlf_topo_label(None, None, 0, None, None, None) == NLF_EBADARG
    assert lib.nlf_topo_remove_floating(None, None, None, None, None, None) == NLF_EBADARG
    u = np.zeros(8)
    assert lib.nlf_upsample_sym(4, 2, 4, u.ctypes.data, u.ctypes.data, None) == NLF_EBADARG
    assert lib.nlf_upsample_sym(3, 2, 1, u.ctypes.data, u.ctypes.data, None) == NLF_EBADARG
    assert lib.nlf_quantile_linear(0, 0.5, u.ctypes.data, ctypes.byref(out)) == NLF_EBADARG
    assert lib.nlf_quantile_linear(3, float("nan"), u.ctypes.data, ctypes.byref(out)) == NLF_EBADARG


def test_connectivity_structures():
    """nlfiber/topology.py:8 periodic_label(b, connectivity): the full neighbourhood (None or all ones) or the
    face structure; anything else is refused."""
    from scipy import ndimage
    from nlfiber_b200.topology import _structure_faces
    b = np.zeros((4, 4, 4), bool)
    assert _structure_faces(b, None) is False
    assert _structure_faces(b, np.ones((3, 3, 3), bool)) is False
    assert _structure_faces(b, ndimage.generate_binary_structure(3, 1)) is True
    assert _structure_faces(np.zeros((5, 5), bool), ndimage.generate_binary_structure(2, 1)) is True
    try:
        _structure_faces(b, ndimage.generate_binary_structure(3, 2))
    except ValueError:
        pass
    else:
        raise AssertionError("edge connectivity must be refused")


def _bfs_components(b, faces=False):
    """Periodic connected components by breadth-first search on the torus (independent of scipy's labelling and
    of the pad-and-merge construction of nlfiber/topology.py:8-43)."""
    d = b.ndim
    offs = [o for o in np.ndindex(*(3,) * d) if any(x != 1 for x in o)]
    offs = [tuple(x - 1 for x in o) for o in offs]
    if faces:
        offs = [o for o in offs if sum(abs(x) for x in o) == 1]
    lab = np.zeros(b.shape, dtype=np.int64)
    n = 0
    for start in zip(*np.nonzero(b)):
        if lab[start]:
            continue
        n += 1
        lab[start] = n
        queue = [start]
        while queue:
            cur = queue.pop()
            for o in offs:
                nb = tuple((c + x) % s for c, x, s in zip(cur, o, b.shape))
                if b[nb] and not lab[nb]:
                    lab[nb] = n
                    queue.append(nb)
    return lab, n


def test_oracle_labelling_matches_breadth_first_search():
    """The oracle's labelling (the checker of the GPU union-find) gives the components of a breadth-first search
    on the torus, for both connectivities, cubes and squares, odd and tiny sides."""
    rng = np.random.default_rng(11)
    for shape, p in (((6, 6, 6), 0.3), ((5, 7, 4), 0.35), ((2, 2, 2), 0.5), ((9, 9), 0.45), ((3, 11), 0.4)):
        b = rng.random(shape) < p
        for faces in (False, True):
            lab, n = OD.periodic_label(b, faces=faces)
            ref, nr = _bfs_components(b, faces)
            assert n == nr
            pairs = set(zip(lab[b].tolist(), ref[b].tolist()))
            assert len(pairs) == n and len({a for a, _ in pairs}) == n and len({c for _, c in pairs}) == n
