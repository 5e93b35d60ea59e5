"""GPU: the C assembly entry point that allocates nothing (nlf_bilinear_noalloc) gives the same C as the
regular entry point (nlf_bilinear), on two calls in a row through the C ABI.

The no-allocation variant exists for callers that may not call cudaMalloc while they run (a handler inside a
framework that owns all device memory, code inside another library's callback, a service with pre-reserved
memory). They pass device arrays; the variant keeps its partial sums in a fixed device array shared by all
calls. Two calls in a row check that the second call does not see the first call's leftovers: the first is the
larger one (5 cells of 16^3, 6 cases), so it fills partial-sum slots with nonzero values that the second, smaller
call (2 cells of 8^3, 4 cases) reads again after writing its own. This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from oracle import density_ref as OD

pytestmark = pytest.mark.gpu


def _case(seed, shape, m, ncell):
    rng = np.random.default_rng(seed)
    rho = np.stack([OD.random_cell(seed + i, n_o=shape[0] // 2, beta=8.0)[0] for i in range(ncell)])
    s = 1e-3 + (1 - 1e-3) * np.clip(rho, 0, 1) ** 3
    u = rng.standard_normal((ncell, m) + shape + (3,)) * 0.1
    Es = rng.standard_normal((m, 6))
    return s, Es, u


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    from nlfiber_b200 import _lib
    from nlfiber_b200 import linear as L

    E, nu = 1.0, 0.3
    for seed, shape, m, ncell in ((11, (16, 16, 16), 6, 5), (23, (8, 8, 8), 4, 2)):
        lh = L.LinearHomogenization(shape, E=E, nu=nu)
        s, Es, u = _case(seed, shape, m, ncell)
        C_ref = np.stack([lh.bilinear(s[i], Es, u[i]) for i in range(ncell)])  # nlf_bilinear
        s_d = torch.from_numpy(s).cuda()
        u_d = torch.from_numpy(u).cuda()
        C_d = torch.full((ncell, m, m), float("nan"), dtype=torch.float64, device="cuda")
        Es_h = np.ascontiguousarray(Es)
        st = _lib.lib.nlf_bilinear_noalloc(*shape, E, nu, ncell, s_d.data_ptr(), Es_h.ctypes.data, m,
                                           u_d.data_ptr(), C_d.data_ptr(), None)
        assert st == 0, _lib.lib.nlf_last_error()
        torch.cuda.synchronize()
        C = C_d.cpu().numpy()
        assert np.abs(C - C_ref).max() < 1e-13 * np.abs(C_ref).max()


def test_noalloc_rejects_oversize_and_host_arrays():
    import torch
    from nlfiber_b200 import _lib

    s = torch.ones((65, 4, 4, 4), dtype=torch.float64, device="cuda")
    u = torch.zeros((65, 1, 4, 4, 4, 3), dtype=torch.float64, device="cuda")
    C = torch.zeros((65, 1, 1), dtype=torch.float64, device="cuda")
    Es = np.eye(6)[:1].copy()
    st = _lib.lib.nlf_bilinear_noalloc(4, 4, 4, 1.0, 0.3, 65, s.data_ptr(), Es.ctypes.data, 1, u.data_ptr(),
                                       C.data_ptr(), None)
    assert st == _lib.NLF_EBADARG and b"at most 64 cells" in _lib.lib.nlf_last_error()
    s_h = np.ones((1, 4, 4, 4))
    st = _lib.lib.nlf_bilinear_noalloc(4, 4, 4, 1.0, 0.3, 1, s_h.ctypes.data, Es.ctypes.data, 1, u.data_ptr(),
                                       C.data_ptr(), None)
    assert st == _lib.NLF_EBADARG and b"device pointers" in _lib.lib.nlf_last_error()
