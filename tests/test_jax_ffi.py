"""The XLA FFI custom call of the corrector solve (nlfiber_b200.jax_ffi, csrc/jax/nlf_jax_ffi.cc).

Where JAX and the built target are absent (this build environment has no jaxlib), the module reports itself
unavailable and refuses to register; where they exist, the custom call inside jax.jit gives the same correctors
as the ctypes path."""
import numpy as np
import pytest


def test_unavailable_without_jax_or_target_refuses_cleanly():
    from nlfiber_b200 import jax_ffi
    if jax_ffi.available():
        pytest.skip("JAX and the FFI target are present; covered by the GPU test")
    with pytest.raises(RuntimeError, match="XLA FFI target needs JAX"):
        jax_ffi.register()


@pytest.mark.gpu
def test_custom_call_matches_ctypes_solve():
    from nlfiber_b200 import jax_ffi
    if not jax_ffi.available():
        pytest.skip("JAX or lib/libnlf_jax.so not present on this machine")
    import jax
    jax.config.update("jax_enable_x64", True)
    from nlfiber_b200 import linear as L
    from oracle import density_ref as OD
    rho = OD.grey_cell(4)
    lh = L.LinearHomogenization(rho.shape, tol=1e-10)
    s = lh.stiffness_scale(rho)
    Es = np.eye(6)[[0, 3]]
    u_ref, it_ref = lh.solve(s, Es)
    f = jax.jit(lambda s_, e_, u_: jax_ffi.linear_solve(s_, e_, u_, tol=1e-10))
    u, it = f(s[None], Es, np.zeros((1, 2) + rho.shape + (3,)))
    assert int(it[0]) == it_ref
    assert np.abs(np.asarray(u)[0] - u_ref).max() <= 1e-12 * np.abs(u_ref).max()
