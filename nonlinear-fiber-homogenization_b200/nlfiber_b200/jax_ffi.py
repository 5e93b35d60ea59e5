"""The corrector solve as an XLA FFI custom call, for callers traced by jax.jit / jax.vjp.

nlfiber's Fiber (nlfiber/fiber.py:27-39) calls LinearHomogenization.invariants inside jax.jit and jax.vjp, with
the solve under stop_gradient (nlfiber/linear.py:259-264). `linear_solve` is that solve as the custom call
"nlf_linear_solve" of lib/libnlf_jax.so (csrc/jax/nlf_jax_ffi.cc), which hands XLA's device buffers to
libnlf.so's C ABI in place: no host round trip, unlike jax.pure_callback.

The target is built by `make -C nonlinear-fiber-homogenization_b200 jax` where jaxlib's FFI headers exist. Without
JAX or without the built target, `available()` is False and `linear_solve` raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
JAX_LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libnlf_jax.so")
_registered = False


def available():
    """JAX is importable and the FFI target has been built."""
    try:
        import jax  # noqa: F401
    except ImportError:
        return False
    return os.path.exists(JAX_LIB_PATH)


def register():
    """Register "nlf_linear_solve" with XLA for the CUDA platform (once per process)."""
    global _registered
    if _registered:
        return
    if not available():
        raise RuntimeError(f"the XLA FFI target needs JAX and {JAX_LIB_PATH} (make -C ... jax)")
    import jax
    lib = ctypes.CDLL(JAX_LIB_PATH)
    jax.ffi.register_ffi_target("nlf_linear_solve", jax.ffi.pycapsule(lib.NlfLinearSolve), platform="CUDA")
    _registered = True


def linear_solve(s, Es, u0, E=1.0, nu=0.3, emin=1e-3, p=3.0, tol=1e-9, maxit=4000, precond="fft", slots=0):
    """nlfiber/linear.py:205-217 solve(s, Es, u0) for a batch of cells inside a JAX trace: s (ncell, nx, ny, nz),
    Es (m, 6), u0 (ncell, m, nx, ny, nz, 3), all float64 on the GPU. Returns (u, iterations per cell). The
    reference wraps its solve in stop_gradient (nlfiber/linear.py:263); so does this (the custom call has no
    derivative rule)."""
    import jax
    import jax.numpy as jnp
    register()
    s, Es, u0 = (jax.lax.stop_gradient(jnp.asarray(a, dtype=jnp.float64)) for a in (s, Es, u0))
    out = (jax.ShapeDtypeStruct(u0.shape, jnp.float64), jax.ShapeDtypeStruct((s.shape[0],), jnp.int32))
    call = jax.ffi.ffi_call("nlf_linear_solve", out, vmap_method="sequential")
    return call(s, Es, u0, E=float(E), nu=float(nu), emin=float(emin), p=float(p), tol=float(tol),
                maxit=int(maxit), precond=1 if precond == "scaled" else 0, slots=int(slots))
