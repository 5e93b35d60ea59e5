"""ctypes binding of libnlf.so (the C ABI declared in include/nlf.h).

The library is the only compute path: importing this module raises if libnlf.so is missing or cannot be
loaded, and every call that fails on the device raises with the library's own message. There is no CPU
fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("NLF_LIB", os.path.join(os.path.dirname(_HERE), "lib", "libnlf.so"))

NLF_OK, NLF_NOT_CONVERGED, NLF_BREAKDOWN = 0, 1, 2
NLF_EBADARG, NLF_ECUDA, NLF_ETIMEOUT = -1, -2, -3
PREC_FP64, PREC_MIXED = 0, 1
PC_FFT, PC_FFT_SCALED = 0, 1

EXPORTS = (
    "nlf_last_error", "nlf_version", "nlf_default_opts", "nlf_linear_create", "nlf_linear_destroy",
    "nlf_stiffness_scale", "nlf_apply_K", "nlf_load", "nlf_precond", "nlf_linear_solve", "nlf_linear_solve_rhs",
    "nlf_bilinear", "nlf_dC_drho", "nlf_C_full", "nlf_precond_symbol", "nlf_apply_K_ex", "nlf_precond_ex",
    "nlf_profile", "nlf_profile_report", "nlf_profile_name", "nlf_bilinear_noalloc",
    "nlf_mech_create", "nlf_mech_destroy", "nlf_mech_set_rho", "nlf_mech_energy", "nlf_mech_hvp",
    "nlf_mech_precond_w", "nlf_mech_grad_w", "nlf_mech_cg", "nlf_mech_set_precond",
    "nlf_unet_create", "nlf_unet_destroy", "nlf_unet_param_count", "nlf_unet_get_params", "nlf_unet_set_params",
    "nlf_unet_forward", "nlf_unet_backward", "nlf_unet_adam_step",
    "nlf_density_create", "nlf_density_create_d", "nlf_density_destroy", "nlf_density_orbits", "nlf_density_rho", "nlf_density_vjp",
    "nlf_correctors_vjp", "nlf_mech_toec",
    "nlf_apply_variants", "nlf_linear_set_apply_variant", "nlf_linear_get_apply_variant", "nlf_linear_autotune",
    "nlf_linear_set_kinv_mode", "nlf_linear_get_kinv_mode", "nlf_linear_set_fft_twiddles",
    "nlf_linear_get_fft_twiddles",
    "nlf_topo_create", "nlf_topo_destroy", "nlf_topo_label", "nlf_topo_remove_floating", "nlf_topo_select",
    "nlf_topo_binary", "nlf_upsample_sym", "nlf_quantile_linear",
)


class SolveOpts(ctypes.Structure):
    """nlf_solve_opts (include/nlf.h)."""
    _fields_ = [
        ("precision", ctypes.c_int), ("precond", ctypes.c_int), ("tol", ctypes.c_double),
        ("maxit", ctypes.c_int), ("inner_tol", ctypes.c_double), ("inner_maxit", ctypes.c_int),
        ("max_sweeps", ctypes.c_int), ("check_every", ctypes.c_int), ("use_graphs", ctypes.c_int),
        ("slots", ctypes.c_int), ("scale_x0", ctypes.c_int), ("energy_tol", ctypes.c_double),
        ("per_case", ctypes.c_int),
    ]


class NlfError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"libnlf status {status}: {msg}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libnlf.so not found at {LIB_PATH}: build it with `make -C "
                          f"{os.path.dirname(os.path.dirname(LIB_PATH))}` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, D, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, None
    sig = {
        "nlf_last_error": (ctypes.c_char_p, []),
        "nlf_version": (ctypes.c_char_p, []),
        "nlf_default_opts": (V, [P]),
        "nlf_linear_create": (I, [ctypes.POINTER(P), I, I, I, D, D, D, D, D, I]),
        "nlf_linear_destroy": (I, [P]),
        "nlf_stiffness_scale": (I, [P, I, P, P, P]),
        "nlf_apply_K": (I, [P, P, I, P, P, P]),
        "nlf_apply_K_ex": (I, [P, P, I, P, P, I, P]),
        "nlf_precond_ex": (I, [P, I, P, P, I, I, P, P]),
        "nlf_load": (I, [P, P, P, I, P, P]),
        "nlf_precond": (I, [P, I, P, P, P]),
        "nlf_linear_solve": (I, [P, I, P, P, I, P, P, P, P, P]),
        "nlf_linear_solve_rhs": (I, [P, I, P, I, P, P, P, P, P]),
        "nlf_bilinear": (I, [P, I, P, P, I, P, P, P]),
        "nlf_dC_drho": (I, [P, I, P, P, I, P, P, P]),
        "nlf_C_full": (I, [P, I, P, P, P, P, P, P, P, P]),
        "nlf_precond_symbol": (I, [P, P]),
        "nlf_profile": (I, [I]),
        "nlf_profile_report": (I, [P, P, P, I]),
        "nlf_profile_name": (ctypes.c_char_p, [I]),
        "nlf_bilinear_noalloc": (I, [I, I, I, D, D, I, P, P, I, P, P, P]),
        "nlf_mech_create": (I, [ctypes.POINTER(P), I, I, I, D, D, I, D, D, D, D]),
        "nlf_mech_destroy": (I, [P]),
        "nlf_mech_set_rho": (I, [P, P, P, P, P, P]),
        "nlf_mech_energy": (I, [P, P, P, P, P, P, P]),
        "nlf_mech_hvp": (I, [P, P, P, P, P, P, P, P]),
        "nlf_mech_precond_w": (I, [P, P, P, P]),
        "nlf_mech_grad_w": (I, [P, P, P, P]),
        "nlf_mech_cg": (I, [P, P, P, I, P, P, P, D, D, I, P, P, P, P, I, P]),
        "nlf_mech_set_precond": (I, [P, I]),
        "nlf_unet_create": (I, [ctypes.POINTER(P), I, I, I, ctypes.c_ulonglong]),
        "nlf_unet_destroy": (I, [P]),
        "nlf_unet_param_count": (ctypes.c_longlong, [P]),
        "nlf_unet_get_params": (I, [P, P, P]),
        "nlf_unet_set_params": (I, [P, P, P]),
        "nlf_unet_forward": (I, [P, I, I, I, I, P, P, P]),
        "nlf_unet_backward": (I, [P, I, I, I, I, P, P, P, P, P, P]),
        "nlf_unet_adam_step": (I, [P, D, D, D, D, P]),
        "nlf_density_create": (I, [ctypes.POINTER(P), I, D]),
        "nlf_density_create_d": (I, [ctypes.POINTER(P), I, I, D]),
        "nlf_density_destroy": (I, [P]),
        "nlf_density_orbits": (I, [P]),
        "nlf_density_rho": (I, [P, I, P, P, D, P, P, P, P]),
        "nlf_density_vjp": (I, [P, I, I, P, P, D, P, P, P]),
        "nlf_correctors_vjp": (I, [P, I, P, P, P, I, P, P, P, P, P, P, P]),
        "nlf_mech_toec": (I, [P, P, P, P, P]),
        "nlf_apply_variants": (I, [I]),
        "nlf_linear_set_apply_variant": (I, [P, I, I]),
        "nlf_linear_get_apply_variant": (I, [P, I, P, P, P, P]),
        "nlf_linear_autotune": (I, [P, I, I, I, I, P, P]),
        "nlf_linear_set_kinv_mode": (I, [P, I]),
        "nlf_linear_get_kinv_mode": (I, [P]),
        "nlf_linear_set_fft_twiddles": (I, [P, I]),
        "nlf_linear_get_fft_twiddles": (I, [P]),
        "nlf_topo_create": (I, [ctypes.POINTER(P), I, I]),
        "nlf_topo_destroy": (I, [P]),
        "nlf_topo_label": (I, [P, P, I, P, P, P]),
        "nlf_topo_remove_floating": (I, [P, P, P, P, P, P]),
        "nlf_topo_select": (I, [P, P, P, ctypes.c_longlong, P, P]),
        "nlf_topo_binary": (I, [P, P, D, I, P, P, P]),
        "nlf_upsample_sym": (I, [I, I, I, P, P, P]),
        "nlf_quantile_linear": (I, [ctypes.c_longlong, D, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(status, allow_not_converged=True):
    """Raise for errors (status < 0); not-converged and breakdown are returned (the reference returns silently
    with it == maxit, nlfiber/linear.py:188,217)."""
    if status < 0:
        raise NlfError(status, lib.nlf_last_error().decode(errors="replace"))
    if status == NLF_NOT_CONVERGED and not allow_not_converged:
        raise NlfError(status, "not converged")
    return status


def default_opts(**kw):
    o = SolveOpts()
    lib.nlf_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        if v is not None:
            setattr(o, k, v)
    return o


def ptr(a):
    """Address of a C-contiguous float64/int32 NumPy array or of a CUDA torch tensor (device pointer)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):  # torch tensor (device or pinned host)
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


def as_f64(a):
    if hasattr(a, "data_ptr") and not isinstance(a, np.ndarray):
        import torch
        if a.dtype != torch.float64:
            raise TypeError("device tensors must be float64")
        return a.contiguous()
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def profile(on=True):
    """Turn the library's kernel profiler on (and reset it) or off."""
    check(lib.nlf_profile(1 if on else 0))


def profile_report():
    """{kernel class: (total_ms, launches, units)} of the launches recorded since profile(True)."""
    n = 32
    ms = np.zeros(n)
    la = np.zeros(n, dtype=np.int64)
    un = np.zeros(n, dtype=np.uint64)
    k = check(lib.nlf_profile_report(ms.ctypes.data, la.ctypes.data, un.ctypes.data, n))
    return {lib.nlf_profile_name(i).decode(): (float(ms[i]), int(la[i]), int(un[i])) for i in range(k)}
