"""CPU tests of the C ABI boundary: libnlf.so loads and exports every entry point declared in include/*.h.
No compute call is made (there may be no GPU)."""
import ctypes
import glob
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"NLF_API\s+[\w\s\*]+?\b(nlf_\w+)\s*\(", src))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    from nlfiber_b200 import _lib
    syms = declared_symbols()
    assert len(syms) >= 15
    for name in syms:
        assert hasattr(_lib.lib, name), name
    assert set(_lib.EXPORTS) <= syms


def test_default_opts_and_version_need_no_device():
    from nlfiber_b200 import _lib
    o = _lib.default_opts()
    assert o.precision == _lib.PREC_FP64 and o.precond == _lib.PC_FFT and o.tol < 0 and o.maxit < 0
    assert b"sm_100a" in _lib.lib.nlf_version()


def test_library_is_a_plain_c_abi():
    """The exported names are unmangled C symbols (a ctypes / cgo / JNI binding can bind them by name)."""
    from nlfiber_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared_symbols():
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value
