"""Python binding of the B200 FFT library (libaoclfftz_gpu.so).

The product is the C ABI in include/aoclfftz.h; this package only loads the
shared object and mirrors the ABI with ctypes for Python callers, tests and
benchmarks. There is no Python or CPU fallback: if the library is missing,
load() raises.
"""
import ctypes
import os

from . import abi, synthetic  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(os.path.dirname(_HERE))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libaoclfftz_gpu.so")
_lib = None


def load(path=None):
    """Loads and binds libaoclfftz_gpu.so (built by `make -C aocl-fftz_b200`)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libaoclfftz_gpu.so not built: %s (run make -C aocl-fftz_b200)" % p)
    lib = abi.bind_gpu(ctypes.CDLL(p))
    if path is None:
        _lib = lib
    return lib
