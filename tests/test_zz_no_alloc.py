"""The no-allocation entry point, aoclfftz_gpu_execute_noalloc_c2c_f.

It serves callers that may not allocate device memory when they transform
(another allocator owns the device's memory, or cudaFree's device-wide
synchronisation is too costly in their loop): its scratch is a static device
array instead of plan memory. These tests check it through the C ABI against
the plan-based entry point (aoclfftz_setup_f + aoclfftz_execute) on the same
inputs, within the rel-L2 bound the other tests use, on calls made back to
back so that the shared scratch is reused. The file name sorts last, so a run
that stops at the first failure has run every other test before this one."""
import ctypes as C
import math

import numpy as np
import pytest

import aoclfftz_b200
from aoclfftz_b200 import abi

pytestmark = pytest.mark.gpu

MAX_ELEMS = 1 << 22  # complex elements of the static scratch array
INVALID_INPUT = -3


def _lib():
    lib = aoclfftz_b200.load()
    f = lib.aoclfftz_gpu_execute_noalloc_c2c_f
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_void_p]
    f.restype = C.c_int
    return lib


def _input(n, howmany, seed):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, (howmany, n)) + 1j * rng.uniform(-1, 1, (howmany, n))).astype(np.complex64)


def _plan_result(lib, x, direction):
    """Output of the plan-based entry point on device buffers."""
    import torch
    howmany, n = x.shape
    din = torch.from_numpy(x.view(np.float32).ravel().copy()).cuda()
    dout = torch.zeros_like(din)
    desc, keep = abi.make_desc(din.data_ptr(), dout.data_ptr(), [(n, 1, 1)], [(howmany, n, n)], 0, direction, 1)
    h = abi.setup(lib, desc, "f32")
    assert h, lib.aoclfftz_gpu_last_error().decode()
    try:
        assert lib.aoclfftz_execute(h) == 0
        torch.cuda.synchronize()
    finally:
        lib.aoclfftz_destroy(h)
    return dout.cpu().numpy().view(np.complex64).reshape(howmany, n)


def _noalloc(lib, x, direction, inplace=False):
    import torch
    howmany, n = x.shape
    din = torch.from_numpy(x.view(np.float32).ravel().copy()).cuda()
    dout = din if inplace else torch.zeros_like(din)
    torch.cuda.synchronize()
    rc = lib.aoclfftz_gpu_execute_noalloc_c2c_f(din.data_ptr(), dout.data_ptr(), n, howmany, direction,
                                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.aoclfftz_gpu_last_error().decode()
    torch.cuda.synchronize()
    return dout.cpu().numpy().view(np.complex64).reshape(howmany, n)


def _rel_l2(a, b):
    a = a.astype(np.complex128)
    b = b.astype(np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _tol(n):
    """4 log2(N) eps of float32, the bound used throughout the tests."""
    return 4 * math.log2(n) * float(np.finfo(np.float32).eps)


@pytest.mark.parametrize("n,howmany,direction", [(1 << 15, 4, 0), (1 << 16, 3, 1), (1 << 18, 2, 0),
                                                 (1 << 21, 2, 1), (1 << 22, 1, 0)])
def test_two_calls_in_a_row_match_plan(n, howmany, direction):
    """Two consecutive calls on different inputs (the second reuses the scratch
    that the first left behind) each match the plan-based entry point."""
    lib = _lib()
    for seed in (1, 2):
        x = _input(n, howmany, seed + n)
        ref = _plan_result(lib, x, direction)
        got = _noalloc(lib, x, direction)
        err = _rel_l2(got, ref)
        assert err <= _tol(n), (seed, err)


def test_alternating_sizes_and_in_place():
    """Calls of different lengths back to back share the scratch; in == out is
    allowed because the column pass reads all input before the row pass writes."""
    lib = _lib()
    for i, (n, hm) in enumerate([(1 << 20, 4), (1 << 15, 128), (1 << 17, 8)]):
        x = _input(n, hm, 100 + i)
        ref = _plan_result(lib, x, i % 2)
        got = _noalloc(lib, x, i % 2, inplace=(i == 1))
        assert _rel_l2(got, ref) <= _tol(n)


def test_rejects_sizes_beyond_the_maximum():
    import torch
    lib = _lib()
    buf = torch.zeros(2 * MAX_ELEMS + 2, dtype=torch.float32, device="cuda")
    p = buf.data_ptr()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    f = lib.aoclfftz_gpu_execute_noalloc_c2c_f
    assert f(p, p, 1 << 22, 2, 0, st) == INVALID_INPUT
    assert "exceeds the static scratch" in lib.aoclfftz_gpu_last_error().decode()
    assert f(p, p, 1 << 23, 1, 0, st) == INVALID_INPUT
    # not a power of two, too short, bad direction, empty batch, host memory
    assert f(p, p, 3 << 14, 1, 0, st) == INVALID_INPUT
    assert f(p, p, 1 << 14, 1, 0, st) == INVALID_INPUT
    assert f(p, p, 1 << 16, 1, 2, st) == INVALID_INPUT
    assert f(p, p, 1 << 16, 0, 0, st) == INVALID_INPUT
    host = np.zeros(2 << 16, dtype=np.float32)
    assert f(host.ctypes.data, p, 1 << 16, 1, 0, st) == INVALID_INPUT
    torch.cuda.synchronize()
