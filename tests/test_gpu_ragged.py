"""GPU parity of ragged batches (aoclfftz_gpu_ragged_*): transforms of mixed
lengths (powers of two, 7-smooth composites, primes through Bluestein, and
lengths that need the four-step split) in one persistent launch under a CUDA
graph, against the FP64 oracle; repeated executes are bitwise identical.
Bound per transform: 4 * log2(N) * eps of the dtype."""
import ctypes as C

import numpy as np
import pytest

import aoclfftz_b200
import oracle
from aoclfftz_b200 import synthetic

pytestmark = pytest.mark.gpu


def run_ragged(sizes, dtype, direction, repeat=1, in_offsets=None, out_offsets=None):
    import torch
    lib = aoclfftz_b200.load()
    cd = np.complex64 if dtype == "f32" else np.complex128
    total_in = (max(o + n for o, n in zip(in_offsets, sizes)) if in_offsets else sum(sizes))
    total_out = (max(o + n for o, n in zip(out_offsets, sizes)) if out_offsets else sum(sizes))
    x = synthetic.complex_normal(21, total_in, cd)
    tdt = torch.float32 if dtype == "f32" else torch.float64
    din = torch.from_numpy(x.view(x.real.dtype).copy()).to("cuda")
    dout = torch.zeros(2 * total_out, dtype=tdt, device="cuda")
    arr = (C.c_int64 * len(sizes))(*sizes)
    io = (C.c_int64 * len(sizes))(*in_offsets) if in_offsets else None
    oo = (C.c_int64 * len(sizes))(*out_offsets) if out_offsets else None
    h = lib.aoclfftz_gpu_ragged_setup(0 if dtype == "f32" else 1, direction, len(sizes), arr, io, oo)
    assert h, lib.aoclfftz_gpu_last_error().decode()
    outs = []
    try:
        for _ in range(repeat):
            assert lib.aoclfftz_gpu_ragged_execute(h, C.c_void_p(din.data_ptr()), C.c_void_p(dout.data_ptr())) == 0
            assert lib.aoclfftz_gpu_synchronize(h) == 0, lib.aoclfftz_gpu_last_error().decode()
            outs.append(dout.cpu().numpy().view(cd).copy())
    finally:
        lib.aoclfftz_destroy(h)
    return x, outs


def check(sizes, dtype, direction, in_offsets=None, out_offsets=None):
    x, outs = run_ragged(sizes, dtype, direction, 1, in_offsets, out_offsets)
    y = outs[0]
    ip = np.cumsum([0] + sizes[:-1]) if in_offsets is None else in_offsets
    op = np.cumsum([0] + sizes[:-1]) if out_offsets is None else out_offsets
    worst = 0.0
    for n, a, b in zip(sizes, ip, op):
        ref = oracle.fft(x[a:a + n], -1 if direction == 0 else +1)
        e = oracle.rel_l2(y[b:b + n], ref)
        worst = max(worst, e / oracle.tol(n, dtype))
        assert e <= oracle.tol(n, dtype), "n=%d rel-L2 %.3e" % (n, e)
    return worst


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_ragged_log_uniform_mix(dtype):
    sizes = synthetic.ragged_sizes(5, 96, 2, 65536)
    check(sizes, dtype, 0)
    check(sizes[::-1], dtype, 1)


def test_ragged_classes_and_offsets():
    sizes = [2, 3, 16, 17, 60, 97, 1024, 4096, 4099, 5000, 8192, 16384, 65521, 65536, 1]
    check(sizes, "f32", 0)
    gap_in = list(np.cumsum([0] + [n + 7 for n in sizes[:-1]]))
    gap_out = list(np.cumsum([0] + [n + 3 for n in sizes[:-1]]))
    check(sizes, "f64", 1, in_offsets=gap_in, out_offsets=gap_out)


def test_ragged_bit_reproducible():
    sizes = synthetic.ragged_sizes(6, 64, 2, 65536)
    _, outs = run_ragged(sizes, "f32", 0, repeat=4)
    for o in outs[1:]:
        assert o.tobytes() == outs[0].tobytes()
