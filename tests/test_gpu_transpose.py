"""The standalone transpose (aoclfftz_gpu_transpose), through the C ABI:
element (r, c) from in[r * row_is + c * col_is] to out[r * row_os + c * col_os]
-- the problem of the reference's transpose solver (core/solvers/
transpose_solver.c:97-141: out of place, in place square, in place
rectangular). Elements move as raw words, so every case must equal numpy's
result byte for byte: plain transposes of every element type, ragged tile
edges, padded rows, general strides, in place square and rectangular, and the
rejected inputs."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TYPES = {("f32", 0): np.complex64, ("f32", 1): np.float32, ("f64", 0): np.complex128, ("f64", 1): np.float64}


def _lib():
    import aoclfftz_b200
    return aoclfftz_b200.load()


def _rand(shape, dt, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    if np.issubdtype(dt, np.complexfloating):
        a = a + 1j * rng.standard_normal(shape)
    return a.astype(dt)


def _run(lib, dtype, real, d_in, d_out, rows, cols, ris, cis, ros, cos):
    rc = lib.aoclfftz_gpu_transpose(0 if dtype == "f32" else 1, real, C.c_void_p(d_in.data_ptr()),
                                    C.c_void_p(d_out.data_ptr()), rows, cols, ris, cis, ros, cos, None)
    return rc


def _torch_buf(a):
    import torch
    raw = np.ascontiguousarray(a).view(np.uint8)
    return torch.from_numpy(raw.copy()).to("cuda")


@pytest.mark.parametrize("dtype,real", list(TYPES))
@pytest.mark.parametrize("rows,cols", [(1, 1), (7, 13), (32, 32), (33, 65), (1000, 33), (4096, 1024)])
def test_transpose_out_of_place(dtype, real, rows, cols):
    import torch
    dt = TYPES[(dtype, real)]
    lib = _lib()
    a = _rand((rows, cols), dt, rows * 7 + cols)
    d_in = _torch_buf(a)
    d_out = torch.zeros(rows * cols * np.dtype(dt).itemsize, dtype=torch.uint8, device="cuda")
    assert _run(lib, dtype, real, d_in, d_out, rows, cols, cols, 1, 1, rows) == 0
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().view(dt).reshape(cols, rows)
    assert got.tobytes() == np.ascontiguousarray(a.T).tobytes()


@pytest.mark.parametrize("dtype,real", [("f32", 0), ("f64", 1)])
def test_transpose_general_strides(dtype, real):
    """Padded input rows, output rows padded too, and a strided (non-unit)
    column stride on the input side."""
    import torch
    dt = TYPES[(dtype, real)]
    lib = _lib()
    rows, cols, pad_in, pad_out = 300, 70, 5, 3
    big = _rand((rows, 2 * (cols + pad_in)), dt, 5)
    a = big[:, 0:2 * cols:2]  # element (r, c) at r * 2 (cols + pad_in) + 2 c
    d_in = _torch_buf(big)
    ld_out = rows + pad_out
    d_out = torch.zeros(cols * ld_out * np.dtype(dt).itemsize, dtype=torch.uint8, device="cuda")
    assert _run(lib, dtype, real, d_in, d_out, rows, cols, 2 * (cols + pad_in), 2, 1, ld_out) == 0
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().view(dt).reshape(cols, ld_out)[:, :rows]
    assert got.tobytes() == np.ascontiguousarray(a.T).tobytes()
    assert not d_out.cpu().numpy().view(dt).reshape(cols, ld_out)[:, rows:].any()


@pytest.mark.parametrize("n", [1, 31, 32, 100, 1024])
@pytest.mark.parametrize("dtype,real", [("f32", 0), ("f32", 1), ("f64", 0)])
def test_transpose_in_place_square(n, dtype, real):
    import torch
    dt = TYPES[(dtype, real)]
    lib = _lib()
    a = _rand((n, n), dt, n)
    d = _torch_buf(a)
    assert _run(lib, dtype, real, d, d, n, n, n, 1, 1, n) == 0
    torch.cuda.synchronize()
    assert d.cpu().numpy().view(dt).reshape(n, n).tobytes() == np.ascontiguousarray(a.T).tobytes()


@pytest.mark.parametrize("rows,cols", [(3, 5), (100, 37), (512, 2048)])
def test_transpose_in_place_rectangular(rows, cols):
    import torch
    dt = np.complex64
    lib = _lib()
    a = _rand((rows, cols), dt, rows + cols)
    d = _torch_buf(a)
    assert _run(lib, "f32", 0, d, d, rows, cols, cols, 1, 1, rows) == 0
    torch.cuda.synchronize()
    assert d.cpu().numpy().view(dt).reshape(cols, rows).tobytes() == np.ascontiguousarray(a.T).tobytes()


def test_transpose_rejects_bad_input():
    import torch
    lib = _lib()
    d = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    h = np.zeros(1024, dtype=np.uint8)
    bad = [(2, 0, d, d, 4, 4, 4, 1, 1, 4), (0, 2, d, d, 4, 4, 4, 1, 1, 4), (0, 0, d, d, 0, 4, 4, 1, 1, 4),
           (0, 0, d, d, 4, 4, 4, -1, 1, 4)]
    for dt, re, i, o, *args in bad:
        assert lib.aoclfftz_gpu_transpose(dt, re, C.c_void_p(i.data_ptr()), C.c_void_p(o.data_ptr()), *args,
                                          None) != 0
        assert lib.aoclfftz_gpu_last_error()
    # host memory is refused, NULL too
    assert lib.aoclfftz_gpu_transpose(0, 0, C.c_void_p(h.ctypes.data), C.c_void_p(d.data_ptr()), 4, 4, 4, 1, 1,
                                      4, None) != 0
    assert lib.aoclfftz_gpu_transpose(0, 0, None, C.c_void_p(d.data_ptr()), 4, 4, 4, 1, 1, 4, None) != 0


def test_transpose_bandwidth():
    """4096 x 4096 complex float (128 MiB each way, > L2), timed with CUDA
    events over 20 launches after warm-up; prints the bandwidth (one read +
    one write of the array per launch). Checked against numpy first."""
    import torch
    lib = _lib()
    n = 4096
    a = _rand((n, n), np.complex64, 1)
    d_in = _torch_buf(a)
    d_out = torch.empty_like(d_in)
    assert _run(lib, "f32", 0, d_in, d_out, n, n, n, 1, 1, n) == 0
    torch.cuda.synchronize()
    assert d_out.cpu().numpy().view(np.complex64).reshape(n, n).tobytes() == np.ascontiguousarray(a.T).tobytes()
    for _ in range(3):
        _run(lib, "f32", 0, d_in, d_out, n, n, n, 1, 1, n)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(20):
        _run(lib, "f32", 0, d_in, d_out, n, n, n, 1, 1, n)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 20
    print("transpose 4096 x 4096 c64: %.4f ms, %.1f GB/s" % (ms, 2 * n * n * 8 / (ms * 1e-3) / 1e9))
