"""Real 3-D transforms at the full sizes of the real-transform workload: fp64,
512^3 and 256 x 256 x 1024 (FFTW order, last dimension innermost), in place,
innermost rows padded to 2 (n0/2 + 1) reals, r2c then c2r through the C ABI on
device buffers.

Checked, as for the reference's own large-size runs, by size-independent
properties plus exact sums where they are affordable:
* round trip: || c2r(r2c(x)) / N - x || / || x || <= 4 log2(N) eps;
* a 64^3 sub-block of the r2c output against separable FP64 DFT sums over the
  whole input (twiddles from exactly reduced integer indices), within the
  same bound;
* Hermitian edge: bins k0 = 0 and k0 = n0/2 of the (k2, k1) = (0, 0) line are
  real up to rounding.
"""
import ctypes as C
import math

import numpy as np
import pytest

import aoclfftz_b200
from aoclfftz_b200 import abi

pytestmark = pytest.mark.gpu


def _dft_cols(n, ks):
    """n x len(ks) matrix of exp(-2 pi i (j k mod n) / n), FP64, exact index."""
    j = np.arange(n, dtype=np.int64)[:, None]
    r = (j * np.asarray(ks, dtype=np.int64)[None, :]) % n
    return np.exp(-2j * np.pi * (r.astype(np.float64) / n))


def _run(lib, buf, shape, direction):
    n2, n1, n0 = shape
    h0 = n0 // 2 + 1
    rrow = 2 * h0
    if direction == 0:  # r2c: real strides in, complex strides out
        dims = [(n0, 1, 1), (n1, rrow, h0), (n2, rrow * n1, h0 * n1)]
        vecs = [(1, rrow * n1 * n2, h0 * n1 * n2)]
    else:
        dims = [(n0, 1, 1), (n1, h0, rrow), (n2, h0 * n1, rrow * n1)]
        vecs = [(1, h0 * n1 * n2, rrow * n1 * n2)]
    desc, keep = abi.make_desc(buf.data_ptr(), buf.data_ptr(), dims, vecs, 1, direction, 0)
    h = abi.setup(lib, desc, "f64")
    assert h, lib.aoclfftz_gpu_last_error().decode()
    try:
        assert lib.aoclfftz_execute(h) == 0, lib.aoclfftz_gpu_last_error().decode()
        import torch
        torch.cuda.synchronize()
    finally:
        lib.aoclfftz_destroy(h)


@pytest.mark.parametrize("shape", [(512, 512, 512), (256, 256, 1024)])
def test_real3d_inplace_padded_fp64(shape):
    import torch
    lib = aoclfftz_b200.load()
    n2, n1, n0 = shape
    h0 = n0 // 2 + 1
    N = n0 * n1 * n2
    tol = 4 * math.log2(N) * float(np.finfo(np.float64).eps)
    g = torch.Generator(device="cuda").manual_seed(20261203)
    x = torch.randn((n2, n1, n0), dtype=torch.float64, device="cuda", generator=g)
    buf = torch.zeros((n2, n1, 2 * h0), dtype=torch.float64, device="cuda")
    buf[:, :, :n0] = x
    _run(lib, buf, shape, 0)
    X = buf.view(torch.complex128)  # (n2, n1, h0) half-complex spectrum

    # 64^3 sub-block of bins against separable exact sums over the whole input
    k0 = np.arange(0, h0, max(1, h0 // 64))[:64]
    k1 = (np.arange(64) * 7 + 3) % n1
    k2 = (np.arange(64) * 11 + 5) % n2
    xc = x.cpu().numpy()
    a = xc.reshape(-1, n0) @ _dft_cols(n0, k0)  # (n2*n1, 64)
    a = a.reshape(n2, n1, len(k0))
    a = np.einsum("zyk,yl->zlk", a, _dft_cols(n1, k1), optimize=True)
    a = np.einsum("zlk,zm->mlk", a, _dft_cols(n2, k2), optimize=True)
    got = X[torch.as_tensor(k2, device="cuda")][:, torch.as_tensor(k1, device="cuda")][
        :, :, torch.as_tensor(k0, device="cuda")].cpu().numpy()
    err = float(np.linalg.norm(got - a) / np.linalg.norm(a))
    assert err <= tol, "r2c 64^3 sub-block rel-L2 %.3e > %.3e" % (err, tol)

    line = X[0, 0].cpu().numpy()
    scale = float(np.abs(line).max())
    assert abs(line[0].imag) <= 64 * tol * scale and abs(line[h0 - 1].imag) <= 64 * tol * scale

    # round trip
    _run(lib, buf, shape, 1)
    y = buf[:, :, :n0] / N
    rt = (torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)).item()
    assert rt <= tol, "round trip rel-L2 %.3e > %.3e" % (rt, tol)
