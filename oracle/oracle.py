"""Oracle for the FFT plan-execution path: TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use
this module, and only as the checker. It exposes:

  * the C restatement in dft_oracle.c (naive FP64 DFT with exact index
    reduction and long-double accumulation; a restated mixed-radix/Bluestein
    FFT and packed real transforms), built into oracle/_build/liboracle.so;
  * the reference library itself (AOCL-FFTZ compiled from its own sources by
    oracle/Makefile into oracle/_ref/libaocl_fftz.so), driven through the same
    aoclfftz.h descriptors as the GPU library.

Pinning: tests/test_oracle.py checks the restatement against the golden
vectors in tests/golden/ (outputs of the reference library on seeded inputs,
written by tests/golden/make_golden.py) and, where the reference library is
present, against live reference runs.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libaocl_fftz.so")
REF_FFTW_SO = os.path.join(HERE, "_ref", "libfftw3_ref.so")

_olib = None
_rlib = None

_dp = C.POINTER(C.c_double)
_i64 = C.c_int64


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    """The C restatement (builds it on first use if needed)."""
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_dft_1d.argtypes = [_i64, C.c_int, _dp, _i64, _i64, _dp, _i64, _i64, _i64]
        L.orc_dft_bins.argtypes = [_i64, C.c_int, _dp, _i64, C.POINTER(_i64), _dp]
        L.orc_dft_nd.argtypes = [C.c_int, C.POINTER(_i64), C.c_int, _dp]
        L.orc_fft.argtypes = [_i64, C.c_int, _dp, _dp]
        L.orc_fft.restype = C.c_int
        L.orc_fft_batch.argtypes = [_i64, C.c_int, _dp, _dp, _i64]
        L.orc_fft_batch.restype = C.c_int
        L.orc_fft_nd.argtypes = [C.c_int, C.POINTER(_i64), C.c_int, _dp]
        L.orc_fft_nd.restype = C.c_int
        L.orc_rfft_packed.argtypes = [_i64, _dp, _dp]
        L.orc_rfft_packed.restype = C.c_int
        L.orc_irfft_packed.argtypes = [_i64, _dp, _dp]
        L.orc_irfft_packed.restype = C.c_int
        L.orc_pow2_radix_balanced.argtypes = [_i64, C.POINTER(_i64)]
        L.orc_pow2_radix_balanced.restype = C.c_int
        L.orc_pow2_balanced_split.argtypes = [_i64, C.POINTER(_i64), C.POINTER(_i64)]
        L.orc_pow2_balanced_split.restype = C.c_int
        L.orc_bluestein_extended_length.argtypes = [_i64]
        L.orc_bluestein_extended_length.restype = _i64
        L.orc_bluestein_chirp.argtypes = [_i64, _i64, _dp]
        _olib = L
    return _olib


def _p(a):
    return a.ctypes.data_as(_dp)


def _c128(x):
    return np.ascontiguousarray(x, dtype=np.complex128)


# ------------------------------------------------------------------ restatement

def dft(x, sign=-1):
    """Naive DFT along the last axis (exact index reduction, long double sums)."""
    x = _c128(x)
    n = x.shape[-1]
    howmany = x.size // n if n else 0
    out = np.empty_like(x)
    lib().orc_dft_1d(n, sign, _p(x), 1, n, _p(out), 1, n, howmany)
    return out


def dft_bins(x, bins, sign=-1):
    x = _c128(x)
    b = np.ascontiguousarray(bins, dtype=np.int64)
    out = np.empty(len(b), dtype=np.complex128)
    lib().orc_dft_bins(x.size, sign, _p(x), len(b), b.ctypes.data_as(C.POINTER(_i64)), _p(out))
    return out


def dft_nd(x, sign=-1):
    """Exact N-D DFT over all axes of a C-ordered array (last axis innermost)."""
    a = _c128(x).copy()
    dims = np.array(a.shape[::-1], dtype=np.int64)
    lib().orc_dft_nd(len(dims), dims.ctypes.data_as(C.POINTER(_i64)), sign, _p(a))
    return a


def fft(x, sign=-1):
    """Restated fast FFT in double along the last axis."""
    x = _c128(x)
    n = x.shape[-1]
    out = np.empty_like(x)
    rc = lib().orc_fft_batch(n, sign, _p(x), _p(out), x.size // n)
    if rc:
        raise RuntimeError("orc_fft failed")
    return out


def fft_nd(x, sign=-1):
    a = _c128(x).copy()
    dims = np.array(a.shape[::-1], dtype=np.int64)
    if lib().orc_fft_nd(len(dims), dims.ctypes.data_as(C.POINTER(_i64)), sign, _p(a)):
        raise RuntimeError("orc_fft_nd failed")
    return a


def rfft_packed(x):
    """r2c along the last axis: packed restatement for even n, full complex
    transform of the real input (first n/2+1 bins) for odd n."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    if n % 2:
        return fft(x.astype(np.complex128))[..., : n // 2 + 1]
    out = np.empty(x.shape[:-1] + (n // 2 + 1,), dtype=np.complex128)
    xs, os_ = x.reshape(-1, n), out.reshape(-1, n // 2 + 1)
    for i in range(xs.shape[0]):
        if lib().orc_rfft_packed(n, _p(xs[i]), _p(os_[i])):
            raise RuntimeError("orc_rfft_packed failed")
    return out


def irfft_packed(X, n):
    """c2r along the last axis (unnormalised): packed restatement for even n,
    Hermitian completion and a full complex transform for odd n."""
    X = _c128(X)
    if n % 2:
        full = np.empty(X.shape[:-1] + (n,), dtype=np.complex128)
        h = n // 2 + 1
        full[..., :h] = X[..., :h]
        full[..., h:] = np.conj(X[..., 1:n - h + 1][..., ::-1])
        return fft(full, sign=+1).real.copy()
    out = np.empty(X.shape[:-1] + (n,), dtype=np.float64)
    xs, os_ = X.reshape(-1, X.shape[-1]), out.reshape(-1, n)
    for i in range(xs.shape[0]):
        if lib().orc_irfft_packed(n, _p(np.ascontiguousarray(xs[i])), _p(os_[i])):
            raise RuntimeError("orc_irfft_packed failed")
    return out


def rfftn(x, rank=None):
    """Real N-D forward transform over the last `rank` axes (all by default):
    packed r2c along the last axis, then complex transforms along the others
    (what the reference's packed 3-D path computes,
    core/solvers/real/packed_solver_rdft.c:154-186)."""
    rank = x.ndim if rank is None else rank
    h = rfft_packed(x)
    for ax in range(x.ndim - rank, x.ndim - 1):
        h = np.moveaxis(fft(np.moveaxis(h, ax, -1)), -1, ax)
    return h


def irfftn(X, n_last, rank=None):
    rank = X.ndim if rank is None else rank
    h = _c128(X)
    for ax in range(X.ndim - rank, X.ndim - 1):
        h = np.moveaxis(fft(np.moveaxis(h, ax, -1), sign=+1), -1, ax)
    return irfft_packed(h, n_last)


def pow2_radix_balanced(n):
    r = (_i64 * 64)()
    s = lib().orc_pow2_radix_balanced(n, r)
    return [r[i] for i in range(s)]


def pow2_balanced_split(n):
    a, b = _i64(), _i64()
    ok = lib().orc_pow2_balanced_split(n, C.byref(a), C.byref(b))
    return (a.value, b.value) if ok else None


def bluestein_extended_length(n):
    return lib().orc_bluestein_extended_length(n)


def bluestein_chirp(n, m):
    b = np.empty(m, dtype=np.complex128)
    lib().orc_bluestein_chirp(n, m, _p(b))
    return b


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128).ravel()
    b = np.asarray(b, dtype=np.complex128).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def tol(n, dtype):
    """rel-L2 bound 4 * log2(N) * eps of the working dtype."""
    eps = np.finfo(np.float32 if dtype in ("f32", np.float32, np.complex64) else np.float64).eps
    return 4.0 * max(1.0, np.log2(max(n, 2))) * eps


# ------------------------------------------------------------ reference library

def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    """The reference AOCL-FFTZ library compiled from its own sources."""
    global _rlib
    if _rlib is None:
        import importlib
        abi = importlib.import_module("aoclfftz_b200.abi")
        _rlib = abi.bind(C.CDLL(REF_SO))
    return _rlib


def ref_execute(dtype, dims, vecs, x_in, out_shape_elems, fft_type=0, direction=0, placement=1, num_threads=1,
                opt_level=3):
    """Runs the reference on host buffers. x_in: numpy array holding the raw
    input buffer (complex64/128 or float32/64); returns the raw output buffer
    (same real dtype family, out_shape_elems scalars)."""
    import importlib
    abi = importlib.import_module("aoclfftz_b200.abi")
    real = np.float32 if dtype == "f32" else np.float64
    xin = np.ascontiguousarray(x_in).view(real).copy()
    if placement == 0:
        buf = np.zeros(max(xin.size, out_shape_elems), dtype=real)
        buf[: xin.size] = xin
        pin = pout = buf.ctypes.data
        out = buf
    else:
        out = np.zeros(out_shape_elems, dtype=real)
        pin, pout = xin.ctypes.data, out.ctypes.data
    desc, keep = abi.make_desc(pin, pout, dims, vecs, fft_type, direction, placement, num_threads=num_threads,
                               opt_level=opt_level)
    L = ref_lib()
    h = abi.setup(L, desc, dtype)
    if not h:
        raise RuntimeError("reference setup failed")
    try:
        rc = L.aoclfftz_execute(h)
        if rc != 0:
            raise RuntimeError("reference execute failed: %d" % rc)
    finally:
        L.aoclfftz_destroy(h)
    return out[:out_shape_elems].copy()
