"""GPU parity of real transforms (r2c forward, c2r backward) through the C ABI
against the FP64 oracle (packed r2c restated from
core/solvers/real/packed_solver_rdft.c) and the reference library.

Bound: rel-L2 <= 4 * log2(N) * eps of the working dtype (N = product of dims).
Layouts follow docs/rst/data_layout_conventions.rst of the reference: the
real side counts real elements, the half-complex side n0/2+1 complex bins;
in-place rows are padded to 2 (n0/2 + 1) reals.
"""
import numpy as np
import pytest

import oracle
from aoclfftz_b200 import synthetic
from fftz_helpers import gather, real_dtype, run_gpu, scatter, span

pytestmark = pytest.mark.gpu


def real_problem(shape, batch, inplace):
    """FFTW-order shape (outermost first) -> dims/vecs for r2c and c2r."""
    rdims = list(reversed(shape))  # dims[0] innermost
    n0 = rdims[0]
    h0 = n0 // 2 + 1
    rrow = 2 * h0 if inplace else n0
    r_str, c_str = [1], [1]
    for i in range(1, len(rdims)):
        r_str.append(r_str[-1] * (rrow if i == 1 else rdims[i - 1]))
        c_str.append(c_str[-1] * (h0 if i == 1 else rdims[i - 1]))
    rtot = r_str[-1] * (rrow if len(rdims) == 1 else rdims[-1])
    ctot = c_str[-1] * (h0 if len(rdims) == 1 else rdims[-1])
    return rdims, r_str, c_str, rtot, ctot


def check_real(dtype, shape, batch=1, inplace=False, seed=3, compare_ref=True):
    rdims, r_str, c_str, rtot, ctot = real_problem(shape, batch, inplace)
    n0 = rdims[0]
    h0 = n0 // 2 + 1
    N = int(np.prod(shape))
    tol = oracle.tol(N, dtype)
    x = synthetic.normal(seed, batch * N).reshape([batch] + list(shape)).astype(real_dtype(dtype))
    # forward r2c
    dims = [(rdims[i], r_str[i], c_str[i]) for i in range(len(rdims))]
    vecs = [(batch, rtot, ctot)]
    pl = 0 if inplace else 1
    in_sc = span(dims, vecs, "in")
    out_sc = 2 * span(dims, vecs, "out", n0=h0)
    raw = scatter(x, [(d[0], d[1]) for d in dims], [(batch, rtot)], max(in_sc, out_sc) if inplace else in_sc, dtype,
                  complex_side=False)
    out_raw, plan = run_gpu(dtype, dims, vecs, raw, out_sc, 1, 0, pl)
    X = gather(out_raw, [(d[0], d[2]) for d in dims], [(batch, ctot)], dtype, n0=h0)
    ref = oracle.rfftn(x.astype(np.float64), rank=len(shape))
    err = oracle.rel_l2(X, ref)
    assert err <= tol, "r2c rel-L2 %.3e > %.3e; plan %s" % (err, tol, plan)
    if compare_ref and oracle.ref_available():
        r_raw = oracle.ref_execute(dtype, dims, vecs, raw, out_sc, 1, 0, pl)
        R = gather(r_raw, [(d[0], d[2]) for d in dims], [(batch, ctot)], dtype, n0=h0)
        # the reference's own error vs the exact DFT widens the bound where it exceeds the
        # dtype bound (the reference's f64 r2c of odd length 15 is off by 8e-13 relative)
        assert oracle.rel_l2(X, R) <= 2 * tol + oracle.rel_l2(R, ref)
    # backward c2r of the oracle spectrum
    cdims = [(rdims[i], c_str[i], r_str[i]) for i in range(len(rdims))]
    cvecs = [(batch, ctot, rtot)]
    cin_sc = 2 * span(cdims, cvecs, "in", n0=h0)
    cout_sc = span(cdims, cvecs, "out")
    craw = scatter(ref.astype(np.complex64 if dtype == "f32" else np.complex128), [(d[0], d[1]) for d in cdims],
                   [(batch, ctot)], max(cin_sc, cout_sc) if inplace else cin_sc, dtype, n0=h0)
    y_raw, plan2 = run_gpu(dtype, cdims, cvecs, craw, cout_sc, 1, 1, pl)
    y = gather(y_raw, [(d[0], d[2]) for d in cdims], [(batch, rtot)], dtype, complex_side=False)
    err2 = oracle.rel_l2(y, x.astype(np.float64) * N)
    assert err2 <= tol, "c2r rel-L2 %.3e > %.3e; plan %s" % (err2, tol, plan2)
    return err, err2


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [2, 4, 6, 16, 18, 64, 100, 512, 1024, 4096, 8192])
def test_r2c_c2r_1d_even(dtype, n):
    check_real(dtype, [n], batch=3)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [1, 3, 5, 15, 17, 99, 255])
def test_r2c_c2r_1d_odd(dtype, n):
    check_real(dtype, [n], batch=2)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_r2c_c2r_inplace_padded(dtype):
    check_real(dtype, [50], batch=4, inplace=True)
    check_real(dtype, [16, 16, 16], batch=1, inplace=True)
    check_real(dtype, [8, 12, 32], batch=2, inplace=True)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_r2c_c2r_nd(dtype):
    check_real(dtype, [16, 32], batch=2)
    check_real(dtype, [6, 10, 14], batch=1)
    check_real(dtype, [64, 64, 64], batch=1)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [34, 1018, 16384, 65536, 1 << 18, 200003])
def test_r2c_c2r_multipass_lines(dtype, n):
    """Real lengths one CTA cannot hold (long packed lines, odd lengths and
    halves with prime factors > 13): widen, complex line algorithm, recombine."""
    check_real(dtype, [n], batch=2)


def test_r2c_c2r_multipass_inplace_nd():
    check_real("f32", [4, 34], batch=2, inplace=True)
    check_real("f64", [3, 17], batch=1)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [16, 256, 1024])
def test_r2c_c2r_interleaved_batch(dtype, n):
    """Transforms interleaved element by element (element stride = batch,
    distance 1): the real lines take a column lane map, so the compile-time
    real-line kernel runs the generic load and store phases around its
    stages. Both directions against the oracle."""
    B = 8
    h0 = n // 2 + 1
    tol = oracle.tol(n, dtype)
    x = synthetic.normal(11, B * n).reshape(B, n).astype(real_dtype(dtype))
    dims, vecs = [(n, B, B)], [(B, 1, 1)]
    in_sc = span(dims, vecs, "in")
    out_sc = 2 * span(dims, vecs, "out", n0=h0)
    raw = scatter(x, [(n, B)], [(B, 1)], in_sc, dtype, complex_side=False)
    out_raw, plan = run_gpu(dtype, dims, vecs, raw, out_sc, 1, 0, 1)
    X = gather(out_raw, [(n, B)], [(B, 1)], dtype, n0=h0)
    ref = oracle.rfftn(x.astype(np.float64), rank=1)
    err = oracle.rel_l2(X, ref)
    assert err <= tol, "r2c rel-L2 %.3e > %.3e; plan %s" % (err, tol, plan)
    cin_sc = 2 * span(dims, vecs, "in", n0=h0)
    cout_sc = span(dims, vecs, "out")
    craw = scatter(ref.astype(np.complex64 if dtype == "f32" else np.complex128), [(n, B)], [(B, 1)], cin_sc, dtype,
                   n0=h0)
    y_raw, plan2 = run_gpu(dtype, dims, vecs, craw, cout_sc, 1, 1, 1)
    y = gather(y_raw, [(n, B)], [(B, 1)], dtype, complex_side=False)
    err2 = oracle.rel_l2(y, x.astype(np.float64) * n)
    assert err2 <= tol, "c2r rel-L2 %.3e > %.3e; plan %s" % (err2, tol, plan2)
