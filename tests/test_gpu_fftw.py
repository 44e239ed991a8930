"""GPU parity of the FFTW3-compatible surface (include/fftw3.h) against the
reference's own FFTW wrapper (wrappers/fftw, built into oracle/_ref/) on the
same host buffers, and against the FP64 oracle. Host numpy buffers exercise the
library's host-staging path. Bound: 4 * log2(N) * eps of the dtype (vs the
oracle), twice that plus the reference's own error (vs the reference)."""
import ctypes as C

import numpy as np
import pytest

import aoclfftz_b200
import oracle
from aoclfftz_b200 import synthetic

pytestmark = pytest.mark.gpu

FWD, BWD = -1, +1
EST = 1 << 6


def _bind(lib):
    for pre in ("fftw", "fftwf"):
        for nm in ("plan_dft", "plan_dft_1d", "plan_dft_2d", "plan_dft_3d", "plan_many_dft", "plan_guru_dft",
                   "plan_dft_r2c", "plan_dft_r2c_1d", "plan_dft_r2c_3d", "plan_dft_c2r", "plan_dft_c2r_1d",
                   "plan_dft_c2r_3d", "plan_many_dft_r2c", "plan_r2r_1d"):
            getattr(lib, pre + "_" + nm).restype = C.c_void_p
        for nm in ("execute", "destroy_plan"):
            getattr(lib, pre + "_" + nm).argtypes = [C.c_void_p]
        for nm in ("execute_dft", "execute_dft_r2c", "execute_dft_c2r"):
            getattr(lib, pre + "_" + nm).argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


@pytest.fixture(scope="module")
def libs():
    ours = _bind(aoclfftz_b200.load())
    ref = _bind(C.CDLL(oracle.REF_FFTW_SO)) if oracle.ref_available() else None
    return ours, ref


def P(a):
    return C.c_void_p(a.ctypes.data)


def run_both(libs, pre, planner, args_fn, inp, out_len, out_dtype):
    """args_fn(in_ptr, out_ptr) -> args of the planner. Returns (ours, ref)."""
    results = []
    for lib in libs:
        if lib is None:
            results.append(None)
            continue
        x = inp.copy()
        y = np.zeros(out_len, dtype=out_dtype) if out_len else x
        plan = getattr(lib, pre + "_" + planner)(*args_fn(P(x), P(y)))
        assert plan, "planner returned NULL"
        getattr(lib, pre + "_execute")(C.c_void_p(plan))
        getattr(lib, pre + "_destroy_plan")(C.c_void_p(plan))
        results.append(y.copy())
    return results


def check(ours, ref, exact, n, dtype):
    tol = oracle.tol(n, dtype)
    assert oracle.rel_l2(ours, exact) <= tol
    if ref is not None:
        assert oracle.rel_l2(ours, ref) <= 2 * tol + oracle.rel_l2(ref, exact)


@pytest.mark.parametrize("pre,dt", [("fftwf", "f32"), ("fftw", "f64")])
def test_plan_dft_1d_2d_3d(libs, pre, dt):
    cd = np.complex64 if dt == "f32" else np.complex128
    x = synthetic.complex_uniform(3, 1024, cd)
    o, r = run_both(libs, pre, "plan_dft_1d", lambda a, b: (1024, a, b, FWD, EST), x, 1024, cd)
    check(o, r, oracle.fft(x), 1024, dt)
    x2 = synthetic.complex_uniform(4, 32 * 48, cd)
    o, r = run_both(libs, pre, "plan_dft_2d", lambda a, b: (32, 48, a, a, BWD, EST), x2, 0, cd)  # in place
    check(o, r, oracle.fft_nd(x2.reshape(32, 48), +1).ravel(), 32 * 48, dt)
    x3 = synthetic.complex_uniform(5, 8 * 16 * 12, cd)
    o, r = run_both(libs, pre, "plan_dft_3d", lambda a, b: (8, 16, 12, a, b, FWD, EST), x3, x3.size, cd)
    check(o, r, oracle.fft_nd(x3.reshape(8, 16, 12)).ravel(), x3.size, dt)


@pytest.mark.parametrize("pre,dt", [("fftwf", "f32"), ("fftw", "f64")])
def test_plan_many_dft_with_embeds(libs, pre, dt):
    cd = np.complex64 if dt == "f32" else np.complex128
    n = (C.c_int * 2)(8, 10)
    inembed = (C.c_int * 2)(10, 12)  # padded input rows
    howmany, idist, odist = 3, 10 * 12, 80
    x = synthetic.complex_uniform(6, howmany * idist, cd)
    o, r = run_both(libs, pre, "plan_many_dft",
                    lambda a, b: (2, n, howmany, a, inembed, 1, idist, b, None, 1, odist, FWD, EST),
                    x, howmany * odist, cd)
    logical = x.reshape(howmany, 10, 12)[:, :8, :10]
    exact = np.stack([oracle.fft_nd(logical[i]) for i in range(howmany)]).ravel()
    check(o, r, exact, 80, dt)


@pytest.mark.parametrize("pre,dt", [("fftwf", "f32"), ("fftw", "f64")])
def test_plan_r2c_c2r(libs, pre, dt):
    rd = np.float32 if dt == "f32" else np.float64
    cd = np.complex64 if dt == "f32" else np.complex128
    # 1-D out of place
    x = synthetic.normal(7, 50).astype(rd)
    o, r = run_both(libs, pre, "plan_dft_r2c_1d", lambda a, b: (50, a, b, EST), x, 26, cd)
    X = oracle.rfft_packed(x.astype(np.float64))
    check(o, r, X, 50, dt)
    o, r = run_both(libs, pre, "plan_dft_c2r_1d", lambda a, b: (50, a, b, EST), X.astype(cd), 50, rd)
    check(o, r, 50 * x.astype(np.float64), 50, dt)
    # 3-D in place with padded rows
    shp = (8, 8, 16)
    h = shp[-1] // 2 + 1
    xr = synthetic.normal(8, 8 * 8 * 16).reshape(shp).astype(rd)
    buf = np.zeros((8, 8, 2 * h), dtype=rd)
    buf[:, :, :16] = xr
    o, r = run_both(libs, pre, "plan_dft_r2c_3d", lambda a, b: (8, 8, 16, a, a, EST), buf.ravel(), 0, rd)
    Xr = oracle.rfftn(xr.astype(np.float64))
    check(o.view(cd).reshape(8, 8, h), None if r is None else r.view(cd).reshape(8, 8, h), Xr, 1024, dt)
    cbuf = Xr.astype(cd).ravel().view(rd).copy()
    o, r = run_both(libs, pre, "plan_dft_c2r_3d", lambda a, b: (8, 8, 16, a, a, EST), cbuf, 0, rd)
    got = o.reshape(8, 8, 2 * h)[:, :, :16]
    check(got, None if r is None else r.reshape(8, 8, 2 * h)[:, :, :16], 1024 * xr.astype(np.float64), 1024, dt)


def test_execute_dft_new_buffers_and_guru(libs):
    ours, ref = libs
    n = 256
    a = synthetic.complex_uniform(9, n, np.complex128)
    b = np.zeros(n, dtype=np.complex128)
    plan = ours.fftw_plan_dft_1d(n, P(a), P(b), FWD, EST)
    assert plan
    a2 = synthetic.complex_uniform(10, n, np.complex128)
    b2 = np.zeros(n, dtype=np.complex128)
    ours.fftw_execute_dft(C.c_void_p(plan), P(a2), P(b2))
    ours.fftw_destroy_plan(C.c_void_p(plan))
    assert oracle.rel_l2(b2, oracle.fft(a2)) <= oracle.tol(n, "f64")

    class IoDim(C.Structure):
        _fields_ = [("n", C.c_int), ("is", C.c_int), ("os", C.c_int)]

    dims = (IoDim * 1)(IoDim(64, 2, 2))
    hdims = (IoDim * 1)(IoDim(3, 128, 128))
    x = synthetic.complex_uniform(11, 3 * 128, np.complex64)
    y = np.zeros_like(x)
    plan = ours.fftwf_plan_guru_dft(1, dims, 1, hdims, P(x), P(y), BWD, EST)
    assert plan
    ours.fftwf_execute(C.c_void_p(plan))
    ours.fftwf_destroy_plan(C.c_void_p(plan))
    got = y.reshape(3, 128)[:, ::2]
    assert oracle.rel_l2(got, oracle.fft(x.reshape(3, 128)[:, ::2], +1)) <= oracle.tol(64, "f32")


def test_r2r_unsupported(libs):
    ours, _ = libs
    a = np.zeros(8)
    assert not ours.fftw_plan_r2r_1d(8, P(a), P(a), 0, EST)


@pytest.mark.parametrize("pre", ["fftw", "fftwf"])
def test_introspection_wisdom_and_threads(libs, pre):
    """The ancillary FFTW calls: sprint_plan describes the GPU plan (a string
    the caller frees), flops / cost report 5 N log2 N for the plan's batch,
    alignment_of is the address modulo 16, wisdom export succeeds with nothing
    written and import reports nothing loaded (as the reference wrapper), the
    thread calls are accepted, and every r2r planner returns NULL."""
    ours, ref = libs
    f = lambda nm: getattr(ours, pre + "_" + nm)
    esz = 8 if pre == "fftwf" else 16
    a = np.zeros(2 * 4096 * 3, dtype=np.float32 if pre == "fftwf" else np.float64)
    b = np.zeros_like(a)
    n = (C.c_int * 1)(4096)
    f("plan_many_dft").restype = C.c_void_p
    p = f("plan_many_dft")(1, n, 3, P(a), None, 1, 4096, P(b), None, 1, 4096, -1, EST)
    assert p
    try:
        f("sprint_plan").restype = C.c_void_p
        sp = f("sprint_plan")(C.c_void_p(p))
        text = C.cast(sp, C.c_char_p).value.decode()
        assert "4096" in text, text
        C.CDLL(None).free(C.c_void_p(sp))
        add, mul, fma = C.c_double(), C.c_double(), C.c_double()
        f("flops")(C.c_void_p(p), C.byref(add), C.byref(mul), C.byref(fma))
        assert abs(add.value + mul.value - 5 * 4096 * 12 * 3) < 1e-6 and fma.value == 0
        f("cost").restype = C.c_double
        assert f("cost")(C.c_void_p(p)) == pytest.approx(5 * 4096 * 12 * 3)
    finally:
        f("destroy_plan")(C.c_void_p(p))
    assert f("alignment_of")(C.c_void_p(a.ctypes.data + esz // 2)) == (a.ctypes.data + esz // 2) % 16
    assert f("export_wisdom_to_filename")(b"/nonexistent/wisdom") == 1
    f("export_wisdom_to_string").restype = C.c_void_p
    ws = f("export_wisdom_to_string")()
    assert C.cast(ws, C.c_char_p).value == b""
    C.CDLL(None).free(C.c_void_p(ws))
    assert f("import_system_wisdom")() == 0
    assert f("import_wisdom_from_string")(b"(fftw-3.3 wisdom)") == 0
    assert f("init_threads")() == 1
    f("plan_with_nthreads")(4)
    assert f("planner_nthreads")() == 4
    f("make_planner_thread_safe")()
    f("forget_wisdom")()
    for nm in ("plan_r2r_2d", "plan_r2r_3d", "plan_many_r2r", "plan_guru_r2r", "plan_guru64_r2r"):
        f(nm).restype = C.c_void_p
    c = np.zeros(64)
    assert not f("plan_r2r_2d")(8, 8, P(c), P(c), 0, 0, EST)
    assert not f("plan_r2r_3d")(4, 4, 4, P(c), P(c), 0, 0, 0, EST)
    assert (C.c_char * 16).in_dll(ours, pre + "_version").value.startswith(b"AOCL-FFTZ")


def test_fortran_interface(libs):
    """The Fortran-callable planners (arguments by reference, dimensions in
    Fortran order): 2-D, many and guru plans of a column-major nx x ny array
    against the oracle's 2-D DFT of the same memory viewed as [ny][nx]."""
    ours, _ = libs
    ref = lambda x, sg=-1: oracle.fft_nd(x.astype(np.complex128), sign=sg)
    nx, ny, batch = 48, 20, 3
    ip = lambda v: C.byref(C.c_int(v))
    for fpre, dt, cd in (("dfftw", "f64", np.complex128), ("dfftwf", "f32", np.complex64)):
        x = synthetic.complex_uniform(7, batch * nx * ny, cd)
        y = np.zeros_like(x)
        plan = C.c_void_p()
        getattr(ours, fpre + "_plan_dft_2d_")(C.byref(plan), ip(nx), ip(ny), P(x), P(y), ip(-1), ip(EST))
        assert plan.value
        getattr(ours, fpre + "_execute_")(C.byref(plan))
        getattr(ours, fpre + "_destroy_plan_")(C.byref(plan))
        r = ref(x[: nx * ny].reshape(ny, nx))
        assert oracle.rel_l2(y[: nx * ny].reshape(ny, nx), r) <= oracle.tol(nx * ny, dt)
        # guru: n = (nx, ny), strides (1, nx), one batch dimension of distance nx * ny
        y[:] = 0
        n = (C.c_int * 2)(nx, ny)
        st = (C.c_int * 2)(1, nx)
        hn, hs = (C.c_int * 1)(batch), (C.c_int * 1)(nx * ny)
        getattr(ours, fpre + "_plan_guru_dft_")(C.byref(plan), ip(2), n, st, st, ip(1), hn, hs, hs, P(x), P(y),
                                                ip(-1), ip(EST))
        assert plan.value
        getattr(ours, fpre + "_execute_")(C.byref(plan))
        cost = C.c_double()
        getattr(ours, fpre + "_cost_")(C.byref(cost), C.byref(plan))
        assert cost.value > 0
        getattr(ours, fpre + "_destroy_plan_")(C.byref(plan))
        for b in range(batch):
            s_ = slice(b * nx * ny, (b + 1) * nx * ny)
            assert oracle.rel_l2(y[s_].reshape(ny, nx), ref(x[s_].reshape(ny, nx))) <= oracle.tol(nx * ny, dt)
        # many: rank 2, n in Fortran order, batch distance nx * ny
        y[:] = 0
        getattr(ours, fpre + "_plan_many_dft_")(C.byref(plan), ip(2), n, ip(batch), P(x), None, ip(1),
                                                ip(nx * ny), P(y), None, ip(1), ip(nx * ny), ip(+1), ip(EST))
        assert plan.value
        getattr(ours, fpre + "_execute_")(C.byref(plan))
        getattr(ours, fpre + "_destroy_plan_")(C.byref(plan))
        rb = np.stack([ref(v, +1) for v in x.reshape(batch, ny, nx)])
        assert oracle.rel_l2(y.reshape(batch, ny, nx), rb) <= oracle.tol(nx * ny, dt)

