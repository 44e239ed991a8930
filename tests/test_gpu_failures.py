"""GPU failure paths and concurrency, in the forms that fault and hang no GPU.

* Every device wait in the library is bounded and ends in an error status the
  host reads (the library's failure detection):
  a TMA tile wait that runs out (its mbarrier is made to expect more bytes
  than the copies deliver) and a ragged dependency wait that cannot complete
  (its count is raised past the predecessor's tiles) are reported by
  aoclfftz_gpu_synchronize, once, and the GPU stays usable.
* A device allocation that fails during setup returns NULL, as the reference's
  setup does on MEMORY_FAILURE (api/aoclfftz.h:60-68, selector/selector.c:
  1617-1619); the failure is injected on the host.
* aoclfftz_execute_io is safe from several threads on one handle
  (api/aoclfftz_api.c:86-135: one caller owns the plan's scratch, the others
  take per-call scratch).
* Executing restores the caller's current device.
"""
import ctypes as C
import threading

import numpy as np
import pytest

import aoclfftz_b200
import oracle
from aoclfftz_b200 import abi, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture
def lib():
    lib = aoclfftz_b200.load()
    lib.aoclfftz_gpu_inject_fault(abi.FAULT_NONE, 0)
    yield lib
    lib.aoclfftz_gpu_inject_fault(abi.FAULT_NONE, 0)
    lib.aoclfftz_gpu_set_hints(None)


def device_plan(lib, n, batch, direction=0, dtype="f32"):
    import torch
    cd = np.complex64 if dtype == "f32" else np.complex128
    x = synthetic.complex_uniform(3, n * batch, cd)
    din = torch.from_numpy(x.view(x.real.dtype).copy()).to("cuda")
    dout = torch.zeros_like(din)
    desc, keep = abi.make_desc(din.data_ptr(), dout.data_ptr(), [(n, 1, 1)], [(batch, n, n)], 0, direction, 1)
    h = abi.setup(lib, desc, dtype)
    return h, x, din, dout, keep


def check_output(dout, x, n, batch, dtype="f32"):
    cd = np.complex64 if dtype == "f32" else np.complex128
    y = dout.cpu().numpy().view(cd).reshape(batch, n)
    ref = oracle.fft(x.reshape(batch, n))
    err = oracle.rel_l2(y, ref)
    assert err <= oracle.tol(n, dtype), err


def test_execute_restores_current_device(lib):
    import torch
    before = torch.cuda.current_device()
    h, x, din, dout, keep = device_plan(lib, 4096, 8)
    assert h
    try:
        assert lib.aoclfftz_execute(h) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == 0
        assert torch.cuda.current_device() == before
    finally:
        lib.aoclfftz_destroy(h)


def test_setup_returns_null_when_a_device_allocation_fails(lib):
    assert lib.aoclfftz_gpu_inject_fault(abi.FAULT_ALLOC, 1) == 0
    h, x, din, dout, keep = device_plan(lib, 1 << 20, 1)
    assert not h
    assert b"allocation" in lib.aoclfftz_gpu_last_error()
    # the injected failure is consumed: the next setup succeeds and computes
    h, x, din, dout, keep = device_plan(lib, 1 << 20, 1)
    assert h, lib.aoclfftz_gpu_last_error()
    try:
        assert lib.aoclfftz_execute(h) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == 0
        check_output(dout, x, 1 << 20, 1)
    finally:
        lib.aoclfftz_destroy(h)


def test_tma_tile_wait_runs_out_and_is_reported(lib):
    """Split-kernel row tiles (kernel family 9, 4096-point rows) whose tile
    barrier expects 16 bytes more than the copies deliver: every CTA's bounded
    wait runs out, synchronize reports it once, and the next execute of the
    same plan is correct."""
    h_ = abi.Hints()
    h_.kernel_family = 9
    lib.aoclfftz_gpu_set_hints(C.byref(h_))
    h, x, din, dout, keep = device_plan(lib, 4096, 64)
    lib.aoclfftz_gpu_set_hints(None)
    assert h, lib.aoclfftz_gpu_last_error()
    try:
        txt = C.create_string_buffer(2048)
        lib.aoclfftz_gpu_describe(h, txt, 2048)
        assert b"tma-split" in txt.value, txt.value
        assert lib.aoclfftz_gpu_inject_fault(abi.FAULT_TMA_SHORT, 16) == 0
        assert lib.aoclfftz_execute(h) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == abi.AOCLFFTZ_EXECUTION_FAILURE
        assert b"gave up waiting" in lib.aoclfftz_gpu_last_error()
        assert lib.aoclfftz_gpu_inject_fault(abi.FAULT_NONE, 0) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == 0  # reported once
        dout.zero_()
        assert lib.aoclfftz_execute(h) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == 0
        check_output(dout, x, 4096, 64)
    finally:
        lib.aoclfftz_destroy(h)


def ragged(lib, sizes, dtype="f32"):
    import torch
    cd = np.complex64 if dtype == "f32" else np.complex128
    x = synthetic.complex_normal(5, sum(sizes), cd)
    din = torch.from_numpy(x.view(x.real.dtype).copy()).to("cuda")
    dout = torch.zeros_like(din)
    arr = (C.c_int64 * len(sizes))(*sizes)
    h = lib.aoclfftz_gpu_ragged_setup(0 if dtype == "f32" else 1, 0, len(sizes), arr, None, None)
    return h, x, din, dout


def test_ragged_dependency_wait_gives_up_and_is_reported_once(lib):
    """A ragged plan whose first dependent tile waits for one tile more than
    its predecessor has, with a short wait limit: the wait gives up, the
    executor finishes, synchronize reports the failure once (the flag is read
    and cleared), and a correct ragged plan then runs on the same GPU."""
    sizes = [65536, 1000, 97, 4096]  # 65536 runs as a multi-pass plan: tiles with dependencies
    assert lib.aoclfftz_gpu_inject_fault(abi.FAULT_RAGGED_WAIT, 2000) == 0
    assert lib.aoclfftz_gpu_inject_fault(abi.FAULT_RAGGED_DEP, 1) == 0
    h, x, din, dout = ragged(lib, sizes)
    assert lib.aoclfftz_gpu_inject_fault(abi.FAULT_RAGGED_DEP, 0) == 0
    assert h, lib.aoclfftz_gpu_last_error()
    try:
        assert lib.aoclfftz_gpu_ragged_execute(h, C.c_void_p(din.data_ptr()), C.c_void_p(dout.data_ptr())) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == abi.AOCLFFTZ_EXECUTION_FAILURE
        assert b"dependency wait gave up" in lib.aoclfftz_gpu_last_error()
        assert lib.aoclfftz_gpu_synchronize(h) == 0
    finally:
        lib.aoclfftz_destroy(h)
    assert lib.aoclfftz_gpu_inject_fault(abi.FAULT_NONE, 0) == 0
    h, x, din, dout = ragged(lib, sizes)
    assert h, lib.aoclfftz_gpu_last_error()
    try:
        assert lib.aoclfftz_gpu_ragged_execute(h, C.c_void_p(din.data_ptr()), C.c_void_p(dout.data_ptr())) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == 0, lib.aoclfftz_gpu_last_error()
        y = dout.cpu().numpy().view(np.complex64)
        off = 0
        for n in sizes:
            e = oracle.rel_l2(y[off:off + n], oracle.fft(x[off:off + n]))
            assert e <= oracle.tol(n, "f32"), (n, e)
            off += n
    finally:
        lib.aoclfftz_destroy(h)


def test_execute_io_from_two_threads_on_one_handle(lib):
    """Two host threads call aoclfftz_execute_io on one plan (a 2^20 four-step
    with plan scratch) with their own device buffers, 20 times each; one holds
    the plan's scratch per call, the other gets stream-ordered per-call
    scratch. Every result matches the FP64 oracle and is identical across
    iterations."""
    import torch
    n = 1 << 20
    h, x0, din0, dout0, keep = device_plan(lib, n, 1)
    assert h, lib.aoclfftz_gpu_last_error()
    bufs = []
    for t in range(2):
        x = synthetic.complex_uniform(40 + t, n, np.complex64)
        din = torch.from_numpy(x.view(np.float32).copy()).to("cuda")
        bufs.append((x, din, torch.zeros_like(din)))
    results = [[], []]
    errors = []

    def worker(t):
        try:
            x, din, dout = bufs[t]
            for _ in range(20):
                rc = lib.aoclfftz_execute_io(h, C.c_void_p(din.data_ptr()), C.c_void_p(dout.data_ptr()))
                if rc != 0:
                    errors.append((t, rc, lib.aoclfftz_gpu_last_error()))
                    return
                torch.cuda.synchronize()
                results[t].append(dout.cpu().numpy().copy())
        except Exception as e:  # surfaced in the main thread
            errors.append((t, repr(e)))

    try:
        th = [threading.Thread(target=worker, args=(t,)) for t in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join(timeout=300)
        assert not errors, errors
        for t in range(2):
            x = bufs[t][0]
            assert len(results[t]) == 20
            y = results[t][0].view(np.complex64)
            err = oracle.rel_l2(y, oracle.fft(x))
            assert err <= oracle.tol(n, "f32"), (t, err)
            for r in results[t][1:]:
                assert r.tobytes() == results[t][0].tobytes()
    finally:
        lib.aoclfftz_destroy(h)
