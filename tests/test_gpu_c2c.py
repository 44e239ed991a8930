"""GPU parity of complex transforms, through the C ABI (aoclfftz_setup_* /
aoclfftz_execute), against the FP64 oracle and the reference library's own
output on the same seeded inputs.

Bound (written here, used by every case): rel-L2 <= 4 * log2(N) * eps of the
working dtype, N = product of the transform dims; eps = 2^-23 (f32), 2^-52 (f64).
Cases follow the reference's test design: every radix and the pow2 iterative,
four-step, Cooley-Tukey and Bluestein paths (test/bench/CMakeLists.txt:55-124),
strided and batched layouts, in- and out-of-place, both directions.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from aoclfftz_b200 import synthetic
from fftz_helpers import cplx_dtype, gather, run_gpu, scatter, span

pytestmark = pytest.mark.gpu


def oracle_c2c(x, rank, sign):
    y = np.asarray(x, dtype=np.complex128)
    for k in range(rank):
        ax = y.ndim - 1 - k
        y = np.moveaxis(oracle.fft(np.moveaxis(y, ax, -1), sign=sign), -1, ax)
    return y


def bound(dims, dtype):
    N = int(np.prod([d[0] for d in dims]))
    return oracle.tol(N, dtype)


def check_c2c(dtype, dims, vecs, direction=0, placement=1, seed=1, host=False, compare_ref=True, ilp64=False,
              pinned=False):
    rank = len(dims)
    lshape = [v[0] for v in reversed(vecs)] + [d[0] for d in reversed(dims)]
    total = int(np.prod(lshape))
    x = synthetic.complex_uniform(seed, total, cplx_dtype(dtype)).reshape(lshape)
    in_sc = 2 * span(dims, vecs, "in")
    out_sc = 2 * span(dims, vecs, "out")
    raw_in = scatter(x, [(d[0], d[1]) for d in dims], [(v[0], v[1]) for v in vecs], in_sc, dtype)
    out_raw, plan = run_gpu(dtype, dims, vecs, raw_in, out_sc, 0, direction, placement, host=host, ilp64=ilp64,
                            pinned=pinned)
    y = gather(out_raw, [(d[0], d[2]) for d in dims], [(v[0], v[2]) for v in vecs], dtype)
    ref = oracle_c2c(x, rank, -1 if direction == 0 else +1)
    err = oracle.rel_l2(y, ref)
    assert err <= bound(dims, dtype), "rel-L2 %.3e > %.3e vs FP64 oracle; plan: %s" % (err, bound(dims, dtype), plan)
    if compare_ref and oracle.ref_available():
        r_raw = oracle.ref_execute(dtype, dims, vecs, raw_in, out_sc, 0, direction, placement)
        r = gather(r_raw, [(d[0], d[2]) for d in dims], [(v[0], v[2]) for v in vecs], dtype)
        # both sides carry rounding error of the working dtype: compare with twice the bound
        e2 = oracle.rel_l2(y, r)
        lim = 2 * bound(dims, dtype) + oracle.rel_l2(r, ref)
        assert e2 <= lim, "rel-L2 %.3e vs reference library; plan: %s" % (e2, plan)
    return err, plan


POW2 = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192]


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", POW2)
@pytest.mark.parametrize("direction", [0, 1])
def test_pow2_contiguous_batch(dtype, n, direction):
    b = 3
    check_c2c(dtype, [(n, 1, 1)], [(b, n, n)], direction)


def test_pow2_16384_f32():
    check_c2c("f32", [(16384, 1, 1)], [(2, 16384, 16384)], 0)
    check_c2c("f32", [(16384, 1, 1)], [(2, 16384, 16384)], 1)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [3, 5, 6, 7, 9, 10, 11, 12, 13, 15, 24, 49, 60, 100, 121, 169, 210, 1000, 1155, 2310])
def test_mixed_radix(dtype, n):
    check_c2c(dtype, [(n, 1, 1)], [(4, n, n)], 0)
    check_c2c(dtype, [(n, 1, 1)], [(2, n, n)], 1)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [17, 19, 97, 127, 251, 1009, 4099])
def test_bluestein_one_kernel(dtype, n):
    check_c2c(dtype, [(n, 1, 1)], [(3, n, n)], 0)
    check_c2c(dtype, [(n, 1, 1)], [(2, n, n)], 1)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [32768, 65536, 3 ** 10, 2 ** 10 * 3 ** 5])
def test_fourstep(dtype, n):
    check_c2c(dtype, [(n, 1, 1)], [(2, n, n)], 0)
    check_c2c(dtype, [(n, 1, 1)], [(1, n, n)], 1)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_bluestein_multipass(dtype):
    n = 65521  # largest prime below 2^16: m = 2^17 needs the four-pass form
    check_c2c(dtype, [(n, 1, 1)], [(1, n, n)], 0)
    check_c2c(dtype, [(n, 1, 1)], [(1, n, n)], 1)


def test_strided_and_inplace():
    # element stride 3, batch stride 1 (column-major batches), in and out of place
    n, b = 256, 3
    check_c2c("f32", [(n, b, b)], [(b, 1, 1)], 0)
    check_c2c("f64", [(n, b, b)], [(b, 1, 1)], 1, placement=0)
    check_c2c("f32", [(100, 2, 3)], [(5, 300, 400)], 0)
    check_c2c("f64", [(64, 1, 1)], [(4, 70, 70)], 0, placement=0)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_multidim(dtype):
    check_c2c(dtype, [(16, 1, 1), (8, 16, 16)], [(2, 128, 128)], 0)
    check_c2c(dtype, [(16, 1, 1), (16, 16, 16), (16, 256, 256)], [(1, 4096, 4096)], 1)
    check_c2c(dtype, [(5, 1, 1), (6, 5, 5), (7, 30, 30)], [(3, 210, 210)], 0)
    check_c2c(dtype, [(32, 1, 1), (17, 32, 32)], [(2, 544, 544)], 0, placement=0)


def test_host_buffers_and_ilp64():
    check_c2c("f32", [(1024, 1, 1)], [(8, 1024, 1024)], 0, host=True)
    check_c2c("f64", [(100, 1, 1)], [(3, 100, 100)], 1, host=True, placement=0)
    check_c2c("f64", [(512, 1, 1)], [(2, 512, 512)], 0, ilp64=True)


def test_pinned_host_buffers_pipelined():
    """Page-locked host buffers take the chunked copy-in / passes / copy-out
    pipeline (three streams); results must match the oracle exactly as the
    device path does. Four-step lines (2^18 f64, 2^22 and 2^24 f32) run their
    last pass in blocks of columns, each copied out behind it."""
    check_c2c("f32", [(4096, 1, 1)], [(64, 4096, 4096)], 0, host=True, pinned=True, compare_ref=False)
    check_c2c("f32", [(1 << 22, 1, 1)], [(3, 1 << 22, 1 << 22)], 0, host=True, pinned=True, compare_ref=False)
    check_c2c("f32", [(1 << 24, 1, 1)], [(2, 1 << 24, 1 << 24)], 1, host=True, pinned=True, compare_ref=False)
    check_c2c("f64", [(1 << 18, 1, 1)], [(4, 1 << 18, 1 << 18)], 1, host=True, pinned=True, compare_ref=False)
    check_c2c("f32", [(100, 1, 1)], [(48, 130, 100)], 0, host=True, pinned=True)
    check_c2c("f64", [(256, 1, 1)], [(12, 256, 256)], 1, placement=0, host=True, pinned=True)
    check_c2c("f32", [(16, 1, 1), (8, 16, 16)], [(6, 128, 128)], 0, host=True, pinned=True)


def test_size_one_and_empty_batch():
    check_c2c("f32", [(1, 1, 1)], [(5, 1, 1)], 0)
    check_c2c("f64", [(1, 1, 1), (8, 1, 1)], [(2, 8, 8)], 0)


def test_config1_shape():
    """The plain c2c workload's shape: 4096-point fp32 transforms, batch 1024,
    out of place, forward then backward, against the FP64 oracle and the
    reference library run on the same seeded inputs."""
    n, b = 4096, 1024
    check_c2c("f32", [(n, 1, 1)], [(b, n, n)], 0)
    check_c2c("f32", [(n, 1, 1)], [(b, n, n)], 1)


def test_config2_transform_against_reference():
    """One transform of the four-step workload: fp32 N = 2^24 (4096 x 4096),
    out of place, both directions, against the FP64 oracle and the reference
    library's own four-step run on the same seeded input."""
    n = 1 << 24
    check_c2c("f32", [(n, 1, 1)], [(1, n, n)], 0)
    check_c2c("f32", [(n, 1, 1)], [(1, n, n)], 1, seed=2)


def test_bit_reproducible():
    """Ten executions give byte-identical output (the reference's
    test/test_bit_repro.c procedure, compared with memcmp semantics)."""
    n = 4096
    x = synthetic.complex_uniform(7, 16 * n, np.complex64)
    outs, _ = run_gpu("f32", [(n, 1, 1)], [(16, n, n)], x, 2 * 16 * n, repeat=10)
    for o in outs[1:]:
        assert o.tobytes() == outs[0].tobytes()
    x = synthetic.complex_uniform(8, 4 * 65521, np.complex128)
    outs, _ = run_gpu("f64", [(65521, 1, 1)], [(4, 65521, 65521)], x, 2 * 4 * 65521, repeat=3)
    for o in outs[1:]:
        assert o.tobytes() == outs[0].tobytes()

@pytest.mark.parametrize("family", [5, 6])
@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n,batch", [(1 << 16, 3), (1 << 20, 2), (1 << 24, 1), (4096, 64), (1024, 40)])
def test_tma_fed_passes(dtype, n, batch, family):
    """Kernel families 5 (tiles fetched by TMA copies) and 6 (persistent CTAs,
    half of the next tile prefetched by TMA during the current one) against
    the oracle, both directions; the four-step passes qualify for column and
    row TMA boxes."""
    if dtype == "f64" and n == 1 << 24:
        n = 1 << 22
    import aoclfftz_b200
    from aoclfftz_b200 import abi
    lib = aoclfftz_b200.load()
    h = abi.Hints()
    h.kernel_family = family
    lib.aoclfftz_gpu_set_hints(C.byref(h))
    try:
        for d in (0, 1):
            if n >= 1 << 20:
                check_c2c(dtype, [(n, 1, 1)], [(batch, n, n)], d, compare_ref=False)
            else:
                check_c2c(dtype, [(n, 1, 1)], [(batch, n, n)], d)
    finally:
        lib.aoclfftz_gpu_set_hints(None)


@pytest.mark.parametrize("n,batch,want", [(1 << 24, 1, 2), (1 << 23, 2, 1), (4096, 64, 1), (4096, 1001, 1),
                                          (1 << 20, 3, 0)])
def test_register_resident_prefetch(n, batch, want):
    """Kernel family 8: 4096-point float passes as persistent CTAs that keep
    the tile in registers and prefetch the whole next tile by TMA. Four-step
    2^24 runs both passes that way (column pass with the four-step twiddle,
    row pass with the transposed store), 2^23 its 4096-point column pass,
    plain 4096-point rows one transform per CTA; 2^20 (1024 x 1024) does not
    qualify and keeps the default kernels. Against the oracle, both
    directions."""
    import aoclfftz_b200
    from aoclfftz_b200 import abi
    lib = aoclfftz_b200.load()
    h = abi.Hints()
    h.kernel_family = 8
    lib.aoclfftz_gpu_set_hints(C.byref(h))
    try:
        for d in (0, 1):
            _, plan = check_c2c("f32", [(n, 1, 1)], [(batch, n, n)], d, compare_ref=n < (1 << 20))
            assert plan.count("tma-prefetch") == want, plan
    finally:
        lib.aoclfftz_gpu_set_hints(None)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n,batch", [(1 << 20, 2), (4096, 64), (512, 100)])
def test_shared_memory_twiddles(dtype, n, batch):
    """Hint twiddles = 2: compile-time passes of >= 512 points read their stage
    twiddles from a shared-memory copy; results against the oracle."""
    import aoclfftz_b200
    from aoclfftz_b200 import abi
    lib = aoclfftz_b200.load()
    h = abi.Hints()
    h.twiddles = 2
    lib.aoclfftz_gpu_set_hints(C.byref(h))
    try:
        for d in (0, 1):
            check_c2c(dtype, [(n, 1, 1)], [(batch, n, n)], d, compare_ref=n < (1 << 20))
    finally:
        lib.aoclfftz_gpu_set_hints(None)



@pytest.mark.parametrize("family,tag", [(9, "tma-split"), (10, "tma-split2"), (11, "tma-split3")])
@pytest.mark.parametrize("n,batch,want", [(1 << 24, 1, 2), (1 << 24, 2, 2), (1 << 23, 2, 1), (4096, 64, 1),
                                          (4096, 1001, 0), (1 << 20, 3, 0)])
def test_split_tiles(family, tag, n, batch, want):
    """Kernel families 9 and 10: 4096-point float passes as 16 x 256 split
    tiles (persistent CTAs, the 64 sub-transforms of a tile in 16-lane groups,
    one exchange across the CTA; 9 exchanges one real component at a time, 10
    full complex values in two rounds with a shared-memory stash, 11 the same
    with the stash in tensor memory). Four-step 2^24 runs both passes that
    way (column tiles with the four-step twiddle, row tiles with the
    transposed store), 2^23 its 4096-point column pass, plain 4096-point rows
    as row tiles with row stores; 1001 rows do not form whole tiles and take
    the register-resident kernel; 2^20 does not qualify. Against the oracle,
    both directions."""
    import aoclfftz_b200
    from aoclfftz_b200 import abi
    lib = aoclfftz_b200.load()
    h = abi.Hints()
    h.kernel_family = family
    lib.aoclfftz_gpu_set_hints(C.byref(h))
    try:
        for d in (0, 1):
            _, plan = check_c2c("f32", [(n, 1, 1)], [(batch, n, n)], d, compare_ref=n < (1 << 20))
            assert plan.count(tag + "]") == want, plan
    finally:
        lib.aoclfftz_gpu_set_hints(None)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n,batch,rs", [(4096, 1024, 0), (4096, 37, 0), (1024, 300, 0), (256, 512, 0),
                                        (8192, 20, 0), (2048, 50, 2), (2048, 50, 1), (1 << 20, 2, 0),
                                        (1 << 24, 1, 0)])
def test_streaming_row_tiles(dtype, n, batch, rs):
    """Kernel family 13: row passes over contiguous lines as persistent
    streaming tiles (each line by one 1-D bulk copy into one of two slots,
    the next tile in flight). Rows `rs` elements apart beyond n: 0 dense, 2
    still 16-byte aligned (f32), 1 not aligned for f32 (the pass runs on the
    one-tile kernel instead). Four-step sizes run their row pass (transposed
    store) this way. Against the oracle and the reference, both directions."""
    if dtype == "f64" and n == 1 << 24:
        n = 1 << 22
    import aoclfftz_b200
    from aoclfftz_b200 import abi
    lib = aoclfftz_b200.load()
    h = abi.Hints()
    h.kernel_family = 13
    lib.aoclfftz_gpu_set_hints(C.byref(h))
    try:
        for d in (0, 1):
            _, plan = check_c2c(dtype, [(n, 1, 1)], [(batch, n + rs, n + rs)], d, compare_ref=n < (1 << 20))
            assert "tma-stream" in plan, plan
    finally:
        lib.aoclfftz_gpu_set_hints(None)


def test_streaming_rows_in_place():
    """Family 13 in place: every tile is staged before its lines are
    overwritten; against the oracle."""
    import aoclfftz_b200
    from aoclfftz_b200 import abi
    lib = aoclfftz_b200.load()
    h = abi.Hints()
    h.kernel_family = 13
    lib.aoclfftz_gpu_set_hints(C.byref(h))
    try:
        for dtype in ("f32", "f64"):
            check_c2c(dtype, [(4096, 1, 1)], [(333, 4096, 4096)], 0, placement=0)
    finally:
        lib.aoclfftz_gpu_set_hints(None)


def test_blocked_fourstep_intermediate_and_unaligned_input():
    """The 2^24 four-step on split tiles keeps its intermediate in 4 x 4
    blocks (both passes marked blk4). An execute whose input is 8 bytes off a
    16-byte boundary cannot feed the column pass by TMA: it runs both passes
    on the plain layout instead, with the same result. Both against the FP64
    oracle."""
    import torch
    import aoclfftz_b200
    from aoclfftz_b200 import abi
    lib = aoclfftz_b200.load()
    n = 1 << 24
    x = synthetic.complex_uniform(9, n, np.complex64)
    ref = oracle.fft(x.astype(np.complex128))
    din = torch.zeros(2 * n + 2, dtype=torch.float32, device="cuda")
    dout = torch.zeros(2 * n, dtype=torch.float32, device="cuda")
    desc, keep = abi.make_desc(din.data_ptr(), dout.data_ptr(), [(n, 1, 1)], [(1, n, n)], 0, 0, 1)
    h = abi.setup(lib, desc, "f32")
    assert h, lib.aoclfftz_gpu_last_error()
    try:
        txt = C.create_string_buffer(2048)
        lib.aoclfftz_gpu_describe(h, txt, 2048)
        assert txt.value.count(b"blk4") == 2, txt.value
        for off in (0, 2):  # floats: 0 aligned, 2 = 8 bytes off
            din.zero_()
            din[off:off + 2 * n] = torch.from_numpy(x.view(np.float32)).to("cuda")
            dout.zero_()
            rc = lib.aoclfftz_execute_io(h, C.c_void_p(din.data_ptr() + 4 * off), C.c_void_p(dout.data_ptr()))
            assert rc == 0, lib.aoclfftz_gpu_last_error()
            assert lib.aoclfftz_gpu_synchronize(h) == 0
            y = dout.cpu().numpy().view(np.complex64)
            err = oracle.rel_l2(y, ref)
            assert err <= oracle.tol(n, "f32"), (off, err)
    finally:
        lib.aoclfftz_destroy(h)
