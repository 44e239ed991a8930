"""Host-side logic of the autotuner and learned plan selector, on the CPU: the
seeded problem generator of the selector workload, the descriptors built for
its problems, the per-candidate feature vector and the regret arithmetic (the
network itself and the timings need the GPU and are tested in
test_gpu_mlp.py)."""
import math

import numpy as np
import pytest

from aoclfftz_b200 import selector, synthetic
from fftz_helpers import span


def _class_ok(n):
    return (n & (n - 1)) == 0 or synthetic._smooth7(n) or synthetic._is_prime(n)


def test_random_problems_are_seeded_and_within_the_workload():
    a = selector.random_problems(123, 200)
    b = selector.random_problems(123, 200)
    assert a == b
    assert a != selector.random_problems(124, 200)
    for p in a:
        dims = p["dims"]
        assert 1 <= len(dims) <= 3
        assert all(n >= 2 and _class_ok(n) for n in dims)
        assert int(np.prod(dims)) <= 1 << 22
        assert 1 <= p["batch"] <= 256
        assert p["batch"] * int(np.prod(dims)) <= 1 << 22
        assert p["kind"] in (0, 1, 2) and p["dtype"] in ("f32", "f64")
        if p["kind"] == 1:
            assert p["direction"] == 0  # r2c is forward
        if p["kind"] == 2:
            assert p["direction"] == 1  # c2r is backward
    kinds = {p["kind"] for p in a}
    ranks = {len(p["dims"]) for p in a}
    assert kinds == {0, 1, 2} and ranks == {1, 2, 3}


@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("strided", [False, True])
def test_descriptor_spans_fit_the_buffers(kind, strided):
    """The extents the descriptor declares (dims and batch, read back from the
    structure) lie inside the buffers sized for it, in scalars of each side."""
    p = dict(dims=[12, 10, 8], kind=kind, dtype="f32", strided=strided, batch=3, direction=1 if kind == 2 else 0)
    desc, keep, in_sc, out_sc = selector.descriptor(p, 0x1000, 0x2000)
    assert desc.dim_rank == 3 and desc.vec_rank == 1
    assert desc.flags.fft_type == (1 if kind else 0) and desc.flags.fft_direction == p["direction"]
    dims = [(desc.dims[i].n, desc.dims[i].in_stride, desc.dims[i].out_stride) for i in range(3)]
    vecs = [(desc.vecs[0].n, desc.vecs[0].in_stride, desc.vecs[0].out_stride)]
    assert [d[0] for d in dims] == p["dims"] and vecs[0][0] == 3
    h0 = p["dims"][0] // 2 + 1
    # scalars per element (complex 2, real 1) and the innermost extent of the
    # half-complex side (n0/2 + 1 bins)
    in_k = 1 if kind == 1 else 2
    out_k = 1 if kind == 2 else 2
    in_n0 = h0 if kind == 2 else None
    out_n0 = h0 if kind == 1 else None
    assert in_k * span(dims, vecs, "in", n0=in_n0) <= in_sc
    assert out_k * span(dims, vecs, "out", n0=out_n0) <= out_sc
    # strided layouts leave every other element unused on both sides
    if strided:
        assert dims[0][1] == 2 and dims[0][2] == 2


def test_features():
    p = dict(dims=[1024, 8], kind=1, dtype="f64", strided=True, batch=4, direction=0)
    passes = [("r2c n=1024 x32", 512, 32, 4), ("fast n=8 x2052", 8, 2052, 32)]
    f = selector.features(p, passes)
    assert f.shape == (selector.NBASE,) and f.dtype == np.float32
    assert f[0] == pytest.approx(math.log2(8192)) and f[1] == pytest.approx(2.0)
    assert (f[2], f[3], f[4]) == (10.0, 3.0, 0.0) and f[5] == 2
    assert (f[6], f[7], f[8], f[9]) == (1.0, 1.0, 0.0, 1.0)
    assert f[10] == 2
    assert f[11 + selector.KINDS.index("r2c")] == 1 and f[11 + selector.KINDS.index("fast")] == 1
    assert f[18] == pytest.approx(9.0) and f[19] == pytest.approx(3.0)
    assert f[22] == pytest.approx(math.log2(512 * 32 + 8 * 2052))
    assert f[23] == pytest.approx(math.log2(8192 * 4) + 3.0)
    assert np.array_equal(f, selector.features(p, passes))


class _Stub:
    def __init__(self, fn):
        self.fn = fn

    def predict(self, X):
        return self.fn(X)


def test_regret_report():
    # three problems, candidates (hints, text, features, ms); feature 0 carries the time
    times = [[2.0, 1.0, 4.0], [1.0, 3.0], [5.0, 5.0, 2.5]]
    data = [[({}, "", np.array([t], dtype=np.float32), t) for t in ts] for ts in times]
    oracle = selector.regret_report(_Stub(lambda X: np.log(X[:, 0])), data)
    assert oracle["mlp_regret_mean"] == pytest.approx(0.0)
    # planner default = the first candidate: regrets 1.0, 0.0, 1.0
    assert oracle["default_regret_mean"] == pytest.approx(2.0 / 3.0)
    worst = selector.regret_report(_Stub(lambda X: -X[:, 0]), data)
    assert worst["mlp_regret_mean"] == pytest.approx((3.0 + 2.0 + 1.0) / 3.0)
    assert worst["problems"] == 3
