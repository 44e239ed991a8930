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


def test_codelet_costs_follow_the_reference_tables():
    """codelet_cost weighs the reference's per-call operation counts (fma,
    mul, add, move, perm, other) by its cycle weights 4, 3, 1, 1, 1, 1: e.g.
    the plain radix-16 codelet {0, 24, 144, 64, 0, 0} -> 280, the twiddled
    one {0, 84, 174, 94, 0, 0} -> 520, the plain radix-2 {0, 0, 4, 8, 0, 0} -> 12."""
    assert selector.codelet_cost(16, True) == 280
    assert selector.codelet_cost(16, False) == 520
    assert selector.codelet_cost(2, True) == 12
    assert selector.codelet_cost(5, False) == 28 * 3 + 40 + 28
    for R in (2, 3, 4, 5, 7, 8, 11, 13, 16):
        # a twiddled call never costs less than the plain one
        assert selector.codelet_cost(R, False) > selector.codelet_cost(R, True)


def test_opcount_cost_of_plans():
    """Per line: n / R_s calls of stage s's codelet, the plain one first;
    linear in the number of lines; a line with no radix split (Bluestein)
    counts its power-of-two convolution twice; elementwise passes 2 n."""
    c16, t16 = selector.codelet_cost(16, True), selector.codelet_cost(16, False)
    one = selector.opcount_cost([("fast", 4096, 1, 1)])
    assert one == 256 * c16 + 2 * 256 * t16
    assert selector.opcount_cost([("fast", 4096, 7, 1)]) == 7 * one
    # 1000 = 8 * 5 * 5 * 5
    c8, t5 = selector.codelet_cost(8, True), selector.codelet_cost(5, False)
    assert selector.opcount_cost([("generic", 1000, 1, 4)]) == 125 * c8 + 3 * 200 * t5
    # prime 1009: m = 2048 = 16 * 16 * 8, twice
    c2048 = 128 * c16 + 128 * t16 + 256 * selector.codelet_cost(8, False)
    assert selector.opcount_cost([("bluestein", 1009, 3, 1)]) == 2 * 3 * c2048
    assert selector.opcount_cost([("elem", 500, 4, 1)]) == 2 * 500 * 4
    # a four-step (two passes) costs more arithmetic than one pass of the same length
    assert selector.opcount_cost([("fast", 64, 64, 1), ("fast", 64, 64, 1)]) > 0


def test_selector_database_layout():
    """The committed autotuner database: 20000 training and 2000 held-out
    problems (seeded draws, so a few repeat within a split) whose problem
    descriptions are disjoint between the splits, every row a distinct plan
    with its candidate's one-hot, a positive median time and op cost."""
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "selector_timings.npz")
    train, test, train_oc, test_oc = selector.load_timings(path)
    assert len(train) == 20000 and len(test) == 2000
    nf = selector.NBASE + len(selector.CANDIDATES)
    for groups, costs in ((train, train_oc), (test, test_oc)):
        for g, c in zip(groups[:500], costs[:500]):
            assert len(g) == len(c) >= 1
            for (_, _, f, ms), oc in zip(g, c):
                assert f.shape == (nf,) and ms > 0 and oc > 0
                assert f[selector.NBASE:].sum() == 1.0
    d = np.load(path)
    probs = json.loads(bytes(d["problems"]).decode())
    u, first = np.unique(d["problem"], return_index=True)
    sp = d["split"][first]
    assert (sp == 0).sum() == 20000 and (sp == 1).sum() == 2000
    tr = {json.dumps(probs[i], sort_keys=True) for i in u[sp == 0]}
    te = {json.dumps(probs[i], sort_keys=True) for i in u[sp == 1]}
    assert not (tr & te)
