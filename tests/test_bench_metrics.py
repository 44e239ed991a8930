"""The bench's metric arithmetic against the per-unit figures the workloads are
specified with (no GPU): flops and algorithmic bytes per direction of each
workload, and the rule that measured DRAM traffic is only reported for the
configuration it was captured on."""
import argparse
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_fourstep_and_batch_metrics():
    # c2c fp32 N = 2^24 batch 4: 8,053,063,680 flop and 1,073,741,824 bytes per direction
    gflops, gbs = bench.step_metrics(1 << 24, 4, 8, 1, 1.0)  # one step = 1 ms
    assert gflops * 1e9 * 1e-3 == pytest.approx(2 * 8053063680)
    assert gbs * 1e9 * 1e-3 == pytest.approx(2 * 1073741824)
    # c2c fp32 N = 4096 batch 1024: 251,658,240 flop and 67,108,864 bytes per direction
    gflops, gbs = bench.step_metrics(4096, 1024, 8, 1, 1.0)
    assert gflops * 1e6 == pytest.approx(2 * 251658240)
    assert gbs * 1e6 == pytest.approx(2 * 67108864)
    # whole-job figures grow with the ranks (weak scaling, same step time)
    assert bench.step_metrics(4096, 1024, 8, 4, 1.0)[0] == pytest.approx(4 * bench.step_metrics(4096, 1024, 8, 1, 1.0)[0])


def test_real3d_metrics():
    # fp64 512^3: 2.5 * 2^27 * 27 = 9,059,696,640 flop per direction and
    # 1,073,741,824 (reals) + 1,077,936,128 (257 x 512 x 512 complex) bytes
    gflops, gbs = bench.real3d_metrics((512, 512, 512), 1.0)
    assert gflops * 1e6 == pytest.approx(2 * 9059696640)
    assert gbs * 1e6 == pytest.approx(2 * (1073741824 + 1077936128))
    # fp64 256 x 256 x 1024: 2.5 * 2^26 * 26 flop, 2^29 + 513 * 65536 * 16 bytes per direction
    gflops, gbs = bench.real3d_metrics((256, 256, 1024), 1.0)
    assert gflops * 1e6 == pytest.approx(2 * 2.5 * 2 ** 26 * 26)
    assert gbs * 1e6 == pytest.approx(2 * (2 ** 29 + 513 * 65536 * 16))


def test_workload_table():
    w = bench.WORKLOADS
    assert w["fourstep24"]["n"] == 1 << 24 and w["fourstep24"]["batch"] == 4 and w["fourstep24"]["dtype"] == "f32"
    assert w["batch4096"]["n"] == 4096 and w["batch4096"]["batch"] == 1024
    for name in ("real3d512", "real3d_256x256x1024"):
        n2, n1, n0 = w[name]["real3d"]
        assert w[name]["n"] == n0 * n1 * n2 and w[name]["dtype"] == "f64"
    assert w["mixed1000"]["n"] == 1000 and w["mixed1000"]["batch"] * 1000 * 8 > 126e6  # larger than L2


def _args(**kw):
    a = argparse.Namespace(family=0, fourstep_n1=0, tpc_col=0, tpc_row=0, twiddles=0)
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def test_measured_traffic_only_for_the_captured_configuration():
    # per transform from the ncu capture, scaled by the transforms of a launch
    assert bench.measured_traffic("fourstep24", _args(), 0, 4) == round(4 * bench.TRAFFIC_PER_TRANSFORM[("fourstep24", 0)])
    assert bench.measured_traffic("fourstep24", _args(), 1, 1) == round(bench.TRAFFIC_PER_TRANSFORM[("fourstep24", 1)])
    # any planner hint or another workload: no traffic figure
    for kw in ({"family": 8}, {"tpc_col": 8}, {"tpc_row": 2}, {"fourstep_n1": 2048}, {"twiddles": 2}):
        assert bench.measured_traffic("fourstep24", _args(**kw), 0, 4) is None
    assert bench.measured_traffic("batch4096", _args(), 0, 1024) is None


def test_ragged_fp64_check_measures_each_transform():
    """The ragged line's FP64 check: exact outputs give errors at the dtype's
    rounding level; one output bin off by 1e-3 of its transform's norm shows
    up as that transform's error above its own bound."""
    import numpy as np
    sizes = [5, 16, 7, 1, 1024, 97, 2, 331]
    offs = np.cumsum([0] + sizes[:-1])
    rng = np.random.default_rng(3)
    x = (rng.standard_normal(sum(sizes)) + 1j * rng.standard_normal(sum(sizes))).astype(np.complex64)
    y = np.concatenate([np.fft.fft(x[o:o + n].astype(np.complex128)).astype(np.complex64)
                        for o, n in zip(offs, sizes)])
    ok = bench.ragged_fp64_check(sizes, offs, x, y, "f32", every=1)
    assert ok["rel_l2"] < 1e-6 and ok["worst_err_over_bound"] < 1.0
    bad = y.copy()
    o, n = int(offs[5]), sizes[5]
    bad[o + 3] += 1e-3 * np.linalg.norm(y[o:o + n])
    res = bench.ragged_fp64_check(sizes, offs, x, bad, "f32", every=1)
    assert res["worst_transform"]["n"] == 97 and res["worst_err_over_bound"] > 100


def test_real3d_fp64_check_against_exact_sums():
    """The real 3-D line's FP64 check: numpy's FP64 rfftn passes at rounding
    level; a perturbed bin in the sub-block is caught."""
    import numpy as np
    x = np.random.default_rng(4).standard_normal((16, 8, 32))
    F = np.fft.rfftn(x)
    k0 = np.arange(0, 17)
    k1 = (np.arange(8) * 7 + 3) % 8
    k2 = (np.arange(16) * 11 + 5) % 16
    got = F[k2][:, k1][:, :, k0]
    ok = bench.real3d_fp64_check(x, got, k0, k1, k2)
    assert ok["rel_l2"] < ok["bound"]
    got[2, 3, 4] += 1e-6 * np.abs(got).max()
    assert bench.real3d_fp64_check(x, got, k0, k1, k2)["rel_l2"] > ok["bound"]
