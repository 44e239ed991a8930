"""Host logic of the multi-GPU bench path on CPU: two gloo ranks.

Transforms are independent, so N GPUs run N replicas of the batch with no
collective on the data path; the only cross-rank steps are the barriers around
the timed region and the maximum of the step time over the ranks. These tests
run that reduction and the whole-job metric on world_size 2 with gloo, and
check that the reference arm prints nothing on ranks other than 0."""
import math
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (ws, rank, rank)
        # each rank times its own replica; the job's time is the slowest rank's
        ms = 1.0 + rank  # rank 1 is the slow one
        dist.barrier()
        got = bench.max_over_ranks(ms, ws, device="cpu")
        value, gbs = bench.step_metrics(4096, 1024, 8, ws, got)
        out.put((rank, got, value, gbs))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_metric_on_two_gloo_ranks():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(ws))
    flops = 2 * 1024 * 5.0 * 4096 * math.log2(4096) * ws
    for rank, got, value, gbs in res:
        assert got == 2.0  # every rank sees the maximum
        assert value == pytest.approx(flops / 2e-3 / 1e9)
        assert gbs == pytest.approx(2 * 1024 * 4096 * 2 * 8 * ws / 2e-3 / 1e9)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    v1, _ = bench.step_metrics(1 << 24, 4, 8, 1, 2.0)
    v2, _ = bench.step_metrics(1 << 24, 4, 8, 2, 2.0)
    assert v2 == pytest.approx(2 * v1)  # weak scaling: per-rank work is fixed


def test_reference_arm_is_silent_off_rank_zero(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class A:
        steps, warmup = 1, 0

    assert bench.run_reference(A(), dict(bench.WORKLOADS["fourstep24"])) is None
