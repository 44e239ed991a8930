#!/usr/bin/env python3
"""Benchmark of the FFT plan-execution path on B200.

Default workload (one step = forward then backward, unnormalised):
  c2c fp32, N = 2^24 = 4096 x 4096 (four-step: two passes through HBM),
  batch 4, out of place; inputs re, im i.i.d. U[-1, 1) from a seed.
Other workloads (--workload): "batch4096" (N = 4096, batch 1024, one pass);
"mixed1000" (N = 1000 = 2^3 5^3, batch 32768, the mixed-radix kernel);
"ragged" / "ragged_f64" (4096 transforms of lengths in [2, 65536] in one
persistent launch); "real3d512" / "real3d_256x256x1024" (fp64 real 3-D, in
place, r2c then c2r, 2.5 N log2 N per direction); "selector" (regret of the
learned plan selector).

Metric: 5 N log2(N) GFLOP/s over all transforms of the step (both directions),
plus HBM GB/s. `value` is measured with inputs resident in HBM; `e2e` runs the
same step through the public C ABI with pinned host buffers (the library
stages them: copy in, transform, copy out). `roofline` describes the dominant
kernel, timed with CUDA events on the plan's stream during the timed region.
`cpu_baseline` times the reference library (built from its sources, OpenMP)
on a bounded sample on this host's cores. `fp64_oracle` states the error of
the timed run's own forward outputs against the FP64 oracle. `copy_ceiling`
(c2c workloads) times plain device copies of the same bytes over the same
buffer rotation: the bandwidth a pass of this size can reach.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun, one process per GPU): every rank runs its own batch
(weak scaling, no collective on the data path); the time is the max over ranks.
"""
import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "aocl-fftz_b200", "python"))

WORKLOADS = {
    "fourstep24": dict(n=1 << 24, batch=4, dtype="f32",
                       desc="c2c fp32 N=2^24 (4096x4096 four-step) batch 4, out-of-place, fwd+bwd"),
    "batch4096": dict(n=4096, batch=1024, dtype="f32",
                      desc="c2c fp32 N=4096 batch 1024, out-of-place, fwd+bwd"),
    "ragged": dict(n=0, batch=4096, dtype="f32", ragged=True,
                   desc="ragged batch of 4096 c2c fp32 transforms, lengths log-uniform in [2, 65536] "
                        "(pow2 / 7-smooth / prime thirds), packed, one persistent launch under a CUDA graph, fwd+bwd"),
    "selector": dict(n=0, batch=0, dtype="mixed", selector=True,
                     desc="learned plan selector: seeded problems (rank 1-3, pow2 / 7-smooth / prime dims, "
                          "c2c/r2c/c2r, f32/f64, unit or strided, batch 1-256, <= 2^22 elements); 2x64 MLP "
                          "trained on the autotuner timings of 20000 problems, regret against exhaustive "
                          "autotuning on 2000 held-out problems (and on fresh problems timed live)"),
    "mixed1000": dict(n=1000, batch=32768, dtype="f32",
                      desc="c2c fp32 N=1000 (2^3 5^3, mixed radix) batch 32768, out-of-place, fwd+bwd"),
    "real3d512": dict(n=512 ** 3, batch=1, dtype="f64", real3d=(512, 512, 512),
                      desc="r2c then c2r fp64 512^3 (FFTW order), in place, innermost rows padded to "
                           "2 (n0/2 + 1) reals, batch 1"),
    "real3d_256x256x1024": dict(n=256 * 256 * 1024, batch=1, dtype="f64", real3d=(256, 256, 1024),
                                desc="r2c then c2r fp64 256 x 256 x 1024 (FFTW order), in place, innermost rows "
                                     "padded to 2 (n0/2 + 1) reals, batch 1"),
    "ragged_f64": dict(n=0, batch=4096, dtype="f64", ragged=True,
                       desc="ragged batch of 4096 c2c fp64 transforms, lengths log-uniform in [2, 65536] "
                            "(pow2 / 7-smooth / prime thirds), packed, one persistent launch under a CUDA graph, "
                            "fwd+bwd"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="fourstep24", choices=sorted(WORKLOADS))
    ap.add_argument("--batch", type=int, default=0, help="override the workload's batch (small profiling cases)")
    ap.add_argument("--fourstep-n1", type=int, default=0, help="planner hint: column length of the split")
    ap.add_argument("--tpc-col", type=int, default=0, help="planner hint: transforms per CTA, column passes")
    ap.add_argument("--tpc-row", type=int, default=0, help="planner hint: transforms per CTA, row passes")
    ap.add_argument("--family", type=int, default=0,
                    help="planner hint: 1 plain tiles, 2 persistent, 5 TMA-fed tiles, 6 persistent half-tile TMA "
                         "prefetch, 7 tensor-core rows, 8 register-resident 4096-point passes everywhere")
    ap.add_argument("--twiddles", type=int, default=0, help="planner hint: 1 global, 2 shared-memory stage twiddles")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--selector-db", default="", help="autotuner timing database of --workload selector "
                                                      "(default: tests/golden/selector_timings.npz)")
    return ap.parse_args()


L2_BYTES = 126 * 1000 * 1000  # B200 L2

# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# default kernels, from one ncu capture of one 2^24-point transform
# (profiles/fourstep24_split_passes_ncu.txt: pass A 212.0 MB, pass B 217.3 MB),
# scaled to a launch over `batch` transforms (the traffic grows with them).
TRAFFIC_PER_TRANSFORM = {("fourstep24", 0): 212.0e6, ("fourstep24", 1): 217.3e6}


def measured_traffic(workload, args, pass_in_direction, batch):
    """ncu-measured DRAM bytes of the dominant launch, or None when the run
    differs from the captured configuration (hints, other workloads)."""
    if args.family or args.fourstep_n1 or args.tpc_col or args.tpc_row or args.twiddles:
        return None
    t = TRAFFIC_PER_TRANSFORM.get((workload, pass_in_direction))
    return None if t is None else round(t * batch)


def max_over_ranks(x, ws, device="cuda"):
    """The largest value of x over all ranks (x itself on a single rank); every
    rank must call it at the same point."""
    if ws <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def step_metrics(n, batch_per_rank, esz, ws, ms):
    """Whole-job 5N log2N GFLOP/s and algorithmic HBM GB/s of one fwd+bwd step
    over ws ranks, each transforming batch_per_rank length-n lines, given the
    step time in ms (the maximum over ranks)."""
    flops = 2 * batch_per_rank * 5.0 * n * math.log2(n) * ws
    alg_bytes = 2 * batch_per_rank * n * 2 * esz * ws  # each direction reads and writes the batch once
    return flops / (ms * 1e-3) / 1e9, alg_bytes / (ms * 1e-3) / 1e9


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """SM clock and throttle reasons sampled during a region: NVML every 2 ms
    (the device found by its PCI bus id), else nvidia-smi every 100 ms.
    Reading only; no GPU setting is changed."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.nv = None
        self.lines = []
        self.samples = []
        self.run = False

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.gpu)
        bus = "%08X:%02X:%02X.0" % (getattr(pr, "pci_domain_id", 0), pr.pci_bus_id, pr.pci_device_id)
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def start(self):
        try:
            self.nv, self.h = self._nvml_handle()
            self.smax = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            self.run = True
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _poll(self):
        nv, h = self.nv, self.h
        get_r = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while self.run:
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(get_r(h))))
            except Exception:
                pass
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nv is not None:
            self.run = False
            self.t.join(timeout=2)
            sm = sorted(c for c, _ in self.samples)
            reasons = sorted({nm for _, r in self.samples for nm, b in self.BITS.items() if r & b})
            return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
                    "samples": len(sm), "sm_mhz_min": sm[0] if sm else None, "source": "NVML, 2 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi, 100 ms"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def make_plan(lib, abi, pin, pout, n, batch, direction, dtype):
    desc, keep = abi.make_desc(pin, pout, [(n, 1, 1)], [(batch, n, n)], 0, direction, 1)
    h = abi.setup(lib, desc, dtype)
    if not h:
        raise RuntimeError("setup failed: %s" % lib.aoclfftz_gpu_last_error().decode())
    return h


def pass_table(lib, h):
    out = []
    k = lib.aoclfftz_gpu_num_launches(h)
    for i in range(k):
        buf = C.create_string_buffer(128)
        ei, eo = C.c_int64(), C.c_int64()
        lib.aoclfftz_gpu_pass_info(h, i, buf, 128, C.byref(ei), C.byref(eo))
        out.append((buf.value.decode(), ei.value, eo.value))
    return out


def run_ours(args, wl):
    import numpy as np
    import torch

    import aoclfftz_b200
    from aoclfftz_b200 import abi, synthetic

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    lib = aoclfftz_b200.load()
    n, b, dtype = wl["n"], wl["batch"], wl["dtype"]
    esz = 8 if dtype == "f32" else 16
    total = n * b
    x = synthetic.complex_uniform(1234 + rank, total, np.complex64 if dtype == "f32" else np.complex128)
    real = x.view(np.float32 if dtype == "f32" else np.float64)
    hx = torch.from_numpy(real).pin_memory()
    # inputs smaller than L2 rotate through enough buffer sets (input,
    # intermediate, output) that a set has left the 126 MB L2 before it is
    # used again: every step reads and writes HBM
    set_bytes = 3 * total * esz
    nsets = 1 if set_bytes >= 3 * L2_BYTES else -(-3 * L2_BYTES // set_bytes)
    sets = []
    for _ in range(nsets):
        sets.append((hx.to("cuda"), torch.empty(2 * total, dtype=hx.dtype, device="cuda"),
                     torch.empty(2 * total, dtype=hx.dtype, device="cuda")))
    dx, dy, dz = sets[0]
    stream = torch.cuda.Stream()
    hints = abi.Hints()
    hints.fourstep_n1, hints.tpc_col, hints.kernel_family = args.fourstep_n1, args.tpc_col, args.family
    hints.tpc_row = args.tpc_row
    hints.twiddles = args.twiddles
    lib.aoclfftz_gpu_set_hints(C.byref(hints))
    pf = make_plan(lib, abi, dx.data_ptr(), dy.data_ptr(), n, b, 0, dtype)
    pb = make_plan(lib, abi, dy.data_ptr(), dz.data_ptr(), n, b, 1, dtype)
    for h in (pf, pb):
        lib.aoclfftz_gpu_set_stream(h, C.c_void_p(stream.cuda_stream))

    cur = [0]

    def step():
        a, b_, c = sets[cur[0]]
        cur[0] = (cur[0] + 1) % nsets
        if (lib.aoclfftz_execute_io(pf, C.c_void_p(a.data_ptr()), C.c_void_p(b_.data_ptr())) or
                lib.aoclfftz_execute_io(pb, C.c_void_p(b_.data_ptr()), C.c_void_p(c.data_ptr()))):
            raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3, nsets)):
            step()
    torch.cuda.synchronize()
    # untimed soak (about half a second of steps) with its own clock record
    soak = ClockSampler(local)
    soak.start()
    t_soak = time.perf_counter()
    with torch.cuda.stream(stream):
        while time.perf_counter() - t_soak < 0.5:
            for _ in range(8):
                step()
            torch.cuda.synchronize()
    clk_soak = soak.stop()
    cur[0] = 0
    # correctness of the round trip on this run's data: z = N x
    zc = dz.view(torch.complex64 if dtype == "f32" else torch.complex128)
    xc = dx.view(zc.dtype)
    rt_err = (torch.linalg.vector_norm(zc / n - xc) / torch.linalg.vector_norm(xc)).item()

    K = args.steps
    lib.aoclfftz_gpu_profile_begin(pf, K)
    lib.aoclfftz_gpu_profile_begin(pb, K)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(K):
            step()
    e1.record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    npf, npb = lib.aoclfftz_gpu_num_launches(pf), lib.aoclfftz_gpu_num_launches(pb)
    tf = (C.c_float * 16)()
    tb = (C.c_float * 16)()
    lib.aoclfftz_gpu_profile_end(pf, tf, 16)
    lib.aoclfftz_gpu_profile_end(pb, tb, 16)
    ms_total = max_over_ranks(ms_total, ws)
    ms = ms_total / K
    value, hbm_gbs = step_metrics(n, b, esz, ws, ms)
    # forward outputs of the first and last transform (set 0) for the FP64 check
    cdt = np.complex64 if dtype == "f32" else np.complex128
    y0 = dy.cpu().numpy().view(cdt)
    fwd_check = (n, dtype, x[:n].copy(), y0[:n].copy(), x[(b - 1) * n:].copy(), y0[(b - 1) * n:].copy())

    # dominant kernel: the pass with the largest summed time
    passes = [("fwd",) + p for p in pass_table(lib, pf)] + [("bwd",) + p for p in pass_table(lib, pb)]
    times = [tf[i] for i in range(npf)] + [tb[i] for i in range(npb)]
    dom = max(range(len(times)), key=lambda i: times[i])
    dom_ms = times[dom] / K
    dom_bytes = (passes[dom][2] + passes[dom][3]) * esz
    peak, peak_kind = load_peaks()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    res = dict(ms=ms, value=value, hbm_gbs=hbm_gbs, rt_err=rt_err, clocks=clk, clocks_soak=clk_soak,
               launches=K * (npf + npb), buffer_bytes=total * esz, nsets=nsets, fwd_check=fwd_check,
               roofline={"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": measured_traffic(args.workload, args, dom % npf if dom < npf else (dom - npf) % npb,
                                                     b),
                         "kernel": "%s %s" % (passes[dom][0], passes[dom][1]),
                         "bytes_per_launch": dom_bytes, "ms_per_launch": round(dom_ms, 5),
                         "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind if peak_kind == "measured"
                         else "fallback 6650 GB/s"},
               passes=[{"pass": "%s %s" % (p[0], p[1]), "ms": round(t / K, 5),
                        "GB/s": round((p[2] + p[3]) * esz / (t / K * 1e-3) / 1e9, 1)}
                       for p, t in zip(passes, times)])

    # the same bytes moved by plain device copies over the same buffer
    # rotation (input -> intermediate -> output, as the two directions do):
    # what a pass of this size can reach, beside the large-copy peak
    def copy_step():
        a, b_, c = sets[cur[0]]
        cur[0] = (cur[0] + 1) % nsets
        b_.copy_(a)
        c.copy_(b_)

    cur[0] = 0
    with torch.cuda.stream(stream):
        for _ in range(max(3, nsets)):
            copy_step()
    torch.cuda.synchronize()
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(K):
            copy_step()
    c1.record(stream)
    torch.cuda.synchronize()
    copy_ms = max_over_ranks(c0.elapsed_time(c1), ws) / K
    res["copy_ceiling"] = {"ms_per_step": round(copy_ms, 5),
                           "GB/s": round(2 * 2 * total * esz / (copy_ms * 1e-3) / 1e9, 1),
                           "fft_step_over_copy_step": round(ms / copy_ms, 3),
                           "how": "torch device copies of the same bytes (in -> mid -> out per step) over the same "
                                  "buffer rotation, CUDA events"}

    # end to end through the C ABI with pinned host buffers
    if not args.no_e2e:
        hy = torch.empty_like(hx).pin_memory()
        hz = torch.empty_like(hx).pin_memory()
        qf = make_plan(lib, abi, hx.data_ptr(), hy.data_ptr(), n, b, 0, dtype)
        qb = make_plan(lib, abi, hy.data_ptr(), hz.data_ptr(), n, b, 1, dtype)
        lib.aoclfftz_gpu_set_hints(None)
        for h in (qf, qb):
            lib.aoclfftz_gpu_set_stream(h, C.c_void_p(stream.cuda_stream))

        def estep():
            if lib.aoclfftz_execute(qf) or lib.aoclfftz_execute(qb):
                raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())

        for _ in range(2):
            estep()
        KE = max(3, min(K, 10))
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(KE):
            estep()
        torch.cuda.synchronize()
        e_ms = (time.perf_counter() - t0) * 1e3 / KE
        e_ms = max_over_ranks(e_ms, ws)
        ez = hz.numpy().view(x.dtype)
        e_err = float(np.linalg.norm(ez / n - x) / np.linalg.norm(x))
        res["e2e"] = {"value": round(step_metrics(n, b, esz, ws, e_ms)[0], 2), "unit": "GFLOP/s",
                      "h2d_bytes_per_step": 2 * b * n * esz, "d2h_bytes_per_step": 2 * b * n * esz,
                      "ms_per_step": round(e_ms, 3), "steps": KE, "round_trip_rel_l2": e_err,
                      "api": "aoclfftz_execute with pinned host in/out (library stages H2D, FFT, D2H)"}
        lib.aoclfftz_destroy(qf)
        lib.aoclfftz_destroy(qb)
    lib.aoclfftz_gpu_set_hints(None)
    lib.aoclfftz_destroy(pf)
    lib.aoclfftz_destroy(pb)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return res


def real3d_desc(abi, ptr, shape, direction, **kw):
    """In-place real 3-D descriptor (dims[0] innermost): r2c reads rows of
    2 (n0/2 + 1) reals and writes n0/2 + 1 complex, c2r the reverse."""
    n2, n1, n0 = shape
    h0 = n0 // 2 + 1
    rrow = 2 * h0
    if direction == 0:
        dims = [(n0, 1, 1), (n1, rrow, h0), (n2, rrow * n1, h0 * n1)]
        vecs = [(1, rrow * n1 * n2, h0 * n1 * n2)]
    else:
        dims = [(n0, 1, 1), (n1, h0, rrow), (n2, h0 * n1, rrow * n1)]
        vecs = [(1, h0 * n1 * n2, rrow * n1 * n2)]
    return abi.make_desc(ptr, ptr, dims, vecs, 1, direction, 0, **kw)


def real3d_metrics(shape, ms):
    """2.5 N log2 N flop per direction (the reference's real-transform
    count); algorithmic bytes per direction = N reals + (n0/2+1) n1 n2 complex."""
    n2, n1, n0 = shape
    N = n0 * n1 * n2
    flop = 2 * 2.5 * N * math.log2(N)
    byts = 2 * (N * 8 + (n0 // 2 + 1) * n1 * n2 * 16)
    return flop / (ms * 1e-3) / 1e9, byts / (ms * 1e-3) / 1e9


def run_real3d(args, wl):
    """Real 3-D fp64 in place: one step = r2c then c2r (unnormalised, so the
    round trip returns N x) through aoclfftz_execute on device buffers."""
    import numpy as np
    import torch

    import aoclfftz_b200
    from aoclfftz_b200 import abi, synthetic

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    lib = aoclfftz_b200.load()
    shape = wl["real3d"]
    n2, n1, n0 = shape
    N = n0 * n1 * n2
    h0 = n0 // 2 + 1
    x = synthetic.complex_uniform(4321 + rank, N // 2, np.complex128).view(np.float64).reshape(n2, n1, n0)
    hx = torch.zeros((n2, n1, 2 * h0), dtype=torch.float64).pin_memory()
    hx[:, :, :n0] = torch.from_numpy(x)
    buf = hx.to("cuda")
    stream = torch.cuda.Stream()
    hints = abi.Hints()
    hints.kernel_family, hints.tpc_col, hints.tpc_row = args.family, args.tpc_col, args.tpc_row
    hints.twiddles = args.twiddles
    lib.aoclfftz_gpu_set_hints(C.byref(hints))
    plans = []
    for d in (0, 1):
        desc, keep = real3d_desc(abi, buf.data_ptr(), shape, d)
        h = abi.setup(lib, desc, "f64")
        if not h:
            raise RuntimeError("setup failed: %s" % lib.aoclfftz_gpu_last_error().decode())
        lib.aoclfftz_gpu_set_stream(h, C.c_void_p(stream.cuda_stream))
        plans.append(h)
    pf, pb = plans

    def step():
        if lib.aoclfftz_execute(pf) or lib.aoclfftz_execute(pb):
            raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())

    with torch.cuda.stream(stream):
        step()
    torch.cuda.synchronize()
    xd = torch.from_numpy(x).cuda()
    rt_err = (torch.linalg.vector_norm(buf[:, :, :n0] / N - xd) / torch.linalg.vector_norm(xd)).item()
    del xd
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            buf[:, :, :n0] *= 1.0 / N  # keep the magnitudes from growing by N per step (outside the timing)
            step()
    buf.copy_(hx)
    K = args.steps
    lib.aoclfftz_gpu_profile_begin(pf, K)
    lib.aoclfftz_gpu_profile_begin(pb, K)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(K):
            step()
    e1.record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), ws) / K
    npf, npb = lib.aoclfftz_gpu_num_launches(pf), lib.aoclfftz_gpu_num_launches(pb)
    tf = (C.c_float * 32)()
    tb = (C.c_float * 32)()
    lib.aoclfftz_gpu_profile_end(pf, tf, 32)
    lib.aoclfftz_gpu_profile_end(pb, tb, 32)
    value, hbm = real3d_metrics(shape, ms)
    passes = [("fwd",) + p for p in pass_table(lib, pf)] + [("bwd",) + p for p in pass_table(lib, pb)]
    times = [tf[i] for i in range(npf)] + [tb[i] for i in range(npb)]
    dom = max(range(len(times)), key=lambda i: times[i])
    dom_ms = times[dom] / K
    dom_bytes = (passes[dom][2] + passes[dom][3]) * 16
    peak, peak_kind = load_peaks()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    res = dict(ms=ms, value=value * ws, hbm_gbs=hbm * ws, rt_err=rt_err, clocks=clk, launches=K * (npf + npb),
               buffer_bytes=buf.numel() * 8,
               roofline={"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "kernel": "%s %s" % (passes[dom][0], passes[dom][1]),
                         "bytes_per_launch": dom_bytes, "ms_per_launch": round(dom_ms, 5),
                         "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind if peak_kind == "measured"
                         else "fallback 6650 GB/s"},
               passes=[{"pass": "%s %s" % (p[0], p[1]), "ms": round(t / K, 5),
                        "GB/s": round((p[2] + p[3]) * 16 / (t / K * 1e-3) / 1e9, 1)}
                       for p, t in zip(passes, times)])
    # FP64 check of the forward transform: one r2c of the original input, a
    # 64^3 sub-block of its half spectrum kept for the CPU leg
    buf.copy_(hx)
    with torch.cuda.stream(stream):
        if lib.aoclfftz_execute(pf):
            raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())
    torch.cuda.synchronize()
    k0 = np.arange(0, h0, max(1, h0 // 64))[:64]
    k1 = (np.arange(64) * 7 + 3) % n1
    k2 = (np.arange(64) * 11 + 5) % n2
    X = buf.view(torch.complex128)
    got = X[torch.as_tensor(k2, device="cuda")][:, torch.as_tensor(k1, device="cuda")][
        :, :, torch.as_tensor(k0, device="cuda")].cpu().numpy()
    res["real3d_check"] = (x, got, k0, k1, k2)
    lib.aoclfftz_gpu_set_hints(None)
    for h in plans:
        lib.aoclfftz_destroy(h)
    del buf, X
    torch.cuda.empty_cache()

    # end to end: the same two plans on the pinned host buffer (the library
    # stages it to the device, transforms, and copies it back)
    if not args.no_e2e:
        eplans = []
        for d in (0, 1):
            desc, keep = real3d_desc(abi, hx.data_ptr(), shape, d)
            h = abi.setup(lib, desc, "f64")
            if not h:
                raise RuntimeError("setup failed: %s" % lib.aoclfftz_gpu_last_error().decode())
            lib.aoclfftz_gpu_set_stream(h, C.c_void_p(stream.cuda_stream))
            eplans.append(h)

        def estep():
            for h in eplans:
                if lib.aoclfftz_execute(h):
                    raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())

        estep()
        torch.cuda.synchronize()
        e_err = float(np.linalg.norm(hx[:, :, :n0].numpy() / N - x) / np.linalg.norm(x))
        KE = max(3, min(K, 5))
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(KE):
            estep()
        torch.cuda.synchronize()
        e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / KE, ws)
        nb = hx.numel() * 8
        res["e2e"] = {"value": round(real3d_metrics(shape, e_ms)[0] * ws, 2), "unit": "GFLOP/s",
                      "h2d_bytes_per_step": 2 * nb, "d2h_bytes_per_step": 2 * nb, "ms_per_step": round(e_ms, 3),
                      "steps": KE, "round_trip_rel_l2": e_err,
                      "api": "aoclfftz_execute with a pinned host buffer, in place (library stages H2D, FFT, D2H)"}
        for h in eplans:
            lib.aoclfftz_destroy(h)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return res


def time_reference_real3d(wl, threads, steps, warmup, min_time=None):
    """The reference's own CPU real 3-D path (r2c then c2r, in place, OpenMP)
    on a host buffer. Returns (seconds per step, steps timed, round-trip error)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from aoclfftz_b200 import abi, synthetic

    L = oracle.ref_lib()
    shape = wl["real3d"]
    n2, n1, n0 = shape
    N = n0 * n1 * n2
    h0 = n0 // 2 + 1
    x = synthetic.complex_uniform(99, N // 2, np.complex128).view(np.float64).reshape(n2, n1, n0)
    buf = np.zeros((n2, n1, 2 * h0))
    buf[:, :, :n0] = x
    plans = []
    for d in (0, 1):
        desc, keep = real3d_desc(abi, buf.ctypes.data, shape, d, num_threads=threads, opt_level=3)
        h = abi.setup(L, desc, "f64")
        if not h:
            raise RuntimeError("reference setup failed")
        plans.append(h)

    def step():
        for h in plans:
            if L.aoclfftz_execute(h) != 0:
                raise RuntimeError("reference execute failed")

    step()
    err = float(np.linalg.norm(buf[:, :, :n0] / N - x) / np.linalg.norm(x))
    for _ in range(warmup):
        buf[:, :, :n0] *= 1.0 / N
        step()
    k = 0
    t0 = time.perf_counter()
    while True:
        step()
        k += 1
        el = time.perf_counter() - t0
        if (steps is not None and k >= steps) or (min_time is not None and el >= min_time):
            break
    for h in plans:
        L.aoclfftz_destroy(h)
    return el / k, k, err


def run_ragged(args, wl):
    """Ragged batch: one graph launch per direction (aoclfftz_gpu_ragged_*)
    against the plain path (one aoclfftz plan per transform, executed back to
    back on the same stream)."""
    import numpy as np
    import torch

    import aoclfftz_b200
    from aoclfftz_b200 import abi, synthetic

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    lib = aoclfftz_b200.load()
    dtype = wl["dtype"]
    dt = 0 if dtype == "f32" else 1
    esz = 8 if dtype == "f32" else 16
    sizes = synthetic.ragged_sizes(4242, wl["batch"], 2, 65536)
    total = int(sum(sizes))
    cd = np.complex64 if dtype == "f32" else np.complex128
    x = synthetic.complex_normal(4243, total, cd)
    dx = torch.from_numpy(x.view(x.real.dtype).copy()).to("cuda")
    dy = torch.empty_like(dx)
    dz = torch.empty_like(dx)
    stream = torch.cuda.Stream()
    arr = (C.c_int64 * len(sizes))(*sizes)
    t0 = time.perf_counter()
    hf = lib.aoclfftz_gpu_ragged_setup(dt, 0, len(sizes), arr, None, None)
    hb = lib.aoclfftz_gpu_ragged_setup(dt, 1, len(sizes), arr, None, None)
    setup_s = time.perf_counter() - t0
    if not hf or not hb:
        raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())
    for h in (hf, hb):
        lib.aoclfftz_gpu_set_stream(h, C.c_void_p(stream.cuda_stream))
    pin, py, pz = C.c_void_p(dx.data_ptr()), C.c_void_p(dy.data_ptr()), C.c_void_p(dz.data_ptr())

    def step():
        if lib.aoclfftz_gpu_ragged_execute(hf, pin, py) or lib.aoclfftz_gpu_ragged_execute(hb, py, pz):
            raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())

    def timed(fn, k):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    for _ in range(max(args.warmup, 3)):
        step()
    if lib.aoclfftz_gpu_synchronize(hf) or lib.aoclfftz_gpu_synchronize(hb):
        raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())
    zc = dz.view(torch.complex64 if dtype == "f32" else torch.complex128).cpu().numpy()
    offs = np.cumsum([0] + sizes[:-1])
    rt = max(float(np.linalg.norm(zc[o:o + n] / n - x[o:o + n]) / max(np.linalg.norm(x[o:o + n]), 1e-30))
             for o, n in zip(offs, sizes))
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ms = timed(step, args.steps)
    clk = clocks.stop()
    # the timed run's forward outputs, for the FP64 check of the CPU leg
    yc = dy.view(torch.complex64 if dtype == "f32" else torch.complex128).cpu().numpy().copy()
    # plain path: one ordinary plan per transform, same stream
    plans = []
    t0 = time.perf_counter()
    for d, a, b in ((0, dx, dy), (1, dy, dz)):
        for o, n in zip(offs, sizes):
            desc, keep = abi.make_desc(a.data_ptr() + int(o) * esz, b.data_ptr() + int(o) * esz, [(n, 1, 1)],
                                       [(1, n, n)], 0, d, 1)
            h = abi.setup(lib, desc, dtype)
            if not h:
                raise RuntimeError(lib.aoclfftz_gpu_last_error().decode())
            lib.aoclfftz_gpu_set_stream(h, C.c_void_p(stream.cuda_stream))
            plans.append(h)
    plain_setup_s = time.perf_counter() - t0
    launches_plain = sum(lib.aoclfftz_gpu_num_launches(h) for h in plans)

    def plain_step():
        for h in plans:
            lib.aoclfftz_execute(h)

    plain_step()
    ms_plain = timed(plain_step, max(2, min(args.steps, 5)))
    for h in plans:
        lib.aoclfftz_destroy(h)
    flops = 2 * sum(5.0 * n * math.log2(n) for n in sizes if n > 1)
    alg_bytes = 2 * 2 * total * esz
    txt = C.create_string_buffer(512)
    lib.aoclfftz_gpu_describe(hf, txt, 512)
    lib.aoclfftz_destroy(hf)
    lib.aoclfftz_destroy(hb)
    peak, peak_kind = load_peaks()
    per_launch = total * 2 * esz  # one read + one write of the packed batch
    achieved = per_launch / (ms / 2 * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": None, "kernel": "fft_ragged_kernel (one launch per direction)",
            "bytes_per_launch": per_launch, "ms_per_launch": round(ms / 2, 5),
            "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind}
    return dict(ms=ms, value=flops / (ms * 1e-3) / 1e9, hbm_gbs=alg_bytes / (ms * 1e-3) / 1e9, rt_err=rt,
                buffer_bytes=total * esz, ragged_check=(sizes, offs, x, yc, dtype),
                clocks=clk, launches=2 * args.steps, roofline=roof,
                extra={"plain_path": {"ms_per_step": round(ms_plain, 4),
                                      "value": round(flops / (ms_plain * 1e-3) / 1e9, 2),
                                      "launches_per_step": launches_plain, "setup_s": round(plain_setup_s, 2)},
                       "speedup_vs_plain": round(ms_plain / ms, 2), "ragged_setup_s": round(setup_s, 2),
                       "plan": txt.value.decode(), "total_elements": total,
                       "sizes": {"count": len(sizes), "min": min(sizes), "max": max(sizes)}})


def run_selector(args, wl):
    """Learned plan selector: the MLP trained on the GPU by the library's own
    kernels on the committed autotuner timings of the training problems
    (tests/golden/selector_timings.npz, made by make_selector_db.py), regret
    against exhaustive autotuning on the held-out problems next to the
    planner's default and the reference's op-count model; plus `--batch` fresh
    problems (default 50) autotuned live on this GPU and scored with the same
    network."""
    import numpy as np
    import torch

    import aoclfftz_b200
    from aoclfftz_b200 import selector

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    lib = aoclfftz_b200.load()
    db = args.selector_db or os.path.join(ROOT, "tests", "golden", "selector_timings.npz")
    t1 = time.perf_counter()
    sel, rep = selector.train_and_evaluate(lib, db, epochs=40)
    fit_s = time.perf_counter() - t1
    nlive = args.batch if args.batch > 0 else 50
    t0 = time.perf_counter()
    live = [selector.time_candidates(lib, p, reps=5) for p in selector.random_problems(20261205, nlive)]
    live = [[c for c in cs] for cs in live if cs]
    tune_s = time.perf_counter() - t0
    live_oc = [[selector.opcount_cost(selector.plan_shape_from_text(c[1])) for c in cs] for cs in live]
    rep_live = selector.regret_report(sel, live, live_oc)
    value = 100.0 * max(0.0, 1.0 - rep["mlp_regret_mean"])
    return dict(ms=fit_s * 1e3, value=value, hbm_gbs=0.0, rt_err=None, clocks={"sm_mhz": None, "sm_max_mhz": None,
                                                                                "reasons": ["not sampled"]},
                launches=0,
                extra={"selector": dict(rep, database=os.path.relpath(db, ROOT), fit_s=round(fit_s, 2)),
                       "selector_live": dict(rep_live, problems_timed=len(live), autotune_s=round(tune_s, 1),
                                             seed=20261205)})


def time_reference(wl, threads, transforms, steps, warmup, min_time=None):
    """The reference library's own CPU path (AOCL-FFTZ compiled from its
    sources into oracle/_ref/, OpenMP) through aoclfftz_setup_f/execute on host
    buffers. One step = forward then backward of `transforms` transforms.
    Returns (seconds per step, steps timed)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from aoclfftz_b200 import abi, synthetic

    L = oracle.ref_lib()
    n, dtype = wl["n"], wl["dtype"]
    cd = np.complex64 if dtype == "f32" else np.complex128
    x = synthetic.complex_uniform(99, n * transforms, cd)
    y = np.empty_like(x)
    z = np.empty_like(x)
    plans = []
    for (a, b_, d) in ((x, y, 0), (y, z, 1)):
        desc, keep = abi.make_desc(a.ctypes.data, b_.ctypes.data, [(n, 1, 1)], [(transforms, n, n)], 0, d, 1,
                                   num_threads=threads, opt_level=3)
        h = abi.setup(L, desc, dtype)
        if not h:
            raise RuntimeError("reference setup failed")
        plans.append(h)

    def step():
        for h in plans:
            if L.aoclfftz_execute(h) != 0:
                raise RuntimeError("reference execute failed")

    for _ in range(warmup):
        step()
    t0 = time.perf_counter()
    k = 0
    while True:
        step()
        k += 1
        el = time.perf_counter() - t0
        if steps is not None and k >= steps:
            break
        if steps is None and el >= min_time:
            break
    for h in plans:
        L.aoclfftz_destroy(h)
    err = float(np.linalg.norm(z / n - x) / np.linalg.norm(x))
    return el / k, k, err


def time_reference_ragged(wl, threads, steps, warmup, min_time=None, sample=None):
    """The reference library on the ragged batch: one reference plan per
    transform (setup not timed), all forward then all backward executes back
    to back -- the reference has no ragged API. `sample` bounds the run to the
    first transforms of the same seeded batch (the setup of the long-prime
    plans alone takes seconds each). Returns (seconds per step, steps timed,
    worst round-trip error, flops per step)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from aoclfftz_b200 import abi, synthetic

    L = oracle.ref_lib()
    dtype = wl["dtype"]
    cd = np.complex64 if dtype == "f32" else np.complex128
    sizes = synthetic.ragged_sizes(4242, wl["batch"], 2, 65536)[:sample]
    total = int(sum(sizes))
    x = synthetic.complex_normal(4243, total, cd)
    y = np.empty_like(x)
    z = np.empty_like(x)
    offs = np.cumsum([0] + sizes[:-1])
    esz = x.itemsize
    plans, keep = [], []
    for a, b_, d in ((x, y, 0), (y, z, 1)):
        for o, n in zip(offs, sizes):
            desc, k = abi.make_desc(a.ctypes.data + int(o) * esz, b_.ctypes.data + int(o) * esz, [(n, 1, 1)],
                                    [(1, n, n)], 0, d, 1, num_threads=threads, opt_level=3)
            h = abi.setup(L, desc, dtype)
            if not h:
                raise RuntimeError("reference setup failed for n=%d" % n)
            plans.append(h)
            keep.append(k)

    def step():
        for h in plans:
            if L.aoclfftz_execute(h) != 0:
                raise RuntimeError("reference execute failed")

    for _ in range(warmup):
        step()
    t0 = time.perf_counter()
    k = 0
    while True:
        step()
        k += 1
        el = time.perf_counter() - t0
        if steps is not None and k >= steps:
            break
        if steps is None and el >= min_time:
            break
    for h in plans:
        L.aoclfftz_destroy(h)
    err = max(float(np.linalg.norm(z[o:o + n] / n - x[o:o + n]) / max(np.linalg.norm(x[o:o + n]), 1e-30))
              for o, n in zip(offs, sizes))
    flops = 2 * sum(5.0 * n * math.log2(n) for n in sizes if n > 1)
    return el / k, k, err, flops


def flops_per_transform(n):
    return 2 * 5.0 * n * math.log2(n)  # forward + backward


def cpu_baseline(wl):
    threads = os.cpu_count() or 1
    if wl.get("ragged"):
        sec, k, err, flops = time_reference_ragged(wl, threads, None, 1, min_time=10.0, sample=512)
        sec1, k1, _, flops1 = time_reference_ragged(wl, 1, None, 0, min_time=5.0, sample=128)
        return {"value": round(flops / sec / 1e9, 3), "unit": "GFLOP/s", "cores": threads, "kind": "reference",
                "sample": "the first 512 of the %d seeded transforms, fwd+bwd per rep as 1024 reference plans "
                          "(one per transform and direction), %d reps (%.1f s), OpenMP %d threads, opt_level 3; "
                          "value_1_thread: the first 128, one thread" % (wl["batch"], k, sec * k, threads),
                "value_1_thread": round(flops1 / sec1 / 1e9, 3), "round_trip_rel_l2": err}
    if wl.get("real3d"):
        sec, k, err = time_reference_real3d(wl, threads, None, 0, min_time=10.0)
        return {"value": round(real3d_metrics(wl["real3d"], sec * 1e3)[0], 3), "unit": "GFLOP/s",
                "cores": threads, "kind": "reference",
                "sample": "the whole %s r2c+c2r per rep, %d reps (%.1f s), OpenMP %d threads, opt_level 3"
                          % ("x".join(map(str, wl["real3d"])), k, sec * k, threads),
                "round_trip_rel_l2": err}
    n = wl["n"]
    t = max(1, min(wl["batch"], (1 << 22) // n)) if n < (1 << 22) else 1
    sec, k, err = time_reference(wl, threads, t, None, 1, min_time=10.0)
    return {"value": round(flops_per_transform(n) * t / sec / 1e9, 3), "unit": "GFLOP/s", "cores": threads,
            "kind": "reference",
            "sample": "%d x %d-point %s c2c fwd+bwd per rep, %d reps (%.1f s), OpenMP %d threads, opt_level 3"
                      % (t, n, wl["dtype"], k, sec * k, threads),
            "round_trip_rel_l2": err}


def run_reference(args, wl):
    ws, rank, local = dist_env()
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "reference library not built (oracle/_ref/libaocl_fftz.so)"}
    threads = os.cpu_count() or 1
    n = wl["n"]
    t = wl["batch"]
    if wl.get("selector"):
        return {"impl": "reference", "unavailable": "the reference has no plan selector to time"}
    if wl.get("ragged"):
        sec, k, err, flops = time_reference_ragged(wl, threads, args.steps, args.warmup, sample=1024)
        v = flops / sec / 1e9
        return {"metric": METRIC, "value": round(v, 3), "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic (splitmix64 N(0,1))",
                "impl": "reference", "config": {"workload": wl["desc"], "batch": wl["batch"]},
                "cpu_baseline": {"value": round(v, 3), "unit": "GFLOP/s", "cores": threads, "kind": "reference",
                                 "sample": "the first 1024 of the %d seeded transforms per step, one reference "
                                           "plan per transform and direction, OpenMP %d threads"
                                           % (wl["batch"], threads)},
                "e2e": {"value": round(v, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "round_trip_rel_l2": err}
    if wl.get("real3d"):
        sec, k, err = time_reference_real3d(wl, threads, args.steps, args.warmup)
        v = real3d_metrics(wl["real3d"], sec * 1e3)[0]
        return {"metric": METRIC, "value": round(v, 3), "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic (splitmix64 U[-1,1))",
                "impl": "reference", "config": {"workload": wl["desc"], "n": n, "batch": 1},
                "cpu_baseline": {"value": round(v, 3), "unit": "GFLOP/s", "cores": threads, "kind": "reference",
                                 "sample": "the whole transform per step, r2c+c2r, OpenMP %d threads" % threads},
                "e2e": {"value": round(v, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "round_trip_rel_l2": err}
    sec1, _, _ = time_reference(wl, threads, t, 1, 0)
    if sec1 * (args.steps + args.warmup) > 150:
        t = max(1, int(t * 150 / (sec1 * (args.steps + args.warmup))))
    sec, k, err = time_reference(wl, threads, t, args.steps, args.warmup)
    v = flops_per_transform(n) * t / sec / 1e9
    base = {"metric": METRIC, "value": round(v, 3), "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic (splitmix64 U[-1,1))", "impl": "reference",
            "config": {"workload": wl["desc"], "n": n, "batch": wl["batch"], "sample_transforms_per_step": t},
            "cpu_baseline": {"value": round(v, 3), "unit": "GFLOP/s", "cores": threads, "kind": "reference",
                             "sample": "%d of %d transforms per step, fwd+bwd, OpenMP %d threads" % (t, wl["batch"],
                                                                                                 threads)},
            "e2e": {"value": round(v, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "round_trip_rel_l2": err}
    return base


def l2_label(r):
    nb = r.get("buffer_bytes", 0)
    if r.get("nsets", 1) > 1:
        return "inputs smaller than L2: %d rotating buffer sets of 3 x %.0f MB (%.0f MB cycled > 126 MB L2)" % (
            r["nsets"], nb / 1e6, 3 * nb * r["nsets"] / 1e6)
    return "inputs larger than L2 (no flush needed)" if nb > L2_BYTES else "inputs fit L2 (no flush)"


def fp64_check(n, dtype, x0, y0, x1, y1):
    """rel-L2 of the GPU's forward outputs in the timed run against the FP64
    oracle: all N bins of the first transform (oracle.fft, itself pinned to
    exact naive sums by the tests), and 32 seeded bins each of the first and
    last transform against exact FP64 naive-DFT sums; with the bound
    4 log2(N) eps of the dtype. About 15 s of host work at N = 2^24."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    e_all = float(oracle.rel_l2(y0, oracle.fft(x0)))
    bins = np.sort(np.random.default_rng(2024).choice(n, size=min(32, n), replace=False))
    e_bins = [float(oracle.rel_l2(y[bins], oracle.dft_bins(x, bins))) for x, y in ((x0, y0), (x1, y1))]
    return {"rel_l2": e_all, "bound": oracle.tol(n, dtype),
            "bins": "all %d bins of the first transform (FP64 fast FFT)" % n,
            "exact_bins_rel_l2": e_bins, "exact_bins": "%d seeded bins of the first and last transform" % len(bins)}


def ragged_fp64_check(sizes, offs, x, y, dtype, every=16):
    """FP64-oracle error of the ragged run's forward outputs: every `every`-th
    transform of the batch against oracle.fft, each against its own bound
    4 log2(n) eps of the dtype; reports the sample's overall rel-L2, the worst
    error / bound ratio and that transform."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    num = den = 0.0
    worst = (0.0, 0, 0.0, 0.0)
    idx = list(range(0, len(sizes), every))
    for i in idx:
        o, n = int(offs[i]), int(sizes[i])
        ref = oracle.fft(np.asarray(x[o:o + n], dtype=np.complex128))
        d = np.asarray(y[o:o + n], dtype=np.complex128) - ref
        num += float(np.vdot(d, d).real)
        den += float(np.vdot(ref, ref).real)
        e = float(oracle.rel_l2(y[o:o + n], ref))
        b = oracle.tol(n, dtype) if n > 1 else oracle.tol(2, dtype)
        if e / b > worst[0]:
            worst = (e / b, n, e, b)
    return {"rel_l2": math.sqrt(num / max(den, 1e-300)), "worst_err_over_bound": round(float(worst[0]), 4),
            "worst_transform": {"n": worst[1], "rel_l2": float(worst[2]), "bound": float(worst[3])},
            "bins": "all bins of every %d-th transform (%d of %d, FP64 fast FFT), each against "
                    "4 log2(n) eps" % (every, len(idx), len(sizes))}


def real3d_fp64_check(x, got, k0, k1, k2):
    """FP64-oracle error of a real 3-D forward transform: a 64^3 sub-block of
    half-spectrum bins against separable exact FP64 sums over the whole input
    (twiddles from exactly reduced integer indices), bound 4 log2(N) eps."""
    import numpy as np

    n2, n1, n0 = x.shape

    def cols(n, ks):
        j = np.arange(n, dtype=np.int64)[:, None]
        r = (j * np.asarray(ks, dtype=np.int64)[None, :]) % n
        return np.exp(-2j * np.pi * (r.astype(np.float64) / n))

    a = (x.reshape(-1, n0) @ cols(n0, k0)).reshape(n2, n1, len(k0))
    a = np.einsum("zyk,yl->zlk", a, cols(n1, k1), optimize=True)
    a = np.einsum("zlk,zm->mlk", a, cols(n2, k2), optimize=True)
    N = n0 * n1 * n2
    return {"rel_l2": float(np.linalg.norm(got - a) / np.linalg.norm(a)),
            "bound": 4 * math.log2(N) * float(np.finfo(np.float64).eps),
            "bins": "64^3 sub-block of the r2c half spectrum (k0 every %d-th, 64 k1, 64 k2) against "
                    "separable exact FP64 sums over the whole input" % max(1, (n0 // 2 + 1) // 64)}


METRIC = "5N·log2N GFLOP/s + HBM GB/s vs plain GPU FFT at stated FP64 err, 1 B200"


def main():
    args = parse()
    wl = dict(WORKLOADS[args.workload])
    if args.batch > 0:
        wl["batch"] = args.batch
        wl["desc"] = wl["desc"].replace("batch %d" % WORKLOADS[args.workload]["batch"], "batch %d" % args.batch)
    ws, rank, local = dist_env()
    if args.impl == "reference":
        out = run_reference(args, wl)
        if out is not None:
            print(json.dumps(out))
        return
    if wl.get("selector"):
        r = run_selector(args, wl)
        if rank == 0:
            print(json.dumps({"metric": "learned plan selector regret vs exhaustive autotuning (held-out)",
                              "value": round(r["value"], 2), "unit": "% of best (100 = always optimal)",
                              "higher_is_better": True, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": round(r["ms"], 1), "scaling": "weak", "vs_baseline": None,
                              "dtype": "mixed", "data": "synthetic", "config": {"workload": wl["desc"]},
                              **r["extra"]}))
        return
    r = run_ragged(args, wl) if wl.get("ragged") else run_real3d(args, wl) if wl.get("real3d") else run_ours(args, wl)
    if rank != 0:
        return
    peak, peak_kind = load_peaks()
    line = {"metric": METRIC, "value": round(r["value"], 2), "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(r["ms"], 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic (splitmix64 U[-1,1))",
            "config": {"workload": wl["desc"], "n": wl["n"], "batch_per_gpu": wl["batch"],
                       "global_batch": wl["batch"] * ws, "l2": l2_label(r),
                       "parallelism": "replicas dp%d" % ws},
            "hbm_gbs": round(r["hbm_gbs"], 1), "hbm_frac_of_measured": round(r["hbm_gbs"] / peak, 4),
            "gpu_launches": r["launches"], "clocks": r["clocks"], "round_trip_rel_l2": r["rt_err"]}
    for key in ("roofline", "passes", "copy_ceiling"):
        if key in r:
            line[key] = r[key]
    line.update(r.get("extra", {}))
    if "e2e" in r:
        line["e2e"] = r["e2e"]
    if "clocks_soak" in r:
        line["clocks_soak"] = r["clocks_soak"]
    if ws == 1 and not args.no_cpu_baseline and not wl.get("selector"):
        # the CPU leg: the reference timed on the host cores, and the FP64
        # oracle as the checker of this run's forward outputs
        if r.get("fwd_check") is not None:
            try:
                line["fp64_oracle"] = fp64_check(*r["fwd_check"])
            except Exception as e:
                line["fp64_oracle"] = {"unavailable": str(e)}
        if r.get("real3d_check") is not None:
            try:
                line["fp64_oracle"] = real3d_fp64_check(*r["real3d_check"])
            except Exception as e:
                line["fp64_oracle"] = {"unavailable": str(e)}
        if r.get("ragged_check") is not None:
            try:
                line["fp64_oracle"] = ragged_fp64_check(*r["ragged_check"])
            except Exception as e:
                line["fp64_oracle"] = {"unavailable": str(e)}
        try:
            line["cpu_baseline"] = cpu_baseline(wl)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
