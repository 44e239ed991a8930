"""The exhaustive autotuner on the GPU (aoclfftz_b200.selector.time_candidates):
for seeded problems of the selector workload it plans every candidate hint
set, times the distinct plans and returns the fastest; the plan it picks must
compute the same transform as every other plan -- checked here against the
FP64 oracle on seeded inputs. Bound: rel-L2 <= 4 log2(N) eps of the dtype."""
import ctypes as C

import numpy as np
import pytest

import aoclfftz_b200
import oracle
from aoclfftz_b200 import abi, selector, synthetic
from fftz_helpers import cplx_dtype, gather, real_dtype, scatter

pytestmark = pytest.mark.gpu


def _problems():
    ps = [p for p in selector.random_problems(777, 400) if p["kind"] == 0 and
          int(np.prod(p["dims"])) * p["batch"] <= (1 << 18)]
    # one of each rank, one strided, both dtypes among them
    out, seen = [], set()
    for p in ps:
        key = (len(p["dims"]), p["strided"], p["dtype"])
        if key not in seen:
            seen.add(key)
            out.append(p)
    return out[:6]


def _oracle(x, rank, sign):
    y = np.asarray(x, dtype=np.complex128)
    for k in range(rank):
        ax = y.ndim - 1 - k
        y = np.moveaxis(oracle.fft(np.moveaxis(y, ax, -1), sign=sign), -1, ax)
    return y


@pytest.mark.parametrize("p", _problems(), ids=lambda p: "%s-%s-b%d-%s%s" % (
    "x".join(map(str, p["dims"])), p["dtype"], p["batch"], "bwd" if p["direction"] else "fwd",
    "-strided" if p["strided"] else ""))
def test_autotuner_choice_computes_the_transform(p):
    import torch
    lib = aoclfftz_b200.load()
    results = selector.time_candidates(lib, p, reps=3)
    assert results, "no candidate planned"
    assert all(ms > 0 for _, _, _, ms in results)
    best = min(results, key=lambda r: r[3])
    dt = p["dtype"]
    desc0, keep0, in_sc, out_sc = selector.descriptor(p, 1, 2)
    dims = [(desc0.dims[i].n, desc0.dims[i].in_stride, desc0.dims[i].out_stride) for i in range(desc0.dim_rank)]
    vecs = [(desc0.vecs[0].n, desc0.vecs[0].in_stride, desc0.vecs[0].out_stride)]
    lshape = [p["batch"]] + list(reversed(p["dims"]))
    x = synthetic.complex_uniform(11, int(np.prod(lshape)), cplx_dtype(dt)).reshape(lshape)
    raw = scatter(x, [(d[0], d[1]) for d in dims], [(v[0], v[1]) for v in vecs], in_sc, dt)
    tdt = torch.float32 if dt == "f32" else torch.float64
    din = torch.from_numpy(np.ascontiguousarray(raw).view(real_dtype(dt))).to("cuda")
    dout = torch.zeros(out_sc, dtype=tdt, device="cuda")
    lib.aoclfftz_gpu_set_hints(C.byref(selector._hints(best[0])))
    desc, keep, _, _ = selector.descriptor(p, din.data_ptr(), dout.data_ptr())
    h = abi.setup(lib, desc, dt)
    lib.aoclfftz_gpu_set_hints(None)
    assert h, lib.aoclfftz_gpu_last_error()
    try:
        assert lib.aoclfftz_execute(h) == 0
        assert lib.aoclfftz_gpu_synchronize(h) == 0
    finally:
        lib.aoclfftz_destroy(h)
    y = gather(dout.cpu().numpy(), [(d[0], d[2]) for d in dims], [(v[0], v[2]) for v in vecs], dt)
    ref = _oracle(x, len(p["dims"]), -1 if p["direction"] == 0 else +1)
    err = oracle.rel_l2(y, ref)
    n = int(np.prod(p["dims"]))
    assert err <= oracle.tol(n, dt), "rel-L2 %.3e with hints %s (plan %s)" % (err, best[0], best[1])
