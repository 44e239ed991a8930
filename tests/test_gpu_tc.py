"""Tensor-core form (kernel family 7): 4096-point float rows computed as two
radix-64 DFT-GEMM stages on tcgen05 with FP32 accumulation, each operand split
into three BF16 terms (24 significant bits) and six products per stage.

Held to the FP32 path's bound against the FP64 oracle: rel-L2 <= 4 log2(N)
eps_f32 (N = 4096 and the 2^24 four-step line); its error is printed next to
the SIMT path's on the same input. The planner never picks it unless asked."""
import ctypes as C

import numpy as np
import pytest

import aoclfftz_b200
import oracle
from aoclfftz_b200 import abi, synthetic
from fftz_helpers import cplx_dtype, run_gpu

pytestmark = pytest.mark.gpu



def _run(family, n, batch, direction, seed):
    lib = aoclfftz_b200.load()
    x = synthetic.complex_uniform(seed, n * batch, np.complex64).reshape(batch, n)
    h = abi.Hints()
    h.kernel_family = family
    lib.aoclfftz_gpu_set_hints(C.byref(h))
    try:
        out, plan = run_gpu("f32", [(n, 1, 1)], [(batch, n, n)], x.view(np.float32).ravel(), 2 * n * batch, 0,
                            direction, 1)
    finally:
        lib.aoclfftz_gpu_set_hints(None)
    return x, out.view(np.complex64).reshape(batch, n), plan


@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("batch", [4, 12])
def test_tc_rows_4096(direction, batch):
    x, y, plan = _run(7, 4096, batch, direction, 11 + batch)
    assert "tc n=4096" in plan, plan
    ref = oracle.fft(x.astype(np.complex128), sign=-1 if direction == 0 else +1)
    err = oracle.rel_l2(y, ref)
    _, y32, _ = _run(0, 4096, batch, direction, 11 + batch)
    err32 = oracle.rel_l2(y32, ref)
    print("rel-L2 vs FP64 oracle: tensor-core %.3e, FP32 SIMT %.3e" % (err, err32))
    assert err <= oracle.tol(4096, "f32"), err
    assert err32 <= oracle.tol(4096, "f32")


def test_tc_fourstep_row_pass():
    """2^24 = 4096 x 4096 four-step (the bench workload's line): its 4096-point
    row pass runs on the tensor cores, the column pass on the FP32 path."""
    n = 1 << 24
    x, y, plan = _run(7, n, 1, 0, 5)
    assert "tc n=4096" in plan, plan
    ref = oracle.fft(x.astype(np.complex128), sign=-1)
    err = oracle.rel_l2(y, ref)
    print("four-step 2^24 with tensor-core row pass: rel-L2 %.3e" % err)
    assert err <= oracle.tol(n, "f32"), err
