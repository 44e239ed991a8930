"""GPU parity against the committed golden fixtures: every case of
tests/golden/reference_outputs.npz (outputs of the reference library on
seeded inputs) runs through the GPU library's C ABI and must agree with the
reference output within 2 * 4 * log2(N) * eps (both sides carry rounding of the
working dtype) and with the FP64 oracle within 4 * log2(N) * eps."""
import json
import os

import numpy as np
import pytest

import golden_cases as G
import oracle
from fftz_helpers import run_gpu

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_outputs.npz")
_d = np.load(GOLD)
GOLDEN = [(c, _d["out_%d" % i]) for i, c in enumerate(json.loads(bytes(_d["cases"]).decode()))]


@pytest.mark.parametrize("idx", range(len(GOLDEN)), ids=[c["name"] for c, _ in GOLDEN])
def test_gpu_matches_reference_golden(idx):
    c, ref_raw = GOLDEN[idx]
    x = G.case_input(c)
    out, plan = run_gpu(c["dtype"], c["dims"], c["vecs"], x, G.out_scalars(c), c["type"], c["dir"], c["placement"])
    y = G.logical_output(c, out)
    tol = G.tolerance(c)
    e_ref = oracle.rel_l2(y, G.logical_output(c, ref_raw))
    e_orc = oracle.rel_l2(y, G.oracle_output(c))
    assert e_ref <= 2 * tol, "vs reference %.3e (tol %.3e) plan %s" % (e_ref, tol, plan)
    assert e_orc <= tol, "vs oracle %.3e (tol %.3e) plan %s" % (e_orc, tol, plan)
