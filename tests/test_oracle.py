"""CPU: the oracle (test infrastructure) pinned against the reference library.

* every golden fixture (outputs of the reference library on seeded inputs,
  tests/golden/reference_outputs.npz) agrees with the restated FP64 oracle
  within 4 * log2(N) * eps of the case's dtype;
* the restated plan-shape helpers reproduce the reference's values
  (core/common/pow2_radix_decompose.c:15-35, :122-150,
  core/common/bluestein_utils.c:39-67, :88-159);
* where the reference library is built in this container, live runs agree too.
"""
import json
import os

import numpy as np
import pytest

import golden_cases as G
import oracle
from aoclfftz_b200 import synthetic

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_outputs.npz")


def load_golden():
    d = np.load(GOLD)
    cases = json.loads(bytes(d["cases"]).decode())
    return [(c, d["out_%d" % i]) for i, c in enumerate(cases)]


GOLDEN = load_golden()


def test_golden_table_matches_case_list():
    assert [c["name"] for c, _ in GOLDEN] == [c["name"] for c in G.CASES]


@pytest.mark.parametrize("idx", range(len(GOLDEN)), ids=[c["name"] for c, _ in GOLDEN])
def test_oracle_matches_reference_golden(idx):
    c, raw = GOLDEN[idx]
    y = G.logical_output(c, raw)
    r = G.oracle_output(c)
    assert oracle.rel_l2(y, r) <= G.tolerance(c)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 16, 17, 60, 97, 128, 243, 1000])
def test_fast_oracle_matches_naive_dft(n):
    x = synthetic.complex_normal(5, 3 * n).reshape(3, n)
    for sign in (-1, +1):
        assert oracle.rel_l2(oracle.fft(x, sign), oracle.dft(x, sign)) < 1e-14


def test_dft_bins_and_nd():
    x = synthetic.complex_normal(6, 4096)
    bins = np.array([0, 1, 7, 100, 2048, 4095])
    assert oracle.rel_l2(oracle.dft_bins(x, bins), oracle.dft(x)[bins]) < 1e-15
    a = synthetic.complex_normal(7, 5 * 6 * 7).reshape(5, 6, 7)
    assert oracle.rel_l2(oracle.fft_nd(a), oracle.dft_nd(a)) < 1e-14


def test_real_restatement_round_trip():
    for n in (2, 6, 16, 50, 99, 1024):
        x = synthetic.normal(8, 3 * n).reshape(3, n)
        X = oracle.rfft_packed(x)
        full = oracle.fft(x.astype(np.complex128))
        assert oracle.rel_l2(X, full[:, : n // 2 + 1]) < 1e-14
        assert oracle.rel_l2(oracle.irfft_packed(X, n), n * x) < 1e-14


def test_plan_shape_helpers_match_reference_values():
    assert oracle.pow2_radix_balanced(512) == [8, 8, 8]
    assert oracle.pow2_radix_balanced(4096) == [16, 16, 16]
    assert oracle.pow2_radix_balanced(2048) == [16, 16, 8]
    assert oracle.pow2_radix_balanced(32) == [8, 4]
    assert oracle.pow2_balanced_split(1 << 24) == (4096, 4096)
    assert oracle.pow2_balanced_split(1 << 13) == (128, 64)
    assert oracle.bluestein_extended_length(17) == 33
    assert oracle.bluestein_extended_length(97) == 195
    assert oracle.bluestein_extended_length(1009) == 2025
    # chirp: b_i = exp(+i pi (i^2 mod 2n) / n), mirrored at m - i
    n, m = 17, 33
    b = oracle.bluestein_chirp(n, m)
    i = np.arange(n)
    want = np.exp(1j * np.pi * ((i * i) % (2 * n)) / n)
    assert np.allclose(b[:n], want, atol=1e-15)
    assert np.allclose(b[m - i[1:]], want[1:], atol=1e-15)
    assert np.all(b[n:m - n + 1] == 0)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [8, 12, 19, 243, 512, 4096, 65536])
def test_live_reference_matches_oracle(dtype, n):
    x = synthetic.complex_uniform(9, 2 * n, G.cplx_dtype(dtype))
    out = oracle.ref_execute(dtype, [(n, 1, 1)], [(2, n, n)], x, 4 * n)
    y = out.view(G.cplx_dtype(dtype)).reshape(2, n)
    assert oracle.rel_l2(y, oracle.fft(x.reshape(2, n))) <= oracle.tol(n, dtype)
