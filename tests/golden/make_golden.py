#!/usr/bin/env python3
"""Writes tests/golden/reference_outputs.npz: outputs of the reference library
(AOCL-FFTZ built from its own sources by oracle/Makefile into oracle/_ref/) on
seeded synthetic inputs, for the layouts the reference's own tests exercise
(test/bench/CMakeLists.txt:55-124: pow2 iterative, Cooley-Tukey radices,
Bluestein primes, col-major batches, multi-dimensional, real packed).

Inputs are not stored: each case's input is regenerated from its seed with
aoclfftz_b200.synthetic (splitmix64), so the file holds only the case table
(JSON) and the reference outputs.

Run in a container that has the reference sources:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "aocl-fftz_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from golden_cases import CASES, case_input, out_scalars  # noqa: E402


def main():
    if not oracle.ref_available():
        raise SystemExit("reference library not built: make -C oracle ref")
    arrays = {}
    table = []
    for i, c in enumerate(CASES):
        x = case_input(c)
        out = oracle.ref_execute(c["dtype"], c["dims"], c["vecs"], x, out_scalars(c), c["type"], c["dir"],
                                 c["placement"])
        arrays["out_%d" % i] = out
        table.append(c)
    arrays["cases"] = np.frombuffer(json.dumps(table).encode(), dtype=np.uint8)
    path = os.path.join(HERE, "reference_outputs.npz")
    np.savez_compressed(path, **arrays)
    print("wrote %s: %d cases, %d bytes" % (path, len(table), os.path.getsize(path)))


if __name__ == "__main__":
    main()
