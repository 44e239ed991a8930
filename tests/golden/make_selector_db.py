"""Generates tests/golden/selector_timings.npz on a B200: the exhaustive
autotuner's timings (aoclfftz_b200.selector.time_candidates: every candidate
hint set planned, each distinct plan timed with CUDA events, median of the
repetitions) for the learned-selector workload --

  training problems   seed 20261203, the first 20000 drawn
  held-out problems   seed 20261204, the first 2000 drawn that differ from
                      every training problem

(rank 1-3, dims powers of two / 7-smooth / primes, c2c / r2c / c2r, f32 /
f64, unit or strided, batch 1-256, at most 2^22 elements per transform batch).

Per problem only distinct plans are kept (candidates whose plan description
matches an earlier one's are the same plan). Stored per row: problem index,
split (0 training, 1 held out), candidate index into selector.CANDIDATES,
plan-structure feature vector, median ms, and the reference-style op-count cost of the plan
(selector.opcount_cost); and the problem descriptions as JSON.

  python tests/golden/make_selector_db.py [--train 20000] [--test 2000]
         [--partial PATH] [--time-limit SECONDS] [--out PATH]

With --partial the run saves its progress every 500 problems and resumes from
that file; --time-limit stops (after saving) when the limit is reached, so a
long generation can span several runs.

  python tests/golden/make_selector_db.py --recost IN [--out PATH]

re-plans every stored (problem, candidate) row of database IN (no timing) and
rewrites its op-count column with the current selector.opcount_cost; every
other column is kept as it is.
"""
import argparse
import ctypes as C
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "aocl-fftz_b200", "python"))

import numpy as np  # noqa: E402

TRAIN_SEED, TEST_SEED = 20261203, 20261204


def problem_list(ntrain, ntest):
    from aoclfftz_b200 import selector
    train = selector.random_problems(TRAIN_SEED, ntrain)
    seen = {json.dumps(p, sort_keys=True) for p in train}
    test = []
    extra = 0
    while len(test) < ntest:
        cand = selector.random_problems(TEST_SEED, ntest + extra)
        test = [p for p in cand if json.dumps(p, sort_keys=True) not in seen][:ntest]
        extra += ntest // 10 + 1
    return train + test, ntrain


def rows_of(index, split, results, candidates):
    from aoclfftz_b200 import selector
    out, texts = [], set()
    for hd, text, feat, ms in results:
        if text in texts:
            continue
        texts.add(text)
        passes = selector.plan_shape_from_text(text)
        # the plan-structure features; the candidate one-hot is rebuilt from cand on load
        out.append((index, split, candidates.index(hd), feat[:selector.NBASE], ms, selector.opcount_cost(passes)))
    return out


def save(path, rows, problems, done):
    np.savez_compressed(path, problem=np.array([r[0] for r in rows], dtype=np.int32),
                        split=np.array([r[1] for r in rows], dtype=np.int8),
                        cand=np.array([r[2] for r in rows], dtype=np.int16),
                        features=np.stack([r[3] for r in rows]).astype(np.float32),
                        ms=np.array([r[4] for r in rows], dtype=np.float32),
                        opcost=np.array([r[5] for r in rows], dtype=np.float64),
                        done=np.array([done], dtype=np.int32),
                        problems=np.frombuffer(json.dumps(problems).encode(), dtype=np.uint8))


def recost(path_in, path_out):
    import torch
    import aoclfftz_b200
    from aoclfftz_b200 import abi, selector

    torch.cuda.set_device(0)
    lib = aoclfftz_b200.load()
    d = np.load(path_in)
    problems = json.loads(bytes(d["problems"]).decode())
    prob, cand = d["problem"], d["cand"]
    opcost = np.zeros(len(prob), dtype=np.float64)
    t0 = time.perf_counter()
    bufs = {}
    for k in range(len(prob)):
        p = problems[int(prob[k])]
        if int(prob[k]) not in bufs:
            bufs.clear()
            _, _, in_sc, out_sc = selector.descriptor(p, 1, 2)
            tdt = torch.float32 if p["dtype"] == "f32" else torch.float64
            bufs[int(prob[k])] = (torch.zeros(in_sc, dtype=tdt, device="cuda"),
                                  torch.zeros(out_sc, dtype=tdt, device="cuda"))
        x, y = bufs[int(prob[k])]
        lib.aoclfftz_gpu_set_hints(C.byref(selector._hints(selector.CANDIDATES[int(cand[k])])))
        desc, keep, _, _ = selector.descriptor(p, x.data_ptr(), y.data_ptr())
        h = abi.setup(lib, desc, p["dtype"])
        lib.aoclfftz_gpu_set_hints(None)
        if not h:
            raise RuntimeError("row %d: %s" % (k, lib.aoclfftz_gpu_last_error().decode()))
        text, passes = selector.plan_shape(lib, h)
        lib.aoclfftz_destroy(h)
        opcost[k] = selector.opcount_cost(passes)
        if (k + 1) % 20000 == 0:
            print("%d rows, %.1f s" % (k + 1, time.perf_counter() - t0), flush=True)
    out = {f: d[f] for f in d.files}
    out["opcost"] = opcost
    np.savez_compressed(path_out, **out)
    print("wrote %s: %d rows re-costed" % (path_out, len(prob)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--test", type=int, default=2000)
    ap.add_argument("--partial", default="")
    ap.add_argument("--time-limit", type=float, default=0.0)
    ap.add_argument("--out", default=os.path.join(HERE, "selector_timings.npz"))
    ap.add_argument("--recost", default="")
    args = ap.parse_args()
    if args.recost:
        recost(args.recost, args.out)
        return
    import torch
    import aoclfftz_b200
    from aoclfftz_b200 import selector

    torch.cuda.set_device(0)
    lib = aoclfftz_b200.load()
    problems, ntrain = problem_list(args.train, args.test)
    rows, start = [], 0
    if args.partial and os.path.exists(args.partial):
        d = np.load(args.partial)
        start = int(d["done"][0])
        rows = [(int(a), int(b), int(c), f, float(m), float(o)) for a, b, c, f, m, o in
                zip(d["problem"], d["split"], d["cand"], d["features"], d["ms"], d["opcost"])]
        print("resuming at problem %d (%d rows)" % (start, len(rows)), flush=True)
    t0 = time.perf_counter()
    i = start
    for i in range(start, len(problems)):
        p = problems[i]
        res = selector.time_candidates(lib, p, reps=5)
        rows += rows_of(i, 0 if i < ntrain else 1, res, selector.CANDIDATES)
        if (i + 1) % 500 == 0:
            el = time.perf_counter() - t0
            print("%d problems, %d rows, %.1f s (%.1f ms per problem)" % (i + 1, len(rows), el,
                                                                         1e3 * el / (i + 1 - start)), flush=True)
            if args.partial:
                save(args.partial, rows, problems, i + 1)
            if args.time_limit and el > args.time_limit:
                print("time limit reached at problem %d" % (i + 1), flush=True)
                return
    save(args.out, rows, problems, len(problems))
    if args.partial:
        save(args.partial, rows, problems, len(problems))
    print("wrote %s: %d problems, %d rows" % (args.out, len(problems), len(rows)), flush=True)


if __name__ == "__main__":
    main()
