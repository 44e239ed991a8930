"""Autotuner and learned plan selector.

The planner of the library makes fixed choices (four-step split, transforms per
CTA, kernel family). The autotuner enumerates alternatives as planner hints
(aoclfftz_gpu_set_hints), builds each candidate plan, times it with CUDA
events and keeps the fastest -- exhaustive search, always correct, costly.
The learned selector predicts each candidate's log time with a small MLP
trained on autotuner timings by the library's own CUDA kernels
(aoclfftz_gpu_mlp_*) and picks the argmin without timing; the exhaustive
autotuner stays its fallback and the yardstick of its regret. No transform result
depends on the selector: every candidate computes the same transform.

The reference's counterpart is a fixed op-count cost model
(core/solvers/solver.c:124-140) and an unimplemented auto-tuner stub
(selector/selector.c:989-1004). Two "methods without the network" stand
beside the MLP: the planner's default choice, and that op-count model
restated over each candidate's passes (opcount_cost).
"""
import ctypes as C
import math

import numpy as np

from . import abi, synthetic

def _is_prime(n):
    return synthetic._is_prime(n)


def _draw_dim(u_class, u_size, lo, hi):
    n0 = int(round(math.exp(math.log(lo) + u_size * (math.log(hi) - math.log(lo)))))
    n0 = max(lo, min(hi, n0))
    cls = int(u_class * 3)
    if cls == 0:
        return synthetic._next_pow2(n0)
    n = n0
    if cls == 1:
        while not synthetic._smooth7(n):
            n += 1
        return n
    while not _is_prime(n):
        n += 1
    return n


def random_problems(seed, count, max_total=1 << 22):
    """Problems of the learned-selector workload: rank 1-3, each dim a power
    of two, a 7-smooth number or a prime; c2c / r2c / c2r; f32 / f64; unit or
    strided element layout; batch 1-256; at most max_total elements."""
    out = []
    i = 0
    while len(out) < count:
        v = synthetic.u01(seed, 16, offset=16 * i)
        i += 1
        rank = 1 + int(v[0] * 3)
        hi = [65536, 2048, 256][rank - 1]
        dims = [_draw_dim(v[1 + 2 * k], v[2 + 2 * k], 2, hi) for k in range(rank)]
        total = int(np.prod(dims))
        if total > max_total:
            continue
        kind = int(v[7] * 3)  # 0 c2c, 1 r2c, 2 c2r
        dtype = "f32" if v[8] < 0.5 else "f64"
        strided = bool(v[9] < 0.3)
        bmax = max(1, min(256, max_total // total))
        batch = max(1, min(bmax, int(round(math.exp(v[10] * math.log(bmax))))))
        direction = 0 if kind != 2 else 1
        if kind == 0 and v[11] < 0.5:
            direction = 1
        out.append(dict(dims=dims, kind=kind, dtype=dtype, strided=strided, batch=batch, direction=direction))
    return out


def descriptor(p, in_ptr, out_ptr):
    """dims / vecs (innermost first) and raw buffer sizes of a problem."""
    dims = p["dims"]
    es = 2 if p["strided"] else 1
    h0 = dims[0] // 2 + 1
    if p["kind"] == 0:
        ins, outs = [], []
        s = es
        for n in dims:
            ins.append(s)
            s *= n
        dist = s
        d = [(n, st, st) for n, st in zip(dims, ins)]
        v = [(p["batch"], dist, dist)]
        in_sc = out_sc = 2 * (dist * p["batch"])
    else:
        rs, cs = [es], [es]
        for k in range(1, len(dims)):
            rs.append(rs[-1] * (dims[0] if k == 1 else dims[k - 1]))
            cs.append(cs[-1] * (h0 if k == 1 else dims[k - 1]))
        rtot = rs[-1] * (dims[0] if len(dims) == 1 else dims[-1])
        ctot = cs[-1] * (h0 if len(dims) == 1 else dims[-1])
        if p["kind"] == 1:
            d = [(n, a, b) for n, a, b in zip(dims, rs, cs)]
            v = [(p["batch"], rtot, ctot)]
            in_sc, out_sc = rtot * p["batch"], 2 * ctot * p["batch"]
        else:
            d = [(n, b, a) for n, a, b in zip(dims, rs, cs)]
            v = [(p["batch"], ctot, rtot)]
            in_sc, out_sc = 2 * ctot * p["batch"], rtot * p["batch"]
    desc, keep = abi.make_desc(in_ptr, out_ptr, d, v, 1 if p["kind"] else 0, p["direction"], 1)
    return desc, keep, in_sc, out_sc


CANDIDATES = [
    dict(),                                   # the planner's default
    dict(tpc_row=1), dict(tpc_row=2), dict(tpc_row=4),
    dict(tpc_col=2), dict(tpc_col=4), dict(tpc_col=8), dict(tpc_col=16),
    dict(kernel_family=1),                    # plain loads everywhere (no TMA-fed column passes)
    dict(kernel_family=2),
    dict(kernel_family=3),                    # generic kernel only
    dict(kernel_family=5),                    # TMA-fed tiles wherever they qualify
    dict(fourstep_n1=256), dict(fourstep_n1=1024), dict(fourstep_n1=4096),
    dict(algorithm=2),                        # force a four-step split where possible
    dict(kernel_family=9),                    # 16 x 256 split tiles for every 4096-point float pass
    dict(kernel_family=12),                   # in-place runtime-radix kernel instead of ping-pong tiles
]


def _hints(h):
    x = abi.Hints()
    for k, val in h.items():
        setattr(x, k, val)
    return x


def plan_shape(lib, h):
    """(plan text, per-pass (kind, n, ntf, tpc)) parsed from the plan description."""
    buf = C.create_string_buffer(4096)
    lib.aoclfftz_gpu_describe(h, buf, 4096)
    text = buf.value.decode()
    return text, plan_shape_from_text(text)


def plan_shape_from_text(text):
    """Per-pass (kind, n, ntf, tpc) of a plan description."""
    passes = []
    for seg in text.split("[")[1:]:
        seg = seg.split("]")[0]
        parts = seg.split()
        kind = parts[0]
        kv = {}
        for t in parts[1:]:
            if "=" in t:
                a, b = t.split("=", 1)
                kv[a] = b
            elif t.startswith("x"):
                kv["x"] = t[1:]
        passes.append((kind, int(kv.get("n", "1")), int(kv.get("x", "1")), int(kv.get("tpc", "1"))))
    return passes


KINDS = ["fast", "pipe", "generic", "bluestein", "elem", "r2c", "c2r"]
NBASE = 24  # plan-structure features


def cand_onehot(index, ncand=None):
    """One-hot of the candidate's hint set: candidates whose plans share the
    same pass structure (TMA use, kernel family) differ only here."""
    v = np.zeros(ncand or len(CANDIDATES), dtype=np.float32)
    v[index] = 1.0
    return v


def features(p, passes):
    """Feature vector of one candidate plan of problem p."""
    dims = p["dims"]
    total = float(np.prod(dims))
    f = np.zeros(NBASE, dtype=np.float32)
    f[0] = math.log2(total)
    f[1] = math.log2(p["batch"])
    for k in range(3):
        f[2 + k] = math.log2(dims[k]) if k < len(dims) else 0.0
    f[5] = len(dims)
    f[6] = 1.0 if p["dtype"] == "f64" else 0.0
    f[7] = 1.0 if p["kind"] == 1 else 0.0
    f[8] = 1.0 if p["kind"] == 2 else 0.0
    f[9] = 1.0 if p["strided"] else 0.0
    f[10] = len(passes)
    for kind, n, ntf, tpc in passes:
        for i, k in enumerate(KINDS):
            if kind.startswith(k):
                f[11 + i] += 1.0
    if passes:
        f[18] = max(math.log2(max(n, 1)) for _, n, _, _ in passes)
        f[19] = min(math.log2(max(n, 1)) for _, n, _, _ in passes)
        f[20] = float(np.mean([math.log2(max(t, 1)) for _, _, _, t in passes]))
        f[21] = max(math.log2(max(t, 1)) for _, _, _, t in passes)
        f[22] = math.log2(sum(max(n, 1) * max(x, 1) for _, n, x, _ in passes))
    f[23] = math.log2(total * p["batch"]) + (3.0 if p["dtype"] == "f64" else 2.0)
    return f


# The reference's op-count cost model. Cycle weights of its operation classes
# (api/aoclfftz_internal.h:201-206): fma, mul, add, move, perm, other.
_W_OPS = (4, 3, 1, 1, 1, 1)
# Operation counts (fma, mul, add, move, perm, other) per call of the
# reference's scalar codelets, as their ops_cnt tables state them: the first
# stage of a line runs the plain codelet (core/kernels/dft/c2c/c/fft<R>c.c),
# every later stage the twiddled one
# (core/kernels/dft/tw_c2c_fwd/c/twid_fwd_fft<R>c.c; the backward tables are
# the same), for the radices this planner uses.
_OPS_FIRST = {2: (0, 0, 4, 8, 0, 0), 3: (0, 4, 12, 12, 0, 0), 4: (0, 0, 16, 16, 0, 0), 5: (0, 12, 32, 20, 0, 0),
              7: (0, 36, 60, 28, 0, 0), 8: (0, 4, 52, 32, 0, 0), 11: (0, 100, 140, 44, 0, 0),
              13: (0, 68, 176, 52, 0, 0), 16: (0, 24, 144, 64, 0, 0)}
_OPS_TW = {2: (0, 4, 6, 10, 0, 0), 3: (0, 12, 16, 16, 0, 0), 4: (0, 12, 22, 22, 0, 0), 5: (0, 28, 40, 28, 0, 0),
           7: (0, 60, 72, 40, 0, 0), 8: (0, 32, 66, 46, 0, 0), 11: (0, 140, 160, 64, 0, 0),
           13: (0, 116, 200, 76, 0, 0), 16: (0, 84, 174, 94, 0, 0)}


def _radices(n):
    """The stage radices the planner uses for a line of length n: 16s (then
    8, 4 or 2) for powers of two, else the balanced power-of-two part and the
    odd factors (csrc/host/plan.c generic_radices)."""
    if n <= 1:
        return []
    if n & (n - 1) == 0:
        out, k = [], n.bit_length() - 1
        st = (k + 3) // 4
        base, extra = k // st, k % st
        return [1 << (base + (1 if i < extra else 0)) for i in range(st)]
    out, k, m = [], 0, n
    while m % 2 == 0:
        m //= 2
        k += 1
    if k:
        st = (k + 3) // 4
        base, extra = k // st, k % st
        out += [1 << (base + (1 if i < extra else 0)) for i in range(st)]
    for q in (13, 11, 7, 5, 3):
        while m % q == 0:
            out.append(q)
            m //= q
    if m != 1:  # Bluestein: count its power-of-two convolution length twice
        return None
    return out


def codelet_cost(R, first):
    """Weighted cycles of one call of the reference's radix-R codelet (core/
    solvers/solver.c:124-140: fma * 4 + mul * 3 + add + move + perm + other)."""
    counts = (_OPS_FIRST if first else _OPS_TW)[R]
    return sum(w * c for w, c in zip(_W_OPS, counts))


def opcount_cost(passes):
    """The reference's fixed cost model restated over a candidate plan's
    passes: a line of length n with stage radices R_0, R_1, ... calls n / R_s
    codelets in stage s, the plain codelet in stage 0 and the twiddled one
    after it, each weighted by its operation counts (codelet_cost); a pass of
    ntf lines costs ntf times that; a line without a radix split (Bluestein)
    counts its power-of-two convolution length twice; elementwise passes 2 n
    per line. It sees the arithmetic only -- not memory traffic, launch shape
    or kernel family."""
    cost = 0.0
    for kind, n, ntf, tpc in passes:
        if kind.startswith("elem"):
            cost += 2.0 * n * max(ntf, 1)
            continue
        rs = _radices(n)
        if rs is None:
            m = 1 << (2 * n - 1).bit_length()
            rs = _radices(m) or [2]
            n = m
            mult = 2.0
        else:
            mult = 1.0
        cost += mult * max(ntf, 1) * sum((n // R) * codelet_cost(R, s == 0) for s, R in enumerate(rs))
    return cost


def time_candidates(lib, p, reps=3, candidates=CANDIDATES):
    """Plans every candidate hint set of problem p, times distinct plans.
    Returns a list of (hints, plan_text, features, ms)."""
    import torch
    tdt = torch.float32 if p["dtype"] == "f32" else torch.float64
    desc0, keep0, in_sc, out_sc = descriptor(p, 1, 2)
    x = torch.randn(in_sc, dtype=tdt, device="cuda")
    y = torch.zeros(out_sc, dtype=tdt, device="cuda")
    seen = {}
    results = []
    for hd in candidates:
        lib.aoclfftz_gpu_set_hints(C.byref(_hints(hd)))
        desc, keep, _, _ = descriptor(p, x.data_ptr(), y.data_ptr())
        h = abi.setup(lib, desc, p["dtype"])
        lib.aoclfftz_gpu_set_hints(None)
        if not h:
            continue
        text, passes = plan_shape(lib, h)
        key = text
        if key in seen:
            lib.aoclfftz_destroy(h)
            results.append((hd, text, features(p, passes), seen[key]))
            continue
        lib.aoclfftz_execute(h)
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            lib.aoclfftz_execute(h)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        lib.aoclfftz_destroy(h)
        ms = float(np.median(ts))
        seen[key] = ms
        results.append((hd, text, features(p, passes), ms))
    # network input: plan structure, then the candidate's one-hot
    return [(hd, text, np.concatenate([f, cand_onehot(candidates.index(hd), len(candidates))]), ms)
            for hd, text, f, ms in results]


class MLPSelector:
    """The 2 x 64 network, trained on the GPU by aoclfftz_gpu_mlp_* kernels."""

    def __init__(self, lib, nfeat=NBASE + len(CANDIDATES), seed=0):
        import torch
        self.lib = lib
        self.F = nfeat
        n = lib.aoclfftz_gpu_mlp_nparams(nfeat)
        rng = np.random.default_rng(seed)
        p = np.zeros(n, dtype=np.float32)
        H = 64
        o = 0
        p[o:o + nfeat * H] = rng.normal(0, math.sqrt(2.0 / nfeat), nfeat * H); o += nfeat * H + H
        p[o:o + H * H] = rng.normal(0, math.sqrt(2.0 / H), H * H); o += H * H + H
        p[o:o + H] = rng.normal(0, math.sqrt(1.0 / H), H)
        self.params = torch.from_numpy(p).cuda()
        self.mu = np.zeros(nfeat, dtype=np.float32)
        self.sd = np.ones(nfeat, dtype=np.float32)

    def _norm(self, X):
        return (np.asarray(X, dtype=np.float32) - self.mu) / self.sd

    def fit(self, X, t, epochs=300, lr=2e-3, batch=256, seed=1):
        import torch
        X = np.asarray(X, dtype=np.float32)
        self.mu = X.mean(0)
        self.sd = X.std(0) + 1e-3
        Xn = torch.from_numpy(self._norm(X)).cuda()
        tt = torch.from_numpy(np.asarray(t, dtype=np.float32)).cuda()
        n = self.params.numel()
        grads = torch.zeros(n, device="cuda")
        m = torch.zeros(n, device="cuda")
        v = torch.zeros(n, device="cuda")
        loss = torch.zeros(1, device="cuda")
        work = torch.zeros(4 * batch * 64 + 2 * batch, device="cuda")
        rng = np.random.default_rng(seed)
        step = 0
        hist = []
        N = Xn.shape[0]
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(N)).cuda()
            tot = 0.0
            for s0 in range(0, N - batch + 1 if N >= batch else 1, batch):
                idx = perm[s0:s0 + batch]
                xb = Xn[idx].contiguous()
                tb = tt[idx].contiguous()
                B = xb.shape[0]
                step += 1
                rc = self.lib.aoclfftz_gpu_mlp_grad(self.params.data_ptr(), self.F, xb.data_ptr(), tb.data_ptr(), B,
                                                    grads.data_ptr(), loss.data_ptr(), work.data_ptr(), None)
                rc |= self.lib.aoclfftz_gpu_mlp_adam(self.params.data_ptr(), grads.data_ptr(), m.data_ptr(),
                                                     v.data_ptr(), n, lr, step, None)
                if rc:
                    raise RuntimeError("mlp kernels failed: %d" % rc)
                tot += float(loss.item()) * B
            hist.append(tot / max(N, 1))
        return hist

    def predict(self, X):
        import torch
        Xn = torch.from_numpy(self._norm(X)).cuda()
        B = Xn.shape[0]
        y = torch.zeros(B, device="cuda")
        work = torch.zeros(2 * B * 64, device="cuda")
        rc = self.lib.aoclfftz_gpu_mlp_forward(self.params.data_ptr(), self.F, Xn.data_ptr(), B, y.data_ptr(),
                                               work.data_ptr(), None)
        if rc:
            raise RuntimeError("mlp forward failed: %d" % rc)
        return y.cpu().numpy()


def regret_report(selector, dataset, opcosts=None):
    """dataset: list of candidate lists (hints, text, features, ms) per
    problem, the planner's default first. Regret = t(chosen) / t(best) - 1 for
    the network, for the planner's default and -- given per-candidate op
    costs -- for the reference's op-count model (ties keep the earlier
    candidate, so an indifferent model falls back to the default)."""
    reg_mlp, reg_def, reg_op = [], [], []
    for i, cands in enumerate(dataset):
        ms = np.array([c[3] for c in cands])
        best = ms.min()
        pred = selector.predict(np.stack([c[2] for c in cands]))
        reg_mlp.append(ms[int(np.argmin(pred))] / best - 1.0)
        reg_def.append(ms[0] / best - 1.0)
        if opcosts is not None:
            reg_op.append(ms[int(np.argmin(np.asarray(opcosts[i])))] / best - 1.0)
    reg_mlp, reg_def = np.array(reg_mlp), np.array(reg_def)
    rep = {"problems": len(dataset),
           "mlp_regret_mean": float(reg_mlp.mean()), "mlp_regret_p95": float(np.percentile(reg_mlp, 95)),
           "default_regret_mean": float(reg_def.mean()), "default_regret_p95": float(np.percentile(reg_def, 95))}
    if opcosts is not None:
        reg_op = np.array(reg_op)
        rep["opcount_regret_mean"] = float(reg_op.mean())
        rep["opcount_regret_p95"] = float(np.percentile(reg_op, 95))
    return rep


def load_timings(path):
    """Autotuner timing database (tests/golden/make_selector_db.py): per
    problem the candidate rows (default plan first). Returns
    (train, test, train_opcost, test_opcost): lists of candidate lists
    (None, None, features, ms) and of per-candidate op costs (None when the
    database has none). Databases without a split field keep the first 80% of
    their problems for training."""
    d = np.load(path)
    prob, feats, ms = d["problem"], d["features"], d["ms"]
    if "cand" in d.files:  # the stored rows hold the plan-structure part only
        feats = np.concatenate([feats, np.eye(len(CANDIDATES), dtype=np.float32)[d["cand"]]], axis=1)
    opc = d["opcost"] if "opcost" in d.files else None
    split = d["split"] if "split" in d.files else None
    order = np.argsort(prob, kind="stable")
    groups, costs, gsplit = [], [], []
    cur = -1
    for k in order:
        if prob[k] != cur:
            cur = prob[k]
            groups.append([])
            costs.append([])
            gsplit.append(int(split[k]) if split is not None else -1)
        groups[-1].append((None, None, feats[k], float(ms[k])))
        costs[-1].append(float(opc[k]) if opc is not None else 0.0)
    if split is None:
        ntrain = int(0.8 * len(groups))
        gsplit = [0] * ntrain + [1] * (len(groups) - ntrain)
    tr = [i for i, s_ in enumerate(gsplit) if s_ == 0]
    te = [i for i, s_ in enumerate(gsplit) if s_ == 1]
    pick = lambda idx, arr: [arr[i] for i in idx]  # noqa: E731
    oc = opc is not None
    return (pick(tr, groups), pick(te, groups), pick(tr, costs) if oc else None, pick(te, costs) if oc else None)


def train_and_evaluate(lib, path, epochs=60, seed=0):
    """Trains the MLP on the database's training problems (log microseconds
    per candidate) and reports held-out regret of the network, the planner's
    default and the op-count model against the exhaustive optimum."""
    train, test, _, test_oc = load_timings(path)
    X = np.stack([c[2] for g in train for c in g])
    y = np.log(np.array([c[3] for g in train for c in g]) * 1e3)
    sel = MLPSelector(lib, nfeat=X.shape[1], seed=seed)
    hist = sel.fit(X, y, epochs=epochs)
    rep = regret_report(sel, test, test_oc)
    rep["train_problems"] = len(train)
    rep["train_rows"] = int(X.shape[0])
    rep["loss_first"], rep["loss_last"] = float(hist[0]), float(hist[-1])
    return sel, rep
