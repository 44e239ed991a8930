"""GPU: the learned plan selector's network, trained by the library's own CUDA
kernels (aoclfftz_gpu_mlp_*), checked against the float64 numpy restatement in
oracle/mlp_oracle.py: forward values and parameter gradients (fp32 vs fp64:
relative error <= 1e-4), one Adam step, and that training lowers the loss.
The end-to-end regret test uses the autotuner timing database committed in
tests/golden/selector_timings.npz when it is present."""
import json
import os

import numpy as np
import pytest

import aoclfftz_b200
import mlp_oracle  # noqa: E402 (oracle/ on sys.path via conftest)
from aoclfftz_b200 import selector

pytestmark = pytest.mark.gpu

F = 24


def _lib():
    return aoclfftz_b200.load()


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def test_forward_and_grad_match_oracle():
    lib = _lib()
    rng = np.random.default_rng(3)
    n = lib.aoclfftz_gpu_mlp_nparams(F)
    assert n == mlp_oracle.nparams(F)
    p = rng.normal(0, 0.2, n).astype(np.float32)
    B = 37
    X = rng.normal(0, 1, (B, F)).astype(np.float32)
    t = rng.normal(0, 1, B).astype(np.float32)
    import torch
    dp, dX, dt = _t(p), _t(X), _t(t)
    y = torch.zeros(B, device="cuda")
    work = torch.zeros(4 * B * 64 + 2 * B, device="cuda")
    assert lib.aoclfftz_gpu_mlp_forward(dp.data_ptr(), F, dX.data_ptr(), B, y.data_ptr(), work.data_ptr(), None) == 0
    y_ref, _, _ = mlp_oracle.forward(p.astype(np.float64), F, X.astype(np.float64))
    assert np.linalg.norm(y.cpu().numpy() - y_ref) / np.linalg.norm(y_ref) < 1e-5
    g = torch.zeros(n, device="cuda")
    loss = torch.zeros(1, device="cuda")
    assert lib.aoclfftz_gpu_mlp_grad(dp.data_ptr(), F, dX.data_ptr(), dt.data_ptr(), B, g.data_ptr(),
                                     loss.data_ptr(), work.data_ptr(), None) == 0
    g_ref, l_ref = mlp_oracle.grad(p.astype(np.float64), F, X.astype(np.float64), t.astype(np.float64))
    gg = g.cpu().numpy()
    assert np.linalg.norm(gg - g_ref) / np.linalg.norm(g_ref) < 1e-4
    assert abs(loss.item() - l_ref) / l_ref < 1e-5


def test_adam_step_matches_formula():
    lib = _lib()
    n = 1000
    rng = np.random.default_rng(4)
    p = rng.normal(size=n).astype(np.float32)
    g = rng.normal(size=n).astype(np.float32)
    dp, dg, dm, dv = _t(p), _t(g), _t(np.zeros(n)), _t(np.zeros(n))
    assert lib.aoclfftz_gpu_mlp_adam(dp.data_ptr(), dg.data_ptr(), dm.data_ptr(), dv.data_ptr(), n, 0.01, 1,
                                     None) == 0
    m = 0.1 * g
    v = 0.001 * g * g
    want = p - 0.01 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.allclose(dp.cpu().numpy(), want, rtol=1e-5, atol=1e-6)


def test_training_lowers_loss():
    lib = _lib()
    rng = np.random.default_rng(5)
    X = rng.normal(size=(2048, F)).astype(np.float32)
    w = rng.normal(size=F)
    t = (np.tanh(X @ w / 4) + 0.1 * (X[:, 0] ** 2)).astype(np.float32)
    sel = selector.MLPSelector(lib, nfeat=F, seed=1)
    hist = sel.fit(X, t, epochs=30, lr=2e-3, batch=256)
    assert hist[-1] < 0.2 * hist[0]
    pred = sel.predict(X[:256])
    assert np.corrcoef(pred, t[:256])[0, 1] > 0.9


DB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "selector_timings.npz")


@pytest.mark.skipif(not os.path.exists(DB), reason="no autotuner timing database committed")
def test_learned_selector_beats_default_on_held_out():
    """Trains on 80% of the committed autotuner timings, evaluates regret
    against exhaustive search on the held-out 20%."""
    d = np.load(DB)
    prob, feats, ms = d["problem"], d["features"], d["ms"]
    nprob = int(prob.max()) + 1
    groups = [[(None, None, feats[k], float(ms[k])) for k in np.nonzero(prob == i)[0]] for i in range(nprob)]
    ntrain = int(0.8 * nprob)
    train, test = groups[:ntrain], groups[ntrain:]
    X = np.stack([c[2] for g in train for c in g])
    y = np.log(np.array([c[3] for g in train for c in g]) * 1e3)
    sel = selector.MLPSelector(_lib(), nfeat=X.shape[1], seed=0)
    sel.fit(X, y, epochs=120)
    rep = selector.regret_report(sel, test)
    assert rep["mlp_regret_mean"] < rep["default_regret_mean"]
    assert rep["mlp_regret_mean"] < 0.10
