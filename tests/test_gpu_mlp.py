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
def test_learned_selector_regret_on_held_out():
    """Trains the network on the committed autotuner timings of the training
    problems (the library's own MLP kernels on the GPU) and measures regret
    against exhaustive autotuning on the held-out problems: at most 5% mean,
    below the planner's default and below the reference's op-count model
    restated over the candidates (the methods without the network)."""
    sel, rep = selector.train_and_evaluate(_lib(), DB, epochs=40)
    assert rep["problems"] >= 2000 and rep["train_problems"] >= 20000, rep
    assert rep["mlp_regret_mean"] <= 0.05, rep
    assert rep["mlp_regret_mean"] < rep["default_regret_mean"], rep
    assert rep["mlp_regret_mean"] < rep["opcount_regret_mean"], rep
