"""The TL surrogate (C5): gradients of the tensor-core network against a CPU
float64 autograd restatement of the same network, a short training run, and
the fallback to the plain FP64 trace."""
import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import surrogate as S
from bellhopcuda_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cpu_net(model, torch):
    """The network's forward in float64 on the CPU from the model's bf16 weights."""
    def lin(l, x):
        w = l.wb.double().cpu().requires_grad_(True)
        b = l.b.double().cpu().requires_grad_(True)
        return w, b, x @ w.T + b

    def mlp(m, x):
        ps = []
        for i, l in enumerate(m.layers):
            w, b, z = lin(l, x)
            ps += [w, b]
            x = torch.nn.functional.gelu(z, approximate="tanh") if l.gelu else z
        return x, ps
    return mlp


def test_gradients_match_cpu_float64():
    import torch
    model = S.Surrogate(seed=3)
    rng = np.random.default_rng(0)
    Bn = 8
    x = torch.tensor(rng.normal(0, 1, (Bn, S.N_IN)).astype(np.float32), device="cuda").bfloat16()
    y = torch.tensor(rng.normal(0, 1, (Bn, S.NP)).astype(np.float32), device="cuda")
    pred = model.forward(x, keep=True)
    dpred = torch.empty((Bn, S.NP), dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    model.ops.mse(pred, y, dpred, loss, 1.0 / (Bn * S.NP))
    model.backward(dpred)
    torch.cuda.synchronize()
    model.ops.check()
    # float64 restatement on the CPU
    mlp = _cpu_net(model, torch)
    b, pb = mlp(model.branch, x.double().cpu())
    t, pt = mlp(model.trunk, model.phi.double().cpu())
    beta = model.pbias.double().cpu().requires_grad_(True)
    p64 = b @ t.T + beta
    # bf16 activations between layers: about 1 % relative, measured on the whole output
    d = pred.cpu().double() - p64.detach()
    assert float(d.norm() / p64.detach().norm()) < 0.02
    l64 = ((p64 - y.double().cpu()) ** 2).mean()
    l64.backward()
    got = []
    for m in (model.branch, model.trunk):
        for l in m.layers:
            got += [l.gw, l.gb]
    ref = pb + pt
    for g, r in zip(got, ref):
        g = g.double().cpu().flatten()
        r = r.grad.flatten()
        cos = float((g @ r) / (g.norm() * r.norm() + 1e-300))
        rel = float((g - r).norm() / (r.norm() + 1e-300))
        assert cos > 0.99 and rel < 0.1, (cos, rel)
    g = model.gpb.double().cpu()
    assert float((g - beta.grad).norm() / beta.grad.norm()) < 0.05


def test_training_reduces_error_and_fallback_is_the_trace(tmp_path):
    import torch
    P = W.c5_params(96, seed=77)
    idx = list(range(96))
    Y = torch.empty((96, S.NP), device="cuda")
    S.trace_tl(P, idx, Y, tmpdir=str(tmp_path))
    X = torch.tensor(S.features(P, idx), device="cuda").bfloat16()
    model = S.Surrogate(seed=1)
    hist = model.train(X[:64], Y[:64], epochs=25, batch=32, lr=1e-3)
    assert hist[-1] < 0.7 * hist[0], hist
    # fallback: threshold 0 sends every field to the FP64 trace
    tl, fb, tm = S.infer(model, P, idx[64:], threshold_db=-1.0, tmpdir=str(tmp_path))
    assert fb.all() and tm["fallback_s"] > 0
    ref = Y[64:] * S.TL_SCALE + S.TL_MEAN
    torch.testing.assert_close(tl, ref, rtol=0, atol=1e-3)
    # no fallback: the surrogate's own prediction
    tl2, fb2, tm2 = S.infer(model, P, idx[64:], threshold_db=1e9, tmpdir=str(tmp_path))
    assert not fb2.any() and tm2["fallback_s"] == 0.0
    assert torch.isfinite(tl2).all()
