"""The TL surrogate (C5): gradients of the tensor-core network against a CPU
float64 autograd restatement of the same network, a short training run, and
the fallback to the plain FP64 trace."""
import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import surrogate as S
from bellhopcuda_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _bf(t):
    """Round a float64 tensor to bfloat16 and back (the GPU's storage points)."""
    return t.to(__import__("torch").bfloat16).double()


def _gelu(z, torch):
    c = 0.7978845608028654   # sqrt(2 / pi), tanh form
    u = c * (z + 0.044715 * z ** 3)
    return 0.5 * z * (1.0 + torch.tanh(u))


def _dgelu(z, torch):
    c = 0.7978845608028654
    u = c * (z + 0.044715 * z ** 3)
    th = torch.tanh(u)
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th ** 2) * c * (1.0 + 3 * 0.044715 * z ** 2)


def _cpu_forward(m, x, torch):
    """One MLP in float64 on the CPU, rounding to bf16 where the GPU stores bf16:
    layer outputs and the kept pre-activations."""
    xs, pres = [], []
    for l in m.layers:
        W = l.wb.double().cpu()
        z = x @ W.T + l.b.double().cpu()
        xs.append(x)
        if l.gelu:
            pres.append(_bf(z))
            x = _bf(_gelu(z, torch))
        else:
            pres.append(None)
            x = _bf(z)
    return x, xs, pres


def _cpu_backward(m, dz, xs, pres, torch):
    """Gradients (gw, gb) of every layer, last to first, with the GPU's bf16
    rounding of the propagated pre-activation gradients."""
    grads = []
    for i in range(len(m.layers) - 1, -1, -1):
        l = m.layers[i]
        grads.append((dz.T @ xs[i], dz.sum(0)))
        if i > 0:
            W = l.wb.double().cpu()
            dz = _bf((dz @ W) * _dgelu(pres[i - 1], torch))
    return grads[::-1]


def test_gradients_match_cpu_float64():
    """Forward and every parameter gradient of the tensor-core network against
    a float64 CPU restatement that rounds to bf16 at the same storage points.
    What remains is FP32 accumulation order and bf16 rounding ties: 1e-2."""
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
    b, bx, bp = _cpu_forward(model.branch, x.double().cpu(), torch)
    t, tx, tp = _cpu_forward(model.trunk, model.phi.double().cpu(), torch)
    p64 = b @ t.T + model.pbias.double().cpu()
    d = pred.cpu().double() - p64
    assert float(d.norm() / p64.norm()) < 1e-2
    # the loss gradient the GPU stored (bf16), propagated on the CPU
    dp = dpred.cpu().double()
    ref_dp = _bf(2.0 * (pred.cpu().double() - y.cpu().double()) / (Bn * S.NP))
    assert float((dp - ref_dp).norm() / ref_dp.norm()) < 1e-2
    db = _bf(dp @ t)
    dt = _bf(dp.T @ b)
    got = []
    for m in (model.branch, model.trunk):
        for l in m.layers:
            got += [l.gw, l.gb]
    ref = []
    for gw, gb in _cpu_backward(model.branch, db, bx, bp, torch) + _cpu_backward(model.trunk, dt, tx, tp, torch):
        ref += [gw, gb]
    for k, (g, r) in enumerate(zip(got, ref)):
        g = g.double().cpu().flatten()
        r = r.flatten()
        rel = float((g - r).norm() / (r.norm() + 1e-300))
        assert rel < 1e-2, (k, rel)
    g = model.gpb.double().cpu()
    assert float((g - dp.sum(0)).norm() / dp.sum(0).norm()) < 1e-3


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


def test_trained_surrogate_gains_over_the_plain_trace(tmp_path):
    """The C5 pipeline on 30,000 incoherent Gaussian-beam fields (27,000 for
    training, 30 epochs) judged at a 2 dB acceptance bound: part of the test
    split is answered by the network, what is returned stays within the bound,
    and the surrogate with its fallback costs less than the plain FP64 trace of
    the same fields. (The full C5 run, 100,000 fields at the 1 dB bound, is
    reported by bench.py's `surrogate` key.)"""
    o = S.run_c5(n=30000, epochs=30, threshold_db=2.0, tmpdir=str(tmp_path))
    assert o["surrogate_only_rms_db_mean"] < 3.0, o["surrogate_only_rms_db_mean"]
    assert o["fallback_rate"] < 0.95, o["fallback_rate"]
    assert o["returned_within_threshold"] >= 0.95, o["returned_within_threshold"]
    assert o["speedup_accounted"] > 1.0, o["speedup_accounted"]
