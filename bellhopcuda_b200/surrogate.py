"""Neural-operator TL surrogate for the 2-D surrogate workload (C5).

The fields are incoherent Gaussian-beam TL (RunType 'IB') by default, or
coherent hat-beam TL ('CG'). A coherent field on the 128 x 256 grid is
sampled far below the Nyquist rate of its interference fringes (wavelengths of
3-30 m against receiver spacings of 39 m in depth and 78 m in range), so at a
receiver it behaves like a Rayleigh-faded amplitude about the incoherent mean,
whose 20 log10 spread is about 5.6 dB: the error floor of any predictor that
varies smoothly with the environment. The incoherent field is the learnable
quantity.

A DeepONet-style operator maps an environment to its TL grid:

    TL(z_i, r_j) = sum_k  b_k(env) * t_k(z_i / D, r_j)  +  beta(z_i, r_j)

* branch net: 128 environment features -> 4 GELU layers of width 1024 -> 512
  coefficients b_k (the SSP sampled at 64 normalised depths, water depth,
  bottom speed, source depth, frequency);
* trunk net: 128 Fourier features of the normalised receiver coordinates ->
  3 layers of width 512 -> 512 basis values t_k per receiver (the same
  128 x 256 normalised grid for every environment, so one trunk pass serves a
  whole batch);
* error head: features -> 256 GELU -> predicted log RMS error (dB) of the
  surrogate for that environment; fields whose predicted error exceeds the
  threshold are recomputed by the plain FP64 tracer (the fallback).

Every GEMM (forward and backward) runs in the library's tcgen05 tensor-core
kernel (bhcb_nn_gemm: BF16 operands, FP32 accumulation in tensor memory) and
the element-wise work in its own kernels (bhcb_nn_*); PyTorch only provides
device memory and the stream. About 4.9 M parameters, FP32 master weights and
Adam states, BF16 weights and activations.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import tempfile
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import BhcbError, PREC_FP64, Tracer, load_library
from . import workloads as W
from .envfile import write_env

NZ, NR = W.C5_NZ, W.C5_NR
NP = NZ * NR
N_IN = 128
N_TRUNK_IN = 128
TL_LO, TL_HI = 30.0, 130.0       # clamp of the training targets (dB)
TL_MEAN, TL_SCALE = 80.0, 20.0   # normalisation of the network output

EPI_F32, EPI_BF16, EPI_GELU, EPI_DGELU = 0, 1, 2, 3


def _torch():
    import torch
    return torch


# ----------------------------------------------------------------- features
def features(P: Dict[str, np.ndarray], idx: Sequence[int]) -> np.ndarray:
    """(len(idx), 128) float32 network inputs of environments idx of c5_params P."""
    idx = np.asarray(idx)
    x = np.zeros((len(idx), N_IN), np.float32)
    for row, i in enumerate(idx):
        _, c = W.c5_ssp(float(P["depth"][i]), P["a"][i])
        x[row, :64] = (c - 1500.0) / 30.0
    x[:, 64] = (P["depth"][idx] - 3000.0) / 2000.0
    x[:, 65] = (P["cp"][idx] - 1650.0) / 150.0
    x[:, 66] = (P["zs"][idx] - 255.0) / 245.0
    x[:, 67] = P["zs"][idx] / P["depth"][idx] * 10.0
    lf = np.log(P["f"][idx] / 50.0) / math.log(10.0)
    x[:, 68] = lf * 2.0 - 1.0
    for k in range(1, 5):
        x[:, 68 + 2 * k - 1] = np.sin(k * math.pi * lf)
        x[:, 68 + 2 * k] = np.cos(k * math.pi * lf)
    return x


def trunk_inputs() -> np.ndarray:
    """(NP, 128) float32 Fourier features of the normalised (depth, range) grid:
    geometric frequency ladders up to the grid's Nyquist rate in each axis."""
    u = np.repeat(np.linspace(0.0, 1.0, NZ), NR)
    v = np.tile(np.linspace(0.0, 1.0, NR), NZ)
    f = [u * 2 - 1, v * 2 - 1]
    for k in np.geomspace(1.0, NZ / 2.0, 24):
        f += [np.sin(k * math.pi * u), np.cos(k * math.pi * u)]
    for k in np.geomspace(1.0, NR / 2.0, 39):
        f += [np.sin(k * math.pi * v), np.cos(k * math.pi * v)]
    return np.stack(f, 1).astype(np.float32)


# ------------------------------------------------------------------- layers
class _Ops:
    """Thin wrappers of the library's surrogate kernels on torch buffers."""

    def __init__(self):
        self.lib = load_library()
        self.torch = _torch()

    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr()) if t is not None else None

    def gemm(self, A, Bm, out, epi, bias=None, aux_in=None, aux_out=None):
        M, K = A.shape
        N = Bm.shape[0]
        assert Bm.shape[1] == K and out.shape[0] == M and out.shape[1] == N
        rc = self.lib.bhcb_nn_gemm(self._p(A), self._p(Bm), self._p(out), M, N, K, epi, self._p(bias),
                                   self._p(aux_in), self._p(aux_out), self._s())
        if rc != 0:
            raise BhcbError(rc, "bhcb_nn_gemm failed (M %d N %d K %d epi %d)" % (M, N, K, epi))

    def T(self, x, out=None):
        R, Cc = x.shape
        if out is None:
            out = self.torch.empty((Cc, R), dtype=x.dtype, device=x.device)
        rc = self.lib.bhcb_nn_transpose(self._p(x), self._p(out), R, Cc, self._s())
        if rc != 0:
            raise BhcbError(rc, "transpose failed")
        return out

    def colsum(self, dy, out):
        M, N = dy.shape
        rc = self.lib.bhcb_nn_colsum(self._p(dy), M, N, self._p(out), self._s())
        if rc != 0:
            raise BhcbError(rc, "colsum failed")

    def adam(self, w, g, m, v, step, lr, wb=None, wt=None, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        rows, cols = (w.shape[0], w.shape[1]) if w.dim() == 2 else (1, w.shape[0])
        rc = self.lib.bhcb_nn_adam(self._p(w), self._p(g), self._p(m), self._p(v), rows, cols, lr, b1, b2, eps,
                                   step, wd, self._p(wb), self._p(wt), self._s())
        if rc != 0:
            raise BhcbError(rc, "adam failed")

    def to_bf16(self, x, out):
        rc = self.lib.bhcb_nn_to_bf16(self._p(x), self._p(out), x.numel(), self._s())
        if rc != 0:
            raise BhcbError(rc, "to_bf16 failed")

    def mse(self, pred, target, grad, loss, scale):
        rc = self.lib.bhcb_nn_mse(self._p(pred), self._p(target), pred.numel(), scale, self._p(grad),
                                  self._p(loss), self._s())
        if rc != 0:
            raise BhcbError(rc, "mse failed")

    def row_rms(self, pred, target, out):
        rc = self.lib.bhcb_nn_row_rms(self._p(pred), self._p(target), pred.shape[0], pred.shape[1],
                                      self._p(out), self._s())
        if rc != 0:
            raise BhcbError(rc, "row_rms failed")

    def affine(self, x, a, b):
        rc = self.lib.bhcb_nn_affine(self._p(x), x.numel(), a, b, self._s())
        if rc != 0:
            raise BhcbError(rc, "affine failed")

    def tl_db(self, field_ptr, out, n):
        rc = self.lib.bhcb_nn_tl_db(C.c_void_p(field_ptr), self._p(out), n, TL_LO, TL_HI, self._s())
        if rc != 0:
            raise BhcbError(rc, "tl_db failed")

    def check(self):
        err = C.c_int32()
        self.lib.bhcb_nn_status(C.byref(err), 1)
        if err.value:
            raise BhcbError(3, "a tensor-core GEMM timed out waiting on its pipeline")


class Linear:
    """y = act(x W^T + b): FP32 master weights with Adam states, bf16 W and W^T."""

    def __init__(self, ops: _Ops, n_out: int, n_in: int, gelu: bool, rng: np.random.Generator, gain: float = 1.0):
        torch = ops.torch
        self.ops, self.n_out, self.n_in, self.gelu = ops, n_out, n_in, gelu
        bound = gain * math.sqrt(6.0 / n_in) / (math.sqrt(2.0) if not gelu else 1.0)
        w = rng.uniform(-bound, bound, (n_out, n_in)).astype(np.float32)
        dev = "cuda"
        self.w = torch.tensor(w, device=dev)
        self.b = torch.zeros(n_out, device=dev)
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.wb = torch.empty((n_out, n_in), dtype=torch.bfloat16, device=dev)
        self.wt = torch.empty((n_in, n_out), dtype=torch.bfloat16, device=dev)
        self.refresh()

    def refresh(self):
        self.ops.to_bf16(self.w, self.wb)
        self.ops.T(self.wb, self.wt)

    def params(self):
        return self.w.numel() + self.b.numel()

    def forward(self, x, keep: bool):
        """x bf16 [M][n_in] -> (y bf16 [M][n_out], pre-activation or None)."""
        torch = self.ops.torch
        M = x.shape[0]
        y = torch.empty((M, self.n_out), dtype=torch.bfloat16, device=x.device)
        pre = None
        if self.gelu:
            pre = torch.empty_like(y) if keep else None
            self.ops.gemm(x, self.wb, y, EPI_GELU, bias=self.b, aux_out=pre)
        else:
            self.ops.gemm(x, self.wb, y, EPI_BF16, bias=self.b)
        return y, pre

    def backward(self, x, dz, pre_in):
        """dz bf16 [M][n_out] (gradient of the pre-activation); x the layer input;
        pre_in the pre-activation that produced x (None for the first layer).
        Accumulates gw, gb; returns the gradient of pre_in (or None)."""
        torch = self.ops.torch
        M = x.shape[0]
        dzt = self.ops.T(dz)                       # [n_out][M]
        xt = self.ops.T(x)                         # [n_in][M]
        self.ops.gemm(dzt, xt, self.gw, EPI_F32)   # gw = dz^T x
        self.ops.colsum(dz, self.gb)
        if pre_in is None:
            return None
        dpre = torch.empty((M, self.n_in), dtype=torch.bfloat16, device=x.device)
        self.ops.gemm(dz, self.wt, dpre, EPI_DGELU, aux_in=pre_in)   # (dz W) * gelu'(pre_in)
        return dpre

    def step(self, t: int, lr: float, wd: float = 0.0):
        self.ops.adam(self.w, self.gw, self.mw, self.vw, t, lr, wb=self.wb, wt=self.wt, wd=wd)
        self.ops.adam(self.b, self.gb, self.mb, self.vb, t, lr)


class MLP:
    def __init__(self, ops, sizes: List[int], rng, last_linear=True):
        self.layers = [Linear(ops, sizes[i + 1], sizes[i], gelu=not (last_linear and i == len(sizes) - 2), rng=rng)
                       for i in range(len(sizes) - 1)]

    def params(self):
        return sum(l.params() for l in self.layers)

    def forward(self, x, keep: bool):
        self.xs, self.pres = [], []
        for l in self.layers:
            y, pre = l.forward(x, keep)
            self.xs.append(x)
            self.pres.append(pre)
            x = y
        return x

    def backward(self, dz):
        for i in range(len(self.layers) - 1, -1, -1):
            pre_in = self.pres[i - 1] if i > 0 else None
            dz = self.layers[i].backward(self.xs[i], dz, pre_in)

    def step(self, t, lr, wd=0.0):
        for l in self.layers:
            l.step(t, lr, wd)


# ------------------------------------------------------------------ network
class Surrogate:
    def __init__(self, width: int = 1024, depth: int = 4, p: int = 512, twidth: int = 512, tdepth: int = 3,
                 seed: int = 0):
        torch = _torch()
        self.ops = _Ops()
        rng = np.random.Generator(np.random.PCG64(seed))
        self.branch = MLP(self.ops, [N_IN] + [width] * depth + [p], rng)
        self.trunk = MLP(self.ops, [N_TRUNK_IN] + [twidth] * tdepth + [p], rng)
        self.err_head = MLP(self.ops, [N_IN, 256, 8], rng)
        self.p = p
        self.pbias = torch.zeros(NP, device="cuda")
        self.gpb = torch.zeros_like(self.pbias)
        self.mpb, self.vpb = torch.zeros_like(self.pbias), torch.zeros_like(self.pbias)
        phi = torch.tensor(trunk_inputs(), device="cuda")
        self.phi = torch.empty(phi.shape, dtype=torch.bfloat16, device="cuda")
        self.ops.to_bf16(phi, self.phi)
        self.t = 0
        self.t_err = 0

    def params(self) -> int:
        return self.branch.params() + self.trunk.params() + self.err_head.params() + NP

    # --- forward / backward of the TL operator
    def forward(self, x_bf16, keep: bool = False):
        """x bf16 [B][128] -> normalised TL prediction float [B][NP]."""
        torch = self.ops.torch
        b = self.branch.forward(x_bf16, keep)           # [B][p]
        tb = self.trunk.forward(self.phi, keep)         # [NP][p]
        pred = torch.empty((x_bf16.shape[0], NP), device="cuda")
        self.ops.gemm(b, tb, pred, EPI_F32, bias=self.pbias)
        if keep:
            self._b, self._tb = b, tb
        return pred

    def backward(self, dpred):
        """dpred bf16 [B][NP]: gradients of every parameter (overwritten)."""
        torch = self.ops.torch
        B = dpred.shape[0]
        self.ops.colsum(dpred, self.gpb)
        tbt = self.ops.T(self._tb)                      # [p][NP]
        db = torch.empty((B, self.p), dtype=torch.bfloat16, device="cuda")
        self.ops.gemm(dpred, tbt, db, EPI_BF16)         # dL/db = dpred t
        dpt = self.ops.T(dpred)                         # [NP][B]
        bt = self.ops.T(self._b)                        # [p][B]
        dt = torch.empty((NP, self.p), dtype=torch.bfloat16, device="cuda")
        self.ops.gemm(dpt, bt, dt, EPI_BF16)            # dL/dt = dpred^T b
        self.branch.backward(db)
        self.trunk.backward(dt)

    def step(self, lr: float, wd: float = 0.0):
        self.t += 1
        self.branch.step(self.t, lr, wd)
        self.trunk.step(self.t, lr, wd)
        self.ops.adam(self.pbias, self.gpb, self.mpb, self.vpb, self.t, lr)

    # --- training on device-resident data
    def train(self, X, Y, epochs: int = 10, batch: int = 256, lr: float = 1e-3, log=None, seed: int = 0) -> List[float]:
        """X bf16 [n][128], Y normalised TL float [n][NP], both on the GPU."""
        torch = self.ops.torch
        n = X.shape[0]
        steps = max(1, (n // batch)) * epochs
        g = torch.Generator(device="cpu").manual_seed(seed)
        loss_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
        dpred = torch.empty((batch, NP), dtype=torch.bfloat16, device="cuda")
        hist = []
        t0 = time.time()
        k = 0
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).cuda()
            loss_dev.zero_()
            nb = max(1, n // batch)
            for i in range(nb):
                idx = perm[i * batch:(i + 1) * batch]
                xb, yb = X[idx], Y[idx]
                pred = self.forward(xb, keep=True)
                self.ops.mse(pred, yb, dpred[:xb.shape[0]], loss_dev, 1.0 / float(xb.shape[0] * NP))
                self.backward(dpred[:xb.shape[0]])
                lr_k = lr * 0.5 * (1.0 + math.cos(math.pi * k / steps))
                self.step(lr_k)
                k += 1
            torch.cuda.synchronize()
            self.ops.check()
            rms_db = math.sqrt(loss_dev.item() / (nb * batch * NP)) * TL_SCALE
            hist.append(rms_db)
            if log:
                log("epoch %d  train TL rms %.3f dB  (%.1f s)" % (ep, rms_db, time.time() - t0))
        return hist

    # --- predicted error (fallback decision)
    def train_error_head(self, X, rms_db, epochs: int = 20, batch: int = 512, lr: float = 1e-3):
        """Fit log(RMS error in dB) of each training field from its features."""
        torch = self.ops.torch
        n = X.shape[0]
        target = torch.zeros((n, 8), device="cuda")
        target[:, 0] = torch.log(rms_db.clamp_min(1e-3))
        target[:, 1:] = 0.0
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        grad = torch.empty((batch, 8), dtype=torch.bfloat16, device="cuda")
        g = torch.Generator(device="cpu").manual_seed(1)
        nb = max(1, n // batch)
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).cuda()
            for i in range(nb):
                idx = perm[i * batch:(i + 1) * batch]
                out = self.err_head.forward(X[idx], keep=True)
                o32 = torch.empty(out.shape, device="cuda")
                o32.copy_(out)
                self.ops.mse(o32, target[idx], grad[:len(idx)], loss, 1.0 / float(len(idx)))
                self.err_head.backward(grad[:len(idx)])
                self.t_err += 1
                self.err_head.step(self.t_err, lr * 0.5 * (1.0 + math.cos(math.pi * ep / epochs)))
        torch.cuda.synchronize()
        self.ops.check()

    def predict_error(self, X):
        out = self.err_head.forward(X, keep=False)
        return out[:, 0].float().exp()

    # --- persistence
    def state(self) -> Dict[str, np.ndarray]:
        s = {"pbias": self.pbias.cpu().numpy()}
        for name, mlp in (("branch", self.branch), ("trunk", self.trunk), ("err", self.err_head)):
            for i, l in enumerate(mlp.layers):
                s["%s%d_w" % (name, i)] = l.w.cpu().numpy()
                s["%s%d_b" % (name, i)] = l.b.cpu().numpy()
        return s

    def load(self, s: Dict[str, np.ndarray]):
        torch = self.ops.torch
        self.pbias.copy_(torch.tensor(s["pbias"]))
        for name, mlp in (("branch", self.branch), ("trunk", self.trunk), ("err", self.err_head)):
            for i, l in enumerate(mlp.layers):
                l.w.copy_(torch.tensor(s["%s%d_w" % (name, i)]))
                l.b.copy_(torch.tensor(s["%s%d_b" % (name, i)]))
                l.refresh()


# ---------------------------------------------------------- data and fallback
def trace_tl(P, idx: Sequence[int], out_rows, chunk: int = 1024, tmpdir: Optional[str] = None,
             max_memory: int = 64 << 30, log=None) -> Dict[str, float]:
    """Plain FP64 traces of environments idx written as normalised TL rows into
    out_rows (a float [len(idx)][NP] GPU tensor). Returns timing."""
    ops = _Ops()
    t_total = 0.0
    d = tmpdir or tempfile.mkdtemp(prefix="c5_")
    pos = 0
    for c0 in range(0, len(idx), chunk):
        sub = list(idx[c0:c0 + chunk])
        roots = [write_env(W.c5_env(P, i), os.path.join(d, "e%d" % i)) for i in sub]
        t0 = time.time()
        with Tracer(precision=PREC_FP64, max_memory=max_memory) as t:
            for r in roots:
                t.add_env(r)
            t.run()
            for k in range(len(sub)):
                ops.tl_db(t.field_device_ptr(k, 0), out_rows[pos + k], NP)
            ops.torch.cuda.synchronize()
        t_total += time.time() - t0
        pos += len(sub)
        for r in roots:
            for ext in (".env",):
                try:
                    os.remove(r + ext)
                except OSError:
                    pass
        if log:
            log("traced %d / %d environments (%.1f s)" % (pos, len(idx), t_total))
    ops.affine(out_rows, 1.0 / TL_SCALE, -TL_MEAN / TL_SCALE)
    return {"trace_s": t_total}


def infer(model: Surrogate, P, idx: Sequence[int], threshold_db: float = 1.0, margin: float = 1.0,
          batch: int = 4096, fallback: bool = True, tmpdir: Optional[str] = None):
    """TL (dB) of environments idx: surrogate prediction, and the plain FP64
    trace for the environments whose predicted error (x margin) exceeds
    threshold_db. Returns (tl float [n][NP] on the GPU, fallback mask, timing)."""
    torch = model.ops.torch
    n = len(idx)
    out = torch.empty((n, NP), device="cuda")
    X = torch.tensor(features(P, idx), device="cuda").bfloat16()
    torch.cuda.synchronize()
    t0 = time.time()
    fb = torch.zeros(n, dtype=torch.bool, device="cuda")
    for c0 in range(0, n, batch):
        xb = X[c0:c0 + batch]
        pred = model.forward(xb, keep=False)
        out[c0:c0 + xb.shape[0]].copy_(pred)
        fb[c0:c0 + xb.shape[0]] = model.predict_error(xb) * margin > threshold_db
    model.ops.affine(out, TL_SCALE, TL_MEAN)
    torch.cuda.synchronize()
    t_sur = time.time() - t0
    t_fb = 0.0
    fb_idx = torch.nonzero(fb).flatten().cpu().numpy()
    if fallback and len(fb_idx):
        rows = torch.empty((len(fb_idx), NP), device="cuda")
        tt = trace_tl(P, [idx[i] for i in fb_idx], rows, tmpdir=tmpdir)
        model.ops.affine(rows, TL_SCALE, TL_MEAN)
        out[torch.tensor(fb_idx, device="cuda")] = rows
        t_fb = tt["trace_s"]
    model.ops.check()
    return out, fb.cpu().numpy(), {"surrogate_s": t_sur, "fallback_s": t_fb}


# ------------------------------------------------------------ calibration
ACCEPT_PRECISION = 0.975   # accepted fields within the threshold, on the validation split


def calibrate_margin(pred_err: np.ndarray, err: np.ndarray, threshold_db: float,
                     precision: float = ACCEPT_PRECISION, min_accept: int = 50) -> float:
    """The margin m of the fallback rule (a field falls back when m x its
    predicted error exceeds threshold_db), from the validation split's
    predicted and actual errors: the fields are accepted in order of predicted
    error up to the largest count (at least min_accept) whose actual errors
    stay within threshold_db for a `precision` fraction of them, and m puts
    the cut at that count's predicted error. Without such a count, m is the
    95th percentile of actual / predicted error (accepted fields then stay
    within the threshold in about 95 % of cases)."""
    order = np.argsort(pred_err, kind="stable")
    ok = err[order] <= threshold_db
    prec = np.cumsum(ok) / np.arange(1, len(ok) + 1)
    good = np.nonzero(prec[min_accept - 1:] >= precision)[0] if len(ok) >= min_accept else np.zeros(0, int)
    if len(good):
        k = int(good[-1]) + min_accept
        cut = float(pred_err[order][k - 1])
        if cut > 0.0:
            return threshold_db / cut * (1.0 - 1e-6)
    return float(np.quantile(err / np.maximum(pred_err, 1e-6), 0.95))


# ------------------------------------------------------------ C5 end to end
def run_c5(n: int = 100000, seed: int = 1005, run_type: str = "IB", fan_deg: float = W.C5_FAN_DEG,
           epochs: int = 40, batch: int = 256, lr: float = 1e-3, threshold_db: float = 1.0,
           infer_batch: int = 4096, chunk: int = 2048, tmpdir: str = "", log=None, save: str = "") -> Dict:
    """Generate n fields with the plain FP64 tracer, train on the first 90 %,
    calibrate the fallback margin on the next 5 % and evaluate on the last
    5 %: the surrogate's own errors, the fallback rate at threshold_db, the
    errors of the returned fields, and the time of the surrogate with its
    fallback against the plain FP64 trace of the same test fields through
    the same call (trace_tl)."""
    torch = _torch()
    P = W.c5_params(n, seed, run_type, fan_deg)
    n_tr, n_va = int(n * 0.90), int(n * 0.05)
    tr, va, te = list(range(n_tr)), list(range(n_tr, n_tr + n_va)), list(range(n_tr + n_va, n))
    tmp = tmpdir or tempfile.mkdtemp(prefix="c5_")
    Y = torch.empty((n, NP), device="cuda")
    gen = trace_tl(P, list(range(n)), Y, chunk=chunk, tmpdir=tmp, log=log)
    X = torch.tensor(features(P, list(range(n))), device="cuda").bfloat16()
    model = Surrogate(seed=0)
    if log:
        log("parameters %d" % model.params())
    t0 = time.time()
    hist = model.train(X[:n_tr], Y[:n_tr], epochs=epochs, batch=batch, lr=lr, log=log)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    # error head on the training fields' actual errors
    rms = torch.empty(n_tr, device="cuda")
    for c0 in range(0, n_tr, infer_batch):
        xb = X[c0:c0 + infer_batch]
        pred = model.forward(xb, keep=False)
        model.ops.row_rms(pred, Y[c0:c0 + xb.shape[0]], rms[c0:c0 + xb.shape[0]])
    rms *= TL_SCALE
    model.train_error_head(X[:n_tr], rms)
    # calibrate the acceptance on the validation split
    pv = model.predict_error(X[n_tr:n_tr + n_va])
    tv = torch.empty(n_va, device="cuda")
    pred = model.forward(X[n_tr:n_tr + n_va], keep=False)
    model.ops.row_rms(pred, Y[n_tr:n_tr + n_va], tv)
    tv *= TL_SCALE
    margin = calibrate_margin(pv.cpu().numpy(), tv.cpu().numpy(), threshold_db)
    # test split: the plain FP64 trace and the surrogate with its fallback,
    # each timed three times, interleaved (the fastest counts: both go through
    # files and the reader, whose time varies by tens of per cent)
    plain_rows = torch.empty((len(te), NP), device="cuda")
    t_plain, t_with = [], []
    for _ in range(3):
        t_plain.append(trace_tl(P, te, plain_rows, tmpdir=tmp)["trace_s"])
        tl, fb, tm = infer(model, P, te, threshold_db=threshold_db, margin=margin, batch=infer_batch, tmpdir=tmp)
        t_with.append(tm["surrogate_s"] + tm["fallback_s"])
    ref = Y[n_tr + n_va:] * TL_SCALE + TL_MEAN
    err = torch.empty(len(te), device="cuda")
    model.ops.row_rms(tl, ref, err)
    err = err.cpu().numpy()
    sur_only, _, tm0 = infer(model, P, te, threshold_db=1e9, batch=infer_batch, tmpdir=tmp)
    e0 = torch.empty(len(te), device="cuda")
    model.ops.row_rms(sur_only, ref, e0)
    e0 = e0.cpu().numpy()
    phi = float(fb.mean())
    out = {
        "fields": n, "run_type": run_type, "fan_deg": fan_deg, "train_fields": n_tr, "test_fields": len(te),
        "params": model.params(), "generate_s": gen["trace_s"], "generate_fields_per_s": n / gen["trace_s"],
        "train_s": t_train, "epochs": epochs, "train_rms_db": hist,
        "surrogate_only_fields_per_s": len(te) / tm0["surrogate_s"], "surrogate_only_rms_db_mean": float(e0.mean()),
        "surrogate_only_rms_db_median": float(np.median(e0)),
        "surrogate_only_within_1db": float((e0 <= 1.0).mean()),
        "threshold_db": threshold_db, "margin": margin, "fallback_rate": phi,
        "fields_per_s_with_fallback": len(te) / min(t_with), "with_fallback_s": t_with,
        "plain_fp64_fields_per_s": len(te) / min(t_plain), "plain_s": t_plain,
        "speedup_with_fallback": min(t_plain) / min(t_with),
        # the same from the per-field costs: the surrogate pass for every
        # field plus the plain trace's time for the fallback fraction
        "speedup_accounted": 1.0 / (tm0["surrogate_s"] / min(t_plain) + phi),
        "returned_rms_db_mean": float(err.mean()), "returned_rms_db_p95": float(np.quantile(err, 0.95)),
        "returned_within_1db": float((err <= 1.0).mean()),
        "returned_within_threshold": float((err <= threshold_db).mean()),
        "accepted_rms_db_mean": float(e0[~fb].mean()) if (~fb).any() else None,
        "accepted_within_1db": float((e0[~fb] <= 1.0).mean()) if (~fb).any() else None,
    }
    pe = (model.predict_error(X[n_tr + n_va:]) * margin).cpu().numpy()
    for thr in (2.0, 3.0, 6.0):
        acc = pe <= thr
        out["accepted_at_%gdb" % thr] = float(acc.mean())
        out["accepted_rms_db_mean_at_%gdb" % thr] = float(e0[acc].mean()) if acc.any() else None
    if save:
        np.savez_compressed(save, **model.state())
    return out


# ---------------------------------------------------------------------- CLI
def main(argv=None):
    """Generate fields with the plain FP64 tracer, train, evaluate on the test
    split (90/5/5 by seed order), report one JSON line."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=100000, help="environments (train + val + test)")
    ap.add_argument("--seed", type=int, default=1005)
    ap.add_argument("--run-type", default="IB", help="RunType of the fields: IB (incoherent Gaussian beams) or CG")
    ap.add_argument("--fan-deg", type=float, default=W.C5_FAN_DEG, help="launch angles -fan .. fan (degrees)")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--threshold-db", type=float, default=1.0)
    ap.add_argument("--infer-batch", type=int, default=4096)
    ap.add_argument("--chunk", type=int, default=2048, help="environments per trace launch")
    ap.add_argument("--save", default="", help="write the weights (.npz)")
    ap.add_argument("--tmpdir", default="")
    a = ap.parse_args(argv)
    out = run_c5(a.n, a.seed, a.run_type, a.fan_deg, a.epochs, a.batch, a.lr, a.threshold_db, a.infer_batch,
                 a.chunk, a.tmpdir, log=lambda m: print(m, flush=True), save=a.save)
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
