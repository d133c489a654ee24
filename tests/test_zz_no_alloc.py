"""Allocation-free entry point bhcb_run_noalloc against the regular run.

Callers that cannot allocate device memory while running (a fixed budget owned
by another allocator, allocation-free real-time loops) prepare a context once
and then call bhcb_run_noalloc with their own output buffer; the entry point
keeps its scratch in a static device array and runs on the context's GPU. This file is collected last so that a run stopping at the first failure
has already run every other test; it also passes alone in a fresh process
(the first call on the device performs the one-time scratch set-up).
"""
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import write_env

pytestmark = pytest.mark.gpu

TL_MAX = 100.0      # compare where TL < 100 dB
TL_RMS_DB = 0.5     # the parity tolerance used by the other GPU tests


def tl_rms(got, ref):
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < TL_MAX
    d = np.abs(a[m] - b[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2))), int(m.sum())


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
@pytest.mark.parametrize("beam", ["G", "B"])
def test_noalloc_matches_regular_run_two_calls(precision, beam, tmp_path):
    import torch
    spec = W.rd_gauss(nalpha=301, nrz=51, nrr=201, nbty=40) if beam == "B" else W.munk_tl(
        nalpha=301, nrz=51, nrr=201)
    root = write_env(spec, os.path.join(str(tmp_path), "na_" + beam))
    with B.Tracer(precision=precision) as t:
        t.setup(root).run()                      # regular entry point (allocates)
        ref = t.field(0, 0)
        # caller-owned output buffer; the entry point itself allocates nothing
        out = torch.empty(ref.shape, dtype=torch.complex64, device="cuda")
        for call in range(2):
            out.fill_(complex(1e30, 1e30))       # stale contents must be overwritten
            torch.cuda.synchronize()
            t.run_noalloc(out.data_ptr(), out.numel() * 8)
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            rms, n = tl_rms(got[0], ref[0])
            print("call %d precision %d beam %s: TL rms %.5f dB over %d receivers" % (call, precision, beam, rms, n))
            assert n > 100
            assert rms < TL_RMS_DB
            assert rms < 0.05   # same math, only the float summation order differs


def test_noalloc_rejects_fields_over_the_static_limit(tmp_path):
    spec = W.munk_tl(nalpha=5, nrz=2049, nrr=1025)   # 2,100,225 receivers > 2**21
    root = write_env(spec, os.path.join(str(tmp_path), "big"))
    with B.Tracer() as t:
        t.setup(root)
        t.prepare()
        with pytest.raises(B.BhcbError, match="static scratch limit") as ei:
            t.run_noalloc(1 << 40, 1 << 40)   # never dereferenced: rejected before any work
        assert ei.value.code == 1


@pytest.mark.parametrize("beam", ["G", "B"])
def test_noalloc_irregular_grid(beam, tmp_path):
    """Irregular receiver grid (one receiver per range, at depth rz[ir])."""
    import torch
    spec = W.munk_tl(nalpha=301, nrz=201, nrr=201, beam=beam)
    spec.run_type = "C%s RI " % beam
    root = write_env(spec, os.path.join(str(tmp_path), "irr_" + beam))
    with B.Tracer(precision=B.PREC_MIXED) as t:
        t.setup(root).run()
        ref = t.field(0, 0)
        out = torch.empty(ref.shape, dtype=torch.complex64, device="cuda")
        for call in range(2):
            out.fill_(complex(1e30, 1e30))
            torch.cuda.synchronize()
            t.run_noalloc(out.data_ptr(), out.numel() * 8)
            rms, n = tl_rms(out.cpu().numpy()[0], ref[0])
            print("irregular %s call %d: TL rms %.5f dB over %d receivers" % (beam, call, rms, n))
            assert n > 50
            assert rms < 0.05


def test_noalloc_rejects_non_tl_context(tmp_path):
    """A context prepared for arrivals has no TL field to compute."""
    spec = W.munk_tl(nalpha=21, nrz=11, nrr=21)
    spec.run_type = "aG RR "
    root = write_env(spec, os.path.join(str(tmp_path), "arr"))
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup(root)
        t.prepare()
        with pytest.raises(B.BhcbError, match="not a TL field") as ei:
            t.run_noalloc(1 << 40, 1 << 40)   # rejected before any work
        assert ei.value.code == 6


def test_noalloc_keeps_the_callers_device(tmp_path):
    """The call runs on the context's GPU and leaves the caller's current
    device as it was; with two GPUs the context lives on the one that is not
    current."""
    import torch
    ngpu = torch.cuda.device_count()
    gpu = 1 if ngpu > 1 else 0
    spec = W.munk_tl(nalpha=101, nrz=31, nrr=101)
    root = write_env(spec, os.path.join(str(tmp_path), "dev"))
    torch.cuda.set_device(0)
    with B.Tracer(gpu=gpu, precision=B.PREC_MIXED) as t:
        t.setup(root).run()
        ref = t.field(0, 0)
        out = torch.empty(ref.shape, dtype=torch.complex64, device="cuda:%d" % gpu)
        torch.cuda.set_device(0)
        t.run_noalloc(out.data_ptr(), out.numel() * 8)
        assert torch.cuda.current_device() == 0
        rms, n = tl_rms(out.cpu().numpy()[0], ref[0])
        print("context on GPU %d of %d: TL rms %.5f dB" % (gpu, ngpu, rms))
        assert n > 50 and rms < 0.05
