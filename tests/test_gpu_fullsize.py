"""GPU parity at the full sizes of the benchmark configurations.

The reduced parity cases elsewhere pin the arithmetic; these run the real
shapes through the same calls a user (and bench.py) makes and compare with the
oracle run over the whole ray fan on the host's threads:

* C1 — Munk, 2001 hat beams, 201 x 1001 receivers: FP64 and mixed TL; the FP64
  trace takes exactly the oracle's ray steps and applies exactly its
  beam-receiver contributions.
* C2 — range-dependent Gaussian beams, 20001 rays, 501 x 2001 receivers, 10
  frequencies sharing one trajectory, run as the benchmark runs it (prepare,
  autotune, launch: trace, influence and scale, replayed from a CUDA graph);
  the 50 Hz and 500 Hz fields against the oracle, and the FP64 trace's step
  count equal to the oracle's.
* C3 — the 256-environment batch in one run; the first four seeded
  environments of the batch against the oracle.

Tolerances: TL = -20 log10|p| within 0.5 dB RMS over receivers
where the oracle TL < 100 dB (mixed precision), 0.1 dB RMS for the FP64 path.
"""
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import write_env
import oracle_ctypes

pytestmark = pytest.mark.gpu

TL_MAX = 100.0
RMS_FP64 = 0.1
RMS_MIXED = 0.5


def tl_err(got, ref):
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < TL_MAX
    d = np.abs(a[m] - b[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2))), float(d.max()), int(m.sum())


_ORACLE = {}


def oracle_field(key, spec):
    """Oracle run of the whole fan (cached per session: several tests share it)."""
    if key not in _ORACLE:
        _ORACLE[key] = oracle_ctypes.run_threaded(spec)
    return _ORACLE[key]


@pytest.mark.parametrize("precision", [B.PREC_FP64, B.PREC_MIXED])
def test_c1_full(precision, workdir):
    spec = W.munk_tl()
    assert (spec.nalpha, spec.nrz, spec.nrr) == (2001, 201, 1001)
    ref = oracle_field("c1", spec)
    root = write_env(spec, os.path.join(workdir, "c1_full_%d" % precision))
    with B.Tracer(precision=precision) as t:
        t.setup(root).run()
        got = t.field()[0]
        st = t.stats()
    rms, mx, n = tl_err(got, ref["field"][0])
    print("C1 prec %d: rms %.5f dB max %.3f dB over %d receivers; steps %d/%d evals %d/%d" % (
        precision, rms, mx, n, st["steps"], ref["nsteps"], st["evals"], ref["nevals"]))
    assert st["err_bits"] == 0
    assert n > 100000
    if precision == B.PREC_FP64:
        assert rms < RMS_FP64
        assert st["steps"] == ref["nsteps"]
        assert st["evals"] == ref["nevals"]
    else:
        assert rms < RMS_MIXED
        assert st["steps"] == ref["nsteps"]


def test_c2_full_bench_sequence(workdir):
    """The benchmark's own sequences on the full C2 workload: one step at a
    time (direct, captured, replayed) and its headline, pipelined launches
    (five back to back after the warm-up, the last one's fields checked)."""
    spec = W.rd_gauss()
    freqs = W.rd_gauss_freqs()
    assert (spec.nalpha, spec.nrz, spec.nrr, len(freqs)) == (20001, 501, 2001, 10)
    root = write_env(spec, os.path.join(workdir, "c2_full"))
    runs = {}
    for pipe in (False, True):
        with B.Tracer(precision=B.PREC_MIXED, pipeline=pipe) as t:
            t.setup(root)
            t.set_frequencies(0, freqs)
            t.prepare()
            t.autotune(repeats=2)
            for _ in range(3):   # serial: direct, captured, replayed
                t.launch()
                t.sync()
            if pipe:
                for _ in range(5):
                    t.launch()
                t.sync()
            st = t.stats()
            runs[pipe] = (st, {i: t.field(0, i)[0] for i in (0, len(freqs) - 1)})
    for pipe, (st, fields) in runs.items():
        assert st["err_bits"] == 0
        assert st["fields"] == 10 and st["groups"] == 1   # one shared trajectory
        for i in (0, len(freqs) - 1):
            s = W.rd_gauss(freq=freqs[i])
            ref = oracle_field("c2_%d" % i, s)
            rms, mx, n = tl_err(fields[i], ref["field"][0])
            print("C2 mixed%s %.1f Hz: rms %.4f dB max %.2f dB over %d receivers; steps %d/%d" % (
                " pipelined" if pipe else "", freqs[i], rms, mx, n, st["steps"], ref["nsteps"]))
            assert n > 300000   # 1.0 M receivers, about half of them above 100 dB at 500 Hz
            assert rms < RMS_MIXED
            assert st["steps"] == ref["nsteps"]


def test_c2_full_fp64(workdir):
    """FP64 trace of the full C2 fan at 500 Hz: steps and contributions equal
    the oracle's, TL within the FP64 bound."""
    freqs = W.rd_gauss_freqs()
    spec = W.rd_gauss(freq=freqs[-1])
    root = write_env(spec, os.path.join(workdir, "c2_full_fp64"))
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup(root).run()
        got = t.field()[0]
        st = t.stats()
    ref = oracle_field("c2_%d" % (len(freqs) - 1), spec)
    rms, mx, n = tl_err(got, ref["field"][0])
    print("C2 FP64 %.1f Hz: rms %.5f dB max %.3f dB; steps %d/%d evals %d/%d" % (
        freqs[-1], rms, mx, st["steps"], ref["nsteps"], st["evals"], ref["nevals"]))
    assert st["err_bits"] == 0
    assert st["steps"] == ref["nsteps"]
    assert rms < RMS_FP64
    assert st["evals"] == ref["nevals"]


def test_c3_batch_envs(workdir):
    """The whole 256-environment batch in one run; four of its environments
    (the first four seeds) against the oracle."""
    envs = W.batch_envs()
    assert len(envs) == 256
    with B.Tracer(precision=B.PREC_MIXED) as t:
        for i, e in enumerate(envs):
            t.add_env(write_env(e, os.path.join(workdir, "c3_%03d" % i)))
        t.run()
        st = t.stats()
        got = {i: t.field(i, 0)[0] for i in range(4)}
    assert st["err_bits"] == 0
    assert st["rays"] == sum(e.nalpha for e in envs)
    for i in range(4):
        ref = oracle_ctypes.run_threaded(envs[i])
        rms, mx, n = tl_err(got[i], ref["field"][0])
        print("C3 env %d (%d rays, %dx%d, %.0f Hz): rms %.4f dB max %.2f dB over %d receivers" % (
            i, envs[i].nalpha, envs[i].nrz, envs[i].nrr, envs[i].freq, rms, mx, n))
        assert n > 1000
        assert rms < RMS_MIXED
