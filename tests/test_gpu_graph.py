"""CUDA-graph capture of one field run (bhcb_graph_*): the captured trace +
influence + scale sequence, replayed several times into a caller-owned buffer,
gives the regular run's field, and replays on a caller stream."""
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import write_env

pytestmark = pytest.mark.gpu


def tl_rms(got, ref):
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < 100.0
    d = np.abs(a[m] - b[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2))), int(m.sum())


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_graph_replays_match_regular_run(precision, tmp_path):
    import torch
    spec = W.rd_gauss(nalpha=301, nrz=51, nrr=201, nbty=40)
    root = write_env(spec, os.path.join(str(tmp_path), "graph"))
    with B.Tracer(precision=precision) as t:
        t.setup(root).run()
        ref = t.field(0, 0)
        out = torch.empty(ref.shape, dtype=torch.complex64, device="cuda")
        with t.graph(out.data_ptr(), out.numel() * 8) as g:
            side = torch.cuda.Stream()
            for k in range(3):
                out.fill_(complex(1e30, 1e30))
                torch.cuda.synchronize()
                if k < 2:
                    g.launch()
                    st = g.status()
                else:   # on a caller stream
                    g.launch(side.cuda_stream)
                    st = g.status(side.cuda_stream)
                assert st["err_bits"] == 0 and st["evals"] > 0
                got = out.cpu().numpy()
                rms, n = tl_rms(got[0], ref[0])
                assert n > 100 and rms < 0.05, (k, rms)


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_batched_step_graph_replays(precision, tmp_path):
    """bhcb_launch on a prepared batch: the first launch runs the kernels
    directly, the second captures the step (several environments, several
    frequencies sharing one trajectory) into a CUDA graph, later launches replay
    it. Every launch gives the fields of a run without graphs."""
    envs = [W.rd_gauss(nalpha=401, nrz=61, nrr=201, nbty=40), W.munk_tl(nalpha=301, nrz=51, nrr=151, beam="B")]
    freqs = [[50.0, 158.1, 500.0], [50.0, 200.0]]
    roots = [write_env(s, os.path.join(str(tmp_path), "b%d" % i)) for i, s in enumerate(envs)]

    def setup(t):
        for i, r in enumerate(roots):
            t.add_env(r)
            t.set_frequencies(i, freqs[i])

    with B.Tracer(precision=precision, graphs=False) as t:
        setup(t)
        t.run()
        ref = [[t.field(i, k) for k in range(len(freqs[i]))] for i in range(len(roots))]
    with B.Tracer(precision=precision) as t:
        setup(t)
        t.prepare()
        for step in range(4):
            t.launch()
            t.sync()
            st = t.stats()
            assert st["err_bits"] == 0 and st["evals"] > 0
            for i in range(len(roots)):
                for k in range(len(freqs[i])):
                    rms, n = tl_rms(t.field(i, k)[0], ref[i][k][0])
                    assert n > 100 and rms < 0.01, (step, i, k, rms)


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_pipelined_launches_match_serial(precision, workdir):
    """BHCB_FLAG_PIPELINE: five launches back to back (the trace of one beside
    the influence of the previous, two buffer slots), one sync; the fields
    equal a serial run's (float atomics: 1e-5 of the field maximum) and the
    counters are the last launch's."""
    spec = W.munk_tl(nalpha=401, nrz=51, nrr=201, beam="B")
    root = write_env(spec, os.path.join(workdir, "pipe_%d" % precision))
    freqs = [50.0, 100.0, 200.0]
    with B.Tracer(precision=precision) as t:
        t.setup(root)
        t.set_frequencies(0, freqs)
        t.run()
        ref = [t.field(0, i) for i in range(len(freqs))]
        st_ref = t.stats()
    with B.Tracer(precision=precision, pipeline=True) as t:
        t.setup(root)
        t.set_frequencies(0, freqs)
        t.prepare()
        for _ in range(5):
            t.launch()
        t.sync()
        st = t.stats()
        got = [t.field(0, i) for i in range(len(freqs))]
        # and again after the sync (the first launch of an epoch)
        t.launch()
        t.sync()
        again = [t.field(0, i) for i in range(len(freqs))]
    assert st["err_bits"] == 0
    assert st["steps"] == st_ref["steps"] and st["segments"] == st_ref["segments"]
    for a, b, c in zip(got, ref, again):
        tol = 1e-5 * np.abs(b).max()
        np.testing.assert_allclose(a, b, rtol=0, atol=tol)
        np.testing.assert_allclose(c, b, rtol=0, atol=tol)
