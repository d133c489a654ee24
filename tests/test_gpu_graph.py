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
