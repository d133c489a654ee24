"""The autotuner (bhcb_autotune): it picks launch shapes from the candidate
sets by timing the prepared TL workload, keeps them in the context, and the
fields computed with the chosen shapes equal the default ones."""
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import write_env

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_autotune_keeps_results(precision, tmp_path):
    spec = W.rd_gauss(nalpha=801, nrz=101, nrr=401, nbty=40)
    root = write_env(spec, os.path.join(str(tmp_path), "tune"))
    with B.Tracer(precision=precision) as t:
        t.setup(root).set_frequencies(0, [60.0, 240.0])
        t.run()
        ref = [t.field(0, i) for i in range(2)]
        tune = t.autotune(repeats=1)
        assert tune["trace_block"] in (32, 64)
        assert tune["influence_ctas_per_sm"] in (2, 3, 4, 5, 6, 8, 10, 12)
        assert tune["stage_kb"] in (0, 32, 64)
        assert 0 < tune["trace_ms"] < 1e4 and 0 < tune["influence_ms"] < 1e4
        t.run()
        got = [t.field(0, i) for i in range(2)]
        for a, b in zip(got, ref):
            np.testing.assert_allclose(a, b, rtol=1e-3, atol=1e-6 * np.abs(b).max())
        with pytest.raises(B.BhcbError):
            t.set_tuning(48, 4)
        with pytest.raises(B.BhcbError):
            t.set_tuning(64, 3, 65)
        for stage_kb in (0, 64):   # tables from global memory, all tables staged
            t.set_tuning(64, 3, stage_kb)
            t.run()
            np.testing.assert_allclose(t.field(0, 0), ref[0], rtol=1e-3, atol=1e-6 * np.abs(ref[0]).max())
