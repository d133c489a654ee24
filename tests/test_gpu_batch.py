"""GPU parity of a batch of uneven environments traced in one launch.

Several environments (different SSP node counts, depths, halfspaces,
frequencies, ray counts and receiver grids; the shape of the 256-environment
batch workload, scaled down) are added to one context and traced together.
Each environment's field is compared with the oracle run on that environment
alone: FP64 within 0.1 dB RMS, mixed within 0.5 dB RMS (TL < 100 dB).
"""
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import write_env
import oracle_ctypes

pytestmark = pytest.mark.gpu


def tl_rms(got, ref):
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < 100.0
    d = np.abs(a[m] - b[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2)))


@pytest.mark.parametrize("precision,tol", [(B.PREC_FP64, 0.1), (B.PREC_MIXED, 0.5)], ids=["fp64", "mixed"])
def test_batch_of_uneven_envs(precision, tol, workdir):
    specs = W.batch_envs(n=6, seed=1003, scale=0.04)
    roots = [write_env(s, os.path.join(workdir, "batch_%d" % i)) for i, s in enumerate(specs)]
    with B.Tracer(precision=precision) as t:
        for r in roots:
            t.add_env(r)
        t.run()
        st = t.stats()
        got = [t.field(i, 0)[0] for i in range(len(specs))]
    assert st["groups"] == len(specs) and st["err_bits"] == 0
    for i, s in enumerate(specs):
        ref = oracle_ctypes.run(s)["field"][0]
        assert got[i].shape == ref.shape
        err = tl_rms(got[i], ref)
        assert err < tol, "env %d: %.3f dB" % (i, err)


def test_batch_in_waves_when_segments_exceed_max_memory(workdir):
    """A max_memory too small for all segments at once: the groups are traced in
    waves; the fields equal a run that fits in one launch."""
    specs = W.batch_envs(n=6, seed=1003, scale=0.04)
    roots = [write_env(s, os.path.join(workdir, "wave_%d" % i)) for i, s in enumerate(specs)]

    def run(max_memory):
        with B.Tracer(precision=B.PREC_FP64, max_memory=max_memory) as t:
            for r in roots:
                t.add_env(r)
            t.run()
            return [t.field(i, 0)[0] for i in range(len(specs))], t.stats()

    full, st = run(0)
    seg_bytes = 192   # FP64 segment record
    small = 8 * 2**20 + st["segments"] * seg_bytes // 3
    waved, st2 = run(small)
    assert st2["segments"] == st["segments"] and st2["evals"] == st["evals"]
    for a, b in zip(waved, full):
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-12 * np.abs(b).max())
