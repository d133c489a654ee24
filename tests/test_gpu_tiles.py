"""The tiled influence of the mixed-precision TL path against the segment-by-
segment influence and against the oracle.

Mixed-precision TL runs on rectilinear receiver grids take the tiled path by
default; ``segment_influence=True`` selects the segment-by-segment kernel.
Both evaluate the same FP32 contribution formula on the same segment records,
so the fields agree to float rounding and the applied contributions almost
exactly (the caustic-branch phase is applied as a rotation, the column phase
as a recurrence on equally spaced ranges). The cases cover several
frequencies sharing one trajectory, several source depths, more receiver
depths than one depth block (256), a column count that is not a multiple of
the column block (4), incoherent TL, hat beams and unequally spaced ranges.
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


def tl_err(got, ref):
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < TL_MAX
    d = np.abs(a[m] - b[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2))), int(m.sum())


def run(root, freqs, segment):
    with B.Tracer(precision=B.PREC_MIXED, segment_influence=segment) as t:
        t.setup(root)
        if freqs:
            t.set_frequencies(0, freqs)
        t.run()
        nf = len(freqs) if freqs else 1
        return [t.field(0, i) for i in range(nf)], t.stats()


def _multi_source():
    s = W.munk_tl(nalpha=401, nrz=101, nrr=201)
    s.nsz = 3
    s.sz = (500.0, 1000.0, 1500.0)
    return s


def _incoherent():
    s = W.munk_tl(nalpha=401, nrz=61, nrr=201, beam="B")
    s.run_type = "IB RR "
    return s


def _unequal_ranges():
    s = W.munk_tl(nalpha=401, nrz=61, nrr=97, beam="B")
    r = np.sort(np.concatenate([[0.0, 100.0], np.random.default_rng(7).uniform(0.0, 100.0, 95)]))
    s.rr_km = tuple(float(x) for x in r)
    return s


CASES = {
    "rd_gauss_3freq_301z_203r": (W.rd_gauss(nalpha=801, nrz=301, nrr=203, nbty=40), [50.0, 158.1, 500.0]),
    "munk_hat_3sources": (_multi_source(), None),
    "munk_gauss_incoherent": (_incoherent(), None),
    "munk_gauss_unequal_ranges": (_unequal_ranges(), None),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tiled_matches_segment_influence(name, workdir):
    spec, freqs = CASES[name]
    root = write_env(spec, os.path.join(workdir, "tiles_" + name))
    tiled, st_t = run(root, freqs, segment=False)
    seg, st_s = run(root, freqs, segment=True)
    assert st_t["err_bits"] == 0 and st_s["err_bits"] == 0
    assert st_t["steps"] == st_s["steps"]
    for i, (a, b) in enumerate(zip(tiled, seg)):
        assert a.shape == b.shape
        rms, n = tl_err(a, b)
        print("%s f%d: tiled vs segment rms %.5f dB over %d receivers; evals %d vs %d" % (
            name, i, rms, n, st_t["evals"], st_s["evals"]))
        assert n > 100
        assert rms < 0.01
    assert abs(st_t["evals"] - st_s["evals"]) <= 1e-4 * st_s["evals"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_tiled_matches_oracle(name, workdir):
    spec, freqs = CASES[name]
    root = write_env(spec, os.path.join(workdir, "tiles_o_" + name))
    tiled, st = run(root, freqs, segment=False)
    for i, f in enumerate(freqs or [spec.freq]):
        s2 = spec
        if freqs:
            import copy
            s2 = copy.deepcopy(spec)
            s2.freq = f
        ref = oracle_ctypes.run(s2)["field"]
        for isz in range(ref.shape[0]):
            rms, n = tl_err(tiled[i][isz], ref[isz])
            print("%s %.1f Hz source %d: rms %.4f dB over %d receivers" % (name, f, isz, rms, n))
            assert n > 100
            assert rms < 0.5
