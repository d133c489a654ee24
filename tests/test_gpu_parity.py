"""GPU parity: the product (through the C ABI) against the oracle.

Tolerance: TL = -20 log10|p| within 0.5 dB RMS over receivers where
the oracle TL < 100 dB; the FP64 tracer is also held to a tighter RMS bound.
"""
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import EnvSpec, write_env
import oracle_ctypes

pytestmark = pytest.mark.gpu

TL_MAX = 100.0


def tl_err(got, ref):
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < TL_MAX
    d = np.abs(a[m] - b[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2))), float(np.percentile(d, 99)), int(m.sum())


def run_product(spec, root, precision, freqs=None):
    write_env(spec, root)
    with B.Tracer(precision=precision) as t:
        t.setup(root)
        if freqs is not None:
            t.set_frequencies(0, freqs)
        t.run()
        nf = len(freqs) if freqs is not None else 1
        out = [t.field(0, i)[0] for i in range(nf)]
        return out, t.stats()


def _irregular(beam):
    s = W.munk_tl(nalpha=301, nrz=201, nrr=201, beam=beam)
    s.run_type = "C%s RI " % beam
    return s


def _steep():
    s = W.munk_tl(nalpha=301, nrz=51, nrr=201, beam="B")
    s.alpha = (-75.0, 75.0)
    return s


CASES = {
    "munk_irregular_hat": _irregular("G"),
    "munk_irregular_gauss": _irregular("B"),
    "munk_steep_gauss": _steep(),
    "munk_hat": W.munk_tl(nalpha=301, nrz=51, nrr=201),
    "munk_gauss": W.munk_tl(nalpha=301, nrz=51, nrr=201, beam="B"),
    "rd_pchip_gauss": W.rd_gauss(nalpha=401, nrz=61, nrr=201, nbty=60),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", [B.PREC_FP64, B.PREC_MIXED])
def test_tl_matches_oracle(name, precision, workdir):
    spec = CASES[name]
    ref = oracle_ctypes.run(spec)
    got, st = run_product(spec, os.path.join(workdir, "%s_%d" % (name, precision)), precision)
    rms, p99, n = tl_err(got[0], ref["field"][0])
    print(name, precision, "rms %.4f p99 %.3f n %d steps %d/%d evals %d/%d" % (
        rms, p99, n, st["steps"], ref["nsteps"], st["evals"], ref["nevals"]))
    assert n > 100
    assert rms < (0.1 if precision == B.PREC_FP64 else 0.5)
    assert st["err_bits"] == 0
