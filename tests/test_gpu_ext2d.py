"""GPU parity of the 2-D options that the oracle restatement does not cover
(quad SSP, ...) against the reference itself.

The fixtures tests/golden/x2d_*.npz hold each case's input files and the field
the reference's own bellhopcxx computed single-threaded (made by
tests/golden/make_golden_ext.py). The product runs the same files through the
C ABI. Tolerance: TL = -20 log10|p| within 0.1 dB RMS (FP64 tracer) and
0.5 dB RMS (mixed tracer) over receivers where the reference's TL < 100 dB.
"""
import glob
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = sorted(p for p in glob.glob(os.path.join(HERE, "golden", "x2d_*.npz"))
              if not os.path.basename(p).startswith(("x2d_arr_", "x2d_eig_")))   # TL fixtures
TL_MAX = 100.0


def write_case(npz, root):
    for k in npz.files:
        if k.startswith("file_"):
            with open(root + "." + k[5:], "w") as f:
                f.write(str(npz[k]))


def tl_err(got, ref):
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < TL_MAX
    d = np.abs(a[m] - b[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2))), int(m.sum())


@pytest.mark.parametrize("precision", [B.PREC_FP64, B.PREC_MIXED])
@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_field_matches_reference(path, precision, workdir):
    g = np.load(path)
    root = os.path.join(workdir, "%s_%d" % (os.path.basename(path)[:-4], precision))
    write_case(g, root)
    with B.Tracer(precision=precision) as t:
        t.setup(root)
        t.run()
        u = t.field(0, 0)
        st = t.stats()
    assert st["err_bits"] == 0
    ref = g["field"]
    assert u.shape == ref.shape
    err, n = tl_err(u, ref)
    print(os.path.basename(path), precision, "rms %.4f dB over %d" % (err, n))
    assert n > 100
    assert err < (0.1 if precision == B.PREC_FP64 else 0.5), "TL RMS %.3f dB" % err
