"""The full-size 3-D workload (C4) against the reference's own runs, on a
subset of the receiver bearings.

Environment, ray fan (144 bearings x 361 elevations = 51,984 rays), source and
receiver depths / ranges are the full C4 ones (``workloads.c4_3d``); the
receiver bearings are two of the 36 (0 and 180 degrees), so every ray of the
full fan is traced. Fixtures come from ``tests/golden/make_golden_c4.py``
(the reference's bellhopcxx) and hold the sha256 of the input files, which the
tests regenerate from the seeded generator.

* TL ('CB   3'): within 0.1 dB RMS of the reference over receivers where its
  TL < 100 dB (FP64 on both sides; float atomics add in another order).
* Arrivals ('aB   3', merging as the reference's single-threaded run merges):
  the per-receiver counts equal on every receiver; the arrivals of every
  997th receiver equal in bounce counts, delays within 1e-6 relative,
  amplitudes within 1e-4 relative.
"""
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def write_files(files, root):
    for suffix, text in files.items():
        with open(root + suffix, "w") as f:
            f.write(text)


def files_sha(files):
    import hashlib
    h = hashlib.sha256()
    for suffix in sorted(files):
        h.update(suffix.encode())
        h.update(files[suffix].encode())
    return h.hexdigest()


@pytest.mark.parametrize("precision", [B.PREC_FP64, B.PREC_MIXED])
def test_c4_bearings_tl(precision, workdir):
    """FP64 within 0.1 dB of the reference; the mixed precision (FP32
    contributions) within the 0.5 dB TL bound."""
    g = np.load(os.path.join(GOLD, "c4_bearings_tl.npz"))
    files = W.c4_3d(run_type="CB   3", ntheta=2)
    assert files_sha(files) == str(g["sha"]), "the seeded C4 generator no longer gives the fixture's inputs"
    root = os.path.join(workdir, "c4_tl_%d" % precision)
    write_files(files, root)
    with B.Tracer(precision=precision) as t:
        t.setup3d(root)
        t.run()
        u = t.field3d(0)
        st = t.stats()
    assert st["err_bits"] == 0
    assert st["rays"] == 144 * 361
    got = np.transpose(u, (1, 2, 3, 0, 4, 5))   # [isz][isx][isy][itheta] -> .shd order
    ref = g["field"]
    assert got.shape == ref.shape == (1, 1, 2, 1, 101, 501)
    a, b = B.tl_db(got), B.tl_db(ref)
    m = b < 100.0
    d = np.abs(a[m] - b[m])
    rms = float(np.sqrt(np.mean(d ** 2)))
    print("C4 2-bearing TL, precision %d: rms %.2e dB over %d receivers, steps %d" % (
        precision, rms, int(m.sum()), st["steps"]))
    assert m.sum() > 50000
    assert rms < (0.1 if precision == B.PREC_FP64 else 0.5)


def test_c4_bearings_arrivals(workdir):
    g = np.load(os.path.join(GOLD, "c4_bearings_arr.npz"))
    files = W.c4_3d(run_type="aB   3", ntheta=2)
    assert files_sha(files) == str(g["sha"])
    root = os.path.join(workdir, "c4_arr")
    write_files(files, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.set_arrival_options(int(g["maxn"]), True)
        t.setup3d(root)
        t.run()
        narr, arr = t.arrivals()
        st = t.stats()
    assert st["err_bits"] == 0
    narr = narr.reshape(-1)
    ref_n = g["narr"].astype(np.int32)
    diff = np.nonzero(narr != ref_n)[0]
    print("C4 2-bearing arrivals: %d receivers, %d arrivals, %d counts differ" % (
        narr.size, int(narr.sum()), diff.size))
    np.testing.assert_array_equal(narr, ref_n)
    arr = arr.reshape(narr.size, -1)
    idx = g["sample_idx"]
    got = np.concatenate([arr[i, :narr[i]] for i in idx])
    ref = g["sample_arr"]
    assert len(got) == len(ref) > 0
    np.testing.assert_array_equal(got["NTopBnc"], ref[:, 8].astype(np.int32))
    np.testing.assert_array_equal(got["NBotBnc"], ref[:, 9].astype(np.int32))
    np.testing.assert_allclose(got["delay_re"], ref[:, 2], rtol=1e-6)
    np.testing.assert_allclose(got["a"], ref[:, 0], rtol=1e-4)
