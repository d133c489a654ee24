"""The oracle (C restatement) against the reference itself.

Golden fixtures in tests/golden/ were produced by the reference's own
bellhopcxx, compiled from its unmodified sources (tests/golden/make_golden.py).
The oracle must reproduce them bit-for-bit. When the reference build is present
(oracle/_ref), a second check runs it live on a fresh randomised case.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle_ctypes  # noqa: E402
from cases import CASES  # noqa: E402
from bellhopcuda_b200.envfile import write_env  # noqa: E402
from bellhopcuda_b200.shdfile import read_shd  # noqa: E402

REF_EXE = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "bellhopcxx")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(name):
    gold = np.load(os.path.join(HERE, "golden", name + ".npz"))
    res = oracle_ctypes.run(CASES[name]())
    assert res["err_bits"] == 0
    got = res["field"]
    ref = gold["field"]
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(res["rr"], gold["rr"])
    np.testing.assert_array_equal(res["rz"], gold["rz"])


@pytest.mark.skipif(not os.path.exists(REF_EXE), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5, 6, 7, 8])
def test_oracle_matches_reference_live(seed, workdir):
    from bellhopcuda_b200 import workloads as W
    rng = np.random.Generator(np.random.PCG64(seed))
    spec = W.rd_gauss(seed=100 + seed, nalpha=int(rng.integers(51, 201)), nrz=int(rng.integers(11, 41)),
                      nrr=int(rng.integers(21, 121)), nbty=int(rng.integers(5, 60)))
    spec.freq = float(rng.uniform(30, 400))
    spec.run_type = ["CG RR ", "CB RR ", "IB RR ", "SB RR ", "SG RR ", "IG RR "][seed % 6]
    spec.ssp_type = ["P", "C", "S", "N"][seed % 4]   # PCHIP, c-linear, spline, n2-linear
    root = write_env(spec, os.path.join(workdir, "live%d" % seed))
    subprocess.run([REF_EXE, "-2", "-1", root], check=True, capture_output=True)
    ref = read_shd(root + ".shd")["field"][0, 0, 0]
    got = oracle_ctypes.run(spec)["field"]
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("seed,run_type", [(1002, "aG RR "), (1003, "aB RR "), (1004, "aB RR ")])
def test_oracle_arrivals_match_reference_counts(seed, run_type, workdir):
    """Arrivals (merging, one thread) of the oracle and of the reference's own
    run: per receiver the count, amplitudes, delays and bounce counts equal."""
    if not os.path.exists(REF_EXE):
        pytest.skip("reference build (oracle/_ref) not present")
    import re
    from bellhopcuda_b200 import workloads as W
    from bellhopcuda_b200.arrfile import read_arr_binary
    spec = W.rd_gauss(seed=seed, nalpha=151, nrz=7, nrr=15, nbty=20)
    spec.run_type = run_type
    root = write_env(spec, os.path.join(workdir, "arr"))
    subprocess.run([REF_EXE, "-2", "-1", root], check=True, capture_output=True)
    A = read_arr_binary(root + ".arr")
    mx = int(re.search(r"Maximum # of arrivals = *(\d+)", open(root + ".prt").read()).group(1))
    o = oracle_ctypes.run(spec, max_narr=mx, allow_merging=1)
    for k, arrs in enumerate(A["sources"][0]["arrivals"]):
        iz, ir = divmod(k, spec.nrr)
        n = o["narr"][0, iz, ir]
        assert n == len(arrs)
        oa = o["arr"][0, iz, ir, :n]
        np.testing.assert_array_equal(oa["a"], arrs[:, 0])
        np.testing.assert_array_equal(oa["delay_re"], arrs[:, 2])
        np.testing.assert_array_equal(oa["NTopBnc"].astype(np.float32), arrs[:, 6])
        np.testing.assert_array_equal(oa["NBotBnc"].astype(np.float32), arrs[:, 7])


@pytest.mark.parametrize("seed,run_type", [(1002, "EG RR "), (1005, "EB RR ")])
def test_oracle_eigen_hits_match_reference(seed, run_type, workdir):
    """Eigen hits (RecordEigenHit) of the oracle against the reference's own
    single-threaded run: the reference writes one re-traced ray per hit, in hit
    order, whose take-off angle and point count (the hit's step + 2) pin the
    hit list."""
    if not os.path.exists(REF_EXE):
        pytest.skip("reference build (oracle/_ref) not present")
    from bellhopcuda_b200 import workloads as W
    from bellhopcuda_b200.rayfile import read_ray
    spec = W.rd_gauss(seed=seed, nalpha=101, nrz=3, nrr=5, nbty=20)
    spec.run_type = run_type
    root = write_env(spec, os.path.join(workdir, "eig"))
    subprocess.run([REF_EXE, "-2", "-1", root], check=True, capture_output=True)
    rays = read_ray(root + ".ray")["rays"]
    o = oracle_ctypes.run(spec)
    hits = o["hits"]
    assert len(hits) == o["neigen"] == len(rays) > 0
    np.testing.assert_array_equal(hits["is"] + 2, [len(r["xy"]) for r in rays])
    fan = np.linspace(spec.alpha[0], spec.alpha[1], spec.nalpha)
    np.testing.assert_allclose(fan[hits["ialpha"]], [r["alpha"] for r in rays], rtol=0, atol=1e-9)


@pytest.mark.parametrize("tag,run_type", [("line", "CB RX "), ("line_hat", "IG RX "), ("irregular", "CB RI ")])
def test_oracle_matches_reference_line_source_and_irregular_grid(tag, run_type, workdir):
    """Line sources (RunType(4) 'X': ScalePressure's line-source constant)
    and an irregular receiver grid (RunType(5) 'I': one depth per range) of
    the oracle against the reference's own single-threaded runs, bit-exact."""
    if not os.path.exists(REF_EXE):
        pytest.skip("reference build (oracle/_ref) not present")
    from bellhopcuda_b200 import workloads as W
    spec = W.rd_gauss(seed=1010, nalpha=121, nrz=60 if tag == "irregular" else 31, nrr=60, nbty=30)
    spec.freq = 120.0
    spec.run_type = run_type
    root = write_env(spec, os.path.join(workdir, tag))
    subprocess.run([REF_EXE, "-2", "-1", root], check=True, capture_output=True)
    ref = read_shd(root + ".shd")["field"][0, 0, 0]
    got = oracle_ctypes.run(spec)["field"]
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got, ref)
