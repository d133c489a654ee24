"""Ray trajectories on the GPU against the reference itself: RunType 'R' (every
ray) and the eigenray re-trace of 'E' runs, through the C ABI, compared with
the .ray files the reference's single-threaded bellhopcxx wrote for the same
inputs (tests/golden/rays_*.npz, made by tests/golden/make_golden_rays.py).
Same rays in the same order with the same take-off angles; on at least 97 % of
them the same number of points and bounce counts and every point within 1 mm
(the rest may take a boundary decision differently at the last floating-point
digit: FP64 on both sides, different operation contraction)."""
import glob
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200.rayfile import read_ray

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = sorted(glob.glob(os.path.join(HERE, "golden", "rays_*.npz")))


def write_case(g, root):
    for k in g.files:
        if k.startswith("file_"):
            with open(root + "." + k[5:], "w") as f:
                f.write(str(g[k]))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[5:-4] for p in GOLD])
def test_rays_match_reference(path, workdir):
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup(root)
        t.run()
        rays = t.rays()
        t.writeout(root + "_gpu")
    ref_n = g["npts"]
    assert len(rays) == len(ref_n) > 0
    np.testing.assert_allclose([r["alpha"] for r in rays], g["alpha"], rtol=1e-9, atol=1e-9)
    offs = np.concatenate([[0], np.cumsum(ref_n)])
    good = 0
    for i, r in enumerate(rays):
        ref = g["rz"][offs[i]:offs[i + 1]]
        if len(r["rz"]) != len(ref):
            continue
        if (r["ntop"], r["nbot"]) != tuple(g["bnc"][i]):
            continue
        if np.max(np.abs(r["rz"] - ref)) <= 1e-3:
            good += 1
    assert good >= 0.97 * len(rays), "%d of %d rays equal" % (good, len(rays))
    # the .ray file holds the same trajectories
    R = read_ray(root + "_gpu.ray")
    assert len(R["rays"]) == len(rays) and R["kind"] == "rz"
    for a, b in zip(R["rays"], rays):
        np.testing.assert_array_equal(a["xy"], b["rz"])
        assert (a["ntop"], a["nbot"]) == (b["ntop"], b["nbot"])
