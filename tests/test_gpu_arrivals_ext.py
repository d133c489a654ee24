"""Arrivals ('a'), eigen hits ('E') and both in one run ('v') of geometric
beams in ray-centred coordinates ('g', 'b'), of simple Gaussian beams ('S')
and (combined run) of Cartesian beams against the reference itself.

The fixtures tests/golden/x2d_arr_*.npz / x2d_eig_*.npz hold each case's
input files and what the reference's own bellhopcxx wrote single-threaded
(the run in which it merges arrivals, src/mode/arr.hpp:78), made by
tests/golden/make_golden_ext.py: the binary .arr records, or the .ray of the
eigen hits re-traced in hit order. FP64: arrival counts and bounce counts
exact, delays within 1e-6 relative, amplitudes within 1e-4 relative, angles
within 1e-3 degrees; eigen hits equal in number and order (ray and step).
"""
import glob
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ARR = sorted(glob.glob(os.path.join(HERE, "golden", "x2d_arr_*.npz")))
EIG = sorted(glob.glob(os.path.join(HERE, "golden", "x2d_eig_*.npz")))


def write_case(npz, root):
    for k in npz.files:
        if k.startswith("file_"):
            with open(root + "." + k[5:], "w") as f:
                f.write(str(npz[k]))


@pytest.mark.parametrize("path", ARR, ids=[os.path.basename(p)[:-4] for p in ARR])
def test_arrivals_match_reference(path, workdir):
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.set_arrival_options(1000, True)
        t.setup(root)
        t.run()
        narr, arr = t.arrivals()
        st = t.stats()
        hits = t.eigen_hits(0) if "eig_alpha" in g.files else None
        if hits is not None:
            t.writeout(root + "_gpu")
    assert st["err_bits"] == 0
    if hits is not None:   # the product writes the .arr and the .ray of the hits
        assert os.path.exists(root + "_gpu.arr") and os.path.exists(root + "_gpu.ray")
    narr = narr.reshape(-1)
    np.testing.assert_array_equal(narr, g["narr"])
    assert narr.sum() > 0
    got = arr.reshape(narr.size, -1)[narr[:, None] > np.arange(arr.shape[-1])]
    ref = g["arr"]
    np.testing.assert_array_equal(got["NTopBnc"], ref[:, 6].astype(np.int32))
    np.testing.assert_array_equal(got["NBotBnc"], ref[:, 7].astype(np.int32))
    np.testing.assert_allclose(got["delay_re"], ref[:, 2], rtol=1e-6)
    np.testing.assert_allclose(got["delay_im"], ref[:, 3], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(got["a"], ref[:, 0], rtol=1e-4)
    np.testing.assert_allclose(got["SrcDeclAngle"], ref[:, 4], rtol=0, atol=1e-3)
    np.testing.assert_allclose(got["RcvrDeclAngle"], ref[:, 5], rtol=0, atol=1e-3)
    ph = np.rad2deg(got["Phase"].astype(np.float64))
    np.testing.assert_allclose(np.rad2deg(np.angle(np.exp(1j * np.deg2rad(ph - ref[:, 1])))), 0.0, atol=1e-3)
    if "eig_alpha" in g.files:   # 'V' / 'v': the run also recorded every contribution's eigen hit
        check_hits(hits, g["eig_alpha"], g["eig_npts"], str(g["file_env"]))


def check_hits(hits, alpha, npts, env_text):
    """Hits in the reference's order: the reference writes one re-traced ray
    per hit, whose take-off angle and point count (the hit's step + 2) give
    each hit's ray and step."""
    assert len(hits) == len(alpha) > 0
    np.testing.assert_array_equal(hits["is"] + 2, npts)
    txt = env_text.splitlines()
    k = [i for i, ln in enumerate(txt) if ln.strip()[:2] in ("'E", "'V", "'v")][0]
    na = int(txt[k + 1].split()[0])
    a1, a2 = (float(v) for v in txt[k + 2].replace("/", " ").split()[:2])
    fan = np.linspace(a1, a2, na)
    np.testing.assert_allclose(fan[hits["ialpha"]], alpha, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("path", EIG, ids=[os.path.basename(p)[:-4] for p in EIG])
def test_eigen_hits_match_reference(path, workdir):
    """The reference writes one re-traced ray per hit, in hit order: its
    take-off angle and point count (the hit's step + 2) give each hit's ray
    and step."""
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup(root)
        t.run()
        hits = t.eigen_hits(0)
        st = t.stats()
    assert st["err_bits"] == 0
    check_hits(hits, g["alpha"], g["npts"], str(g["file_env"]))
