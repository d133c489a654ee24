"""GPU parity of the 3-D (BELLHOP3D) field modes against the reference itself.

The fixtures in tests/golden/*3d*.npz hold each case's input files and the
field the reference's own bellhopcxx computed as a 3-D run (made by
tests/golden/make_golden3d.py). The product runs the same files through the C
ABI. Tolerance: TL = -20 log10|p| within 0.5 dB RMS over receivers where the
reference's TL < 100 dB (the reference's own FP64 runs differ between
thread counts by float atomics; the same bound as the 2-D path).
"""
import glob
import os

import numpy as np
import pytest

import bellhopcuda_b200 as B

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = sorted(glob.glob(os.path.join(HERE, "golden", "*3d*.npz")))
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


def to_file_order(u):
    """product [isz][isx][isy][itheta][iz][ir] -> .shd order [isx][isy][itheta][isz][iz][ir]"""
    return np.transpose(u, (1, 2, 3, 0, 4, 5))


TL3D = [p for p in GOLD if "_arr_" not in p and "_eig_" not in p and "_v_" not in p and not p.endswith("_ray.npz")]


@pytest.mark.parametrize("precision", [B.PREC_FP64, B.PREC_MIXED])
@pytest.mark.parametrize("path", TL3D, ids=[os.path.basename(p)[:-4] for p in TL3D])
def test_3d_field_matches_reference(path, precision, workdir):
    """Both precisions: the mixed one evaluates the Cartesian beams' TL
    contributions in FP32 (the trace stays FP64); same 0.5 dB bound."""
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4] + "_%d" % precision)
    write_case(g, root)
    with B.Tracer(precision=precision) as t:
        t.setup3d(root)
        t.run()
        u = t.field3d(0)
        st = t.stats()
        grid = t.grid3d(0)
    assert st["err_bits"] == 0
    assert st["rays"] > 0 and st["segments"] > 0 and st["evals"] > 0
    np.testing.assert_allclose(grid["rr"], g["rr"])
    np.testing.assert_array_equal(grid["rz"], g["rz"])
    np.testing.assert_allclose(grid["theta"], g["theta"])
    got = to_file_order(u)
    ref = g["field"]
    assert got.shape == ref.shape
    err, n = tl_err(got, ref)
    assert n > 0
    assert err < 0.5, "TL RMS %.3f dB over %d receivers" % (err, n)


def test_3d_writeout_shd(workdir):
    from bellhopcuda_b200.shdfile import read_shd
    path = [p for p in GOLD if "munk3d_sources" in p][0]
    g = np.load(path)
    root = os.path.join(workdir, "wr3d")
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup3d(root)
        t.run()
        u = t.field3d(0)
        t.writeout(root)
    shd = read_shd(root + ".shd")
    np.testing.assert_array_equal(shd["field"], to_file_order(u))
    np.testing.assert_allclose(shd["theta"], g["theta"])
    np.testing.assert_array_equal(shd["sz"], g["sz"])


def test_3d_batch_equals_single_runs(workdir):
    """Several 3-D environments in one launch give each one's own field."""
    names = ["munk3d_hat", "hex3d_gauss", "parabot3d_hat"]
    roots = []
    for n in names:
        g = np.load(os.path.join(HERE, "golden", n + ".npz"))
        root = os.path.join(workdir, "b3_" + n)
        write_case(g, root)
        roots.append(root)
    singles = []
    for r in roots:
        with B.Tracer(precision=B.PREC_FP64) as t:
            t.setup3d(r)
            t.run()
            singles.append(t.field3d(0))
    with B.Tracer(precision=B.PREC_FP64) as t:
        for r in roots:
            t.add_env3d(r)
        t.run()
        batch = [t.field3d(i) for i in range(len(roots))]
        assert t.stats()["groups"] == len(roots)
    for a, b in zip(batch, singles):
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-6 * np.abs(b).max())


def test_3d_small_max_memory_runs_in_waves(workdir):
    g = np.load(os.path.join(HERE, "golden", "munk3d_gauss.npz"))
    root = os.path.join(workdir, "w3d")
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup3d(root)
        t.run()
        full, st = t.field3d(0), t.stats()
    small = st["segments"] * 288 // 3 + (8 << 20) + full.nbytes + (64 << 20)
    with B.Tracer(precision=B.PREC_FP64, max_memory=small) as t:
        t.setup3d(root)
        t.run()
        waved, st2 = t.field3d(0), t.stats()
    assert st2["segments"] == st["segments"]
    np.testing.assert_allclose(waved, full, rtol=1e-4, atol=1e-6 * np.abs(full).max())


ARR3D = sorted(p for p in GOLD if "_arr_" in p)
# fixtures whose rays cross a boundary grid in Nx2D planes (one ray in about a
# hundred differs from the reference's trajectory)
NX2D_GRID_RAY_DIFF = {"seamount3d_nx2d_arr_hat"}
EIG3D = sorted(p for p in GOLD if "_eig_" in p)


@pytest.mark.parametrize("path", ARR3D, ids=[os.path.basename(p)[:-4] for p in ARR3D])
def test_3d_arrivals_match_reference(path, workdir):
    """3-D arrivals (RunType 'a') against the reference's single-threaded run
    (merging on): counts and bounce counts exact, delays within 1e-6 relative,
    amplitudes within 1e-4 relative, angles within 1e-3 degrees."""
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.set_arrival_options(1000, True)
        t.setup3d(root)
        t.run()
        narr, arr = t.arrivals()
        t.writeout(root + "_gpu")
    check_arrivals(narr, arr, g, root, os.path.basename(path)[:-4])


def check_arrivals(narr, arr, g, root, name):
    narr = narr.reshape(-1)
    assert narr.sum() > 0
    if name in NX2D_GRID_RAY_DIFF:
        # Nx2D rays over a boundary grid: about one ray in a hundred leaves the
        # reference's trajectory (see test_3d_rays_match_reference), and its
        # contributions move an arrival between neighbouring receivers. Counts
        # equal on at least 95 % of the receivers; records compared there.
        same = narr == g["narr"]
        assert same.mean() >= 0.95, "%d of %d receivers differ" % ((~same).sum(), same.size)
        assert abs(int(narr.sum()) - int(g["narr"].sum())) <= max(2, 0.02 * g["narr"].sum())
        off_ref = np.concatenate([[0], np.cumsum(g["narr"])])
        keep_ref = np.concatenate([np.arange(off_ref[i], off_ref[i + 1]) for i in np.nonzero(same)[0]])
        narr_eq = np.where(same, narr, 0)
        got = arr.reshape(narr.size, -1)[narr_eq[:, None] > np.arange(arr.shape[-1])]
        ref = g["arr"][keep_ref]
        good = (got["NTopBnc"] == ref[:, 8].astype(np.int32)) & (got["NBotBnc"] == ref[:, 9].astype(np.int32)) \
            & np.isclose(got["delay_re"], ref[:, 2], rtol=1e-6, atol=0)
        assert good.mean() >= 0.95, good.mean()
        return
    np.testing.assert_array_equal(narr, g["narr"])
    got = arr.reshape(narr.size, -1)[narr[:, None] > np.arange(arr.shape[-1])]
    ref = g["arr"]
    np.testing.assert_array_equal(got["NTopBnc"], ref[:, 8].astype(np.int32))
    np.testing.assert_array_equal(got["NBotBnc"], ref[:, 9].astype(np.int32))
    np.testing.assert_allclose(got["delay_re"], ref[:, 2], rtol=1e-6)
    np.testing.assert_allclose(got["delay_im"], ref[:, 3], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(got["a"], ref[:, 0], rtol=1e-4)
    for k, c in (("SrcDeclAngle", 4), ("SrcAzimAngle", 5), ("RcvrDeclAngle", 6), ("RcvrAzimAngle", 7)):
        np.testing.assert_allclose(got[k], ref[:, c], rtol=0, atol=1e-3, err_msg=k)
    # the product's own .arr file holds the same records
    from bellhopcuda_b200.arrfile import read_arr_binary
    A = read_arr_binary(root + "_gpu.arr")
    assert A["dim"] == "'3D'"
    mine = np.concatenate([a for s in A["sources"] for a in s["arrivals"]])
    np.testing.assert_array_equal(mine[:, 2], got["delay_re"])
    np.testing.assert_allclose(mine[:, 1], ref[:, 1], rtol=0, atol=1e-3)   # phase in degrees


@pytest.mark.parametrize("path", EIG3D, ids=[os.path.basename(p)[:-4] for p in EIG3D])
def test_3d_eigen_hits_match_reference(path, workdir):
    """3-D eigen hits ('E') against the reference's single-threaded run: it
    writes one re-traced ray per hit, in hit order, whose take-off angle and
    point count (the hit's step + 2) give each hit's ray and step."""
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup3d(root)
        t.run()
        hits = t.eigen_hits(0)
    check_hits(hits, g, g["alpha"], g["npts"], "'E")


def check_hits(hits, g, alpha, npts, run_tag):
    assert len(hits) == len(alpha) > 0
    np.testing.assert_array_equal(hits["is"] + 2, npts)
    # the take-off angle of each hit's ray: elevation fan from the .env (alpha1, alpha2, n)
    txt = str(g["file_env"]).splitlines()
    k = [i for i, ln in enumerate(txt) if ln.strip().startswith(run_tag)][0]
    na = int(txt[k + 1].split()[0])
    a1, a2 = (float(v) for v in txt[k + 2].replace("/", " ").split()[:2])
    fan = np.deg2rad(np.linspace(a1, a2, na))
    np.testing.assert_allclose(fan[hits["ialpha"]], alpha, rtol=1e-9, atol=1e-12)


RAY3D = sorted(p for p in GOLD if p.endswith("_ray.npz"))


def compare_rays3d(rays, g, frac=0.97):
    """Same rays in the same order (take-off angle, point count, bounce
    counts); on at least frac of the rays whose points the fixture keeps,
    every point within 1 mm (a boundary decision may fall differently at the
    last floating-point digit: FP64 on both sides, different contraction)."""
    assert len(rays) == len(g["npts"]) > 0
    np.testing.assert_allclose(np.deg2rad([r["alpha"] for r in rays]), g["alpha"], rtol=1e-9, atol=1e-12)
    same_n = sum(len(r["rz"]) == n for r, n in zip(rays, g["npts"]))
    assert same_n >= frac * len(rays), "%d of %d point counts equal" % (same_n, len(rays))
    nkeep = int(g["xyz_rays"])
    offs = np.concatenate([[0], np.cumsum(g["npts"][:nkeep])])
    good = 0
    for i in range(nkeep):
        ref = g["xyz"][offs[i]:offs[i + 1]]
        r = rays[i]
        if len(r["rz"]) == len(ref) and (r["ntop"], r["nbot"]) == tuple(g["bnc"][i]) and \
                np.max(np.abs(r["rz"] - ref)) <= 1e-3:
            good += 1
    assert good >= frac * nkeep, "%d of %d rays equal" % (good, nkeep)


@pytest.mark.parametrize("path", RAY3D, ids=[os.path.basename(p)[:-4] for p in RAY3D])
def test_3d_rays_match_reference(path, workdir):
    """3-D ray runs ('R') against the reference's single-threaded .ray output,
    and the product's own .ray file read back."""
    from bellhopcuda_b200.rayfile import read_ray
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup3d(root)
        t.run()
        rays = t.rays(dim=3)
        t.writeout(root + "_gpu")
    compare_rays3d(rays, g)
    R = read_ray(root + "_gpu.ray")
    assert R["kind"] == "xyz" and len(R["rays"]) == len(rays)
    for a, b in zip(R["rays"], rays):
        np.testing.assert_array_equal(a["xy"], b["rz"])
        assert (a["ntop"], a["nbot"]) == (b["ntop"], b["nbot"])


@pytest.mark.parametrize("path", EIG3D, ids=[os.path.basename(p)[:-4] for p in EIG3D])
def test_3d_eigenrays_match_reference(path, workdir):
    """The hit rays re-traced up to their hit (PostProcessEigenrays) against
    the reference's .ray output of the same 3-D eigen run."""
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.setup3d(root)
        t.run()
        rays = t.rays(dim=3)
        t.writeout(root + "_gpu")
    compare_rays3d(rays, g)
    from bellhopcuda_b200.rayfile import read_ray
    assert len(read_ray(root + "_gpu.ray")["rays"]) == len(rays)


V3D = sorted(p for p in GOLD if "_v_" in p)


@pytest.mark.parametrize("path", V3D, ids=[os.path.basename(p)[:-4] for p in V3D])
def test_3d_combined_arrivals_and_eigen_hits(path, workdir):
    """RunType 'v': arrivals and eigen hits of one 3-D / Nx2D run, against
    the reference's .arr and .ray outputs of that run: the arrivals as in
    test_3d_arrivals_match_reference, the hits and their re-traced rays as in
    the eigen tests."""
    g = np.load(path)
    root = os.path.join(workdir, os.path.basename(path)[:-4])
    write_case(g, root)
    with B.Tracer(precision=B.PREC_FP64) as t:
        t.set_arrival_options(1000, True)
        t.setup3d(root)
        t.run()
        narr, arr = t.arrivals()
        hits = t.eigen_hits(0)
        rays = t.rays(dim=3)
        t.writeout(root + "_gpu")
    check_arrivals(narr, arr, g, root, os.path.basename(path)[:-4])
    check_hits(hits, g, g["eig_alpha"], g["eig_npts"], "'v")
    eig = {k[4:]: g[k] for k in g.files if k.startswith("eig_")}
    compare_rays3d(rays, eig)
    from bellhopcuda_b200.rayfile import read_ray
    assert len(read_ray(root + "_gpu.ray")["rays"]) == len(rays)
