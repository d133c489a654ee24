"""Host-side checks that need no GPU: the C ABI library loads and exports every
entry point of include/bhcb.h; the native reader / preprocessing agrees with
the oracle on sizes and rejects invalid inputs with the reference's messages."""
import os
import re
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))

import bellhopcuda_b200 as B  # noqa: E402
import oracle_ctypes  # noqa: E402
from cases import CASES  # noqa: E402
from bellhopcuda_b200.envfile import EnvSpec, write_env  # noqa: E402
from bellhopcuda_b200 import workloads as W  # noqa: E402


def header_functions():
    txt = open(os.path.join(ROOT, "include", "bhcb.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bhcb_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    lib = B.load_library()
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares every one of them
    bound = {n for n, _, _ in B.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_version_string():
    assert b"sm_100a" in B.load_library().bhcb_version()


@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_sizes_match_oracle(name, workdir):
    spec = CASES[name]()
    root = write_env(spec, os.path.join(workdir, "sz_" + name))
    info = B.check_env(root)
    o = oracle_ctypes.run(spec)
    assert info["nsz"] == o["NSz"]
    assert info["nrz"] == o["NRz"]
    assert info["nrr"] == o["NRr"]
    assert info["nalpha"] == o["Nalpha"]


def test_reader_list_directed_syntax(workdir):
    """Repeat counts, commas, '/' terminators and quoted strings."""
    root = os.path.join(workdir, "ld")
    open(root + ".env", "w").write(
        "'list, directed test' ! title\n"
        "100.0\n1\n'CVW'\n"
        "3  0.0  1000.0\n"
        "0.0 1500.0 /\n500.0,1510.0,0.0,1.0 /\n1000.0 1520.0 /\n"
        "'A' 0.0\n1000.0 1600.0 0.0 1.8 0.8 0.0 /\n"
        "1\n500.0 /\n"
        "3\n100.0 2*900.0 /\n"
        "11\n0.0 10.0 /\n"
        "'CG'\n"
        "21\n-10.0 10.0 /\n"
        "0.0 1100.0 10.5\n")
    info = B.check_env(root)
    assert info["nrz"] == 3 and info["nrr"] == 11 and info["nalpha"] == 21
    assert info["freq"] == 100.0 and abs(info["deltas"] - 100.0) < 1e-12


def _write(workdir, name, **kw):
    from bellhopcuda_b200 import workloads as W
    spec = W.munk_tl(nalpha=11, nrz=5, nrr=5)
    for k, v in kw.items():
        setattr(spec, k, v)
    return write_env(spec, os.path.join(workdir, name))


def test_reader_rejects_nonmonotone_ssp(workdir):
    z = np.arange(0.0, 5001.0, 100.0)
    z[10], z[11] = z[11], z[10]
    root = _write(workdir, "nonmono", ssp_z=list(z))
    with pytest.raises(B.BhcbError, match="monotone"):
        B.check_env(root)


def test_reader_rejects_bathymetry_below_ssp(workdir):
    root = _write(workdir, "deep", bty_r=[0.0, 50.0, 100.0], bty_z=[4000.0, 6000.0, 4000.0])
    with pytest.raises(B.BhcbError, match="bathymetry drops below"):
        B.check_env(root)


def test_reader_rejects_bad_box(workdir):
    root = _write(workdir, "box", box_z=0.0)
    with pytest.raises(B.BhcbError, match="beam box"):
        B.check_env(root)


def test_reader_rejects_unsupported_beam(workdir):
    """Cerveny beams are TL-only (as in the reference); ray-centred and simple
    Gaussian beams take arrivals and eigen runs."""
    root = _write(workdir, "cerveny", run_type="AC RR ")
    with pytest.raises(B.BhcbError, match="does not support eigenrays or arrivals"):
        B.check_env(root)
    for rt in ("Ag RR ", "ab RR ", "ES RR "):
        root = _write(workdir, "x_" + rt[:2], run_type=rt)
        assert B.check_env(root)["run_type"].startswith(rt[:2])


def test_reader_missing_file(workdir):
    with pytest.raises(B.BhcbError, match="unable to open"):
        B.check_env(os.path.join(workdir, "does_not_exist"))


def test_open_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(B.BhcbError):
        B.Tracer()


import oracle_ctypes  # noqa: E402  (test infrastructure: locates the reference tree)

REFERENCE_INPUTS = os.path.join(oracle_ctypes.reference_dir(), "test", "in")


@pytest.mark.skipif(not os.path.isdir(REFERENCE_INPUTS), reason="reference inputs not present")
@pytest.mark.parametrize("name", ["Munk", "MunkB_Coh", "MunkB_gb", "DickinsB", "DickinsFlatB", "free",
                                  "GulfB_rd_gb", "GulfB_ri_Cerveny", "MunkB_Coh_CervenyR", "MunkB_Coh_CervenyC",
                                  "DickinsCervenyB", "Gulf_ray_rd"])
def test_reader_accepts_reference_inputs(name, workdir):
    src = os.path.join(REFERENCE_INPUTS, name)
    if not os.path.exists(src + ".env"):
        pytest.skip("no such input")
    import shutil
    for ext in (".env", ".bty", ".ati", ".ssp", ".sbp"):
        if os.path.exists(src + ext):
            shutil.copy(src + ext, os.path.join(workdir, name + ext))
    try:
        B.check_env(os.path.join(workdir, name))
    except B.BhcbError as e:
        assert "not supported" in str(e) or "not a field mode" in str(e), str(e)


# ------------------------------------- 2-D options pinned by reference fixtures
GOLD2D_EXT = sorted(n[:-4] for n in os.listdir(os.path.join(HERE, "golden")) if n.startswith("x2d_")
                    and n.endswith(".npz"))


def write_fixture_files(npz, root):
    for k in npz.files:
        if k.startswith("file_"):
            with open(root + "." + k[5:], "w") as f:
                f.write(str(npz[k]))


@pytest.mark.parametrize("name", GOLD2D_EXT)
def test_reader2d_ext_sizes_match_reference_fixture(name, workdir):
    """The reader accepts the option (quad SSP, ...) and sees the grid the
    reference wrote in its .shd."""
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    root = os.path.join(workdir, name)
    write_fixture_files(g, root)
    info = B.check_env(root)
    if "field" in g.files:          # TL: the .shd grid
        nsz, nrz, nrr = g["field"].shape
        assert (info["nsz"], info["nrz"], info["nrr"]) == (nsz, nrz, nrr)
    elif "narr" in g.files:         # arrivals: the .arr grid
        assert (info["nsz"], info["nrz"], info["nrr"]) == (len(g["sz"]), len(g["rz"]), len(g["rr"]))
    assert info["nalpha"] > 0


def test_reader_rejects_bad_quad_ssp(workdir):
    from cases2d_ext import CASES2D_EXT
    files = CASES2D_EXT["x2d_quad_munk_gauss"]()
    root = os.path.join(workdir, "badquad")
    with open(root + ".env", "w") as f:
        f.write(files[".env"])
    with pytest.raises(B.BhcbError, match="quad SSP"):
        B.check_env(root)                     # no .ssp file
    lines = files[".ssp"].splitlines()
    r = lines[1].split()
    lines[1] = " ".join([r[1], r[0]] + r[2:])
    with open(root + ".ssp", "w") as f:
        f.write("\n".join(lines) + "\n")
    with pytest.raises(B.BhcbError, match="monotone"):
        B.check_env(root)


# ------------------------------------------------------------------ 3-D reader
GOLD3D = sorted(n[:-4] for n in os.listdir(os.path.join(HERE, "golden")) if "3d" in n and n.endswith(".npz"))


@pytest.mark.parametrize("name", GOLD3D)
def test_reader3d_sizes_match_reference_fixture(name, workdir):
    """The 3-D reader sees the grid the reference wrote in its .shd."""
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    root = os.path.join(workdir, "r3_" + name)
    for k in g.files:
        if k.startswith("file_"):
            with open(root + "." + k[5:], "w") as f:
                f.write(str(g[k]))
    info = B.check_env3d(root)
    if "field" in g.files:
        nsx, nsy, nth, nsz, nrz, nrr = g["field"].shape
        assert info["dims"] == (nsz, nsx, nsy, nth, nrz, nrr)
    elif "npts" in g.files:   # eigen fixture: one re-traced ray per hit
        assert len(g["npts"]) == len(g["alpha"]) > 0
    else:   # arrivals fixture: one count per receiver
        d = info["dims"]
        assert (d[0], d[3], d[4], d[5]) == (len(g["sz"]), len(g["theta"]), len(g["rz"]), len(g["rr"]))
        assert int(np.prod(d)) == g["narr"].size
    assert info["nrays"] > 0


def test_reader3d_fixes_360_degree_sweep(workdir):
    """CheckFix360Sweep drops the duplicate bearing of a full 360-degree fan."""
    from cases3d import CASES3D
    root = os.path.join(workdir, "sweep3d")
    for suffix, text in CASES3D["parabot3d_hat"]().items():
        with open(root + suffix, "w") as f:
            f.write(text)
    info = B.check_env3d(root)
    assert info["nrays"] == 61 * 36      # 37 bearings 0..360 -> 36


def test_reader3d_rejects_2d_runs_and_unsupported_beams(workdir):
    from cases3d import CASES3D
    text = CASES3D["munk3d_gauss"]()[".env"]
    root = os.path.join(workdir, "bad3d")
    with open(root + ".env", "w") as f:
        f.write(text.replace("'CB   3'", "'CB    '"))
    with pytest.raises(B.BhcbError, match="RunType"):
        B.check_env3d(root)
    with open(root + ".env", "w") as f:
        f.write(text.replace("'CB   3'", "'CR   3'"))
    with pytest.raises(B.BhcbError, match="not supported"):
        B.check_env3d(root)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_INPUTS), reason="reference inputs not present")
@pytest.mark.parametrize("name", ["Munkslice3dGaussian", "Munkslice3dHatCart", "MunkRot3D", "DoubleSeamount3D",
                                  "PerfectWedge3dHat", "KR3dGaussian", "HyperBot3DHatCart", "KR3d_ray",
                                  "DoubleSeamount3D_ray", "Munkslice2dGaussian"])
def test_reader3d_accepts_reference_inputs(name, workdir):
    src = os.path.join(REFERENCE_INPUTS, name)
    if not os.path.exists(src + ".env"):
        pytest.skip("no such input")
    import shutil
    for ext in (".env", ".bty", ".ati", ".ssp", ".sbp"):
        if os.path.exists(src + ext):
            shutil.copy(src + ext, os.path.join(workdir, name + ext))
    try:
        info = B.check_env3d(os.path.join(workdir, name))
        assert info["nrays"] > 0
    except B.BhcbError as e:
        assert "not supported" in str(e), str(e)


def test_env_desc_reads_file(workdir):
    """bhcb_read_env_desc gives the file's values (ranges in km, angles in degrees)."""
    spec = W.munk_tl(nalpha=301, nrz=51, nrr=201)
    root = write_env(spec, os.path.join(workdir, "desc_munk"))
    with B.EnvDescription(root) as e:
        d = e.desc
        assert d.nsz == 1 and d.nrz == 51 and d.nrr == 201 and d.nalpha == 301
        assert abs(d.rr_km[200] - spec.rr_km[1]) < 1e-9
        assert d.alpha_deg[0] == spec.alpha[0] and d.alpha_deg[300] == spec.alpha[1]
        assert d.nssp == len(spec.ssp_z)
        assert d.run_type[:2] == spec.run_type[:2].encode()
        assert abs(d.freq0 - spec.freq) < 1e-12
    with pytest.raises(B.BhcbError):
        B.EnvDescription(os.path.join(workdir, "no_such_env"))


def test_c5_environments_follow_run_type_and_fan(workdir):
    """The surrogate workload's environments: the same seeded parameters for
    either field type; 'IB' with a +-89 degree fan by default, 'CG' on
    request; the reader takes both."""
    from bellhopcuda_b200 import workloads as W
    P = W.c5_params(4, seed=5)
    Q = W.c5_params(4, seed=5, run_type="CG", fan_deg=60.0)
    for k in ("depth", "cp", "zs", "f", "a"):
        np.testing.assert_array_equal(P[k], Q[k])
    a, b = W.c5_env(P, 1), W.c5_env(Q, 1)
    assert a.run_type.startswith("IB") and b.run_type.startswith("CG")
    assert tuple(a.alpha) == (-89.0, 89.0) and tuple(b.alpha) == (-60.0, 60.0)
    for name, spec in (("ib", a), ("cg", b)):
        info = B.check_env(write_env(spec, os.path.join(workdir, name)))
        assert info["nrz"] == W.C5_NZ and info["nrr"] == W.C5_NR


def test_surrogate_acceptance_calibration():
    """The fallback rule's margin: on the calibration fields, the accepted
    ones (smallest predicted errors) stay within the threshold for at least
    97.5 % of them; without enough such fields the 95th-percentile rule."""
    from bellhopcuda_b200.surrogate import calibrate_margin, ACCEPT_PRECISION
    rng = np.random.default_rng(3)
    pe = rng.uniform(0.5, 3.0, 5000)
    err = pe * rng.lognormal(0.0, 0.2, 5000)
    m = calibrate_margin(pe, err, 1.0)
    acc = pe * m <= 1.0
    assert acc.sum() >= 50 and (err[acc] <= 1.0).mean() >= ACCEPT_PRECISION
    # one more field accepted would break the precision target
    nxt = np.sort(pe[~acc])[0]
    acc2 = pe <= nxt
    assert acc2.sum() == acc.sum() + 1 and (err[acc2] <= 1.0).mean() < ACCEPT_PRECISION
    # no field within the threshold: the 95th-percentile margin accepts none
    m2 = calibrate_margin(pe, err + 5.0, 1.0)
    assert not (pe * m2 <= 1.0).any()


def test_arrivals_ascii_and_binary_files_agree(workdir):
    """The reference's ASCII ('A') and binary ('a') arrivals of one 2-D run
    (tests/golden/make_golden_readout.py) read alike: the same receivers and
    counts, values within the ASCII file's printed digits."""
    from bellhopcuda_b200.arrfile import read_arr_ascii, read_arr_binary
    g = np.load(os.path.join(HERE, "golden", "readout_cases.npz"))
    paths = {}
    for case in ("ro2d_A", "ro2d_a"):
        paths[case] = os.path.join(workdir, case + ".arr")
        with open(paths[case], "wb") as f:
            f.write(g[case + "_out"].tobytes())
    A, Bn = read_arr_ascii(paths["ro2d_A"]), read_arr_binary(paths["ro2d_a"])
    assert A["dim"] == Bn["dim"] == "'2D'" and A["freq"] == Bn["freq"]
    for k in ("sz", "rz", "rr"):
        np.testing.assert_allclose(A[k], Bn[k], rtol=1e-6)
    for sa, sb in zip(A["sources"], Bn["sources"]):
        assert sa["maxn"] == sb["maxn"]
        for a, b in zip(sa["arrivals"], sb["arrivals"]):
            assert a.shape == b.shape
            np.testing.assert_allclose(a, b, rtol=2e-5, atol=1e-6)


def test_every_entry_rejects_null_arguments():
    """The C ABI's error contract without a GPU: every entry point that takes a
    context or buffers returns BHCB_ERR_ARG for null handles and zero sizes
    instead of touching memory (the bhc:: layer above maps it to false)."""
    import ctypes as C
    lib = B.load_library()
    host_only = {"bhcb_version", "bhcb_close", "bhcb_free_env_desc", "bhcb_read_env_desc", "bhcb_check_env",
                 "bhcb_check_env3d", "bhcb_last_error", "bhcb_graph_destroy",
                 "bhcb_nn_status"}   # reads the device's error word: no device here
    checked = 0
    for name, ret, args in B.SIGNATURES:
        if name in host_only or not args or ret is None:
            continue
        vals = []
        for a in args:
            if a in (C.c_float, C.c_double, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_int, C.c_size_t):
                vals.append(a(0))
            else:
                vals.append(None)
        assert getattr(lib, name)(*vals) == 1, name   # BHCB_ERR_ARG
        checked += 1
    assert checked >= 40
