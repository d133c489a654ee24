"""The bhc:: C++ interface (include/bhcb/bhc.hpp) over libbhcb.so, on the CPU.

A program written against the header (tests/bhc_api_check.cpp) is compiled and
linked here; its "params" mode exercises setup from the defaults and from
files, the extsetup_* resizing, writeenv round trips and get_ssp, none of
which needs a GPU. The GPU runs are in test_gpu_bhc_api.py.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from bellhopcuda_b200 import build as BUILD

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build_check(out_dir: str) -> str:
    lib = BUILD.build()
    exe = os.path.join(out_dir, "bhc_api_check")
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "bhc_api_check.cpp"), "-L" + os.path.dirname(lib), "-lbhcb",
                    "-Wl,-rpath," + os.path.dirname(lib), "-o", exe], check=True)
    return exe


def test_header_exports(tmp_path):
    """Every function template of the header is instantiated in the library for
    2-D, Nx2D and 3-D (the program links)."""
    lib = BUILD.build()
    out = subprocess.run(["nm", "-DC", lib], capture_output=True, text=True, check=True).stdout
    for name in ["setup", "run", "postprocess", "writeout", "readout", "finalize", "get_ssp", "echo",
                 "writeenv", "get_percent_progress", "extsetup_sxsy", "extsetup_sz", "extsetup_rcvrranges",
                 "extsetup_rcvrdepths", "extsetup_rcvrbearings", "extsetup_rayelevations",
                 "extsetup_raybearings", "extsetup_sbp", "extsetup_freqvec", "extsetup_altimetry",
                 "extsetup_bathymetry", "extsetup_trc", "extsetup_brc", "extsetup_ssp_quad",
                 "extsetup_ssp_hexahedral", "extsetup_blocking"]:
        assert (" bhc::%s<" % name) in out or (" bhc::%s(" % name) in out, name


def test_params_roundtrip(tmp_path):
    exe = build_check(str(tmp_path))
    r = subprocess.run([exe, "params", str(tmp_path)], capture_output=True, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
    env = open(os.path.join(tmp_path, "edited.env")).read()
    assert "'R~'" in env and os.path.exists(os.path.join(tmp_path, "edited.bty"))


def _arr_ascii(text: str, is3d: bool) -> dict:
    """The ASCII arrivals file as the test reads it: one statement per line."""
    lines = [ln.replace(",", " ").split() for ln in text.splitlines() if ln.strip()]
    k = 2
    dims = []
    for _ in range(6 if is3d else 3):
        dims.append(int(lines[k][0]))
        k += 1
    if is3d:
        nsx, nsy, nsz, nrz, nrr, nth = dims
    else:
        (nsz, nrz, nrr), nsx, nsy, nth = dims, 1, 1, 1
    nf = 10 if is3d else 8
    maxn, recs = [], []
    for _ in range(nsz * nsx * nsy):
        maxn.append(int(lines[k][0]))
        k += 1
        for _ in range(nth * nrz * nrr):
            n = int(lines[k][0])
            k += 1
            for _ in range(n):
                recs.append([float(v) for v in lines[k][:nf]])
                k += 1
    return dict(dims=(nsx, nsy, nsz, nth, nrz, nrr), freq=float(lines[1][0]), maxn=maxn,
                recs=np.array(recs).reshape(-1, nf))


@pytest.mark.parametrize("case", ["ro2d_A", "ro2d_a", "ro2d_R", "ro3d_A", "ro3d_a", "ro3d_R", "ronx_a", "ronx_R"])
def test_readout_reference_files(case, tmp_path):
    """bhc::readout of .arr (ASCII and binary) and .ray files that the
    reference itself wrote (2-D, 3-D, Nx2D; tests/golden/make_golden_readout.py):
    the coordinates, counts and every record come back (sums compared with the
    test's own reading of the file)."""
    from bellhopcuda_b200.arrfile import read_arr_binary
    from bellhopcuda_b200.rayfile import read_ray
    g = np.load(os.path.join(HERE, "golden", "readout_cases.npz"))
    dim, suffix = int(g[case + "_dim"]), str(g[case + "_suffix"])
    root = os.path.join(str(tmp_path), case)
    with open(root + ".env", "w") as f:
        f.write(str(g[case + "_env"]))
    data = g[case + "_out"].tobytes()
    with open(root + suffix, "wb") as f:
        f.write(data)
    exe = build_check(str(tmp_path))
    r = subprocess.run([exe, "readout", str(dim), root], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    out = [ln for ln in r.stdout.splitlines() if ln.startswith(("arr ", "ray "))][0].split()
    is3d = dim != 2
    if suffix == ".arr":
        if case.endswith("_a"):
            A = read_arr_binary(root + ".arr")
            dims = (len(A["sx"]), len(A["sy"]), len(A["sz"]), len(A["theta"]), len(A["rz"]), len(A["rr"]))
            recs = np.concatenate([a for s in A["sources"] for a in s["arrivals"]]).astype(np.float64)
            maxn, freq = [s["maxn"] for s in A["sources"]], A["freq"]
        else:
            A = _arr_ascii(data.decode(), is3d)
            dims, recs, maxn, freq = A["dims"], A["recs"], A["maxn"], A["freq"]
        assert tuple(int(v) for v in out[1:7]) == dims
        assert abs(float(out[7]) - freq) <= 1e-6 * freq
        assert int(out[8]) == len(recs) > 0
        assert int(out[9]) >= max(maxn) and int(out[10]) == max(maxn)
        if not is3d:   # 2-D records carry no azimuths
            z = np.zeros((len(recs), 1))
            recs = np.hstack([recs[:, :5], z, recs[:, 5:6], z, recs[:, 6:]])
        phase = np.float32(np.deg2rad(recs[:, 1]))
        want = [recs[:, 0].astype(np.float32).sum(), phase.astype(np.float64).sum()] + \
            [recs[:, k].astype(np.float32).astype(np.float64).sum() for k in range(2, 10)]
        got = [float(v) for v in out[11:21]]
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-9)
    else:
        R = read_ray(root + ".ray")
        rays = R["rays"]
        assert int(out[1]) == len(rays) > 0
        assert int(out[2]) == sum(len(x["xy"]) for x in rays)
        alpha = sum(np.rad2deg(x["alpha"]) if is3d else x["alpha"] for x in rays)
        sx = sy = sz = 0.0
        for x in rays:
            p = x["xy"]
            if dim == 4:   # Nx2D: range along the plane from the first point, depth
                d = p[-1, :2] - p[0, :2]
                t = d / np.hypot(*d) if np.hypot(*d) > 0 else np.array([1.0, 0.0])
                sx += ((p[:, :2] - p[0, :2]) @ t).sum()
                sy += p[:, 2].sum()
            else:
                sx += p[:, 0].sum()
                sy += p[:, 1].sum()
                sz += p[:, 2].sum() if dim == 3 else 0.0
        got = [float(v) for v in out[3:9]]
        want = [alpha, sx, sy, sz, sum(x["ntop"] for x in rays), sum(x["nbot"] for x in rays)]
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-6 * max(1.0, abs(sx)))


@pytest.mark.parametrize("case", ["seamount3d_gauss", "hex3d_nx2d_hat", "munk3d_gauss"])
def test_writeenv_3d_and_nx2d(case, tmp_path):
    """writeenv of a 3-D / Nx2D setup writes its files under the new root
    (.env and the boundary / SSP files), which set up the same run."""
    g = np.load(os.path.join(HERE, "golden", case + ".npz"))
    root = os.path.join(str(tmp_path), case)
    for k in g.files:
        if k.startswith("file_"):
            with open(root + "." + k[5:], "w") as f:
                f.write(str(g[k]))
    dim = "4" if "nx2d" in case else "3"
    exe = build_check(str(tmp_path))
    new = os.path.join(str(tmp_path), "copy")
    r = subprocess.run([exe, "writeenv", dim, root, new], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
    for k in g.files:
        if k.startswith("file_"):
            assert open(new + "." + k[5:]).read() == str(g[k])


def _hex_table(text):
    """x, y (km), z (m), c[ix, iy, iz] of a hexahedral .ssp file."""
    t = text.split()
    k = 0
    nx = int(t[k]); x = np.array(t[k + 1:k + 1 + nx], float); k += 1 + nx
    ny = int(t[k]); y = np.array(t[k + 1:k + 1 + ny], float); k += 1 + ny
    nz = int(t[k]); z = np.array(t[k + 1:k + 1 + nz], float); k += 1 + nz
    c = np.array(t[k:k + nx * ny * nz], float).reshape(nz, ny, nx).transpose(2, 1, 0)
    return x, y, z, c


def test_get_ssp_3d_and_nx2d(tmp_path):
    """get_ssp of 3-D and Nx2D setups: the hexahedral grid's nodes, a point
    halfway between two nodes in x (the mean of their c), and a 1-D profile's
    nodes and midpoints (c-linear)."""
    exe = build_check(str(tmp_path))

    def ssp(dim, root, *x):
        r = subprocess.run([exe, "ssp", str(dim), root] + ["%.17g" % v for v in x], capture_output=True,
                           text=True, timeout=60)
        assert r.returncode == 0, r.stdout + r.stderr
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("ssp ")][0].split()
        return float(line[2])

    def case(name):
        g = np.load(os.path.join(HERE, "golden", name + ".npz"))
        root = os.path.join(str(tmp_path), name)
        for k in g.files:
            if k.startswith("file_"):
                with open(root + "." + k[5:], "w") as f:
                    f.write(str(g[k]))
        return g, root

    g, root = case("hex3d_gauss")
    xk, yk, zk, c = _hex_table(str(g["file_ssp"]))
    for ix, iy, iz in ((0, 0, 0), (1, 2, 3), (2, 1, 5), (1, 1, 2)):
        got = ssp(3, root, xk[ix] * 1000.0, yk[iy] * 1000.0, zk[iz])
        assert abs(got - c[ix, iy, iz]) <= 1e-3, (ix, iy, iz, got, c[ix, iy, iz])
    got = ssp(3, root, 0.5 * (xk[0] + xk[1]) * 1000.0, yk[1] * 1000.0, zk[4])
    assert abs(got - 0.5 * (c[0, 1, 4] + c[1, 1, 4])) <= 1e-3
    g, root = case("munk3d_gauss")
    env = str(g["file_env"]).splitlines()
    k = [i for i, ln in enumerate(env) if ln.strip().startswith("'CVW")][0]
    prof = []
    for ln in env[k + 2:]:
        vals = ln.replace("/", " ").split()
        if len(vals) < 2 or not vals[0].replace(".", "", 1).isdigit():
            break
        prof.append((float(vals[0]), float(vals[1])))
        if float(vals[0]) >= 5000.0:
            break
    zp, cp = np.array(prof).T
    for i in (0, 10, 20):
        assert abs(ssp(3, root, 100.0, -50.0, zp[i]) - cp[i]) <= 1e-3
        mid = 0.5 * (zp[i] + zp[i + 1])
        assert abs(ssp(3, root, 0.0, 0.0, mid) - 0.5 * (cp[i] + cp[i + 1])) <= 1e-3
    g, root = case("hex3d_nx2d_hat")
    xk, yk, zk, c = _hex_table(str(g["file_ssp"]))
    assert abs(ssp(4, root, xk[2] * 1000.0, zk[3]) - c[2, 1, 3]) <= 1e-3   # (r, 0, z): y = 0 is node 1
