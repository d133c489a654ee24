"""The bhc:: C++ interface on the GPU: a program written against
include/bhcb/bhc.hpp (tests/bhc_api_check.cpp) runs the tracer through
setup / run / writeout / readout and its field is compared with the oracle.

Tolerance: TL RMS over receivers with oracle TL < 100 dB, 0.1 dB for the FP64
tracer (the default), 0.5 dB with BHCB_PRECISION=mixed.
"""
import os
import subprocess

import numpy as np
import pytest

import bellhopcuda_b200 as B
from bellhopcuda_b200 import workloads as W
from bellhopcuda_b200.envfile import EnvSpec, write_env
import oracle_ctypes
from test_bhc_api import build_check
from test_gpu_parity import tl_err

pytestmark = pytest.mark.gpu


def defaults_spec():
    """The modules' defaults as an environment file (src/module/*.hpp Default())."""
    return EnvSpec(title="no env file", bot_bc="R", sz=(567.8,), nrz=11, rz=(0.0, 5000.0), nrr=10,
                   rr_km=(5.0, 50.0), nalpha=0, box_z=6000.0, box_r_km=101.0)


def run_exe(exe, args, precision="fp64"):
    env = dict(os.environ)
    if precision == "mixed":
        env["BHCB_PRECISION"] = "mixed"
    r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=600, env=env)
    print(r.stdout[-2000:], r.stderr[-2000:])
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")


def field_of(path, nrz, nrr):
    u = np.fromfile(path, dtype=np.complex64)
    return u.reshape(-1, nrz, nrr)[0]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_defaults_match_oracle(precision, tmp_path):
    exe = build_check(str(tmp_path))
    out = os.path.join(tmp_path, "def.bin")
    run_exe(exe, ["run", "-", out, os.path.join(tmp_path, "def_out")], precision)
    ref = oracle_ctypes.run(defaults_spec())
    got = field_of(out, 11, 10)
    rms, p99, n = tl_err(got, ref["field"][0])
    print("defaults", precision, rms, p99, n)
    assert n > 50
    assert rms < (0.1 if precision == "fp64" else 0.5)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_file_run_writeout_readout(precision, tmp_path):
    exe = build_check(str(tmp_path))
    spec = W.munk_tl(nalpha=301, nrz=51, nrr=201, beam="B")
    root = os.path.join(tmp_path, "munk")
    write_env(spec, root)
    out = os.path.join(tmp_path, "munk.bin")
    run_exe(exe, ["run", root, out, os.path.join(tmp_path, "munk_out")], precision)
    ref = oracle_ctypes.run(spec)
    rms, p99, n = tl_err(field_of(out, 51, 201), ref["field"][0])
    print("munk", precision, rms, p99, n)
    assert n > 1000
    assert rms < (0.1 if precision == "fp64" else 0.5)
    # the same file through the Python Tracer (file route of the C ABI)
    with B.Tracer() as t:
        t.setup(root)
        t.run()
        same = t.field(0, 0)[0]
    rms2, _, _ = tl_err(field_of(out, 51, 201), same)
    assert rms2 < 0.01 if precision == "fp64" else rms2 < 0.5


def test_nonblocking(tmp_path):
    exe = build_check(str(tmp_path))
    root = os.path.join(tmp_path, "munk_nb")
    write_env(W.munk_tl(nalpha=301, nrz=51, nrr=201), root)
    run_exe(exe, ["nonblocking", root])


def test_desc_route_matches_file_route(tmp_path):
    """An environment handed over in memory (bhcb_add_env_desc) traces the same
    rays as the same environment read from its files: equal step and
    contribution counts (the oracle's) and the same field."""
    spec = W.rd_gauss(nalpha=401, nrz=61, nrr=201, nbty=60)
    root = write_env(spec, os.path.join(tmp_path, "rd"))
    ref = oracle_ctypes.run(spec)
    with B.Tracer() as t:
        t.setup(root)
        t.run()
        a, sa = t.field(0, 0)[0], t.stats()
        t.clear()
        with B.EnvDescription(root) as e:
            assert t.add_env_desc(e) == 0
        t.run()
        b, sb = t.field(0, 0)[0], t.stats()
        c = t.ssp_at(0, 1000.0, spec.ssp_z[1])
    assert sa["steps"] == sb["steps"] == ref["nsteps"]
    assert sa["evals"] == sb["evals"] == ref["nevals"]
    rms, _, n = tl_err(b, a)
    assert n > 1000 and rms < 1e-3
    assert abs(c - spec.ssp_cp[1]) < 1e-6


def test_3d_arrivals_through_bhc(tmp_path):
    """A 3-D arrivals run ('a', munk3d_arr_hat) through bhc::setup<true, true> /
    run: the arrival counts sum to the reference's and MaxNPerSource holds each
    source's largest count over all its bearings and receivers."""
    HERE = os.path.dirname(os.path.abspath(__file__))
    g = np.load(os.path.join(HERE, "golden", "munk3d_arr_hat.npz"))
    root = os.path.join(str(tmp_path), "munk3d_arr_hat")
    for k in g.files:
        if k.startswith("file_"):
            with open(root + "." + k[5:], "w") as f:
                f.write(str(g[k]))
    exe = build_check(str(tmp_path))
    r = subprocess.run([exe, "run3arr", root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("arr3 ")][0].split()
    assert int(line[1]) == 1 and int(line[2]) == int(g["narr"].sum()) > 0
