"""The bhc:: C++ interface (include/bhcb/bhc.hpp) over libbhcb.so, on the CPU.

A program written against the header (tests/bhc_api_check.cpp) is compiled and
linked here; its "params" mode exercises setup from the defaults and from
files, the extsetup_* resizing, writeenv round trips and get_ssp, none of
which needs a GPU. The GPU runs are in test_gpu_bhc_api.py.
"""
import os
import shutil
import subprocess

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
