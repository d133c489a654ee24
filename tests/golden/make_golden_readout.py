"""Generate the readout fixtures: output files written by the reference itself.

Runs the reference's bellhopcxx (compiled from its sources by oracle/Makefile
into oracle/_ref/) on small 2-D, 3-D and Nx2D environments with RunType 'A'
(ASCII arrivals), 'a' (binary arrivals) and 'R' (rays), and stores each
case's .env text and the .arr / .ray file it wrote in
tests/golden/readout_cases.npz. tests/test_bhc_api.py reads those files back
through bhc::readout without the reference or a GPU. Run from the repository
root:

    make -C oracle ref && python tests/golden/make_golden_readout.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from bellhopcuda_b200 import workloads as W  # noqa: E402
from bellhopcuda_b200.envfile import env_text  # noqa: E402
from cases3d import _munk_slice  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "bellhopcxx")


def _env2d(run_type, nalpha=21):
    spec = W.munk_tl(nalpha=nalpha, nrz=5, nrr=6)
    spec.run_type = run_type
    return env_text(spec)


CASES = {
    # name: (dimension flag, .env text, output suffix)
    "ro2d_A": (2, lambda: _env2d("AG RR "), ".arr"),
    "ro2d_a": (2, lambda: _env2d("aG RR "), ".arr"),
    "ro2d_R": (2, lambda: _env2d("RG RR ", nalpha=7), ".ray"),
    "ro3d_A": (3, lambda: _munk_slice("AG   3", alpha=(15, -15.0, 15.0), beta=(5, -6.0, 6.0), theta=[0.0, 3.0],
                                      nrz_range=(3, 800.0, 2800.0), rr_range=(4, 8.0, 26.0))[".env"], ".arr"),
    "ro3d_a": (3, lambda: _munk_slice("aG   3", alpha=(31, -15.0, 15.0), beta=(7, -6.0, 6.0), theta=[0.0, 3.0],
                                      nrz_range=(3, 800.0, 2800.0), rr_range=(4, 8.0, 26.0))[".env"], ".arr"),
    "ro3d_R": (3, lambda: _munk_slice("R    3", alpha=(5, -12.0, 12.0), beta=(2, -6.0, 6.0),
                                      theta=[0.0])[".env"], ".ray"),
    "ronx_a": (4, lambda: _munk_slice("aB   2", alpha=(31, -15.0, 15.0), theta=[0.0, 3.0],
                                      nrz_range=(3, 800.0, 2800.0), rr_range=(4, 8.0, 26.0))[".env"], ".arr"),
    "ronx_R": (4, lambda: _munk_slice("R    2", alpha=(5, -12.0, 12.0), beta=(2, -6.0, 6.0),
                                      theta=[0.0])[".env"], ".ray"),
}


def main():
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, (dim, env, suffix) in CASES.items():
            root = os.path.join(d, name)
            text = env()
            with open(root + ".env", "w") as f:
                f.write(text)
            flag = {2: [], 3: ["-3"], 4: ["-4"]}[dim]
            r = subprocess.run([EXE] + flag + ["-1", root], capture_output=True, text=True)
            if r.returncode != 0:
                raise SystemExit("reference failed on %s:\n%s%s" % (name, r.stdout[-2000:], r.stderr[-2000:]))
            data = open(root + suffix, "rb").read()
            out[name + "_env"] = np.array(text)
            out[name + "_out"] = np.frombuffer(data, np.uint8)
            out[name + "_dim"] = np.int32(dim)
            out[name + "_suffix"] = np.array(suffix)
            print(name, suffix, len(data), "bytes")
    np.savez_compressed(os.path.join(HERE, "readout_cases.npz"), **out)


if __name__ == "__main__":
    main()
