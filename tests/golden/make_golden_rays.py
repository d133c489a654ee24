"""Generate the ray-trajectory fixtures (.ray) from the reference itself.

Runs the reference's own bellhopcxx (compiled from its sources by
oracle/Makefile into oracle/_ref/) single-threaded on ray runs ('R') and
eigenray runs ('E') of the Munk and range-dependent workloads, a quad-SSP case
and a beam-shift case, and stores the
input files and the trajectories as tests/golden/rays_<case>.npz. Run from the
repository root:

    make -C oracle ref && python tests/golden/make_golden_rays.py
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

from bellhopcuda_b200 import workloads as W  # noqa: E402
from bellhopcuda_b200.envfile import write_env  # noqa: E402
from bellhopcuda_b200.rayfile import read_ray  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "bellhopcxx")


def cases():
    munk_r = W.munk_tl(nalpha=41, nrz=11, nrr=21)
    munk_r.run_type = "R      "
    munk_r.alpha = (-14.0, 14.0)
    rd_r = W.rd_gauss(nalpha=31, nrz=11, nrr=21, nbty=30)
    rd_r.run_type = "RB RR "
    munk_e = W.munk_tl(nalpha=401, nrz=3, nrr=5, beam="G")
    munk_e.rz = (500.0, 2500.0)
    munk_e.rr_km = (20.0, 60.0)
    munk_e.run_type = "EG RR "
    rd_e = W.rd_gauss(nalpha=151, nrz=2, nrr=2, nbty=30)
    rd_e.rz = (800.0, 2000.0)
    rd_e.rr_km = (30.0, 60.0)
    rd_e.run_type = "EB RR "
    sys.path.insert(0, HERE)
    from cases2d_ext import CASES2D_EXT
    quad_r = CASES2D_EXT["x2d_quad_shallow_bty"]()
    quad_r[".env"] = quad_r[".env"].replace("'CG RR'", "'R'").replace("\n401\n", "\n41\n")
    shift_r = CASES2D_EXT["x2d_beam_shift_shallow"]()
    shift_r[".env"] = shift_r[".env"].replace("'CB RR S'", "'RB RR S'").replace("\n301\n", "\n31\n")
    return {"munk_ray": munk_r, "rd_ray": rd_r, "munk_eigen": munk_e, "rd_eigen": rd_e,
            "quad_ray": quad_r, "beam_shift_ray": shift_r}


def write_files(files, root):
    for suffix, text in files.items():
        with open(root + suffix, "w") as f:
            f.write(text)
    return root


def main(names=None):
    with tempfile.TemporaryDirectory() as d:
        for name, spec in cases().items():
            if names and name not in names:
                continue
            if isinstance(spec, dict):     # input files as text (tests/golden/cases2d_ext.py)
                root = write_files(spec, os.path.join(d, name))
            else:
                root = write_env(spec, os.path.join(d, name))
            r = subprocess.run([EXE, "-2", "-1", root], capture_output=True, text=True)
            if r.returncode != 0:
                raise SystemExit("reference failed on %s:\n%s" % (name, r.stdout[-2000:]))
            R = read_ray(root + ".ray")
            npts = np.array([len(x["xy"]) for x in R["rays"]], np.int32)
            files = {}
            for ext in (".env", ".bty", ".ati", ".ssp", ".sbp", ".brc", ".trc"):
                if os.path.exists(root + ext):
                    files["file_" + ext[1:]] = np.array(open(root + ext).read())
            np.savez_compressed(os.path.join(HERE, "rays_" + name + ".npz"),
                                alpha=np.array([x["alpha"] for x in R["rays"]]), npts=npts,
                                bnc=np.array([[x["ntop"], x["nbot"]] for x in R["rays"]], np.int32).reshape(-1, 2),
                                rz=np.concatenate([x["xy"] for x in R["rays"]]) if len(npts) else np.zeros((0, 2)),
                                **files)
            print(name, "rays", len(npts), "points", int(npts.sum()))


if __name__ == "__main__":
    main(sys.argv[1:])
