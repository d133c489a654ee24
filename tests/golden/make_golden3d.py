"""Generate the 3-D golden TL fixtures from the reference itself.

Runs the reference's own bellhopcxx (compiled from its sources by
oracle/Makefile into oracle/_ref/) as a 3-D run (-3), or an Nx2D run (-4) for
cases whose RunType(6) is '2', on every case of
tests/golden/cases3d.py and stores, per case, the input files' text and the
scaled complex field (TL runs), the arrivals (RunType 'a'), the rays
('R', 'E') or the arrivals with the hit rays ('v') as
tests/golden/<case>.npz. The GPU tests write the input
files back from the fixture, so they need neither the reference nor this
script at run time. Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden3d.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from bellhopcuda_b200.arrfile import read_arr_binary  # noqa: E402
from bellhopcuda_b200.rayfile import read_ray  # noqa: E402
from bellhopcuda_b200.shdfile import read_shd  # noqa: E402
from cases3d import CASES3D  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "bellhopcxx")


def main(names=None):
    with tempfile.TemporaryDirectory() as d:
        for name, fn in CASES3D.items():
            if names and name not in names:
                continue
            files = fn()
            root = os.path.join(d, name)
            for suffix, text in files.items():
                with open(root + suffix, "w") as f:
                    f.write(text)
            t0 = time.time()
            # RunType(6) '2' selects the reference's Nx2D mode (-4), '3' its 3-D mode
            run_line = [ln for ln in files[".env"].splitlines() if ln.startswith("'") and ln.rstrip().endswith(
                ("3'", "2'"))]
            dim = "-4" if run_line and run_line[-1].rstrip().endswith("2'") else "-3"
            r = subprocess.run([EXE, dim, "-1", root], capture_output=True, text=True)
            if r.returncode != 0:
                raise SystemExit("reference failed on %s:\n%s%s" % (name, r.stdout[-2000:], r.stderr[-2000:]))
            texts = {"file_" + suffix[1:]: np.array(text) for suffix, text in files.items()}
            rays = {}
            if os.path.exists(root + ".ray"):
                # ray runs ('R') and eigen hits ('E', 'V', 'v'): the reference
                # writes the traced rays (eigen: the hit rays re-traced, in hit
                # order, so each ray's take-off angle in radians and point count,
                # the hit's step + 2, pin the hit list) with their points (x, y, z)
                R = read_ray(root + ".ray")
                npts = np.array([len(x["xy"]) for x in R["rays"]], np.int32)
                # points of the first (at most) 64 rays keep the fixture small
                nkeep = min(len(npts), 64)
                rays = dict(alpha=np.array([x["alpha"] for x in R["rays"]]), npts=npts,
                            bnc=np.array([[x["ntop"], x["nbot"]] for x in R["rays"]], np.int32).reshape(-1, 2),
                            xyz=np.concatenate([x["xy"] for x in R["rays"][:nkeep]]) if nkeep
                            else np.zeros((0, 3)), xyz_rays=np.int32(nkeep))
                print(name, "rays", len(R["rays"]), "points", int(npts.sum()), "%.1fs" % (time.time() - t0))
            if os.path.exists(root + ".arr"):
                # arrivals: per receiver (source, bearing, depth, range) the
                # count and the records, flattened with offsets; a combined run
                # ('V', 'v') keeps its hit rays beside them under eig_*
                A = read_arr_binary(root + ".arr")
                narr = np.array([len(a) for src in A["sources"] for a in src["arrivals"]], np.int32)
                recs = np.concatenate([a for src in A["sources"] for a in src["arrivals"]] or
                                      [np.zeros((0, 10), np.float32)])
                eig = {"eig_" + k: v for k, v in rays.items()}
                np.savez_compressed(os.path.join(HERE, name + ".npz"), narr=narr, arr=recs, rr=A["rr"],
                                    rz=A["rz"], sz=A["sz"], theta=A["theta"],
                                    maxn=np.array([s["maxn"] for s in A["sources"]], np.int32), **eig, **texts)
                print(name, "arrivals", int(narr.sum()), "max", int(narr.max()), "%.1fs" % (time.time() - t0))
                continue
            if rays:
                np.savez_compressed(os.path.join(HERE, name + ".npz"), **rays, **texts)
                continue
            shd = read_shd(root + ".shd")
            np.savez_compressed(os.path.join(HERE, name + ".npz"), field=shd["field"],
                                rr=shd["rr"], rz=shd["rz"], sz=shd["sz"], theta=shd["theta"], **texts)
            print(name, shd["field"].shape, "%.3g" % float(np.abs(shd["field"]).max()),
                  "%.1fs" % (time.time() - t0))


if __name__ == "__main__":
    main(sys.argv[1:])
