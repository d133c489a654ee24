"""Generate the fixtures of the 2-D cases in tests/golden/cases2d_ext.py from
the reference itself.

Runs the reference's own bellhopcxx (compiled from its sources by
oracle/Makefile into oracle/_ref/) single-threaded as a 2-D run on every case
and stores, per case, the input files' text and the scaled complex field
[isz][iz][ir] (TL runs), the arrivals (RunType 'a') or the re-traced eigen
hit rays ('E') as tests/golden/<case>.npz. The GPU tests write the input
files back from the fixture, so they need neither the reference nor this
script at run time. Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden_ext.py [case ...]
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
from cases2d_ext import CASES2D_EXT  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "bellhopcxx")


def main(names=None):
    with tempfile.TemporaryDirectory() as d:
        for name, fn in CASES2D_EXT.items():
            if names and name not in names:
                continue
            files = fn()
            root = os.path.join(d, name)
            for suffix, text in files.items():
                with open(root + suffix, "w") as f:
                    f.write(text)
            t0 = time.time()
            r = subprocess.run([EXE, "-2", "-1", root], capture_output=True, text=True)
            if r.returncode != 0 or not any(os.path.exists(root + x) for x in (".shd", ".arr", ".ray")):
                raise SystemExit("reference failed on %s:\n%s%s" % (name, r.stdout[-2000:], r.stderr[-2000:]))
            texts = {"file_" + suffix[1:]: np.array(text) for suffix, text in files.items()}
            extra = {}
            if os.path.exists(root + ".ray") and os.path.exists(root + ".arr"):
                # arrivals and eigen hits ('V' / 'v'): both, the rays' keys prefixed
                R = read_ray(root + ".ray")
                extra = dict(eig_alpha=np.array([x["alpha"] for x in R["rays"]]),
                             eig_npts=np.array([len(x["xy"]) for x in R["rays"]], np.int32))
                print(name, "eigen rays", len(R["rays"]))
            elif os.path.exists(root + ".ray"):
                # eigen hits ('E'): the reference writes the hit rays re-traced,
                # in hit order; each ray's take-off angle (deg) and point count
                # (the hit's step + 2) pin the hit list
                R = read_ray(root + ".ray")
                npts = np.array([len(x["xy"]) for x in R["rays"]], np.int32)
                nkeep = min(len(npts), 64)
                np.savez_compressed(os.path.join(HERE, name + ".npz"),
                                    alpha=np.array([x["alpha"] for x in R["rays"]]), npts=npts,
                                    bnc=np.array([[x["ntop"], x["nbot"]] for x in R["rays"]], np.int32).reshape(-1, 2),
                                    xyz=np.concatenate([x["xy"] for x in R["rays"][:nkeep]]) if nkeep
                                    else np.zeros((0, 2)), xyz_rays=np.int32(nkeep), **texts)
                print(name, "eigen rays", len(R["rays"]), "%.1fs" % (time.time() - t0))
                continue
            if os.path.exists(root + ".arr"):
                # arrivals: per receiver (source, depth, range) the count and
                # the records (a, phase deg, delay re / im, source and receiver
                # declination, top / bottom bounces), flattened
                A = read_arr_binary(root + ".arr")
                narr = np.array([len(a) for src in A["sources"] for a in src["arrivals"]], np.int32)
                recs = np.concatenate([a for src in A["sources"] for a in src["arrivals"]] or
                                      [np.zeros((0, 8), np.float32)])
                np.savez_compressed(os.path.join(HERE, name + ".npz"), narr=narr, arr=recs, rr=A["rr"], rz=A["rz"],
                                    sz=A["sz"], maxn=np.array([s["maxn"] for s in A["sources"]], np.int32), **extra,
                                    **texts)
                print(name, "arrivals", int(narr.sum()), "max", int(narr.max()), "%.1fs" % (time.time() - t0))
                continue
            shd = read_shd(root + ".shd")
            field = shd["field"][0, 0, 0]
            np.savez_compressed(os.path.join(HERE, name + ".npz"), field=field, rr=shd["rr"], rz=shd["rz"],
                                sz=shd["sz"], **texts)
            print(name, field.shape, "%.3g" % float(np.abs(field).max()), "%.1fs" % (time.time() - t0))


if __name__ == "__main__":
    main(sys.argv[1:])
