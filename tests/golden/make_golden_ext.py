"""Generate the fixtures of the 2-D cases in tests/golden/cases2d_ext.py from
the reference itself.

Runs the reference's own bellhopcxx (compiled from its sources by
oracle/Makefile into oracle/_ref/) single-threaded as a 2-D run on every case
and stores, per case, the input files' text and the scaled complex field
[isz][iz][ir] as tests/golden/<case>.npz. The GPU tests write the input
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
            if r.returncode != 0 or not os.path.exists(root + ".shd"):
                raise SystemExit("reference failed on %s:\n%s%s" % (name, r.stdout[-2000:], r.stderr[-2000:]))
            texts = {"file_" + suffix[1:]: np.array(text) for suffix, text in files.items()}
            shd = read_shd(root + ".shd")
            field = shd["field"][0, 0, 0]
            np.savez_compressed(os.path.join(HERE, name + ".npz"), field=field, rr=shd["rr"], rz=shd["rz"],
                                sz=shd["sz"], **texts)
            print(name, field.shape, "%.3g" % float(np.abs(field).max()), "%.1fs" % (time.time() - t0))


if __name__ == "__main__":
    main(sys.argv[1:])
