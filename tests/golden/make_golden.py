"""Generate the golden TL fixtures from the reference itself.

Runs the reference's own bellhopcxx (compiled from its sources by
oracle/Makefile into oracle/_ref/) single-threaded on every case of
tests/golden/cases.py and stores the scaled complex field of each as
tests/golden/<case>.npz. Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py
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

from bellhopcuda_b200.envfile import write_env  # noqa: E402
from bellhopcuda_b200.shdfile import read_shd  # noqa: E402
from cases import CASES  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "bellhopcxx")


def main():
    with tempfile.TemporaryDirectory() as d:
        for name, fn in CASES.items():
            root = write_env(fn(), os.path.join(d, name))
            r = subprocess.run([EXE, "-2", "-1", root], capture_output=True, text=True)
            if r.returncode != 0:
                raise SystemExit("reference failed on %s:\n%s" % (name, r.stdout[-2000:]))
            shd = read_shd(root + ".shd")
            np.savez_compressed(os.path.join(HERE, name + ".npz"), field=shd["field"][0, 0, 0],
                                rr=shd["rr"], rz=shd["rz"], sz=shd["sz"])
            print(name, shd["field"].shape, float(np.abs(shd["field"]).max()))


if __name__ == "__main__":
    main()
