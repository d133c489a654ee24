"""Per-receiver arrival counts of the FULL 3-D workload (C4: 51,984 rays,
36 bearings x 101 depths x 501 ranges = 1,821,636 receivers) on the GPU
against the reference's single-threaded run (counts made by
``make_golden_c4.py counts REF.npz``; about 15 minutes of CPU, so they are
not a committed fixture).

    python tests/golden/check_c4_arrival_counts.py REF.npz

Prints how many receivers differ and exits non-zero if any does.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import bellhopcuda_b200 as B  # noqa: E402
from bellhopcuda_b200 import workloads as W  # noqa: E402
from make_golden_c4 import files_sha  # noqa: E402


def main(ref_path: str) -> int:
    g = np.load(ref_path)
    files = W.c4_3d(run_type="aB   3", ntheta=36)
    if files_sha(files) != str(g["sha"]):
        print("the counts were made from other inputs")
        return 2
    with tempfile.TemporaryDirectory() as d:
        root = os.path.join(d, "c4_full_arr")
        for suffix, text in files.items():
            with open(root + suffix, "w") as f:
                f.write(text)
        with B.Tracer(precision=B.PREC_FP64) as t:
            t.set_arrival_options(int(g["maxn"]), True)
            t.setup3d(root)
            t.run()
            narr, _ = t.arrivals()
            st = t.stats()
    narr = narr.reshape(-1)
    ref = g["narr"].astype(np.int32)
    diff = np.nonzero(narr != ref)[0]
    print("C4 arrivals, MaxNArr %d: %d receivers, %d arrivals (reference %d), %d receivers differ%s; "
          "GPU steps %d, err_bits 0x%x" % (int(g["maxn"]), narr.size, int(narr.sum()), int(ref.sum()), diff.size,
                                          (" (first: %s)" % diff[:10].tolist()) if diff.size else "",
                                          st["steps"], st["err_bits"]))
    return 1 if diff.size or narr.size != ref.size else 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1]))
