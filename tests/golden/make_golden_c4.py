"""Golden fixtures of the full-size 3-D workload (C4) on a subset of bearings,
and the reference's per-receiver arrival counts on the whole receiver grid.

The environment is the full C4 one (``workloads.c4_3d``: hexahedral Munk +
eddy SSP on 41 x 41 x 51 nodes, 101 x 101 bathymetry grid, 144 x 361 rays,
source 500 m, 200 Hz, 101 depths x 501 ranges); only the receiver bearings
are cut to two of its 36 (0 and 180 degrees), so every ray of the full fan is
traced and every bearing plane of the subset sees all of them. The reference
is the reference's own bellhopcxx built by ``oracle/Makefile``.

    python tests/golden/make_golden_c4.py            # both subset fixtures
    python tests/golden/make_golden_c4.py tl|arr     # one of them
    python tests/golden/make_golden_c4.py counts OUT.npz
        # arrival counts of the FULL C4 grid (36 bearings) from the reference's
        # single-threaded run (the mode in which it merges arrivals; about
        # 15 minutes on 8 cores), for tests/golden/check_c4_arrival_counts.py

Fixtures store the sha256 of the input files instead of their text: the GPU
tests regenerate the files from the seeded generator and check the hashes.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bellhopcuda_b200 import workloads as W  # noqa: E402
from bellhopcuda_b200.arrfile import read_arr_binary  # noqa: E402
from bellhopcuda_b200.shdfile import read_shd  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "bellhopcxx")
NTHETA_SUBSET = 2          # bearings 0 and 180 degrees of the 36-bearing grid
SAMPLE_EVERY = 997         # arrival records kept for every 997th receiver


def c4_files(run_type: str, ntheta: int = NTHETA_SUBSET) -> dict:
    return W.c4_3d(run_type=run_type, ntheta=ntheta)


def files_sha(files: dict) -> np.ndarray:
    h = hashlib.sha256()
    for suffix in sorted(files):
        h.update(suffix.encode())
        h.update(files[suffix].encode())
    return np.array(h.hexdigest())


def _run(files: dict, d: str, name: str, single: bool) -> str:
    root = os.path.join(d, name)
    for suffix, text in files.items():
        with open(root + suffix, "w") as f:
            f.write(text)
    cmd = [EXE, "-3"] + (["-1"] if single else []) + [root]
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise SystemExit("reference failed on %s:\n%s%s" % (name, r.stdout[-2000:], r.stderr[-2000:]))
    print(name, "reference run %.1fs" % (time.time() - t0), flush=True)
    return root


def make_tl(d: str) -> None:
    files = c4_files("CB   3")
    root = _run(files, d, "c4_bearings_tl", single=False)
    shd = read_shd(root + ".shd")
    np.savez_compressed(os.path.join(HERE, "c4_bearings_tl.npz"), field=shd["field"].astype(np.complex64),
                        rr=shd["rr"], rz=shd["rz"], theta=shd["theta"], sha=files_sha(files))
    print("c4_bearings_tl", shd["field"].shape)


def _arrivals(root: str):
    A = read_arr_binary(root + ".arr")
    narr = np.array([len(a) for src in A["sources"] for a in src["arrivals"]], np.int32)
    return A, narr


def make_arr(d: str) -> None:
    files = c4_files("aB   3")
    root = _run(files, d, "c4_bearings_arr", single=True)
    A, narr = _arrivals(root)
    flat = [a for src in A["sources"] for a in src["arrivals"]]
    idx = np.arange(0, len(flat), SAMPLE_EVERY, dtype=np.int64)
    recs = np.concatenate([flat[i] for i in idx] or [np.zeros((0, 10), np.float32)])
    np.savez_compressed(os.path.join(HERE, "c4_bearings_arr.npz"), narr=narr.astype(np.int16),
                        maxn=np.int32(A["sources"][0]["maxn"]), sample_idx=idx, sample_arr=recs,
                        rr=A["rr"], rz=A["rz"], theta=A["theta"], sha=files_sha(files))
    print("c4_bearings_arr arrivals", int(narr.sum()), "max", int(narr.max()), "maxn", A["sources"][0]["maxn"])


def make_counts(out: str) -> None:
    files = c4_files("aB   3", ntheta=36)
    with tempfile.TemporaryDirectory() as d:
        root = _run(files, d, "c4_full_arr", single=True)
        A, narr = _arrivals(root)
    np.savez_compressed(out, narr=narr.astype(np.int16), maxn=np.int32(A["sources"][0]["maxn"]),
                        theta=A["theta"], sha=files_sha(files))
    print("full C4 arrival counts:", narr.size, "receivers,", int(narr.sum()), "arrivals, maxn",
          A["sources"][0]["maxn"])


def main(argv):
    if argv and argv[0] == "counts":
        return make_counts(argv[1])
    with tempfile.TemporaryDirectory() as d:
        if not argv or "tl" in argv:
            make_tl(d)
        if not argv or "arr" in argv:
            make_arr(d)


if __name__ == "__main__":
    main(sys.argv[1:])
