"""Run one synthetic workload through the C ABI and print its counters.

    python -m bellhopcuda_b200.run_workload rd_gauss --nalpha 4001 --all-freqs
    python -m bellhopcuda_b200.run_workload munk_tl --precision fp64
    python -m bellhopcuda_b200.run_workload batch --count 256 --scale 1.0

Used for profiling captures (ncu) of a chosen size; writes the input files
under --dir (default: a temporary directory).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import bellhopcuda_b200 as B  # noqa: E402
from bellhopcuda_b200 import workloads as W  # noqa: E402
from bellhopcuda_b200.envfile import write_env  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["rd_gauss", "munk_tl", "batch"])
    ap.add_argument("--nalpha", type=int, default=0, help="rays (0 = the workload's own)")
    ap.add_argument("--all-freqs", action="store_true", help="rd_gauss: evaluate all 10 frequencies")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--dir", default=None)
    ap.add_argument("--count", type=int, default=256, help="batch: environments")
    ap.add_argument("--scale", type=float, default=1.0, help="batch: ray / receiver scale")
    ap.add_argument("--max-memory-gb", type=float, default=0.0, help="device budget (0: library default)")
    a = ap.parse_args(argv)
    d = a.dir or tempfile.mkdtemp()
    prec = B.PREC_FP64 if a.precision == "fp64" else B.PREC_MIXED
    if a.workload == "batch":
        roots = [write_env(s, os.path.join(d, "batch_%d" % i))
                 for i, s in enumerate(W.batch_envs(n=a.count, scale=a.scale))]
        with B.Tracer(precision=prec, max_memory=int(a.max_memory_gb * 2**30)) as t:
            for r in roots:
                t.add_env(r)
            for _ in range(a.repeat):
                t.run()
                print(json.dumps(t.stats()), flush=True)
        return 0
    kw = {"nalpha": a.nalpha} if a.nalpha else {}
    spec = W.rd_gauss(**kw) if a.workload == "rd_gauss" else W.munk_tl(**kw)
    root = write_env(spec, os.path.join(d, a.workload))
    with B.Tracer(precision=prec, max_memory=int(a.max_memory_gb * 2**30)) as t:
        t.setup(root)
        if a.all_freqs and a.workload == "rd_gauss":
            t.set_frequencies(0, W.rd_gauss_freqs())
        for _ in range(a.repeat):
            t.run()
            print(json.dumps(t.stats()), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
