"""ORACLE — test/measurement infrastructure only.

Counts the oracle's ray steps and applied beam-receiver contributions for a
workload, splitting the rays over worker processes (spawned before any GPU
use). The counts are the algorithmic work units of the roofline numbers that
bench.py reports (steps x F_step + contributions x F_infl), so they come from
the oracle and not from the product's own step policy.

    python oracle/count_work.py rd_gauss   # all 10 frequencies
    python oracle/count_work.py munk_tl
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def _count(args):
    name, freq, first, count = args
    import oracle_ctypes
    from bellhopcuda_b200 import workloads as W
    spec = W.rd_gauss(freq=freq) if name == "rd_gauss" else W.munk_tl()
    r = oracle_ctypes.run(spec, rays=(first, count))
    return r["nsteps"], r["nevals"]


def count(name: str, nproc: int = 0) -> dict:
    from bellhopcuda_b200 import workloads as W
    freqs = W.rd_gauss_freqs() if name == "rd_gauss" else [W.munk_tl().freq]
    nrays = 20001 if name == "rd_gauss" else 2001
    chunk = 250
    tasks = [(name, f, a, min(chunk, nrays - a)) for f in freqs for a in range(0, nrays, chunk)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(nproc or os.cpu_count()) as pool:
        res = pool.map(_count, tasks)
    per = {}
    for (n_, f, _, _), (s, e) in zip(tasks, res):
        d = per.setdefault(repr(f), [0, 0])
        d[0] += s
        d[1] += e
    return {"workload": name, "freqs": freqs, "nrays": nrays,
            "steps": {k: v[0] for k, v in per.items()}, "evals": {k: v[1] for k, v in per.items()},
            "steps_total": sum(v[0] for v in per.values()),
            "evals_total": sum(v[1] for v in per.values())}


if __name__ == "__main__":
    out = count(sys.argv[1] if len(sys.argv) > 1 else "rd_gauss")
    print(json.dumps(out, indent=1))
