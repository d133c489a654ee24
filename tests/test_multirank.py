"""Multi-rank host logic of bench.py on CPU: two gloo ranks.

On the GPUs each rank traces its own environment (weak scaling, no data-path
collective); the only collectives are the barrier around the timed region and
the max-over-ranks of the timing. These run here over gloo with world size 2.
"""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import datetime, json, os, sys, tempfile
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
comm = bench.RankComm(dist, "cpu", None)
comm.barrier()
t = comm.max_over_ranks(1.25 + rank)      # per-rank "timed region" seconds
with tempfile.TemporaryDirectory() as tmp:
    spec, root, freqs = bench.make_env(tmp, rank)
    ssp = [round(float(c), 6) for c in spec.ssp_cp[:4]]
v = bench.aggregate_value(world, len(freqs), 5, t)
comm.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": rank, "max": t, "value": v, "ssp": ssp}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_bench_ranks_gloo_world2(tmp_path):
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, ROOT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    # both ranks see the slowest rank's time and the same whole-job value
    assert outs[0]["max"] == outs[1]["max"] == 2.25
    assert outs[0]["value"] == outs[1]["value"] == 2 * 10 * 5 / 2.25
    # each rank traces its own environment (different seeds)
    assert outs[0]["ssp"] != outs[1]["ssp"]


def test_aggregate_value_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_value(1, 10, 5, 0.25) == 200.0
    c = bench.RankComm(None, "cpu", None)
    c.barrier()
    assert c.max_over_ranks(3.0) == 3.0
