#!/usr/bin/env python
"""Benchmark: TL fields/s on one B200 for the range-dependent Gaussian-beam
workload (2-D, PCHIP SSP, 200-point bathymetry, 20001 rays over +-30 deg,
501 x 2001 receivers, 10 log-spaced frequencies 50-500 Hz).

A step is one pass of the hot path over the batch: trace every ray, evaluate
every beam-receiver contribution for all 10 frequencies, post-process the 10
TL fields. Our arm runs the mixed-precision path (FP64 ray trace, FP32
beam-receiver contributions) with the 10 frequencies sharing one trajectory,
successive steps pipelined (two traces side by side, then their influences);
beside it on the same line: the steps one at a time (`serial_steps`), the
FP64 per-frequency tracer (`fp64_trace`), the 3-D workload (`c4_3d_tl`), the
TL surrogate with its FP64 fallback (`surrogate`), the end-to-end rate through
the C ABI with host buffers (`e2e`) and the reference's bellhopcxx on the host
cores (`cpu_baseline`).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank owns a different environment of the same
shape (seed + rank); there is no data-path collective ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TL fields/s on 1 B200: mixed vs FP64 trace, surrogate vs plain, <=0.5 dB TL err"
UNIT = "TL fields/s"
WORKLOAD = "rd_gauss"
# the workload both arms run (identical in both JSON lines)
CONFIG = {"workload": "rd_gauss: 2-D Gaussian-beam TL, PCHIP SSP 64 nodes, 200-pt bathymetry, 20001 rays "
                      "+-30 deg, 501x2001 receivers, 10 freqs 50-500 Hz (log-spaced)",
          "fields": 10, "rays": 20001, "receivers": 501 * 2001}

# Algorithmic work per unit, frozen before the first GPU timing: one 2-D
# oracle ray step (Step + RayUpdate + RayTerminate for a 1-D SSP) and one
# applied beam-receiver contribution (InfluenceGeoCore + ApplyContribution).
F_STEP = 320.0
F_INFL = 40.0
# Oracle counts for this workload (oracle/count_work.py rd_gauss): trajectories
# do not depend on frequency, so steps are per trace; contributions are summed
# over the 10 frequencies.
ORACLE_STEPS_PER_TRACE = 20993289
ORACLE_EVALS_ALL_FREQS = 6440570521
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one full-size
# influence launch (10 frequencies) of the current build: 863.68 MB read +
# 506.92 MB written, from a one-pass ncu capture of the full workload
# summarised in profiles/influence_kernel_rd_gauss.md.
INFLUENCE_DRAM_BYTES = 863.68e6 + 506.92e6


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                      "-lms", "200", "-i", str(self.gpu)], stdout=self.f,
                                     stderr=subprocess.DEVNULL)
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- ranks
class RankComm:
    """Barrier and max-over-ranks around the timed region: NCCL on the GPUs
    (device "cuda"), gloo on CPU in the multi-rank tests (device "cpu")."""

    def __init__(self, dist=None, device="cuda", sync=None):
        self.dist, self.device, self.sync = dist, device, sync

    def barrier(self):
        if self.dist:
            self.dist.barrier()
        if self.sync:
            self.sync()

    def max_over_ranks(self, x):
        if not self.dist:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def aggregate_value(world, fields_per_step, steps, total_s):
    """Whole-job TL fields/s: every rank computes its own environment (weak
    scaling); the job time is the slowest rank's."""
    return world * fields_per_step * steps / total_s


# ------------------------------------------------------------- FP pipe peaks
def probe_fp_peak(gpu):
    """Measured (FP32, FP64) FMA throughput in TFLOP/s from bench_probe.so
    (bench_probe.cu, built by __graft_entry__.build())."""
    lib = ctypes.CDLL(os.path.join(ROOT, "bench_probe.so"))
    lib.bench_probe_fp_peak.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]
    a, b = ctypes.c_double(), ctypes.c_double()
    if lib.bench_probe_fp_peak(gpu, ctypes.byref(a), ctypes.byref(b)) != 0:
        raise RuntimeError("FP peak probe failed")
    return a.value, b.value


# ------------------------------------------------------------- environment
def make_env(tmp, rank, rays=0):
    from bellhopcuda_b200 import workloads as W
    from bellhopcuda_b200.envfile import write_env
    spec = W.rd_gauss(seed=1002 + rank) if not rays else W.rd_gauss(seed=1002 + rank, nalpha=rays)
    root = write_env(spec, os.path.join(tmp, "rd_gauss_%d" % rank))
    return spec, root, W.rd_gauss_freqs()


def tl_rms(a, b):
    import numpy as np
    from bellhopcuda_b200 import tl_db
    ta, tb = tl_db(a), tl_db(b)
    m = tb < 100.0
    d = np.abs(ta[m] - tb[m])
    d = np.where(np.isfinite(d), d, 1e3)
    return float(np.sqrt(np.mean(d ** 2)))


# ------------------------------------------------------------- our arm
def time_arm(B, torch, root, freqs, precision, steps, warmup, gpu, flush, tune=None, pipeline=False):
    """Device time per step of the prepared run (tables resident in HBM).
    Serial: each step replays the CUDA graph of trace + influence + scale that
    the first two launches set up, L2 flushed before each step, timed one by
    one. Pipelined (BHCB_FLAG_PIPELINE): the `steps` launches go back to back,
    the trace of each beside the influence of the previous one, timed as a
    whole from the first launch to the last field; every step writes and reads
    its own 655 MB of segment records (more than the 126 MB L2), and L2 is
    flushed once before the first. tune: None to run the autotuner first
    (untimed), else a shape to apply."""
    t = B.Tracer(gpu=gpu, precision=precision, pipeline=pipeline)
    t.setup(root)
    t.set_frequencies(0, freqs)
    t.prepare()
    if tune is None:
        t.tuning = t.autotune(repeats=2)
    else:
        t.set_tuning(tune["trace_block"], tune["influence_ctas_per_sm"], tune["stage_kb"], tune.get("trace_lanes", 32))
        t.tuning = tune
    s = torch.cuda.ExternalStream(t.stream_ptr(), device=gpu)
    if pipeline and tune is None:
        # concurrent trace and influence share each SM's registers: pick the
        # shape by timing pipelined launches (untimed tuning, like autotune)
        best = None
        base = dict(t.tuning)
        for tb, k in ((base["trace_block"], base["influence_ctas_per_sm"]), (32, 6), (32, 5), (64, 6), (32, 4)):
            t.set_tuning(tb, k, base["stage_kb"], base.get("trace_lanes", 32))
            for _ in range(2):
                t.launch()
            t.sync()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(4):
                t.launch()
            e1.record(s)
            t.sync()
            ms = e0.elapsed_time(e1) / 4
            if best is None or ms < best[0]:
                best = (ms, tb, k)
        t.tuning = dict(base, trace_block=best[1], influence_ctas_per_sm=best[2], chosen_by_pipeline=True)
        t.set_tuning(best[1], best[2], base["stage_kb"], base.get("trace_lanes", 32))
    for _ in range(warmup):
        t.launch()
        t.sync()
    times, stats = [], []
    if pipeline:
        with torch.cuda.stream(s):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            t.launch()
        e1.record(s)
        t.sync()
        total = e0.elapsed_time(e1)
        times = [total / steps] * steps
        stats = [t.stats()]
    else:
        for _ in range(steps):
            with torch.cuda.stream(s):
                flush.zero_()          # evict L2 (256 MiB > 126 MB) outside the timed window
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            t.launch()
            e1.record(s)
            t.sync()
            times.append(e0.elapsed_time(e1))
            stats.append(t.stats())
    fields = [t.field(0, i)[0] for i in range(len(freqs))]
    return t, times, stats, fields


def time_c4(B, tmp, rank, runs=3):
    """The 3-D workload (51,984 rays, 36 bearings x 101 depths x 501 ranges,
    Gaussian beams, hexahedral SSP) as one TL run per step in both precisions:
    the run's own trace and influence times (device events), median of
    `runs` runs after one untimed run. Not part of the headline metric."""
    from bellhopcuda_b200 import workloads as W
    files = W.c4_3d(run_type="CB   3")
    root = os.path.join(tmp, "c4_%d" % rank)
    for suffix, text in files.items():
        with open(root + suffix, "w") as f:
            f.write(text)
    out = {"workload": "C4: 3-D Gaussian-beam TL, 361 x 144 rays, 36 x 101 x 501 receivers, 200 Hz"}
    for name, prec in (("fp64", B.PREC_FP64), ("mixed", B.PREC_MIXED)):
        with B.Tracer(precision=prec) as t:
            t.setup3d(root)
            t.run()
            st = []
            for _ in range(runs):
                t.run()
                st.append(t.stats())
        tot = sorted(x["trace_ms"] + x["influence_ms"] for x in st)[len(st) // 2]
        out[name] = {"run_ms": tot, "trace_ms": statistics.median(x["trace_ms"] for x in st),
                     "influence_ms": statistics.median(x["influence_ms"] for x in st),
                     "contributions": int(st[-1]["evals"])}
    out["mixed_speedup"] = out["fp64"]["run_ms"] / out["mixed"]["run_ms"]
    return out


def run_gemm(dims, warmup, launches=20):
    """The surrogate's tcgen05 GEMM (bhcb_nn_gemm) on random bf16 operands:
    C[M][N] = A[M][K] B[N][K]^T + bias with the given epilogue (default bf16
    output), timed with CUDA events over `launches` launches after `warmup`."""
    import torch
    from bellhopcuda_b200 import surrogate as S
    M, N, K = dims[:3]
    epi = dims[3] if len(dims) > 3 else S.EPI_BF16
    ops = S._Ops()
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    Bm = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    out = torch.empty(M, N, device="cuda", dtype=torch.float32 if epi == S.EPI_F32 else torch.bfloat16)
    bias = torch.zeros(N, device="cuda")
    aux = torch.empty(M, N, device="cuda", dtype=torch.bfloat16) if epi in (S.EPI_GELU, S.EPI_DGELU) else None
    kw = {"aux_out": aux} if epi == S.EPI_GELU else ({"aux_in": aux} if epi == S.EPI_DGELU else {})
    if aux is not None:
        aux.zero_()
    for _ in range(max(warmup, 1)):
        ops.gemm(A, Bm, out, epi, bias=bias, **kw)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(launches):
        ops.gemm(A, Bm, out, epi, bias=bias, **kw)
    e1.record()
    torch.cuda.synchronize()
    ops.check()
    ms = e0.elapsed_time(e1) / launches
    print(json.dumps({"gemm": [M, N, K], "epilogue": epi, "ms": ms, "tflops": 2.0 * M * N * K / (ms * 1e-3) / 1e12,
                      "launches": launches}))
    return 0


def time_e2e(B, torch, root, freqs, steps, gpu, tune=None):
    """Same metric through the public C ABI with host buffers: setup reads the
    files, prepare uploads the tables, run, and every field copied back to
    pinned host memory, all inside the timed window."""
    t = B.Tracer(gpu=gpu, precision=B.PREC_MIXED)
    if tune is not None:
        t.set_tuning(tune["trace_block"], tune["influence_ctas_per_sm"], tune["stage_kb"], tune.get("trace_lanes", 32))
    nf = len(freqs)
    t.setup(root)
    t.set_frequencies(0, freqs)
    t.run()
    _, nsz, nrz, nrr = t.field_shape(0)
    host = [torch.empty((nsz, nrz, nrr), dtype=torch.complex64, pin_memory=True) for _ in range(nf)]
    s = torch.cuda.ExternalStream(t.stream_ptr(), device=gpu)
    times = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        t.setup(root)
        t.set_frequencies(0, freqs)
        t.run()
        for i in range(nf):
            arr = host[i].numpy()
            t.field(0, i, out=arr)
        e1.record(s)
        torch.cuda.synchronize(gpu)
        times.append(e0.elapsed_time(e1))
    st = t.stats()
    d2h = nf * nsz * nrz * nrr * 8
    t.close()
    return times, st["h2d_bytes"], d2h


# ------------------------------------------------------- reference CPU arm
def reference_field(spec, freq, tmp, tag):
    """One whole TL field of the workload (all 20001 rays at one frequency)
    by the reference's own bellhopcxx on all host threads; returns the run's
    own 'Run:' time in seconds (bhc::run only, file reading and writing
    excluded) and the process's wall time."""
    import copy
    from bellhopcuda_b200.envfile import write_env
    exe = os.path.join(ROOT, "oracle", "_ref", "bellhopcxx")
    if not os.path.exists(exe):
        raise FileNotFoundError("oracle/_ref/bellhopcxx not built")
    s2 = copy.deepcopy(spec)
    s2.freq = freq
    root = write_env(s2, os.path.join(tmp, "ref_%s" % tag))
    t0 = time.perf_counter()
    out = subprocess.run([exe, "-2", root], capture_output=True, text=True, timeout=1200)
    wall = time.perf_counter() - t0
    mm = re.search(r"Run:\s*([0-9.eE+-]+)\s*ms", out.stdout)
    if out.returncode != 0 or not mm:
        raise RuntimeError("bellhopcxx failed: " + (out.stdout + out.stderr)[-200:])
    return float(mm.group(1)) / 1000.0, wall


def cpu_baseline(spec, freqs, tmp):
    """Bounded sample for the main line: five whole fields (every other
    frequency of the ten), each the full ray fan and receiver grid."""
    idx = list(range(0, len(freqs), 2))
    try:
        runs = [reference_field(spec, freqs[i], tmp, "cb%d" % i)[0] for i in idx]
    except Exception as e:   # noqa: BLE001 - reported, not fatal to the GPU line
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference", "sample": str(e)}
    return {"value": len(idx) / sum(runs), "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "sample": "reference bellhopcxx (unmodified sources, %d host threads): %d whole TL fields of the "
                      "workload (20001 rays, 501x2001 receivers) at %s Hz; value = fields / sum of the "
                      "runs' own Run: times" % (os.cpu_count(), len(idx),
                                                ", ".join("%.1f" % freqs[i] for i in idx)),
            "run_s": runs}


def run_reference_arm(args, rank, world):
    """The reference's CPU implementation on the same workload: each step is
    one whole TL field (the full 20001-ray fan over the 501 x 2001 grid) at
    one of the ten frequencies. The reference's time per field falls with
    frequency (wider beams at low frequency), so the frequencies are taken
    lowest, highest, second lowest, second highest, ...: every even number of
    steps pairs slow and fast fields, and ten steps cover all ten. Measured,
    not extrapolated."""
    if rank != 0:
        return 0
    from bellhopcuda_b200 import workloads as W
    with tempfile.TemporaryDirectory() as tmp:
        spec = W.rd_gauss()
        ladder = W.rd_gauss_freqs()
        n = len(ladder)
        freqs = [ladder[(k // 2) if k % 2 == 0 else n - 1 - k // 2] for k in range(n)]
        try:
            for i in range(max(args.warmup, 0)):
                reference_field(spec, freqs[i % len(freqs)], tmp, "w%d" % i)
            runs, walls = [], []
            for i in range(args.steps):
                r, w = reference_field(spec, freqs[i % len(freqs)], tmp, "s%d" % i)
                runs.append(r)
                walls.append(w)
        except Exception as e:   # noqa: BLE001 - the arm reports why it cannot run
            print(json.dumps({"impl": "reference", "unavailable": str(e)}))
            return 0
        v = args.steps / sum(runs)
        line = {
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(runs) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dict(CONFIG),
            "step": "one whole TL field per step (frequencies in turn: %s)" % ", ".join(
                "%.1f" % freqs[i % len(freqs)] for i in range(args.steps)),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "sample": "%d whole fields of the workload, the reference's Run: time per field"
                                       % args.steps},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s_per_field": statistics.mean(walls),
        }
        print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ main
def run_surrogate(tmp):
    """C5: 100,000 seeded environments traced by the plain FP64 tracer
    (incoherent Gaussian beams), the neural operator trained on 90 % of them
    (40 epochs, tcgen05 GEMMs), the fallback margin calibrated on 5 %, and the
    last 5 % answered by the surrogate with the FP64 trace as fallback at the
    1 dB bound, timed against the plain trace of the same fields."""
    from bellhopcuda_b200 import surrogate as S
    o = S.run_c5(n=100000, epochs=40, threshold_db=1.0, tmpdir=tmp)
    o["train_rms_db"] = o["train_rms_db"][-1]
    o["workload"] = ("C5: 100,000 fields 128 x 256, 64-node SSP = Munk + 8 modes N(0, 2 m/s), depth 1000-5000 m, "
                     "cp 1500-1800, source 10-500 m, 50-500 Hz; incoherent Gaussian beams, launch angles +-89 deg")
    return o


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the 3-D (C4) TL timing")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the C5 surrogate run (100,000 traced fields, training, test split)")
    ap.add_argument("--serial", action="store_true",
                    help="time the steps one at a time (graph replay) instead of pipelined launches")
    ap.add_argument("--gemm", type=int, nargs="+", metavar="M N K [EPI]",
                    help="time the surrogate's tensor-core GEMM (bhcb_nn_gemm) alone and exit")
    ap.add_argument("--rays", type=int, default=0,
                    help="profiling only: trace this many rays of the fan instead of 20001 (the line says so)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling only: the serial mixed run alone (no e2e, FP64 or CPU legs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.gemm:
        return run_gemm(args.gemm, args.warmup)

    import torch
    import bellhopcuda_b200 as B
    from bellhopcuda_b200 import workloads as W

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    comm = RankComm(dist, "cuda", torch.cuda.synchronize)
    barrier, max_over_ranks = comm.barrier, comm.max_over_ranks

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    fp32_peak, fp64_peak = probe_fp_peak(local)
    with tempfile.TemporaryDirectory() as tmp:
        spec, root, freqs = make_env(tmp, rank, args.rays)
        nf = len(freqs)
        if args.profile:
            # profiling driver: the serial mixed run only (influence after the trace)
            shape = {"trace_block": 32, "influence_ctas_per_sm": 8, "stage_kb": 64}   # fixed: no tuning launches
            t, times, stats, _ = time_arm(B, torch, root, freqs, B.PREC_MIXED, args.steps, args.warmup, local,
                                          flush, tune=shape)
            t.close()
            print(json.dumps({"profile": "serial mixed run", "rays": spec.nalpha, "steps": args.steps,
                              "ms_per_step": statistics.mean(times),
                              "trace_ms": statistics.mean(x["trace_ms"] for x in stats),
                              "influence_ms": statistics.mean(x["influence_ms"] for x in stats),
                              "contributions": stats[-1]["evals"], "segments": stats[-1]["segments"]}))
            return 0
        # ---- headline: mixed precision, shared trajectory
        barrier()
        pipe = not args.serial
        with ClockSampler(local) as clk:
            t, times, stats, fields_mixed = time_arm(B, torch, root, freqs, B.PREC_MIXED, args.steps,
                                                     args.warmup, local, flush, pipeline=pipe)
            barrier()
        clocks = clk.summary()
        total_s = max_over_ranks(sum(times) / 1000.0)
        ms_per_step = 1000.0 * total_s / args.steps
        value = aggregate_value(world, nf, args.steps, total_s)
        st = stats[-1]
        tuning = t.tuning
        t.close()
        # ---- the same steps one at a time (graph replay, L2 flushed before each)
        serial = None
        if pipe:
            ts_, times_s, _, _ = time_arm(B, torch, root, freqs, B.PREC_MIXED, max(2, args.steps // 2),
                                          args.warmup, local, flush, tune=tuning, pipeline=False)
            ts_.close()
            ms_s = max_over_ranks(statistics.mean(times_s))
            serial = {"ms_per_step": ms_s, "value": world * nf * 1000.0 / ms_s,
                      "launch": "one step at a time: CUDA graph replay of memsets + trace + influence + scale"}
        fp64 = None
        if not args.no_fp64:
            t64, times64, stats64, fields64 = time_arm(B, torch, root, freqs, B.PREC_FP64,
                                                       max(2, args.steps // 2), 1, local, flush, pipeline=pipe)
            t64.close()
            ms64 = max_over_ranks(statistics.mean(times64))
            errs = [tl_rms(fields_mixed[i], fields64[i]) for i in range(nf)]
            fp64 = {"value": world * nf * 1000.0 / ms64, "ms_per_step": ms64,
                    "mixed_speedup": (world * nf * 1000.0 / ms64) and value / (world * nf * 1000.0 / ms64),
                    "tl_rms_err_db_mixed_vs_fp64_max_over_freqs": max(errs),
                    "trace_ms": stats64[-1]["trace_ms"], "influence_ms": stats64[-1]["influence_ms"]}
        # ---- the kernels' own times inside the timed steps (events in the graph)
        kernels = {"trace_kernel_ms": statistics.mean(x["trace_ms"] for x in stats),
                   "influence_kernel_ms": statistics.mean(x["influence_ms"] for x in stats)}
        # ---- end to end through the C ABI with host buffers
        e2e_times, h2d, d2h = time_e2e(B, torch, root, freqs, max(1, args.steps), local, tune=tuning)
        e2e_s = max_over_ranks(sum(e2e_times) / 1000.0)
        e2e = {"value": world * nf * len(e2e_times) / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h)}
        # ---- roofline of the dominant kernel, on its own launch time
        infl_ms = kernels["influence_kernel_ms"]
        trace_ms = kernels["trace_kernel_ms"]
        dom = "influence_kernel" if infl_ms >= trace_ms else "trace_kernel"
        if dom == "influence_kernel":
            work = F_INFL * ORACLE_EVALS_ALL_FREQS
            dur = infl_ms
        else:
            work = F_STEP * ORACLE_STEPS_PER_TRACE
            dur = trace_ms
        achieved = work / (dur * 1e-3) / 1e12
        roofline = {"bound": "fp32", "kernel": dom, "achieved": achieved, "peak": fp32_peak,
                    "unit": "TFLOP/s", "frac": achieved / fp32_peak if fp32_peak else None,
                    "traffic": INFLUENCE_DRAM_BYTES if dom == "influence_kernel" else None,
                    "peak_source": "FP32 FMA probe (bench_probe.cu) measured in this run "
                                   "(MEASURED_PEAKS.json has no FP32 figure)",
                    "work": "%s x %d oracle units per launch" % (
                        ("F_infl=%g flop" % F_INFL, ORACLE_EVALS_ALL_FREQS) if dom == "influence_kernel"
                        else ("F_step=%g flop" % F_STEP, ORACLE_STEPS_PER_TRACE)),
                    "kernel_ms": dur,
                    "other_kernel": {"trace_kernel_ms": trace_ms, "trace_achieved_tflops":
                                     F_STEP * ORACLE_STEPS_PER_TRACE / (trace_ms * 1e-3) / 1e12,
                                     "influence_kernel_ms": infl_ms},
                    "fp64_peak_tflops": fp64_peak}
        c4 = None if args.no_c4 else time_c4(B, tmp, rank)
        sur = None
        if rank == 0 and world == 1 and not args.no_surrogate:
            sur = run_surrogate(tmp)
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(spec, freqs, tmp)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 ray trace / f32 beam-receiver contributions", "data": "synthetic",
        "config": dict(CONFIG),
        "detail": {"frequencies_share_one_trajectory": True, "fields_per_step": nf, "rays": int(st["rays"]),
                   "steps_traced": int(st["steps"]), "contributions": int(st["evals"]),
                   "l2": ("each step writes and reads its own 655 MB of segment records (> 126 MB L2); L2 flushed "
                          "(256 MiB write) once before the timed steps") if pipe else
                         "flushed (256 MiB write) before every timed step",
                   "parallelism": "replicas per GPU (one environment per rank)",
                   "launch_shape": {"trace_block": tuning["trace_block"],
                                    "influence_ctas_per_sm": tuning["influence_ctas_per_sm"],
                                    "stage_kb": tuning["stage_kb"],
                                    "trace_lanes": tuning.get("trace_lanes", 32),
                                    "chosen_by": "bhcb_autotune, then timed pipelined launches of five shapes "
                                                 "(before the warm-up, untimed)" if tuning.get("chosen_by_pipeline")
                                    else "bhcb_autotune before the warm-up (untimed)"}},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": 3 * args.steps, "fp64_trace": fp64, "kernels": kernels, "c4_3d_tl": c4,
        "surrogate": sur,
        "launch": ("pipelined launches (BHCB_FLAG_PIPELINE): the trace of step k+1 beside the influence of step k "
                   "on two streams, double-buffered segment records and accumulators; steps timed as a whole")
                  if pipe else "CUDA graph replay of memsets + trace + influence + scale per step",
        "serial_steps": serial,
    }
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
