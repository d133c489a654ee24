"""Build recipe for the native library libbhcb.so (sm_100a).

Compiles the CUDA kernels and the C++ host runtime with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and links them in-tree next to this
file, so the library travels with the repository checkout.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libbhcb.so")
BUILD = os.path.join(ROOT, "_build")

CU_SOURCES = ["kernels2d.cu", "influence_mixed.cu", "arrivals.cu", "kernels3d.cu", "api.cu", "api3d.cu",
              "noalloc.cu", "nn_gemm.cu", "nn_ops.cu", "influence_x.cu", "influence3d_x.cu", "nx2d.cu"]
CPP_SOURCES = ["host/ldi.cpp", "host/env2d.cpp", "host/envdesc.cpp", "host/bhc_cxx.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# FP64 ray tracers (2-D, 3-D, Nx2D, the ray-centred / Cerveny / SGB prologues,
# the allocation-free fused kernel) and the FP64 influence / arrival gathers:
# products and sums rounded separately, as the reference's x86 host build
# computes them. Step-size reductions, boundary snaps and arrival merges are
# decided at tolerance edges, so a contracted multiply-add changes step counts
# and arrival counts of a few rays. The FP32 influence kernel keeps contraction.
NO_FMAD = ("kernels2d.cu", "kernels3d.cu", "nx2d.cu", "influence_x.cu", "influence3d_x.cu", "noalloc.cu",
           "arrivals.cu")
EXTRA = {src: ["-fmad=false"] for src in NO_FMAD}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _deps():
    out = []
    for d, _, files in os.walk(CSRC):
        out += [os.path.join(d, f) for f in files if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    out.append(os.path.join(ROOT, "include", "bhcb.h"))
    return out


def build(verbose: bool = False, force: bool = False, ptxas_v: bool = False) -> str:
    """Compile libbhcb.so if any source is newer than it; returns its path."""
    if not force and not _stale(LIB, _deps()):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    objs, cmds = [], []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
    for src in CU_SOURCES:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        cmd = [cc, *ARCH, "-lineinfo", *common, "--expt-relaxed-constexpr", *EXTRA.get(src, []), "-c",
               os.path.join(CSRC, src), "-o", obj]
        if ptxas_v:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        cmds.append([cc, *common, "-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # translation units compile independently: run them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda c: _run(c, verbose), cmds))
    tmp = LIB + ".tmp"
    _run([cc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], verbose)
    os.replace(tmp, LIB)
    return LIB


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]))
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_v="--ptxas-v" in sys.argv))
