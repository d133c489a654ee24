"""Times the surrogate's tensor-core GEMM (bhcb_nn_gemm) with CUDA events.

    python -m bellhopcuda_b200.nn_bench M N K [EPI [REPS]]

A [M][K] and B [N][K] are random bf16, EPI is one of the BHCB_NN_EPI_*
values (0 FP32 out, 1 bf16, 2 bf16 + GELU, 3 bf16 + GELU'); prints one JSON
line with the time per launch (after three warm-up launches), TFLOP/s and the
output bandwidth.
"""
from __future__ import annotations

import ctypes as C
import json
import sys


def main(argv=None):
    import torch
    from . import load_library
    args = sys.argv[1:] if argv is None else argv
    M, N, K = (int(v) for v in args[:3])
    epi = int(args[3]) if len(args) > 3 else 0
    reps = int(args[4]) if len(args) > 4 else 20
    lib = load_library()
    A = torch.randn(M, K, device="cuda").bfloat16()
    Bm = torch.randn(N, K, device="cuda").bfloat16()
    out = torch.empty(M, N, device="cuda", dtype=torch.float32 if epi == 0 else torch.bfloat16)
    aux = torch.zeros(M, N, device="cuda", dtype=torch.bfloat16) if epi == 3 else None
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run():
        rc = lib.bhcb_nn_gemm(p(A), p(Bm), p(out), M, N, K, epi, None, p(aux), None, s)
        if rc != 0:
            raise RuntimeError("bhcb_nn_gemm returned %d" % rc)

    for _ in range(3):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    res = dict(M=M, N=N, K=K, epi=epi, ms=ms, tflops=2.0 * M * N * K / ms / 1e9,
               out_gbs=out.numel() * out.element_size() / ms / 1e6)
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
