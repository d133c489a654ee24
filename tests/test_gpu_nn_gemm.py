"""The surrogate's tensor-core GEMM (tcgen05 / TMEM, bhcb_nn_gemm) against a
torch FP32 reference of the same op on the same bf16 inputs: every epilogue,
tile-aligned and ragged shapes. Tolerance: FP32 accumulation in a different
order, plus one bf16 rounding of the output for the bf16 epilogues."""
import ctypes as C

import numpy as np
import pytest

import bellhopcuda_b200 as B

pytestmark = pytest.mark.gpu


def gemm(A, Bm, out, epi, bias=None, aux_in=None, aux_out=None):
    import torch
    lib = B.load_library()
    M, K = A.shape
    N = Bm.shape[0]
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    rc = lib.bhcb_nn_gemm(p(A), p(Bm), p(out), M, N, K, epi, p(bias), p(aux_in), p(aux_out),
                          C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    err = C.c_int32()
    assert lib.bhcb_nn_status(C.byref(err), 1) == 0
    assert err.value == 0


def gelu(x):
    import torch
    return torch.nn.functional.gelu(x, approximate="tanh")


SHAPES = [(128, 128, 64), (256, 384, 512), (300, 200, 136), (4096, 1024, 512), (64, 32768, 512), (512, 512, 4096)]


@pytest.mark.parametrize("M,N,K", SHAPES)
def test_gemm_f32_bias(M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    Bm = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    out = torch.full((M, N), float("nan"), device="cuda")
    gemm(A, Bm, out, 0, bias=bias)
    ref = A.float() @ Bm.float().T + bias
    torch.testing.assert_close(out, ref, rtol=1e-4, atol=1e-3 * K ** 0.5)


@pytest.mark.parametrize("M,N,K", SHAPES[:4])
def test_gemm_bf16_gelu_and_dgelu(M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(11 + M + N + K)
    A = (torch.randn(M, K, device="cuda", generator=g) / K ** 0.5).bfloat16()
    Bm = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    out = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    pre = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    gemm(A, Bm, out, 2, bias=bias, aux_out=pre)
    ref_pre = A.float() @ Bm.float().T + bias
    torch.testing.assert_close(pre.float(), ref_pre, rtol=1e-2, atol=2e-2)
    torch.testing.assert_close(out.float(), gelu(ref_pre), rtol=1e-2, atol=2e-2)
    # backward through GELU: acc * gelu'(pre)
    dY = (torch.randn(M, K, device="cuda", generator=g) / K ** 0.5).bfloat16()
    out2 = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    gemm(dY, Bm, out2, 3, aux_in=pre)
    x = pre.float().requires_grad_(True)
    gelu(x).backward(torch.ones_like(x))
    ref2 = (dY.float() @ Bm.float().T) * x.grad
    torch.testing.assert_close(out2.float(), ref2, rtol=2e-2, atol=3e-2)
