// BF16 GEMM on the 5th-generation tensor cores (sm_100a) for the TL surrogate.
//
//   C[M, N] = epilogue(A[M, K] * B[N, K]^T)      A, B row-major bf16 (K-major)
//
// One CTA per 128 x 128 output tile, 128 threads, three CTAs per SM (64 KiB of
// shared memory and 128 tensor-memory columns each), so that one CTA's
// epilogue overlaps the other CTAs' main loops:
//   warp 0 lane 0  TMA producer: 128 x 64 bf16 tiles of A and B per stage into
//                  a 2-stage ring (128-byte swizzle), completion on the stage's
//                  "full" mbarrier (transaction bytes);
//   warp 1 lane 0  MMA issuer: four tcgen05.mma.kind::f16 (M 128, N 128, K 16)
//                  per stage into a 128-column FP32 accumulator in tensor memory;
//                  tcgen05.commit on the stage's "empty" mbarrier frees the slot,
//                  a final commit signals the epilogue;
//   all 4 warps    epilogue: tcgen05.ld of their 32 accumulator lanes (rows),
//                  staged through the (then idle) stage ring so that each store
//                  instruction writes 32 consecutive columns of one row; bias /
//                  GELU / GELU' / conversion on the way out.
// Every mbarrier wait is bounded; a wait that runs out sets the error word,
// the CTA skips its stores, frees its tensor memory and returns. No TMA load
// uses cluster multicast.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/bhcb.h"

namespace bhcb {
namespace {

constexpr int BM = 128, BN = 128, BK = 64, STAGES = 2;
constexpr int GROUP_M = 16;  // tile rows per L2 group of the launch order (8192^3: 1094 -> 1143 TFLOP/s)
constexpr int TILE_A = BM * BK * 2;   // 16 KiB
constexpr int TILE_B = BN * BK * 2;
constexpr int SMEM_BYTES = STAGES * (TILE_A + TILE_B) + 1024 + 256;
constexpr unsigned WAIT_LIMIT = 1u << 24;
// instruction descriptor: FP32 accumulate (bit 4), A and B BF16 (bits 7, 10),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17)
    | ((uint32_t)(BM >> 4) << 24);

__device__ int g_nn_error;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// false when the wait ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    for(unsigned i = 0; i < WAIT_LIMIT; ++i)
        if(mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
                 : "memory");
}
// shared-memory matrix descriptor of a K-major tile with 128-byte rows in the
// 128-byte swizzle (8-row groups 1024 bytes apart)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused when swizzled)
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset
    d |= (uint64_t)1 << 46;             // descriptor version
    d |= (uint64_t)2 << 61;             // 128-byte swizzle
    return d;
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
                 "l"(a), "l"(b), "r"(IDESC), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                   "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
                   "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for(int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// GELU, tanh form, and its derivative
__device__ __forceinline__ float gelu_f(float x)
{
    const float k = 0.7978845608028654f, c = 0.044715f;
    return 0.5f * x * (1.0f + tanhf(k * (x + c * x * x * x)));
}
__device__ __forceinline__ float dgelu_f(float x)
{
    const float k = 0.7978845608028654f, c = 0.044715f;
    const float u = k * (x + c * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k * (1.0f + 3.0f * c * x * x);
}

template<int EPI>
__global__ void __launch_bounds__(128, 3) gemm_tc_kernel(const __grid_constant__ CUtensorMap tmA,
                                                         const __grid_constant__ CUtensorMap tmB, int M, int N,
                                                         int K, void *C, const float *__restrict__ bias,
                                                         const __nv_bfloat16 *__restrict__ aux_in,
                                                         __nv_bfloat16 *aux_out)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t *sA = smem;
    uint8_t *sB = smem + STAGES * TILE_A;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * (TILE_A + TILE_B));
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    __shared__ int s_fail;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // Tile order: the launch order walks groups of GROUP_M tile rows, a column
    // of GROUP_M tiles at a time, so the CTAs resident together share GROUP_M
    // panels of A and a band of B panels that fit in L2 (instead of every B
    // panel against a few A rows).
    int m_t, n_t;
    {
        const int num_m = (int)gridDim.y, num_n = (int)gridDim.x;
        const int t = (int)blockIdx.y * num_n + (int)blockIdx.x;
        const int per_group = GROUP_M * num_n;
        const int first_m = (t / per_group) * GROUP_M;
        const int gsz = min(num_m - first_m, GROUP_M);
        const int r = t - (t / per_group) * per_group;
        m_t = first_m + r % gsz;
        n_t = r / gsz;
    }
    const int m0 = m_t * BM, n0 = n_t * BN;
    const int nk = (K + BK - 1) / BK;
    if(threadIdx.x == 0) {
        s_fail = 0;
        for(int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if(warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if(warp == 0 && lane == 0) {
        // ---- producer
        for(int kb = 0; kb < nk; ++kb) {
            const int s = kb % STAGES, round = kb / STAGES;
            if(kb >= STAGES && !mbar_wait(&empty[s], (round - 1) & 1)) {
                s_fail = 1;
                break;
            }
            mbar_expect_tx(&full[s], TILE_A + TILE_B);
            tma_load_2d(sA + s * TILE_A, &tmA, &full[s], kb * BK, m0);
            tma_load_2d(sB + s * TILE_B, &tmB, &full[s], kb * BK, n0);
        }
    } else if(warp == 1 && lane == 0) {
        // ---- MMA issuer
        bool ok = true;
        for(int kb = 0; kb < nk; ++kb) {
            const int s = kb % STAGES, round = kb / STAGES;
            if(!mbar_wait(&full[s], round & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sA + s * TILE_A), b0 = smem_u32(sB + s * TILE_B);
#pragma unroll
            for(int k = 0; k < BK / 16; ++k)
                umma_bf16(tmem, sw128_desc(a0 + k * 32), sw128_desc(b0 + k * 32), (kb > 0 || k > 0) ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        if(!ok) s_fail = 1;
        umma_commit(done);   // arrives once every MMA issued so far has completed
    }
    // ---- epilogue
    __syncwarp();
    const bool ready = mbar_wait(done, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    const bool good = ready && s_fail == 0;
    if(!good && threadIdx.x == 0) atomicExch(&g_nn_error, 1);
    if(good) {
        // every MMA has completed, so the stage ring is free: each warp stages
        // its 32 rows x 32 columns through shared memory and stores them row by
        // row, one coalesced 32-column segment per instruction
        float *stage = reinterpret_cast<float *>(smem) + warp * (32 * 33);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // after the ring's async-proxy use
#pragma unroll 1
        for(int c = 0; c < BN / 32; ++c) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32), v);
#pragma unroll
            for(int j = 0; j < 32; ++j) stage[lane * 33 + j] = v[j];
            __syncwarp();
            const int col = n0 + c * 32 + lane;
            const bool colok = col < N;
            const float bcol = (bias && colok) ? bias[col] : 0.0f;
#pragma unroll 4
            for(int rr = 0; rr < 32; ++rr) {
                const int row = m0 + warp * 32 + rr;
                if(row >= M) break;
                if(!colok) continue;
                const float acc = stage[rr * 33 + lane];
                const size_t idx = (size_t)row * N + col;
                if(EPI == BHCB_NN_EPI_F32) {
                    reinterpret_cast<float *>(C)[idx] = acc + bcol;
                } else if(EPI == BHCB_NN_EPI_BF16) {
                    reinterpret_cast<__nv_bfloat16 *>(C)[idx] = __float2bfloat16_rn(acc + bcol);
                } else if(EPI == BHCB_NN_EPI_BF16_GELU) {
                    const float pre = acc + bcol;
                    if(aux_out) aux_out[idx] = __float2bfloat16_rn(pre);
                    reinterpret_cast<__nv_bfloat16 *>(C)[idx] = __float2bfloat16_rn(gelu_f(pre));
                } else {   // BHCB_NN_EPI_BF16_DGELU
                    reinterpret_cast<__nv_bfloat16 *>(C)[idx]
                        = __float2bfloat16_rn(acc * dgelu_f(__bfloat162float(aux_in[idx])));
                }
            }
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if(warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if(!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess
           && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// rows x K row-major bf16, boxes of 64 columns x box_rows rows, 128-byte swizzle,
// out-of-range elements read as zero
bool make_map(CUtensorMap *map, const void *ptr, int rows, int K, int box_rows)
{
    EncodeTiledFn enc = encode_fn();
    if(!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template<int EPI> void set_smem_once()
{
    static bool done = false;
    if(!done) {
        cudaFuncSetAttribute(gemm_tc_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
        done = true;
    }
}

} // namespace
} // namespace bhcb

using namespace bhcb;

extern "C" int bhcb_nn_gemm(const void *A, const void *B, void *C, int32_t M, int32_t N, int32_t K, int32_t epi,
                            const float *bias, const void *aux_in, void *aux_out, void *stream)
{
    if(!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return BHCB_ERR_ARG;
    // TMA: 16-byte aligned bases and row strides (K a multiple of 8 bf16)
    if((K % 8) != 0 || (reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15))
        return BHCB_ERR_ARG;
    if(epi == BHCB_NN_EPI_BF16_DGELU && !aux_in) return BHCB_ERR_ARG;
    CUtensorMap ma, mb;
    if(!make_map(&ma, A, M, K, BM) || !make_map(&mb, B, N, K, BN)) return BHCB_ERR_CUDA;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    cudaStream_t st = (cudaStream_t)stream;
    const __nv_bfloat16 *ai = reinterpret_cast<const __nv_bfloat16 *>(aux_in);
    __nv_bfloat16 *ao = reinterpret_cast<__nv_bfloat16 *>(aux_out);
    switch(epi) {
    case BHCB_NN_EPI_F32:
        set_smem_once<BHCB_NN_EPI_F32>();
        gemm_tc_kernel<BHCB_NN_EPI_F32><<<grid, 128, SMEM_BYTES, st>>>(ma, mb, M, N, K, C, bias, ai, ao);
        break;
    case BHCB_NN_EPI_BF16:
        set_smem_once<BHCB_NN_EPI_BF16>();
        gemm_tc_kernel<BHCB_NN_EPI_BF16><<<grid, 128, SMEM_BYTES, st>>>(ma, mb, M, N, K, C, bias, ai, ao);
        break;
    case BHCB_NN_EPI_BF16_GELU:
        set_smem_once<BHCB_NN_EPI_BF16_GELU>();
        gemm_tc_kernel<BHCB_NN_EPI_BF16_GELU><<<grid, 128, SMEM_BYTES, st>>>(ma, mb, M, N, K, C, bias, ai, ao);
        break;
    case BHCB_NN_EPI_BF16_DGELU:
        set_smem_once<BHCB_NN_EPI_BF16_DGELU>();
        gemm_tc_kernel<BHCB_NN_EPI_BF16_DGELU><<<grid, 128, SMEM_BYTES, st>>>(ma, mb, M, N, K, C, bias, ai, ao);
        break;
    default: return BHCB_ERR_ARG;
    }
    return cudaGetLastError() == cudaSuccess ? BHCB_OK : BHCB_ERR_CUDA;
}

extern "C" int bhcb_nn_status(int32_t *error, int32_t clear)
{
    int v = 0;
    if(cudaMemcpyFromSymbol(&v, g_nn_error, sizeof v) != cudaSuccess) return BHCB_ERR_CUDA;
    if(error) *error = v;
    if(clear) {
        int z = 0;
        if(cudaMemcpyToSymbol(g_nn_error, &z, sizeof z) != cudaSuccess) return BHCB_ERR_CUDA;
    }
    return BHCB_OK;
}
