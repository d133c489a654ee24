// Element-wise and reduction kernels of the TL surrogate's training and
// inference (the GEMMs are in nn_gemm.cu): field -> TL(dB) conversion, bf16
// transpose, masked MSE loss and its gradient, bias gradients (column sums),
// Adam updates of FP32 master weights with bf16 (and transposed bf16) copies,
// FP32 -> bf16 conversion and the per-field RMS error used by the fallback.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bhcb.h"

namespace bhcb {
namespace {

// TL = -20 log10 |p| (the reference's definition), clamped to [lo, hi]
__global__ void tl_db_kernel(const float2 *__restrict__ p, float *__restrict__ tl, long long n, float lo, float hi)
{
    for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float2 v = p[i];
        const float a = sqrtf(v.x * v.x + v.y * v.y);
        float t = a > 0.0f ? -20.0f * log10f(a) : hi;
        tl[i] = fminf(fmaxf(t, lo), hi);
    }
}

// out[c][r] = in[r][c], 32 x 32 tiles through shared memory
__global__ void transpose_bf16_kernel(const __nv_bfloat16 *__restrict__ in, __nv_bfloat16 *__restrict__ out, int R,
                                      int Cc)
{
    __shared__ __nv_bfloat16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for(int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if(r < R && c < Cc) t[k][threadIdx.x] = in[(size_t)r * Cc + c];
    }
    __syncthreads();
    for(int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if(c < Cc && r < R) out[(size_t)c * R + r] = t[threadIdx.x][k];
    }
}

// loss = sum over valid (pred - target)^2 (accumulated in FP64), grad = scale * 2 (pred - target)
__global__ void mse_kernel(const float *__restrict__ pred, const float *__restrict__ target, long long n, float scale,
                           __nv_bfloat16 *__restrict__ grad, double *__restrict__ loss)
{
    double acc = 0.0;
    for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = pred[i] - target[i];
        acc += (double)d * d;
        grad[i] = __float2bfloat16_rn(scale * 2.0f * d);
    }
    for(int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// per-row RMS of (pred - target) over ncol columns (one block per row)
__global__ void row_rms_kernel(const float *__restrict__ pred, const float *__restrict__ target, int ncol,
                               float *__restrict__ rms)
{
    __shared__ double part[32];
    const size_t base = (size_t)blockIdx.x * ncol;
    double acc = 0.0;
    for(int j = threadIdx.x; j < ncol; j += blockDim.x) {
        const double d = (double)pred[base + j] - (double)target[base + j];
        acc += d * d;
    }
    for(int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if(threadIdx.x == 0) {
        double s = 0.0;
        for(int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
        rms[blockIdx.x] = (float)sqrt(s / ncol);
    }
}

// db[n] = sum_m dy[m][n]
__global__ void colsum_kernel(const __nv_bfloat16 *__restrict__ dy, int M, int N, float *__restrict__ db)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if(n >= N) return;
    float s = 0.0f;
    for(int m = 0; m < M; ++m) s += __bfloat162float(dy[(size_t)m * N + n]);
    db[n] = s;
}

// Adam (bias-corrected) on FP32 master weights; writes the bf16 copy [R][C]
// and, when wt is not NULL, its transpose [C][R]
__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, long long n, int R, int Cc, float lr, float b1, float b2, float eps,
                            float c1, float c2, float wd, __nv_bfloat16 *__restrict__ wb, __nv_bfloat16 *__restrict__ wt)
{
    for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float wi = w[i] * (1.0f - lr * wd);
        wi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        const __nv_bfloat16 h = __float2bfloat16_rn(wi);
        if(wb) wb[i] = h;
        if(wt) {
            const int r = (int)(i / Cc), c = (int)(i % Cc);
            wt[(size_t)c * R + r] = h;
        }
    }
}

__global__ void f32_to_bf16_kernel(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, long long n)
{
    for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

int grid_for(long long n, int block)
{
    long long g = (n + block - 1) / block;
    if(g > 148LL * 32) g = 148LL * 32;
    return (int)(g < 1 ? 1 : g);
}

} // namespace
} // namespace bhcb

using namespace bhcb;

#define NN_LAUNCH_OK (cudaGetLastError() == cudaSuccess ? BHCB_OK : BHCB_ERR_CUDA)

extern "C" int bhcb_nn_tl_db(const void *field, float *tl, int64_t n, float lo, float hi, void *stream)
{
    if(!field || !tl || n < 0) return BHCB_ERR_ARG;
    tl_db_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>((const float2 *)field, tl, n, lo, hi);
    return NN_LAUNCH_OK;
}

extern "C" int bhcb_nn_transpose(const void *in, void *out, int32_t rows, int32_t cols, void *stream)
{
    if(!in || !out || rows <= 0 || cols <= 0) return BHCB_ERR_ARG;
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    transpose_bf16_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)in,
                                                                          (__nv_bfloat16 *)out, rows, cols);
    return NN_LAUNCH_OK;
}

extern "C" int bhcb_nn_mse(const float *pred, const float *target, int64_t n, float scale, void *grad,
                           double *loss_dev, void *stream)
{
    if(!pred || !target || !grad || !loss_dev || n <= 0) return BHCB_ERR_ARG;
    mse_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(pred, target, n, scale, (__nv_bfloat16 *)grad,
                                                                   loss_dev);
    return NN_LAUNCH_OK;
}

extern "C" int bhcb_nn_row_rms(const float *pred, const float *target, int32_t rows, int32_t cols, float *rms,
                               void *stream)
{
    if(!pred || !target || !rms || rows <= 0 || cols <= 0) return BHCB_ERR_ARG;
    row_rms_kernel<<<rows, 256, 0, (cudaStream_t)stream>>>(pred, target, cols, rms);
    return NN_LAUNCH_OK;
}

extern "C" int bhcb_nn_colsum(const void *dy, int32_t M, int32_t N, float *db, void *stream)
{
    if(!dy || !db || M <= 0 || N <= 0) return BHCB_ERR_ARG;
    colsum_kernel<<<(N + 127) / 128, 128, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)dy, M, N, db);
    return NN_LAUNCH_OK;
}

extern "C" int bhcb_nn_adam(float *w, const float *g, float *m, float *v, int32_t rows, int32_t cols, float lr,
                            float beta1, float beta2, float eps, int32_t step, float weight_decay, void *w_bf16,
                            void *wt_bf16, void *stream)
{
    if(!w || !g || !m || !v || rows <= 0 || cols <= 0 || step <= 0) return BHCB_ERR_ARG;
    const long long n = (long long)rows * cols;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, rows, cols, lr, beta1, beta2, eps,
                                                                    c1, c2, weight_decay, (__nv_bfloat16 *)w_bf16,
                                                                    (__nv_bfloat16 *)wt_bf16);
    return NN_LAUNCH_OK;
}

extern "C" int bhcb_nn_to_bf16(const float *x, void *y, int64_t n, void *stream)
{
    if(!x || !y || n <= 0) return BHCB_ERR_ARG;
    f32_to_bf16_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(x, (__nv_bfloat16 *)y, n);
    return NN_LAUNCH_OK;
}

namespace bhcb {
namespace {
__global__ void affine_kernel(float *__restrict__ x, long long n, float a, float b)
{
    for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = a * x[i] + b;
}
} // namespace
} // namespace bhcb

extern "C" int bhcb_nn_affine(float *x, int64_t n, float a, float b, void *stream)
{
    if(!x || n <= 0) return BHCB_ERR_ARG;
    affine_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(x, n, a, b);
    return NN_LAUNCH_OK;
}
