// Floating-point pipe peak probe used by bench.py (not part of the library):
// the roofline denominator for the tracer's kernels, which are bound by the
// FP32/FP64 pipes rather than by HBM or the tensor cores. Each thread runs
// independent FMA chains; every SM gets many resident warps so the pipes, not
// latency, set the rate. Built by __graft_entry__.build() into bench_probe.so.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

template<typename T, int CHAINS> __global__ void fma_chains(T *out, int iters, T a, T b)
{
    T x[CHAINS];
#pragma unroll
    for(int c = 0; c < CHAINS; ++c) x[c] = (T)(threadIdx.x + c);
    for(int i = 0; i < iters; ++i) {
#pragma unroll
        for(int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for(int c = 0; c < CHAINS; ++c) s += x[c];
    if(s == (T)-1) out[0] = s;   // keeps the chains live
}

template<typename T> double run_probe(int sms)
{
    constexpr int CHAINS = 8;
    T *out = nullptr;
    if(cudaMalloc(&out, sizeof(T)) != cudaSuccess) return 0.0;
    int blocks = sms * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_chains<T, CHAINS><<<blocks, threads>>>(out, 64, (T)0.999, (T)0.001);
    float best = 1e30f;
    for(int r = 0; r < 3; ++r) {
        cudaEventRecord(e0);
        fma_chains<T, CHAINS><<<blocks, threads>>>(out, iters, (T)0.999, (T)0.001);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if(ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    double flops = 2.0 * CHAINS * (double)iters * blocks * threads;
    return flops / (best * 1e-3) / 1e12;
}

} // namespace

// returns 0 on success, 3 (a CUDA error) otherwise
extern "C" int bench_probe_fp_peak(int32_t gpu_index, double *fp32_tflops, double *fp64_tflops)
{
    if(cudaSetDevice(gpu_index) != cudaSuccess) return 3;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, gpu_index);
    if(fp32_tflops) *fp32_tflops = run_probe<float>(sms);
    if(fp64_tflops) *fp64_tflops = run_probe<double>(sms);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
