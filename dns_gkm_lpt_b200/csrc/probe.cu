// FMA throughput probe: the FP64 / FP32 vector peaks that bound the sweep
// kernels (the driver-measured peaks cover HBM copies and bf16 tensor GEMMs
// only).  Independent FMA chains per thread, grid of 8 CTAs per SM, timed with
// CUDA events after one warm-up launch.
#include "gkm_internal.h"

namespace gkm {
namespace {

template <class T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T* out, T a, T b, int iters)
{
    T x[8];
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = T(threadIdx.x) * T(1e-7) + T(c);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < 8; c++) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) s += x[c];
    if (s == T(-12345)) out[0] = s;   // keeps the chains live
}

template <class T>
cudaError_t time_probe(double* tflops)
{
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    T* out = nullptr;
    e = cudaMalloc(&out, sizeof(T));
    if (e != cudaSuccess) return e;
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_probe_kernel<T><<<blocks, threads>>>(out, T(0.999999), T(1e-7), iters);
    cudaEventRecord(e0);
    fma_probe_kernel<T><<<blocks, threads>>>(out, T(0.999999), T(1e-7), iters);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return e;
    const double flops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return cudaGetLastError();
}

}  // namespace

cudaError_t probe_fma_peak(double* fp64_tflops, double* fp32_tflops)
{
    cudaError_t e = time_probe<double>(fp64_tflops);
    if (e == cudaSuccess) e = time_probe<float>(fp32_tflops);
    return e;
}

}  // namespace gkm
