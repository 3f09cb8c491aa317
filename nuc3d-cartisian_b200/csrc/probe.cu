// Pipe-throughput probe: the measured FP64 (or FP32) FMA rate of this GPU,
// used as the roofline denominator of the stencil kernels (which run on the
// FMA pipes, not on tensor cores).  Every thread runs 8 independent FMA chains
// so the pipe, not the dependency latency, limits the rate.
#include <cuda_runtime.h>

#include "nuc3d_b200.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_probe(T *sink, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = T(threadIdx.x + i);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = fma(x[i], a, b);
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == T(-1.2345)) sink[0] = s;  // keeps the chains alive
}

template <typename T>
int probe(double *tflops) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NUC3D_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return NUC3D_ERR_CUDA;
    T *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(T)) != cudaSuccess) return NUC3D_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256, iters = 16384;
    k_fma_probe<T><<<blocks, threads>>>(sink, 256, T(0.999999), T(1e-7));  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        k_fma_probe<T><<<blocks, threads>>>(sink, iters, T(0.999999), T(1e-7));
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return NUC3D_ERR_CUDA;
    double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return NUC3D_OK;
}

}  // namespace

extern "C" NUC3D_API int nuc3d_probe_peak(int precision, double *tflops) {
    if (!tflops) return NUC3D_ERR_INVALID;
    return precision == NUC3D_MIXED ? probe<float>(tflops) : probe<double>(tflops);
}
