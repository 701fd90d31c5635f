// Measured FP64 CUDA-core rate of this GPU: the denominator of the
// factorisation's and substitution's roofline fractions (the pool's
// measured peaks cover copy bandwidth and bf16 tensor throughput only).
// Every thread runs eight independent chains of dependent DFMAs, enough
// warps are resident to cover the DFMA latency, and the device time of one
// launch is taken with CUDA events.
#include <cuda_runtime.h>

#include "common.hpp"
#include "germaine_gpu.h"
#include "kernels.cuh"

namespace gm {

constexpr int PK_ITERS = 2048;
constexpr int PK_CHAINS = 8;

__global__ void __launch_bounds__(256) k_dfma_peak(double seed, double *sink) {
    double a[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) a[c] = seed + threadIdx.x * 1e-9 + c;
    const double m = 1.0 - 1e-12, b = 1e-13;
#pragma unroll 4
    for (int i = 0; i < PK_ITERS; ++i) {
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) a[c] = fma(a[c], m, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += a[c];
    if (s == 12345.678) *sink = s;   // keeps the chains live; never true
}

}  // namespace gm

extern "C" int gm_peak_fp64(int device, double *tflops) {
    if (!tflops) return gm::fail(GM_ERROR_INVALID, "gm_peak_fp64: null output");
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_peak_fp64: bad device");
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_peak_fp64: properties");
    double *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return gm::fail(GM_ERROR_OUT_OF_MEMORY, "gm_peak_fp64: allocation");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = prop.multiProcessorCount * 8;
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {   // the first launches warm the clocks up
        cudaEventRecord(e0, 0);
        gm::k_dfma_peak<<<blocks, 256>>>(1.0, sink);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep >= 2 && ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_peak_fp64: %s", cudaGetErrorString(err));
    const double flops = 2.0 * gm::PK_ITERS * gm::PK_CHAINS * 256.0 * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return GM_OK;
}
