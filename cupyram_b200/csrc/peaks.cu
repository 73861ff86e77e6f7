// peaks.cu - FP64 / FP32 FMA throughput of the device (the ALU roofline of
// the march, whose HBM roofline is the measured copy bandwidth).
//
// Every thread runs kChains independent FMA recurrences a = a * b + c for
// `iters` iterations; b and c are kernel arguments, so nothing folds, and the
// chains' sum is stored once per thread so that nothing is dead.  The grid is
// 8 CTAs of 256 threads per SM.  2 flops per FMA.
#include <cuda_runtime.h>

#include "../../include/cupyram_b200_peaks.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;
constexpr int kBlocksPerSM = 8;

template <typename T>
__global__ void __launch_bounds__(kThreads) fma_chains(T* out, int iters, T b, T c) {
    T a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
#pragma unroll 4
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    out[(size_t)blockIdx.x * kThreads + threadIdx.x] = s;
}

template <typename T>
int run(int iters, double* tflops, double* ms) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CR_PEAKS_ECUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return CR_PEAKS_ECUDA;
    const int blocks = sms * kBlocksPerSM;
    T* out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * (size_t)blocks * kThreads) != cudaSuccess) return CR_PEAKS_ECUDA;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    // b < 1 and c small keep every chain finite for any iteration count
    const T b = (T)0.9999999, c = (T)1e-7;
    if (ce == cudaSuccess) {
        fma_chains<T><<<blocks, kThreads>>>(out, iters, b, c);  // warm-up
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(e0);
    if (ce == cudaSuccess) {
        fma_chains<T><<<blocks, kThreads>>>(out, iters, b, c);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(e1);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float t = 0.f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    if (ce != cudaSuccess) return CR_PEAKS_ECUDA;
    const double flops = 2.0 * kChains * (double)iters * (double)blocks * kThreads;
    *ms = t;
    *tflops = t > 0.f ? flops / (t * 1e-3) * 1e-12 : 0.0;
    return 0;
}

}  // namespace

extern "C" int cr_peak_fma(int fp64, int iters, double* tflops, double* ms) {
    if (iters < 1 || !tflops || !ms) return CR_PEAKS_EINVAL;
    return fp64 ? run<double>(iters, tflops, ms) : run<float>(iters, tflops, ms);
}
