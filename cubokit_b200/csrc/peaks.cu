// CUDA-core FMA rates of this device, measured: the denominators of the compute fractions the measurements report for
// the FP32 forms (FP32 pipe) and the FP64 forms (FP64 pipe).  Each thread runs eight independent multiply-add chains,
// so the pipes see no dependency stalls; the flops are 2 per FMA.
#include <algorithm>

#include "engine.h"

namespace cubo {

namespace {

constexpr int kChains = 8;
constexpr int kPeakThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kPeakThreads) fma_chain_kernel(T *out, int iterations, T x, T y) {
    T acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) acc[c] = (T)(threadIdx.x + c);
    for (int i = 0; i < iterations; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++)
#pragma unroll
            for (int c = 0; c < kChains; c++) acc[c] = fma(acc[c], x, y);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += acc[c];
    if (s == (T)-1.2345) out[0] = s;  // keeps the chains live; never true for these inputs
}

template <typename T>
double measure(cudaStream_t s, int sms, T *sink) {
    const int blocks = sms * 8, iterations = sizeof(T) == 8 ? 256 : 2048;
    const double flops = 2.0 * kChains * 16 * (double)iterations * blocks * kPeakThreads;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best = 0.0;
    for (int rep = 0; rep < 4; rep++) {  // the first launch warms up
        cudaEventRecord(a, s);
        fma_chain_kernel<T><<<blocks, kPeakThreads, 0, s>>>(sink, iterations, (T)0.999999, (T)1e-7);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0 && ms > 0.0f) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

}  // namespace

cudaError_t measure_fma_peaks(cudaStream_t s, int sms, double *fp32_tflops, double *fp64_tflops) {
    double *sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(double));
    if (e != cudaSuccess) return e;
    *fp32_tflops = measure<float>(s, sms, reinterpret_cast<float *>(sink));
    *fp64_tflops = measure<double>(s, sms, sink);
    e = cudaGetLastError();
    cudaFree(sink);
    return e;
}

}  // namespace cubo
