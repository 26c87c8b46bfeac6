// es_probe.cu - measured FMA pipe rates: the denominators of the stage (a)
// rooflines (FP64 for the plain kernel, FP32 for the split kernel's bulk).
// Independent FMA chains, enough warps to cover the FMA latency on every SM,
// timed with CUDA events on a private stream.
#include "es_cuda.h"

#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;
constexpr int kIters = 2048;

template <typename T>
__global__ void __launch_bounds__(256) fma_kernel(T* sink, T a, T b)
{
    T x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c];
    if (s == (T)12345.678) sink[0] = s;  // keeps the chains live
}

template <typename T>
es_status probe(int32_t device_ordinal, double* out_tflops)
{
    if (!out_tflops) return ES_ERR_BAD_ARG;
    if (cudaSetDevice(device_ordinal) != cudaSuccess) return ES_ERR_DEVICE;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ordinal);
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return ES_ERR_LAUNCH;
    T* sink = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    es_status st = ES_OK;
    if (cudaMalloc(&sink, sizeof(T)) != cudaSuccess) st = ES_ERR_OOM;
    const int blocks = sms * 8;
    float best_ms = 1e30f;
    for (int rep = 0; st == ES_OK && rep < 5; rep++) {
        cudaEventRecord(e0, s);
        fma_kernel<T><<<blocks, 256, 0, s>>>(sink, (T)0.999999, (T)1e-9);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = ES_ERR_LAUNCH;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_ms) best_ms = ms;  // first launch is warm-up
    }
    if (st == ES_OK) {
        const double flops = 2.0 * kChains * (double)kIters * 256.0 * blocks;
        *out_tflops = flops / (best_ms * 1e-3) / 1e12;
    }
    cudaFree(sink);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    return st;
}

}  // namespace

extern "C" es_status es_probe_fp64_fma(int32_t device_ordinal, double* out_tflops)
{
    return probe<double>(device_ordinal, out_tflops);
}

extern "C" es_status es_probe_fp32_fma(int32_t device_ordinal, double* out_tflops)
{
    return probe<float>(device_ordinal, out_tflops);
}
