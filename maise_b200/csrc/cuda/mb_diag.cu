/*
 * mb_diag.cu -- FMA throughput probes (FP64 and FP32).  Each thread runs
 * independent FMA chains; the kernel fills every SM with resident warps.
 * The measured rates are the denominators of the FP64 roofline of the
 * descriptor kernels and the FP32 roofline of the batched relax.
 */
#include <cuda_runtime.h>

#include "../../../include/maise_b200.h"

namespace {

constexpr int CHAINS = 8;

template <class T>
__global__ void k_fma_chains(T *out, int iters, T a, T b) {
    T v[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; c++) v[c] = (T)(threadIdx.x * 1e-9 + c);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < CHAINS; c++) v[c] = fma(v[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; c++) s += v[c];
    if (s == (T)12345.678) out[0] = s; /* keeps the chains live */
}

}  // namespace

template <class T>
static int fma_peak(int device, double *tflops) {
    cudaDeviceProp prop;
    T *out = nullptr;
    cudaEvent_t e0, e1;
    const int threads = 256, iters = 4096;
    if (!tflops) return MB_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return MB_ERR_NOGPU;
    int blocks = prop.multiProcessorCount * 8;
    if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return MB_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const T a = (T)0.999999, b = (T)1e-7;
    k_fma_chains<T><<<blocks, threads>>>(out, iters, a, b); /* warm-up */
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        float ms = 0.0f;
        cudaEventRecord(e0);
        k_fma_chains<T><<<blocks, threads>>>(out, iters, a, b);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    int err = (int)cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err) return MB_ERR_CUDA;
    double flops = 2.0 * CHAINS * (double)iters * threads * (double)blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return MB_OK;
}

extern "C" int mb_fp64_peak(int device, double *tflops) { return fma_peak<double>(device, tflops); }

extern "C" int mb_fp32_peak(int device, double *tflops) { return fma_peak<float>(device, tflops); }
