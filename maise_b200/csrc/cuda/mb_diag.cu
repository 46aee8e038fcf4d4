/*
 * mb_diag.cu -- FP64 FMA throughput probe.  Each thread runs independent
 * FMA chains; the kernel fills every SM with resident warps.  The measured
 * rate is the denominator of the FP64 roofline of the descriptor kernel.
 */
#include <cuda_runtime.h>

#include "../../../include/maise_b200.h"

namespace {

constexpr int CHAINS = 8;

__global__ void k_fma_chains(double *out, int iters, double a, double b) {
    double v[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; c++) v[c] = threadIdx.x * 1e-9 + c;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < CHAINS; c++) v[c] = fma(v[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < CHAINS; c++) s += v[c];
    if (s == 12345.678) out[0] = s; /* keeps the chains live */
}

}  // namespace

extern "C" int mb_fp64_peak(int device, double *tflops) {
    cudaDeviceProp prop;
    double *out = nullptr;
    cudaEvent_t e0, e1;
    const int threads = 256, iters = 4096;
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return MB_ERR_NOGPU;
    int blocks = prop.multiProcessorCount * 8;
    if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return MB_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_chains<<<blocks, threads>>>(out, iters, 0.999999, 1e-7); /* warm-up */
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        float ms = 0.0f;
        cudaEventRecord(e0);
        k_fma_chains<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
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
