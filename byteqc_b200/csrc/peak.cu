// FP64 FMA throughput microbenchmark: the roofline denominator of the J/K
// kernels (the FP64 pipe of the CUDA cores; no tensor cores).
#include "bqc.h"

__global__ void dfma_kernel(double *out, int iters, double a, double b) {
    // 8 independent FMA chains per thread hide the pipe latency
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678) out[0] = s;   // keeps the chains alive
}

extern "C" int BQCfp64_fma_peak(double *flops_per_s, float *ms_out) {
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    double *out = nullptr;
    if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return 1;
    const int threads = 512, blocks = nsm * 4, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    dfma_kernel<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);   // warm-up
    cudaEventRecord(e0);
    dfma_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    *flops_per_s = flops / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
