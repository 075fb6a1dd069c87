// peak_fp64.cu -- measures the device's FP64 FMA throughput (roofline denominator for
// the FP64 contraction kernel; the driver's measured peaks cover HBM and BF16 only).
// Each thread runs 8 independent DFMA chains; grid = 4 CTAs of 256 threads per SM.
#include "rbc.h"
#include <cuda_runtime.h>

__global__ void __launch_bounds__(256) k_dfma_peak(double* out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = threadIdx.x * 1e-3 + i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = fma(x[i], a, b);
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == 12345.678) out[blockIdx.x] = s; // keeps the chains live; never true in practice
}

extern "C" rbc_status rbc_measure_fp64_peak(int device, double* tflops)
{
    if (!tflops) return RBC_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return RBC_ERR_CUDA;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * nsm * 4) != cudaSuccess) return RBC_ERR_OUT_OF_MEMORY;
    const int iters = 20000;
    const int grid = nsm * 4;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_dfma_peak<<<grid, 256>>>(out, 100, 0.999999, 1e-7);
    cudaEventRecord(a);
    k_dfma_peak<<<grid, 256>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess || ms <= 0) return RBC_ERR_CUDA;
    const double flops = 2.0 * 8.0 * iters * (double)grid * 256.0;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return RBC_OK;
}
