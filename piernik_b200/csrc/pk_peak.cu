// pk_peak.cu -- measurement utility: the FP64 FMA throughput of the device.
//
// The sweep kernels are bound by FP64 issue, not by HBM, so their roofline
// denominator is the device's dependent-free DFMA rate: 32 independent fused
// multiply-add chains per thread, enough warps per SM to hide the pipe's
// latency, timed with CUDA events.
#include <cuda_runtime.h>

#include "../../include/piernik_b200.h"

namespace {

constexpr int CHAINS = 32;

__global__ void __launch_bounds__(256) k_dfma_peak(double* out, int iters, double b, double c)
{
    double a[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) a[k] = threadIdx.x * 1.0e-3 + k;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < CHAINS; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += a[k];
    if (s == 1.2345e300) out[threadIdx.x] = s;   // keeps the chains live; never true for these inputs
}

}  // namespace

extern "C" int pk_fp64_peak(double* tflops)
{
    if (!tflops) return PK_E_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PK_E_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return PK_E_CUDA;
    double* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = PK_OK;
    const int blocks = sms * 8, threads = 256, iters = 512;
    if (cudaMalloc(&out, sizeof(double) * threads) != cudaSuccess) return PK_E_NOMEM;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = PK_E_CUDA;
    float best = 1e30f;
    for (int rep = 0; rc == PK_OK && rep < 4; ++rep) {   // the first launch warms up
        cudaEventRecord(e0);
        k_dfma_peak<<<blocks, threads>>>(out, iters, 0.999999999, 1.0e-9);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = PK_E_CUDA;
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    if (rc == PK_OK) {
        const double flops = 2.0 * CHAINS * (double)iters * blocks * threads;
        *tflops = flops / (best * 1e-3) / 1e12;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    return rc;
}
