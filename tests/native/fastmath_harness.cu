// Device harness for the tolerance arithmetic's branch-free reciprocal,
// quotient and reciprocal square root (piernik_b200/csrc/pk_fast.cuh): each evaluated
// on n operand pairs next to CUDA's correctly rounded division and square
// root, for the GPU test of their error in units in the last place.
#include <cuda_runtime.h>

#include "../../piernik_b200/csrc/pk_fast.cuh"

__global__ void k_fastmath(const double* a, const double* b, int n, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = a[i], y = b[i];
    double* o = out + 8 * (long long)i;
    o[0] = pk::rcp_nr(y);
    o[1] = 1.0 / y;
    o[2] = pk::div_nr(x, y);
    o[3] = x / y;
    o[4] = pk::rsqrt_nr(y) * y;
    o[5] = sqrt(y);
    o[6] = pk::rsqrt_nr(y);
    o[7] = 1.0 / sqrt(y);
}

// a, b, out: host arrays (n, n, 8n doubles); returns a cudaError_t
extern "C" int fastmath_eval(const double* a, const double* b, int n, double* out)
{
    double *da = nullptr, *db = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&da, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&db, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * 8 * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(da, a, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(db, b, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_fastmath<<<(n + 255) / 256, 256>>>(da, db, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 8 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(da);
    cudaFree(db);
    cudaFree(dout);
    return (int)e;
}
