// FP64 pipe throughput probe: the denominator of the roofline of the
// FP64-bound stages (AABB enclosures, narrow phase).  Eight independent DFMA
// chains per thread on every SM; the result is the device's DFMA issue rate.
#include <cstdint>

#include "kernels.cuh"

namespace mzb
{

__global__ void __launch_bounds__(256) k_dfma_chains(double *out, int iters)
{
    const unsigned g = blockIdx.x * blockDim.x + threadIdx.x;
    double a0 = g * 1e-12, a1 = a0 + 1e-13, a2 = a0 + 2e-13, a3 = a0 + 3e-13;
    double a4 = a0 + 4e-13, a5 = a0 + 5e-13, a6 = a0 + 6e-13, a7 = a0 + 7e-13;
    const double m = 0.9999999999, c = 1e-9;
    for (int i = 0; i < iters; ++i) {
        a0 = fma(a0, m, c);
        a1 = fma(a1, m, c);
        a2 = fma(a2, m, c);
        a3 = fma(a3, m, c);
        a4 = fma(a4, m, c);
        a5 = fma(a5, m, c);
        a6 = fma(a6, m, c);
        a7 = fma(a7, m, c);
    }
    out[g] = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
}

cudaError_t measure_dfma_rate(double *per_second)
{
    int dev = 0, n_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const unsigned blocks = unsigned(n_sm) * 8, threads = 256;
    const int iters = 8192;
    double *out = nullptr;
    e = cudaMalloc(&out, sizeof(double) * blocks * threads);
    if (e != cudaSuccess) return e;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    k_dfma_chains<<<blocks, threads>>>(out, iters); // warm-up
    cudaEventRecord(t0);
    k_dfma_chains<<<blocks, threads>>>(out, iters);
    cudaEventRecord(t1);
    e = cudaEventSynchronize(t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(out);
    if (e != cudaSuccess) return e;
    *per_second = double(blocks) * threads * iters * 8 / (ms * 1e-3);
    return cudaGetLastError();
}

} // namespace mzb
