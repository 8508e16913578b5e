// Arithmetic-peak microbenchmarks: the roofline denominators for the FP64 / FP32 SIMT
// kernels (the HBM and bf16 tensor peaks come from the pool's own measurement).
// Each thread runs 8 independent FMA chains; the grid fills every SM several times.
#include <cuda_runtime.h>

#include "../../../include/gfnff_b200.h"

namespace {

template <class T>
__global__ void k_fma_peak(T* out, int iters, T a, T b)
{
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)1234.5678) out[0] = s;   // keeps the chains alive
}

template <class T>
double run(int device)
{
    if (cudaSetDevice(device) != cudaSuccess) return -1.0;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    T* out = nullptr;
    if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return -1.0;
    const int threads = 256, blocks = sms * 8, iters = 2048;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        k_fma_peak<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
        if (rep > 0 && ms > 0.f) best = fmax(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return cudaGetLastError() == cudaSuccess ? best : -1.0;
}

}  // namespace

extern "C" double gfnff_fma_peak_tflops(int device, int fp64)
{
    return fp64 ? run<double>(device) : run<float>(device);
}
