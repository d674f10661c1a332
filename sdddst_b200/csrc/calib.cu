// Roofline denominators of the CUDA-core pipes: sustained FP64 and FP32 FMA
// throughput of this GPU, measured with long chains of independent FMAs
// (8 accumulators per thread, 8 resident CTAs of 256 threads per SM), best
// of three timed launches.
#include "engine.h"

#include <cuda_runtime.h>

namespace sd {

template <typename T>
__global__ void fma_peak_kernel(T *out, int iters, T a, T b)
{
    T r0 = (T)threadIdx.x, r1 = r0 + (T)1, r2 = r0 + (T)2, r3 = r0 + (T)3;
    T r4 = r0 + (T)4, r5 = r0 + (T)5, r6 = r0 + (T)6, r7 = r0 + (T)7;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            r0 = r0 * a + b;
            r1 = r1 * a + b;
            r2 = r2 * a + b;
            r3 = r3 * a + b;
            r4 = r4 * a + b;
            r5 = r5 * a + b;
            r6 = r6 * a + b;
            r7 = r7 * a + b;
        }
    }
    T s = r0 + r1 + r2 + r3 + r4 + r5 + r6 + r7;
    if (s == (T)-12345.0) out[blockIdx.x] = s; // keeps the chains live
}

template <typename T>
static double run_peak(int device, int iters)
{
    cudaDeviceProp dp;
    cudaGetDeviceProperties(&dp, device);
    const int blocks = dp.multiProcessorCount * 8;
    T *out = nullptr;
    cudaMalloc(&out, sizeof(T) * blocks);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fma_peak_kernel<T><<<blocks, 256>>>(out, iters / 4, (T)0.999999, (T)1e-7); // warm-up
    // best of three timed launches: the attainable rate, not one sample of it
    float ms = 0;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(a);
        fma_peak_kernel<T><<<blocks, 256>>>(out, iters, (T)0.999999, (T)1e-7);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        if (t > 0 && (ms == 0 || t < ms)) ms = t;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    double flops = 2.0 * 8.0 * 16.0 * (double)iters * 256.0 * blocks;
    return ms > 0 ? flops / (ms * 1e-3) / 1e12 : 0.0;
}

} // namespace sd

extern "C" int sdddst_vector_peaks(int device, double *fp64_tflops, double *fp32_tflops)
{
    if (cudaSetDevice(device) != cudaSuccess) return SDDDST_ERR_CUDA;
    if (fp64_tflops) *fp64_tflops = sd::run_peak<double>(device, 4096);
    if (fp32_tflops) *fp32_tflops = sd::run_peak<float>(device, 8192);
    return cudaDeviceSynchronize() == cudaSuccess ? SDDDST_OK : SDDDST_ERR_CUDA;
}
