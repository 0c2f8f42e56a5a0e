// Measurement helpers: the FP32 FMA throughput of the device (the roofline
// denominator of the FP32-pipe-bound PP kernel), timed with CUDA events.
#include "p3m_kernels.h"

namespace p3m {

// 8 independent FMA chains per thread; 2 FLOP per FMA.
__global__ void __launch_bounds__(256) k_fma_peak(float *out, int iters, float a, float b)
{
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    float x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1234.5f) out[blockIdx.x] = s;  // keeps the chains live
}

double fp32_fma_tflops(int device)
{
    cudaSetDevice(device);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = 2048;
    float *out = nullptr;
    if (cudaMalloc(&out, sizeof(float) * blocks) != cudaSuccess) return -1.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_peak<<<blocks, threads>>>(out, 64, 0.999f, 1e-3f);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        k_fma_peak<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace p3m
