// k_peak.cu -- FP64 FMA throughput of this GPU, measured: the denominator of
// the solve stage's roofline (its work runs on the FP64 pipes).  Each thread
// advances 8 independent fused multiply-add chains; the grid covers every SM
// several times over.  2 flops per FMA.
#include <cuda_runtime.h>

#include "yspec_gpu.h"

namespace {

__global__ void k_fp64_fma(double* out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
    double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
    for (int i = 0; i < iters; i++) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1.2345) out[blockIdx.x] = s;   // keeps the chains live; never true in practice
}

}  // namespace

extern "C" int ysg_fp64_peak(int device, double* tflops)
{
    if (!tflops) return YSG_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return YSG_ERR_CUDA;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    double* out = nullptr;
    if (cudaMalloc(&out, (size_t)nsm * 16 * sizeof(double)) != cudaSuccess) return YSG_ERR_CUDA;
    const int blocks = nsm * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fp64_fma<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);   // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        k_fp64_fma<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return YSG_ERR_CUDA;
    const double flops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return YSG_OK;
}
