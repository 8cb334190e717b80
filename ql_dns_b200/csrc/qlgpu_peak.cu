// qlgpu_peak.cu -- FP64 FMA throughput of the device, the denominator of the
// FP64 roofline reported for the DNS transforms (bench.py).  Independent FMA
// chains per thread, 8 resident blocks of 256 threads per SM, timed with CUDA
// events; no memory traffic besides one store per thread.
#include <cuda_runtime.h>

#include "../../include/qlgpu.h"

namespace {

constexpr int CHAINS = 8;

__global__ void __launch_bounds__(256) fma_loop(int iters, double b, double c, double* out) {
    double a[CHAINS];
#pragma unroll
    for (int i = 0; i < CHAINS; ++i) a[i] = 1e-3 * (threadIdx.x + i);
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int i = 0; i < CHAINS; ++i) a[i] = fma(a[i], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < CHAINS; ++i) s += a[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int qlgpu_fp64_peak(int device, double* tflops) {
    if (!tflops) return QLGPU_ERR_ARG;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return QLGPU_ERR_CUDA;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return QLGPU_ERR_NODEVICE;
    const int blocks = sms * 8, threads = 256, iters = 4096;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return QLGPU_ERR_CUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_loop<<<blocks, threads>>>(iters, 0.999999, 1e-7, out);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(e0);
        fma_loop<<<blocks, threads>>>(iters, 0.999999, 1e-7, out);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return QLGPU_ERR_CUDA;
    *tflops = 2.0 * CHAINS * (double)iters * blocks * threads / (best * 1e-3) / 1e12;
    return QLGPU_OK;
}
