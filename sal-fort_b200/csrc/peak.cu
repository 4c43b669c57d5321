// FMA-pipe throughput microbenchmark: the FP64 / FP32 roofline denominators
// (the measured HBM and bf16 tensor peaks do not cover the CUDA-core pipes).
#include <cuda_runtime.h>

#include <string>

#include "../../include/salgpu.h"

namespace sal {
int set_error(int code, const std::string &msg);
}

template <class T>
__global__ void __launch_bounds__(256) fma_kernel(T *out, int iters, T a, T b) {
    // 8 independent chains per thread hide the FMA latency
    T x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = (T)(threadIdx.x + i);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = x[i] * a + b;
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == (T)12345.678) out[0] = s;  // keeps the chains alive
}

extern "C" int sal_fma_peak(int32_t precision, double *tflops) {
    if (!tflops || (precision != 64 && precision != 32)) return sal::set_error(SAL_EINVAL, "precision must be 64 or 32");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return sal::set_error(SAL_ENODEV, "no CUDA device");
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void *out = nullptr;
    if (cudaMalloc(&out, 16) != cudaSuccess) return sal::set_error(SAL_ENOMEM, "cudaMalloc failed");
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        if (precision == 64) fma_kernel<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
        else fma_kernel<float><<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return sal::set_error(SAL_ECUDA, cudaGetErrorString(e));
    const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return SAL_OK;
}
