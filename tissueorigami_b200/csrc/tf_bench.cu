// tf_bench.cu -- measurement hook: the FP64 FMA throughput of the device, the ceiling of the
// element kernel (whose closed-form tangent makes it compute-bound, ~15 kflop per prism).
//
// Every thread runs kChains independent chains of dependent FMAs (x = x * a + b), enough
// independent work per warp to keep the FP64 pipe busy; the grid fills every SM several times.
// The result is written out so the chains cannot be removed. Timed with CUDA events on a private
// stream after one warm-up launch.
#include <cuda_runtime.h>

#include "../../include/tf_b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_fp64_fma(int iters, double a, double b, double* out) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (double)(threadIdx.x + c) * 1e-3;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int tf_measure_fp64(int32_t device, double* tflops) {
    if (!tflops) return TF_ERR_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return TF_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return TF_ERR_CUDA;
    const int blocks = sms * 8, iters = 1 << 14;
    double* out = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = TF_OK;
    if (cudaMalloc(&out, sizeof(double) * (size_t)blocks * kThreads) != cudaSuccess) return TF_ERR_OUT_OF_MEMORY;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess)
        rc = TF_ERR_CUDA;
    float ms = 0.0f;
    if (rc == TF_OK) {
        // a = 1 - 2^-30, b = 2^-30: the chains stay bounded and finite for any iteration count
        const double a = 1.0 - 9.313225746154785e-10, b = 9.313225746154785e-10;
        k_fp64_fma<<<blocks, kThreads, 0, s>>>(iters, a, b, out);
        cudaEventRecord(e0, s);
        k_fp64_fma<<<blocks, kThreads, 0, s>>>(iters, a, b, out);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
            cudaGetLastError() != cudaSuccess)
            rc = TF_ERR_CUDA;
    }
    if (rc == TF_OK) {
        const double flops = 2.0 * kChains * (double)iters * blocks * kThreads;
        *tflops = flops / (ms * 1e-3) / 1e12;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaFree(out);
    return rc;
}
