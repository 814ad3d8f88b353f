// Calibration probes (the reference's device microbenchmarks,
// src/kernels/cuda/device_benchmarks.h:30-67, measured for the planner's CUDA
// time model): the device's FP64 add/multiply issue rate and its
// device-to-device copy bandwidth, both timed with CUDA events.
#include <cuda_runtime.h>

#include <cstdint>

#include "mb2_internal.h"

namespace mb2 {
namespace {

// Eight independent DMUL/DADD chains per thread; `iters` rounds of 16 FP64
// instructions each.  The result is stored so nothing is dead code.
__global__ void __launch_bounds__(256) k_fp64_probe(double* out, int iters, double x) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = x + i + threadIdx.x;
    const double m = 1.0000000001, c = 1e-9;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            a[i] = __dmul_rn(a[i], m);
            a[i] = __dadd_rn(a[i], c);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

int probe_rates(int sm_count, double* fp64_per_s, double* copy_gbs) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * 256 * 64 * 1024) != cudaSuccess) return MB2_ERR_RESOURCE;
    const int blocks = sm_count * 8, iters = 4096;
    k_fp64_probe<<<blocks, 256>>>(out, 16, 1.0);  // warm-up
    cudaEventRecord(e0);
    k_fp64_probe<<<blocks, 256>>>(out, iters, 1.0);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *fp64_per_s = static_cast<double>(blocks) * 256.0 * iters * 16.0 / (ms * 1e-3);
    cudaFree(out);
    const size_t bytes = size_t{1} << 31;  // 2 GiB each way
    void *a = nullptr, *b = nullptr;
    *copy_gbs = 0.0;
    if (cudaMalloc(&a, bytes) == cudaSuccess && cudaMalloc(&b, bytes) == cudaSuccess) {
        cudaMemcpy(b, a, bytes, cudaMemcpyDeviceToDevice);
        float best = 1e30f;
        for (int r = 0; r < 5; ++r) {
            cudaEventRecord(e0);
            cudaMemcpy(b, a, bytes, cudaMemcpyDeviceToDevice);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) best = ms;
        }
        *copy_gbs = 2.0 * static_cast<double>(bytes) / (best * 1e-3) / 1e9;
    }
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaGetLastError() == cudaSuccess ? MB2_OK : MB2_ERR_CUDA;
}

}  // namespace mb2
