// Kernels of the batched parameter sweep: many bindings of one circuit,
// their states back to back in one buffer (binding b at b * 2^n).
//
// k_batch_init: every binding's state to exp(i*phase)|0...0>.
// k_batch_expect: one thread-block cluster of 8 CTAs per binding.  The
// binding's state is read from HBM once into the cluster's shared memory
// (each CTA holds 2^(n-3) amplitudes: 128 KiB at 16 qubits); every Pauli
// term then pairs amplitudes across the cluster through distributed shared
// memory, and <H> = sum_t coef_t <P_t> is formed in term order by rank 0.
// Reductions run in a fixed order (threads, warps, ranks, terms), so a
// binding's value does not depend on the grid or on its neighbours.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "mb2_internal.h"

namespace cg = cooperative_groups;

namespace mb2 {
namespace {

constexpr int kThreads = 256;
constexpr int kCluster = 8;

template <typename A>
__device__ __forceinline__ A make_amp(double re, double im);
template <>
__device__ __forceinline__ double2 make_amp<double2>(double re, double im) { return make_double2(re, im); }
template <>
__device__ __forceinline__ float2 make_amp<float2>(double re, double im) {
    return make_float2(static_cast<float>(re), static_cast<float>(im));
}
__device__ __forceinline__ double2 as_d2(double2 a) { return a; }
__device__ __forceinline__ double2 as_d2(float2 a) { return make_double2(a.x, a.y); }

template <typename A>
__global__ void k_batch_init(A* st, uint64_t total, uint32_t n, double re, double im) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t mask = (uint64_t{1} << n) - 1;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride)
        st[i] = (i & mask) == 0 ? make_amp<A>(re, im) : make_amp<A>(0.0, 0.0);
}

__device__ __forceinline__ void block_sum2(double& re, double& im, double* sh) {
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        sh[2 * w] = re;
        sh[2 * w + 1] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        re = 0.0;
        im = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
            re += sh[2 * k];
            im += sh[2 * k + 1];
        }
    }
}

template <typename A>
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kThreads)
    k_batch_expect(const A* __restrict__ st, uint32_t n, const uint64_t* __restrict__ xs,
                   const uint64_t* __restrict__ zs, const double* __restrict__ coefs, uint32_t num_terms,
                   double* __restrict__ out) {
    extern __shared__ double2 slice[];
    __shared__ double part[2 * kMaxBatchTerms];
    __shared__ double red[2 * (kThreads / 32)];
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank();
    const uint64_t b = blockIdx.x / kCluster;
    const uint32_t sl = n - 3;
    const uint32_t S = 1u << sl;
    const A* src = st + (b << n) + (static_cast<uint64_t>(rank) << sl);
    for (uint32_t i = threadIdx.x; i < S; i += kThreads) slice[i] = as_d2(src[i]);
    cluster.sync();
    for (uint32_t t = 0; t < num_terms; ++t) {
        const uint64_t x = xs[t], z = zs[t];
        double re = 0.0, im = 0.0;
        if (x == 0) {
            for (uint32_t i = threadIdx.x; i < S; i += kThreads) {
                const uint64_t m = (static_cast<uint64_t>(rank) << sl) | i;
                const double2 a = slice[i];
                const double p = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
                re = (__popcll(z & m) & 1) ? __dsub_rn(re, p) : __dadd_rn(re, p);
            }
        } else {
            const uint32_t h = 63 - __clzll(static_cast<long long>(x));
            for (uint32_t i = threadIdx.x; i < S; i += kThreads) {
                const uint64_t m = (static_cast<uint64_t>(rank) << sl) | i;
                if ((m >> h) & 1u) continue;
                const uint64_t m2 = m ^ x;
                const uint32_t r2 = static_cast<uint32_t>(m2 >> sl);
                const uint32_t i2 = static_cast<uint32_t>(m2) & (S - 1);
                const double2* other = r2 == rank ? slice : cluster.map_shared_rank(slice, r2);
                const double2 a = slice[i], c = other[i2];
                const double tr = __dadd_rn(__dmul_rn(a.x, c.x), __dmul_rn(a.y, c.y));
                const double ti = __dsub_rn(__dmul_rn(a.x, c.y), __dmul_rn(a.y, c.x));
                const bool neg2 = __popcll(z & m2) & 1;
                const bool neg1 = __popcll(z & m) & 1;
                re = neg2 ? __dsub_rn(re, tr) : __dadd_rn(re, tr);
                im = neg2 ? __dsub_rn(im, ti) : __dadd_rn(im, ti);
                re = neg1 ? __dsub_rn(re, tr) : __dadd_rn(re, tr);
                im = neg1 ? __dadd_rn(im, ti) : __dsub_rn(im, ti);
            }
        }
        block_sum2(re, im, red);
        if (threadIdx.x == 0) {
            part[2 * t] = re;
            part[2 * t + 1] = im;
        }
    }
    cluster.sync();
    if (rank == 0 && threadIdx.x == 0) {
        double total = 0.0;
        for (uint32_t t = 0; t < num_terms; ++t) {
            double re = 0.0, im = 0.0;
            for (uint32_t r = 0; r < kCluster; ++r) {
                const double* p = cluster.map_shared_rank(part, r);
                re += p[2 * t];
                im += p[2 * t + 1];
            }
            // i^popcount(x & z) * (re, im); only the real part enters <H>.
            const int ph = __popcll(xs[t] & zs[t]) & 3;
            const double value_re = ph == 0 ? re : ph == 1 ? -im : ph == 2 ? -re : im;
            total += coefs[t] * value_re;
        }
        out[b] = total;
    }
    cluster.sync();  // rank 0 reads the others' partials before they exit
}

}  // namespace

int launch_batch_init(void* amps, uint32_t n, uint64_t bindings, double re, double im, void* stream,
                      int precision) {
    const uint64_t total = bindings << n;
    const uint64_t blocks = (total + 255) / 256;
    const unsigned grid = static_cast<unsigned>(blocks < 148ull * 16 ? blocks : 148ull * 16);
    if (precision == MB2_C64)
        k_batch_init<float2><<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<float2*>(amps), total, n,
                                                                                 re, im);
    else
        k_batch_init<double2><<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<double2*>(amps), total,
                                                                                  n, re, im);
    note_launches(1);
    return launch_status();
}

int launch_batch_expect(const void* amps, uint32_t n, uint64_t bindings, const uint64_t* dev_x,
                        const uint64_t* dev_z, const double* dev_coefs, uint32_t num_terms, double* dev_out,
                        void* stream, int precision) {
    if (n < 3 || n > 16 || num_terms > kMaxBatchTerms) return MB2_ERR_INVALID;
    const size_t smem = (size_t{1} << (n - 3)) * sizeof(double2);
    static const bool attr = [] {  // once, thread-safe
        const int most = static_cast<int>((size_t{1} << 13) * sizeof(double2));
        return cudaFuncSetAttribute(k_batch_expect<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, most) ==
                   cudaSuccess &&
               cudaFuncSetAttribute(k_batch_expect<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, most) ==
                   cudaSuccess;
    }();
    if (!attr) return launch_status();
    const unsigned grid = static_cast<unsigned>(bindings * kCluster);
    const auto s = static_cast<cudaStream_t>(stream);
    if (precision == MB2_C64)
        k_batch_expect<float2><<<grid, kThreads, smem, s>>>(static_cast<const float2*>(amps), n, dev_x, dev_z,
                                                            dev_coefs, num_terms, dev_out);
    else
        k_batch_expect<double2><<<grid, kThreads, smem, s>>>(static_cast<const double2*>(amps), n, dev_x, dev_z,
                                                             dev_coefs, num_terms, dev_out);
    note_launches(1);
    return launch_status();
}

}  // namespace mb2
