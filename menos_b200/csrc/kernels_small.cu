// Kernels of the small-request batch (small_batch.cpp): many complex128
// states of at most 2^16 amplitudes, each step one launch for all of them.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_math.cuh"
#include "mb2_internal.h"

namespace mb2 {
namespace {
using dev::cadd;
using dev::cmul;

constexpr int kThreads = 256;

// |initial phase> on every state: amplitude 0 of state j is vals[j] (the
// states were zeroed with one memset).
__global__ void k_init_jobs(double2* __restrict__ base, const uint64_t* __restrict__ offsets,
                            const double2* __restrict__ vals, uint32_t count) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
        base[offsets[j]] = vals[j];
}

// One CTA per (state, Pauli term): sum over m of conj(a[m ^ x]) (-1)^{|m & z|}
// a[m] (a fixed order: per thread in steps of the block, then the block's
// warps), times i^{|x & z|}: <psi|P|psi> for P = i^{|x&z|} X^x Z^z.
__global__ void __launch_bounds__(kThreads) k_expect_jobs(const ExpectJob* __restrict__ jobs,
                                                         double* __restrict__ out) {
    const ExpectJob J = jobs[blockIdx.x];
    const double2* __restrict__ a = static_cast<const double2*>(J.st);
    const uint64_t na = uint64_t{1} << J.n;
    double re = 0.0, im = 0.0;
    for (uint64_t m = threadIdx.x; m < na; m += kThreads) {
        const double2 v = a[m], w = a[m ^ J.x];
        // conj(w) * v
        double pr = __dadd_rn(__dmul_rn(w.x, v.x), __dmul_rn(w.y, v.y));
        double pi = __dsub_rn(__dmul_rn(w.x, v.y), __dmul_rn(w.y, v.x));
        if (__popcll(m & J.z) & 1) {
            re = __dsub_rn(re, pr);
            im = __dsub_rn(im, pi);
        } else {
            re = __dadd_rn(re, pr);
            im = __dadd_rn(im, pi);
        }
    }
    __shared__ double sre[kThreads / 32], sim[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        re = __dadd_rn(re, __shfl_down_sync(0xffffffffu, re, o));
        im = __dadd_rn(im, __shfl_down_sync(0xffffffffu, im, o));
    }
    if ((threadIdx.x & 31u) == 0) {
        sre[threadIdx.x >> 5] = re;
        sim[threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0, i = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) {
            r = __dadd_rn(r, sre[w]);
            i = __dadd_rn(i, sim[w]);
        }
        const int ph = __popcll(J.x & J.z) & 3;  // times i^ph
        out[2 * blockIdx.x] = ph == 0 ? r : ph == 1 ? -i : ph == 2 ? -r : i;
        out[2 * blockIdx.x + 1] = ph == 0 ? i : ph == 1 ? r : ph == 2 ? -i : -r;
    }
}

// One CTA per state: the reference's walk (src/engines/dense/sample.cpp:
// 55-69) -- cumulative += |a_b|^2 in index order, shot s goes to the first b
// with u[s] < cumulative (the last state when none does) -- done by one
// thread, exactly; the block's other threads stage the next amplitudes'
// probabilities in shared memory.
__global__ void __launch_bounds__(kThreads) k_walk_jobs(const WalkJob* __restrict__ jobs) {
    const WalkJob J = jobs[blockIdx.x];
    const double2* __restrict__ a = static_cast<const double2*>(J.st);
    const uint64_t na = uint64_t{1} << J.n;
    __shared__ double p[2][kThreads];
    double cumulative = 0.0;
    uint64_t s = 0;
    auto stage = [&](uint64_t base, int buf) {
        const uint64_t b = base + threadIdx.x;
        if (b < na) {
            const double2 v = a[b];
            p[buf][threadIdx.x] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
        }
    };
    stage(0, 0);
    __syncthreads();
    int cur = 0;
    for (uint64_t base = 0; base < na; base += kThreads) {
        if (base + kThreads < na) stage(base + kThreads, cur ^ 1);
        if (threadIdx.x == 0) {
            const uint64_t lim = na - base < kThreads ? na - base : kThreads;
            for (uint64_t i = 0; i < lim && s < J.shots; ++i) {
                cumulative = __dadd_rn(cumulative, p[cur][i]);
                while (s < J.shots && J.u[s] < cumulative) J.basis[s++] = base + i;
            }
        }
        __syncthreads();
        cur ^= 1;
    }
    if (threadIdx.x == 0)
        for (; s < J.shots; ++s) J.basis[s] = na - 1;
}

}  // namespace

int launch_init_jobs(void* base, const uint64_t* dev_offsets, const double* dev_vals, uint32_t count, void* stream) {
    if (count == 0) return MB2_OK;
    k_init_jobs<<<(count + kThreads - 1) / kThreads, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(base), dev_offsets, reinterpret_cast<const double2*>(dev_vals), count);
    note_launches(1);
    return launch_status();
}

int launch_expect_jobs(const ExpectJob* dev_jobs, uint32_t count, double* dev_out, void* stream) {
    if (count == 0) return MB2_OK;
    k_expect_jobs<<<count, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(dev_jobs, dev_out);
    note_launches(1);
    return launch_status();
}

int launch_walk_jobs(const WalkJob* dev_jobs, uint32_t count, void* stream) {
    if (count == 0) return MB2_OK;
    k_walk_jobs<<<count, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(dev_jobs);
    note_launches(1);
    return launch_status();
}

}  // namespace mb2
