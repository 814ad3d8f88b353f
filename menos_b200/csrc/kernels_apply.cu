// sm_100a gate kernels of the plain complex128 path.
//
// Bitwise contract (the reference's generic kernel,
// src/kernels/cpu/dense_kernels.cpp:465-524): each output amplitude is
//     (+0) + m[out][0]*a[0] + m[out][1]*a[1] + ...   (increasing `in`)
// with the product (mr*ar - mi*ai, mr*ai + mi*ar), every multiply and add
// rounded on its own (built with -fmad=false and written with __dmul_rn /
// __dadd_rn / __dsub_rn, which are never contracted).  Two rewrites keep the
// result identical and save FP64 issue slots:
//   * the leading "(+0) +" only turns a -0.0 into +0.0, and the sign of a
//     zero never changes a later non-zero sum, so it is dropped inside the
//     arithmetic and applied once, as canon(), where an amplitude is stored;
//   * a product term whose matrix entry is exactly zero (either sign) is a
//     signed zero and changes nothing but a zero's sign, so it is skipped;
//     an entry with zero imaginary part contributes (mr*ar, mr*ai).
// Both hold for finite amplitudes, the reference kernels' own precondition
// (src/kernels/dense_kernels.h:105-124).
#include <cuda_runtime.h>

#include <cstdint>

#include "device_math.cuh"
#include "mb2_internal.h"

namespace mb2 {
namespace {

using namespace dev;

// ---------------------------------------------------------------- init
__global__ void k_init_c128(double2* st, uint64_t n_amps, double re, double im) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps; i += stride)
        st[i] = (i == 0) ? make_double2(re, im) : make_double2(0.0, 0.0);
}
__global__ void k_init_c64(float2* st, uint64_t n_amps, float re, float im) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps; i += stride)
        st[i] = (i == 0) ? make_float2(re, im) : make_float2(0.0f, 0.0f);
}

// ---------------------------------------------------------------- per-gate kernels
struct M8 {
    double v[8];
};
struct M32 {
    double v[32];
};
struct D128 {
    double v[128];
};

// One pair (i0, i0 | 2^q) per thread iteration: the reference's 1-qubit
// contract (dense_kernels.cpp:227-273).
__global__ void __launch_bounds__(256) k_apply_1q(double2* __restrict__ st, uint64_t npairs, uint32_t q, M8 m) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t bit = uint64_t{1} << q;
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < npairs; p += stride) {
        const uint64_t i0 = insert_zero(p, q);
        const double2 a0 = st[i0];
        const double2 a1 = st[i0 | bit];
        st[i0] = canon(cadd(cmul(m.v[0], m.v[1], a0), cmul(m.v[2], m.v[3], a1)));
        st[i0 | bit] = canon(cadd(cmul(m.v[4], m.v[5], a0), cmul(m.v[6], m.v[7], a1)));
    }
}

// One group of four per thread iteration; local bit j = operand j
// (dense_kernels.cpp:275-297).
__global__ void __launch_bounds__(256) k_apply_2q(double2* __restrict__ st, uint64_t ngroups, uint32_t q0,
                                                  uint32_t q1, M32 m) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint32_t lo = q0 < q1 ? q0 : q1;
    const uint32_t hi = q0 < q1 ? q1 : q0;
    const uint64_t b0 = uint64_t{1} << q0, b1 = uint64_t{1} << q1;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < ngroups; g += stride) {
        const uint64_t base = insert_zero(insert_zero(g, lo), hi);
        const uint64_t idx[4] = {base, base | b0, base | b1, base | b0 | b1};
        double2 a[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = st[idx[i]];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            double2 s = cmul(m.v[8 * o], m.v[8 * o + 1], a[0]);
#pragma unroll
            for (int i = 1; i < 4; ++i) s = cadd(s, cmul(m.v[8 * o + 2 * i], m.v[8 * o + 2 * i + 1], a[i]));
            st[idx[o]] = canon(s);
        }
    }
}

// Diagonal matrices: each amplitude times its entry (dense_kernels.cpp:299-363).
__global__ void __launch_bounds__(256) k_apply_diag(double2* __restrict__ st, uint64_t n_amps, uint32_t k,
                                                    uint32_t q0, uint32_t q1, uint32_t q2, uint32_t q3,
                                                    uint32_t q4, uint32_t q5, D128 d) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint32_t q[6] = {q0, q1, q2, q3, q4, q5};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps; i += stride) {
        uint32_t e = 0;
        for (uint32_t j = 0; j < k; ++j) e |= static_cast<uint32_t>((i >> q[j]) & 1u) << j;
        st[i] = canon(scale_entry(d.v[2 * e], d.v[2 * e + 1], st[i]));
    }
}

// The generic k-operand kernel (dense_kernels.cpp:465-524), cooperative per
// CTA: a batch of groups is gathered into shared memory, each thread then
// forms whole outputs (sum over `in` in increasing order) and stores them.
// Dynamic shared memory: the matrix (dim^2, transposed) then the batch (kGenBatch amps).
constexpr uint32_t kGenBatch = 1024;
__global__ void __launch_bounds__(256) k_apply_generic(double2* __restrict__ st, uint32_t n, uint32_t k,
                                                       uint32_t q0, uint32_t q1, uint32_t q2, uint32_t q3,
                                                       uint32_t q4, uint32_t q5,
                                                       const double2* __restrict__ matrix) {
    extern __shared__ double2 smem[];
    const uint32_t dim = 1u << k;
    double2* mat = smem;
    double2* buf = smem + dim * dim;
    const uint32_t q[6] = {q0, q1, q2, q3, q4, q5};
    // The operands in increasing order: a group's base index is its number
    // with a zero bit inserted at each of them, lowest first (k steps, not
    // one per free qubit).
    uint32_t qs[6] = {q0, q1, q2, q3, q4, q5};
    for (uint32_t a = 1; a < k; ++a)
        for (uint32_t b = a; b > 0 && qs[b - 1] > qs[b]; --b) {
            const uint32_t t = qs[b];
            qs[b] = qs[b - 1];
            qs[b - 1] = t;
        }
    auto group_base = [&](uint64_t g) {
        for (uint32_t j = 0; j < k; ++j) g = insert_zero(g, qs[j]);
        return g;
    };
    // Transposed in shared memory (mat[in * dim + out]): the lanes of a
    // quarter-warp form consecutive outputs, so their reads of one input's
    // column are contiguous instead of dim entries apart (one bank).
    for (uint32_t i = threadIdx.x; i < dim * dim; i += blockDim.x) mat[(i % dim) * dim + i / dim] = matrix[i];
    const uint64_t ngroups = (uint64_t{1} << n) >> k;
    const uint32_t per_batch = kGenBatch >> k;  // groups per batch (k <= 6 -> >= 16)
    const uint64_t nbatches = (ngroups + per_batch - 1) / per_batch;
    for (uint64_t bt = blockIdx.x; bt < nbatches; bt += gridDim.x) {
        __syncthreads();
        // gather
        for (uint32_t s = threadIdx.x; s < kGenBatch; s += blockDim.x) {
            const uint64_t g = bt * per_batch + (s >> k);
            if (g >= ngroups) continue;
            const uint32_t local = s & (dim - 1);
            uint64_t idx = group_base(g);
            for (uint32_t j = 0; j < k; ++j)
                if ((local >> j) & 1u) idx |= uint64_t{1} << q[j];
            buf[s] = st[idx];
        }
        __syncthreads();
        for (uint32_t s = threadIdx.x; s < kGenBatch; s += blockDim.x) {
            const uint64_t g = bt * per_batch + (s >> k);
            if (g >= ngroups) continue;
            const uint32_t out = s & (dim - 1);
            const double2* grp = buf + (s & ~(dim - 1));
            double2 acc = cmul(mat[out].x, mat[out].y, grp[0]);
            for (uint32_t in = 1; in < dim; ++in) acc = cadd(acc, cmul(mat[in * dim + out].x, mat[in * dim + out].y, grp[in]));
            uint64_t idx = group_base(g);
            for (uint32_t j = 0; j < k; ++j)
                if ((out >> j) & 1u) idx |= uint64_t{1} << q[j];
            st[idx] = canon(acc);
        }
    }
}

// The generic kernel for 7..10 operands (a density matrix's superoperator of
// a 4- or 5-qubit channel): one CTA per group of 2^k amplitudes, gathered
// into shared memory; thread `out` forms sum over `in` (increasing) of
// m[out][in] * a[in] exactly as k_apply_generic, reading the matrix
// transposed (mt[in * dim + out], so a warp's reads are contiguous) from
// global memory, where it stays in L2.
struct Q10 {
    uint32_t q[10];
};

__global__ void __launch_bounds__(256) k_apply_wide(double2* __restrict__ st, uint32_t n, uint32_t k, Q10 ops,
                                                    const double2* __restrict__ mt) {
    extern __shared__ double2 grp[];
    const uint32_t dim = 1u << k;
    uint64_t opmask = 0;
    for (uint32_t j = 0; j < k; ++j) opmask |= uint64_t{1} << ops.q[j];
    const uint64_t rest = ((uint64_t{1} << n) - 1) & ~opmask;
    const uint64_t ngroups = (uint64_t{1} << n) >> k;
    for (uint64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const uint64_t base = pdep64(g, rest);
        __syncthreads();
        for (uint32_t l = threadIdx.x; l < dim; l += blockDim.x) {
            uint64_t idx = base;
            for (uint32_t j = 0; j < k; ++j)
                if ((l >> j) & 1u) idx |= uint64_t{1} << ops.q[j];
            grp[l] = st[idx];
        }
        __syncthreads();
        for (uint32_t out = threadIdx.x; out < dim; out += blockDim.x) {
            double2 acc = cmul(mt[out].x, mt[out].y, grp[0]);
            for (uint32_t in = 1; in < dim; ++in) {
                const double2 e = mt[static_cast<size_t>(in) * dim + out];
                acc = cadd(acc, cmul(e.x, e.y, grp[in]));
            }
            uint64_t idx = base;
            for (uint32_t j = 0; j < k; ++j)
                if ((out >> j) & 1u) idx |= uint64_t{1} << ops.q[j];
            st[idx] = canon(acc);
        }
    }
}

int grid_for(uint64_t work, int threads) {
    const uint64_t blocks = (work + threads - 1) / threads;
    return static_cast<int>(blocks < 148ull * 16 ? (blocks == 0 ? 1 : blocks) : 148ull * 16);
}


}  // namespace

int launch_init(void* amps, uint64_t n_amps, int precision, double re, double im, void* stream) {
    const auto s = static_cast<cudaStream_t>(stream);
    if (precision == MB2_C64)
        k_init_c64<<<grid_for(n_amps, 256), 256, 0, s>>>(static_cast<float2*>(amps), n_amps, static_cast<float>(re),
                                                        static_cast<float>(im));
    else
        k_init_c128<<<grid_for(n_amps, 256), 256, 0, s>>>(static_cast<double2*>(amps), n_amps, re, im);
    note_launches(1);
    return launch_status();
}

int launch_apply_1q(void* amps, uint32_t n, uint32_t q, const double* m8, void* stream) {
    M8 m;
    for (int i = 0; i < 8; ++i) m.v[i] = m8[i];
    const uint64_t npairs = (uint64_t{1} << n) >> 1;
    k_apply_1q<<<grid_for(npairs, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<double2*>(amps),
                                                                                    npairs, q, m);
    note_launches(1);
    return launch_status();
}

int launch_apply_2q(void* amps, uint32_t n, uint32_t q0, uint32_t q1, const double* m32, void* stream) {
    M32 m;
    for (int i = 0; i < 32; ++i) m.v[i] = m32[i];
    const uint64_t ng = (uint64_t{1} << n) >> 2;
    k_apply_2q<<<grid_for(ng, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<double2*>(amps), ng, q0,
                                                                                q1, m);
    note_launches(1);
    return launch_status();
}

int launch_apply_diag(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* diag, void* stream) {
    D128 d;
    const uint32_t dim = 1u << k;
    for (uint32_t i = 0; i < 2 * dim; ++i) d.v[i] = diag[i];
    uint32_t qq[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t j = 0; j < k; ++j) qq[j] = q[j];
    const uint64_t na = uint64_t{1} << n;
    k_apply_diag<<<grid_for(na, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(amps), na, k, qq[0], qq[1], qq[2], qq[3], qq[4], qq[5], d);
    note_launches(1);
    return launch_status();
}

int launch_apply_generic(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* dev_matrix,
                         void* stream) {
    uint32_t qq[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t j = 0; j < k; ++j) qq[j] = q[j];
    const uint32_t dim = 1u << k;
    const size_t smem = (size_t{dim} * dim + kGenBatch) * sizeof(double2);
    static const bool attr_set = [] {  // once, thread-safe
        return cudaFuncSetAttribute(k_apply_generic, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024) ==
               cudaSuccess;
    }();
    if (!attr_set) return launch_status();
    const uint64_t ngroups = (uint64_t{1} << n) >> k;
    const uint64_t nb = (ngroups + (kGenBatch >> k) - 1) / (kGenBatch >> k);
    const int grid = static_cast<int>(nb < 148ull * 4 ? nb : 148ull * 4);
    k_apply_generic<<<grid, 256, smem, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(amps), n, k, qq[0], qq[1], qq[2], qq[3], qq[4], qq[5],
        reinterpret_cast<const double2*>(dev_matrix));
    note_launches(1);
    return launch_status();
}

int launch_apply_wide(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* dev_matrix_t,
                      void* stream) {
    if (k < 1 || k > 10 || k > n) return MB2_ERR_INVALID;
    Q10 ops{};
    for (uint32_t j = 0; j < k; ++j) ops.q[j] = q[j];
    const uint64_t ngroups = (uint64_t{1} << n) >> k;
    const int grid = static_cast<int>(ngroups < 148ull * 8 ? ngroups : 148ull * 8);
    k_apply_wide<<<grid, 256, (size_t{1} << k) * sizeof(double2), static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(amps), n, k, ops, reinterpret_cast<const double2*>(dev_matrix_t));
    note_launches(1);
    return launch_status();
}

int launch_tile_pass(void* amps, uint32_t n, const TilePass& pass, const uint32_t* dev_words,
                     const double* dev_sdata, const double* dev_gdata, int sm_count, void* stream,
                     const BatchLayout* batch) {
    if (pass.m > kMaxTileQubits || pass.m < kMinTileQubits) return MB2_ERR_INVALID;
    if ((pass.word_count & 3u) != 0 || (pass.param_len != 0 && batch == nullptr)) return MB2_ERR_INVALID;
    const size_t staged = size_t{pass.word_count} * 4 + (size_t{pass.sdata_count} + pass.param_len) * sizeof(double);
    TileLaunch L;
    L.amps = amps;
    L.m = pass.m;
    L.smask = pass.smask;
    L.gmask = pass.gmask;
    L.words = dev_words + pass.word_begin;
    L.nwords = pass.word_count;
    L.sdata = dev_sdata + pass.sdata_begin;
    L.nsdata = pass.sdata_count;
    L.gdata = dev_gdata;
    L.pdata = batch ? batch->pdata : nullptr;
    L.pstride = batch ? batch->pstride : 0u;
    L.param_lo = pass.param_lo;
    L.param_len = pass.param_len;
    L.bshift = n - pass.m;
    L.stream = stream;
    L.threads = 1u << (pass.m - kRegQubits);
    // 12-qubit tiles keep three tile buffers (two tiles in flight), smaller
    // ones two; the instance launchers size the grid (CTAs per SM).
    L.stages = pass.m == kMaxTileQubits ? 3u : 2u;
    L.smem = L.stages * (size_t{1} << pass.m) * sizeof(double2) + staged;
    L.sm_count = sm_count;
    L.heavy = pass.heavy;
    // A batch adds the bindings above the n qubits: ntiles counts every
    // binding's tiles, and n grows to the bits the binding index occupies.
    L.ntiles = (uint64_t{1} << n) >> pass.m;
    L.n_all = n;
    if (batch != nullptr) {
        L.ntiles *= batch->bindings;
        while ((uint64_t{1} << (L.n_all - n)) < batch->bindings) ++L.n_all;
    }
    const int rc = pass.m == 11 ? launch_tile_m11(L) : pass.m == 12 ? launch_tile_m12(L) : launch_tile_generic(L);
    note_launches(1);
    return rc;
}

namespace {
// The error of the last failed launch on this thread: cudaGetLastError
// clears the error it reports, so the launch wrappers keep it for the
// message the caller builds.
thread_local cudaError_t t_launch_error = cudaSuccess;
}  // namespace

int launch_status() {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return MB2_OK;
    t_launch_error = e;
    return MB2_ERR_CUDA;
}

int record_cuda_error(int cuda_error) {
    const auto e = static_cast<cudaError_t>(cuda_error);
    if (e == cudaSuccess) return MB2_OK;
    cudaGetLastError();  // clear a non-sticky error; the message is kept here
    t_launch_error = e;
    return MB2_ERR_CUDA;
}

const char* last_cuda_error_string() {
    cudaError_t e = t_launch_error;
    t_launch_error = cudaSuccess;
    if (e == cudaSuccess) e = cudaGetLastError();
    return cudaGetErrorString(e);
}

}  // namespace mb2
