// Device counts sampler with the reference's exact results.
//
// The reference (src/engines/dense/sample.cpp:24-75) sorts `shots` uniforms
// and walks the basis states once, cumulative = fl(cumulative + |a_i|^2)
// strictly in index order; shot s lands on the first basis state i whose
// running sum c_i exceeds u_s, and shots past the end go to the last state.
// The running sum drifts from the exact prefix sum by up to ~N ulps, so a
// plain parallel scan would move shots.  This sampler reproduces the chain
// c_i bit for bit in parallel:
//
// Within one binade [2^e, 2^(e+1)) every c is M*u with u = 2^(e-52) and
// M in [2^52, 2^53).  Adding p = (k + f) u (k integer, 0 <= f < 1, exact
// since p/u is a power-of-two scaling) rounds to (M + k) u for f < 1/2,
// (M + k + 1) u for f > 1/2 and, on a tie, to whichever of the two has an
// even M.  So each element is a map from the parity of M to (increment, new
// parity); those maps compose associatively, and a chunk of 4096 elements
// reduces to one such map.  Chunks whose run stays inside one binade are
// advanced in O(1) from their exact start value; chunks that cross a binade
// boundary (the first few dozen, while the sum is small, and one per
// boundary) are walked with the reference's own FP64 adds.  The chunk's
// binade is guessed from an approximate prefix sum; a wrong guess only
// costs the sequential walk, never the result.
//
// |a|^2 is re*re + im*im with each product and the sum rounded (std::norm,
// no FMA).
#include <cuda_runtime.h>

#include <cstdint>

#include "mb2_internal.h"

namespace mb2 {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = kSampleChunk / kThreads;  // 16

__device__ __forceinline__ double prob(double2 a) { return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y)); }
// A complex64 amplitude's probability in FP64 (the squares of FP32 values are exact).
__device__ __forceinline__ double prob(float2 a) {
    return __dadd_rn(__dmul_rn(static_cast<double>(a.x), static_cast<double>(a.x)),
                     __dmul_rn(static_cast<double>(a.y), static_cast<double>(a.y)));
}

// Step A: approximate chunk sums (any order; only used to guess binades).
template <typename A>
__global__ void __launch_bounds__(kThreads) k_chunk_sums(const A* __restrict__ st, uint64_t n_amps,
                                                         uint32_t chunk, double* __restrict__ sums) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * chunk;
    double s = 0.0;
    for (uint32_t i = threadIdx.x; i < chunk; i += kThreads)
        if (base + i < n_amps) s += prob(st[base + i]);
    __shared__ double sh[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
        sums[blockIdx.x] = t;
    }
}

// Step B: exclusive scan of the chunk sums, one CTA (approximate).
__global__ void __launch_bounds__(1024) k_scan_sums(const double* __restrict__ sums, uint64_t nchunks,
                                                    double* __restrict__ starts) {
    __shared__ double part[1024];
    const uint64_t per = (nchunks + 1023) / 1024;
    const uint64_t b = threadIdx.x * per;
    double s = 0.0;
    for (uint64_t i = b; i < b + per && i < nchunks; ++i) s += sums[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double run = 0.0;
        for (int t = 0; t < 1024; ++t) {
            const double v = part[t];
            part[t] = run;
            run += v;
        }
    }
    __syncthreads();
    double run = part[threadIdx.x];
    for (uint64_t i = b; i < b + per && i < nchunks; ++i) {
        starts[i] = run;
        run += sums[i];
    }
}

// The per-element parity map of binade e, as (inc if parity 0, inc if parity 1).
struct PMap {
    long long inc0, inc1;
    int par0, par1;  // parity after, from parity 0 / 1
};

__device__ __forceinline__ PMap compose(const PMap& a, const PMap& b) {
    // a then b
    PMap r;
    r.inc0 = a.inc0 + (a.par0 ? b.inc1 : b.inc0);
    r.par0 = a.par0 ? b.par1 : b.par0;
    r.inc1 = a.inc1 + (a.par1 ? b.inc1 : b.inc0);
    r.par1 = a.par1 ? b.par1 : b.par0;
    return r;
}

__device__ __forceinline__ PMap element_map(double p, int e) {
    // q = p / u with u = 2^(e-52): an exact power-of-two scaling.
    const double q = ldexp(p, 52 - e);
    const double kf = floor(q);
    const double f = q - kf;
    const long long k = static_cast<long long>(kf);
    PMap m;
    if (f < 0.5) {
        m.inc0 = k;
        m.inc1 = k;
    } else if (f > 0.5) {
        m.inc0 = k + 1;
        m.inc1 = k + 1;
    } else {  // tie: the even of M + k, M + k + 1
        m.inc0 = (k & 1) ? k + 1 : k;
        m.inc1 = (k & 1) ? k : k + 1;
    }
    m.par0 = static_cast<int>((m.inc0) & 1);
    m.par1 = static_cast<int>((1 + m.inc1) & 1);
    return m;
}

__device__ __forceinline__ int binade_of(double c) {
    int e;
    frexp(c, &e);  // c = f * 2^e, f in [0.5, 1): binade 2^(e-1)
    return e - 1;
}

// Step C: each chunk's composed map for the binade its approximate start
// lies in.  A chunk whose approximate range is not safely inside one binade
// is marked for the sequential walk.
struct ChunkMap {
    long long inc0, inc1;
    int par0, par1;
    int e;      // binade the map is for
    int valid;  // 0: walk sequentially
};

template <typename A>
__global__ void __launch_bounds__(kThreads) k_chunk_maps(const A* __restrict__ st, uint64_t n_amps,
                                                         uint32_t chunk, const double* __restrict__ starts,
                                                         const double* __restrict__ sums,
                                                         ChunkMap* __restrict__ maps) {
    const uint64_t j = blockIdx.x;
    const uint64_t base = j * chunk;
    const double a = starts[j];
    const double hi = a + sums[j];
    // Generous drift allowance (relative): the chain's rounding drift plus
    // the approximate scan's error.
    const double slack = (static_cast<double>(base + chunk) + 1.0e6) * 2.3e-16;
    const int e = a > 0.0 ? binade_of(a) : -2000;
    const double lo_edge = ldexp(1.0, e), hi_edge = ldexp(1.0, e + 1);
    const bool ok = a > 0.0 && e > -1000 && a * (1.0 - slack) > lo_edge && hi * (1.0 + slack) < hi_edge;
    __shared__ int s_ok;
    if (threadIdx.x == 0) s_ok = ok;
    __syncthreads();
    if (!s_ok) {
        if (threadIdx.x == 0) {
            ChunkMap m{};
            m.valid = 0;
            m.e = e;
            maps[j] = m;
        }
        return;
    }
    // Each thread composes its contiguous run of 16 elements in order.
    PMap acc{0, 0, 0, 1};
    const uint64_t my = base + static_cast<uint64_t>(threadIdx.x) * kPerThread;
#pragma unroll 4
    for (int i = 0; i < kPerThread; ++i) {
        const uint64_t idx = my + i;
        const double p = idx < n_amps ? prob(st[idx]) : 0.0;
        acc = compose(acc, element_map(p, e));
    }
    // Ordered reduction across the block: warp shuffles (lane order), then warps.
    for (int o = 1; o < 32; o <<= 1) {
        PMap other;
        other.inc0 = __shfl_down_sync(0xffffffffu, acc.inc0, o);
        other.inc1 = __shfl_down_sync(0xffffffffu, acc.inc1, o);
        other.par0 = __shfl_down_sync(0xffffffffu, acc.par0, o);
        other.par1 = __shfl_down_sync(0xffffffffu, acc.par1, o);
        if ((threadIdx.x & 31) % (2 * o) == 0) acc = compose(acc, other);
    }
    __shared__ PMap wm[kThreads / 32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        PMap t = wm[0];
        for (int w = 1; w < kThreads / 32; ++w) t = compose(t, wm[w]);
        ChunkMap m;
        m.inc0 = t.inc0;
        m.inc1 = t.inc1;
        m.par0 = t.par0;
        m.par1 = t.par1;
        m.e = e;
        m.valid = 1;
        maps[j] = m;
    }
}

// Step D: the exact chain at every chunk start.
//
// D1 (one CTA): chunks whose maps are valid for the same binade form
// segments; a segmented scan gives each chunk the composition of the
// segment's chunks before it (`excl`) and each segment head the whole
// segment's map and length.
// D2 (one warp): walks the segments in order with the exact running value
// c.  A segment is crossed in O(1) when c lies in its binade and the
// segment does not leave it; otherwise its chunks are taken one at a time
// (O(1) per chunk under the same checks, or the reference's FP64 adds over
// the chunk's elements).
// D3 (all chunks): the start of every chunk inside a crossed segment,
// exactly, from the segment's start value and `excl`.
// cstart[j] = the chain before chunk j; cstart[nchunks] = the final sum;
// seq[j] = 1 when chunk j was walked element by element.
struct SMap {
    long long inc0, inc1;
    int par0, par1;
    unsigned count;
    unsigned pad;
};

__device__ __forceinline__ SMap sm_identity() { return SMap{0, 0, 0, 1, 0, 0}; }

__device__ __forceinline__ SMap sm_compose(const SMap& a, const SMap& b) {
    SMap r;
    r.inc0 = a.inc0 + (a.par0 ? b.inc1 : b.inc0);
    r.par0 = a.par0 ? b.par1 : b.par0;
    r.inc1 = a.inc1 + (a.par1 ? b.inc1 : b.inc0);
    r.par1 = a.par1 ? b.par1 : b.par0;
    r.count = a.count + b.count;
    r.pad = 0;
    return r;
}

__device__ __forceinline__ bool seg_head(const ChunkMap* maps, uint64_t j) {
    if (j == 0 || !maps[j].valid || !maps[j - 1].valid) return true;
    return maps[j].e != maps[j - 1].e;
}

__device__ __forceinline__ SMap sm_of(const ChunkMap& m) {
    return SMap{m.inc0, m.inc1, m.par0, m.par1, 1, 0};
}

__global__ void __launch_bounds__(1024) k_seg_scan(const ChunkMap* __restrict__ maps, uint64_t nchunks,
                                                   SMap* __restrict__ excl, SMap* __restrict__ seg_total) {
    __shared__ SMap agg[1024];
    __shared__ unsigned char agg_head[1024];
    const uint64_t per = (nchunks + 1023) / 1024;
    const uint64_t b = threadIdx.x * per, e = b + per < nchunks ? b + per : nchunks;
    // Pass 1: this range's segmented aggregate.
    SMap v = sm_identity();
    bool any_head = false;
    for (uint64_t j = b; j < e; ++j) {
        if (seg_head(maps, j)) {
            v = sm_of(maps[j]);
            any_head = true;
        } else {
            v = sm_compose(v, sm_of(maps[j]));
        }
    }
    agg[threadIdx.x] = v;
    agg_head[threadIdx.x] = any_head ? 1 : 0;
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive segmented scan of the 1024 aggregates
        SMap run = sm_identity();
        for (int t = 0; t < 1024; ++t) {
            const SMap a = agg[t];
            const bool h = agg_head[t] != 0;
            agg[t] = run;
            run = h ? a : sm_compose(run, a);
        }
    }
    __syncthreads();
    // Pass 2: per chunk, within-segment exclusive prefix; segment totals at heads.
    SMap run = agg[threadIdx.x];
    for (uint64_t j = b; j < e; ++j) {
        if (seg_head(maps, j)) run = sm_identity();
        excl[j] = run;
        run = sm_compose(run, sm_of(maps[j]));
        const bool last = (j + 1 == nchunks) || seg_head(maps, j + 1);
        if (last) seg_total[j + 1 - run.count] = run;
    }
}

__device__ __forceinline__ bool advance_exact(double& c, int e, long long inc0, long long inc1) {
    if (!(c > 0.0) || binade_of(c) != e) return false;
    const double u = ldexp(1.0, e - 52);
    const long long M = static_cast<long long>(c / u);  // exact: c is on the grid
    const long long M2 = M + ((M & 1) ? inc1 : inc0);
    if (M2 >= (1LL << 53)) return false;
    c = static_cast<double>(M2) * u;  // exact: M2 < 2^53
    return true;
}

template <typename A>
__global__ void __launch_bounds__(32) k_seg_chain(const A* __restrict__ st, uint64_t n_amps, uint32_t chunk,
                                                  uint64_t nchunks, const ChunkMap* __restrict__ maps,
                                                  const SMap* __restrict__ seg_total, double* __restrict__ cstart,
                                                  unsigned char* __restrict__ seq, unsigned char* __restrict__ direct,
                                                  double* __restrict__ seg_c) {
    __shared__ double buf[kSampleChunk];
    const int lane = threadIdx.x;
    double c = 0.0;
    uint64_t j = 0;
    while (j < nchunks) {
        const ChunkMap m = maps[j];
        const bool head = seg_head(maps, j);
        if (head && m.valid) {
            const SMap t = seg_total[j];
            double c2 = c;
            if (advance_exact(c2, m.e, t.inc0, t.inc1)) {
                if (lane == 0) seg_c[j] = c;
                c = c2;
                j += t.count;
                continue;
            }
        }
        // This chunk on its own.
        if (lane == 0) {
            cstart[j] = c;
            direct[j] = 1;
        }
        double c2 = c;
        if (m.valid && advance_exact(c2, m.e, m.inc0, m.inc1)) {
            c = c2;
            if (lane == 0) seq[j] = 0;
        } else {
            const uint64_t base = j * chunk;
            for (uint32_t i = lane; i < chunk; i += 32) buf[i] = (base + i < n_amps) ? prob(st[base + i]) : 0.0;
            __syncwarp();
            double cc = c;
            if (lane == 0)
                for (uint32_t i = 0; i < chunk; ++i) cc = __dadd_rn(cc, buf[i]);
            c = __shfl_sync(0xffffffffu, cc, 0);
            __syncwarp();
            if (lane == 0) seq[j] = 1;
        }
        ++j;
    }
    if (lane == 0) cstart[nchunks] = c;
}

__global__ void __launch_bounds__(kThreads) k_seg_fill(uint64_t nchunks, const ChunkMap* __restrict__ maps,
                                                       const SMap* __restrict__ excl,
                                                       const unsigned char* __restrict__ direct,
                                                       const double* __restrict__ seg_c, double* __restrict__ cstart,
                                                       unsigned char* __restrict__ seq) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= nchunks || direct[j]) return;
    const SMap x = excl[j];
    const uint64_t h = j - x.count;
    const double c = seg_c[h];
    const double u = ldexp(1.0, maps[j].e - 52);
    const long long M = static_cast<long long>(c / u);
    cstart[j] = static_cast<double>(M + ((M & 1) ? x.inc1 : x.inc0)) * u;
    seq[j] = 0;
}

// Number of sorted uniforms strictly below x.
__device__ __forceinline__ uint64_t count_below(const double* __restrict__ u, uint64_t shots, double x) {
    uint64_t lo = 0, hi = shots;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (u[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Each chunk boundary's shot index: bounds[j] = the uniforms below
// cstart[j] (j = 0..nchunks), one thread per boundary, so the searches'
// dependent loads overlap across the grid.
__global__ void k_shot_bounds(const double* __restrict__ cstart, uint64_t nchunks, const double* __restrict__ u,
                              uint64_t shots, uint64_t* __restrict__ bounds) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j <= nchunks) bounds[j] = count_below(u, shots, cstart[j]);
}

// Step E: per chunk, the exact running sums of its elements, then each of
// its shots placed on the first element whose sum exceeds the uniform.
template <typename A>
__global__ void __launch_bounds__(kThreads) k_assign(const A* __restrict__ st, uint64_t n_amps,
                                                     uint32_t chunk, const ChunkMap* __restrict__ maps,
                                                     const double* __restrict__ cstart,
                                                     const unsigned char* __restrict__ seq,
                                                     const double* __restrict__ u, const uint64_t* __restrict__ bounds,
                                                     uint64_t* __restrict__ basis) {
    __shared__ double cs[kSampleChunk];
    const uint64_t j = blockIdx.x;
    const uint64_t base = j * chunk;
    const double c0 = cstart[j];
    const uint64_t lo = bounds[j], hi = bounds[j + 1];
    if (lo >= hi) return;  // (uniform over the CTA)
    if (seq[j]) {
        // The reference's own adds, in order.
        for (uint32_t i = threadIdx.x; i < chunk; i += kThreads) cs[i] = (base + i < n_amps) ? prob(st[base + i]) : 0.0;
        __syncthreads();
        if (threadIdx.x == 0) {
            double c = c0;
            for (uint32_t i = 0; i < chunk; ++i) {
                c = __dadd_rn(c, cs[i]);
                cs[i] = c;
            }
        }
        __syncthreads();
    } else {
        // c_i = c0 + (prefix increment) * u: each thread composes its run,
        // the runs' maps are scanned in order, then each element's value.
        const ChunkMap m = maps[j];
        const double uu = ldexp(1.0, m.e - 52);
        const long long M0 = static_cast<long long>(c0 / uu);
        __shared__ PMap runs[kThreads];
        PMap acc{0, 0, 0, 1};
        const uint64_t my = base + static_cast<uint64_t>(threadIdx.x) * kPerThread;
        double p[kPerThread];
#pragma unroll
        for (int i = 0; i < kPerThread; ++i) {
            p[i] = (my + i < n_amps) ? prob(st[my + i]) : 0.0;
            acc = compose(acc, element_map(p[i], m.e));
        }
        // The runs' maps composed in thread order (exact integer maps, so
        // any grouping gives the same result): an inclusive scan within
        // each warp by shuffles, the warps' totals in order, then each
        // thread's exclusive prefix.
        const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
        PMap inc = acc;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            PMap prev;
            prev.inc0 = __shfl_up_sync(0xffffffffu, inc.inc0, o);
            prev.inc1 = __shfl_up_sync(0xffffffffu, inc.inc1, o);
            prev.par0 = __shfl_up_sync(0xffffffffu, inc.par0, o);
            prev.par1 = __shfl_up_sync(0xffffffffu, inc.par1, o);
            if (lane >= o) inc = compose(prev, inc);
        }
        if (lane == 31) runs[warp] = inc;
        __syncthreads();
        if (threadIdx.x == 0) {
            PMap run{0, 0, 0, 1};
            for (uint32_t w = 0; w < kThreads / 32; ++w) {
                const PMap v = runs[w];
                runs[w] = run;
                run = compose(run, v);
            }
        }
        __syncthreads();
        PMap ex;  // this thread's runs before it within the warp
        ex.inc0 = __shfl_up_sync(0xffffffffu, inc.inc0, 1);
        ex.inc1 = __shfl_up_sync(0xffffffffu, inc.inc1, 1);
        ex.par0 = __shfl_up_sync(0xffffffffu, inc.par0, 1);
        ex.par1 = __shfl_up_sync(0xffffffffu, inc.par1, 1);
        if (lane == 0) ex = PMap{0, 0, 0, 1};
        const PMap before = compose(runs[warp], ex);
        int par = static_cast<int>(M0 & 1);
        long long M = M0 + (par ? before.inc1 : before.inc0);
        par = static_cast<int>(M & 1);
#pragma unroll
        for (int i = 0; i < kPerThread; ++i) {
            const PMap em = element_map(p[i], m.e);
            M += par ? em.inc1 : em.inc0;
            par = static_cast<int>(M & 1);
            cs[threadIdx.x * kPerThread + i] = static_cast<double>(M) * uu;
        }
        __syncthreads();
    }
    for (uint64_t s = lo + threadIdx.x; s < hi; s += kThreads) {
        const double x = u[s];
        uint32_t a = 0, b = chunk;  // first i with x < cs[i]
        while (a < b) {
            const uint32_t mid = (a + b) >> 1;
            if (x < cs[mid]) b = mid;
            else a = mid + 1;
        }
        basis[s] = base + a;
    }
}

// Shots at or past the final sum go to the last basis state.
__global__ void k_leftover(const uint64_t* __restrict__ bounds, uint64_t nchunks, uint64_t shots, uint64_t last,
                           uint64_t* __restrict__ basis) {
    for (uint64_t s = bounds[nchunks] + threadIdx.x; s < shots; s += blockDim.x) basis[s] = last;
}

}  // namespace

size_t sample_scratch_bytes(uint32_t n, uint64_t shots) {
    const uint64_t na = uint64_t{1} << n;
    const uint32_t chunk = static_cast<uint32_t>(na < kSampleChunk ? na : kSampleChunk);
    const uint64_t nchunks = na / chunk;
    auto al = [](size_t b) { return (b + 255) & ~size_t{255}; };
    (void)shots;
    return 2 * al(nchunks * 8) + al((nchunks + 1) * 8) + al(nchunks * sizeof(ChunkMap)) + al(nchunks) +
           2 * al(nchunks * sizeof(SMap)) + al(nchunks) + al(nchunks * 8) + al((nchunks + 1) * 8);
}

template <typename A>
int launch_sample_t(const void* amps, uint32_t n, const double* dev_uniforms_sorted, uint64_t shots, void* scratch,
                    uint64_t* dev_basis, void* stream) {
    const auto s = static_cast<cudaStream_t>(stream);
    const auto* st = static_cast<const A*>(amps);
    const uint64_t na = uint64_t{1} << n;
    const uint32_t chunk = static_cast<uint32_t>(na < kSampleChunk ? na : kSampleChunk);
    const uint64_t nchunks = na / chunk;
    auto al = [](size_t b) { return (b + 255) & ~size_t{255}; };
    auto* p = static_cast<unsigned char*>(scratch);
    auto* sums = reinterpret_cast<double*>(p);
    p += al(nchunks * 8);
    auto* starts = reinterpret_cast<double*>(p);
    p += al(nchunks * 8);
    auto* cst = reinterpret_cast<double*>(p);
    p += al((nchunks + 1) * 8);
    auto* maps = reinterpret_cast<ChunkMap*>(p);
    p += al(nchunks * sizeof(ChunkMap));
    auto* seq = reinterpret_cast<unsigned char*>(p);
    p += al(nchunks);
    auto* excl = reinterpret_cast<SMap*>(p);
    p += al(nchunks * sizeof(SMap));
    auto* seg_total = reinterpret_cast<SMap*>(p);
    p += al(nchunks * sizeof(SMap));
    auto* direct = reinterpret_cast<unsigned char*>(p);
    p += al(nchunks);
    auto* seg_c = reinterpret_cast<double*>(p);
    p += al(nchunks * 8);
    auto* bounds = reinterpret_cast<uint64_t*>(p);
    k_chunk_sums<<<static_cast<unsigned>(nchunks), kThreads, 0, s>>>(st, na, chunk, sums);
    k_scan_sums<<<1, 1024, 0, s>>>(sums, nchunks, starts);
    k_chunk_maps<<<static_cast<unsigned>(nchunks), kThreads, 0, s>>>(st, na, chunk, starts, sums, maps);
    cudaMemsetAsync(direct, 0, nchunks, s);
    k_seg_scan<<<1, 1024, 0, s>>>(maps, nchunks, excl, seg_total);
    k_seg_chain<<<1, 32, 0, s>>>(st, na, chunk, nchunks, maps, seg_total, cst, seq, direct, seg_c);
    k_seg_fill<<<static_cast<unsigned>((nchunks + kThreads - 1) / kThreads), kThreads, 0, s>>>(nchunks, maps, excl,
                                                                                                direct, seg_c, cst,
                                                                                                seq);
    k_shot_bounds<<<static_cast<unsigned>((nchunks + 1 + kThreads - 1) / kThreads), kThreads, 0, s>>>(
        cst, nchunks, dev_uniforms_sorted, shots, bounds);
    k_assign<<<static_cast<unsigned>(nchunks), kThreads, 0, s>>>(st, na, chunk, maps, cst, seq,
                                                                 dev_uniforms_sorted, bounds, dev_basis);
    k_leftover<<<1, 256, 0, s>>>(bounds, nchunks, shots, na - 1, dev_basis);
    return launch_status();
}

// The exact chain alone (steps A-D): the reference's sequential sum of
// |a_i|^2 over the whole state is its final value, cstart[nchunks].
template <typename A>
int launch_exact_norm_t(const void* amps, uint32_t n, void* scratch, double* host_total, void* stream) {
    const auto s = static_cast<cudaStream_t>(stream);
    const auto* st = static_cast<const A*>(amps);
    const uint64_t na = uint64_t{1} << n;
    const uint32_t chunk = static_cast<uint32_t>(na < kSampleChunk ? na : kSampleChunk);
    const uint64_t nchunks = na / chunk;
    auto al = [](size_t b) { return (b + 255) & ~size_t{255}; };
    auto* p = static_cast<unsigned char*>(scratch);
    auto* sums = reinterpret_cast<double*>(p);
    p += al(nchunks * 8);
    auto* starts = reinterpret_cast<double*>(p);
    p += al(nchunks * 8);
    auto* cst = reinterpret_cast<double*>(p);
    p += al((nchunks + 1) * 8);
    auto* maps = reinterpret_cast<ChunkMap*>(p);
    p += al(nchunks * sizeof(ChunkMap));
    auto* seq = reinterpret_cast<unsigned char*>(p);
    p += al(nchunks);
    auto* excl = reinterpret_cast<SMap*>(p);
    p += al(nchunks * sizeof(SMap));
    auto* seg_total = reinterpret_cast<SMap*>(p);
    p += al(nchunks * sizeof(SMap));
    auto* direct = reinterpret_cast<unsigned char*>(p);
    p += al(nchunks);
    auto* seg_c = reinterpret_cast<double*>(p);
    k_chunk_sums<<<static_cast<unsigned>(nchunks), kThreads, 0, s>>>(st, na, chunk, sums);
    k_scan_sums<<<1, 1024, 0, s>>>(sums, nchunks, starts);
    k_chunk_maps<<<static_cast<unsigned>(nchunks), kThreads, 0, s>>>(st, na, chunk, starts, sums, maps);
    cudaMemsetAsync(direct, 0, nchunks, s);
    k_seg_scan<<<1, 1024, 0, s>>>(maps, nchunks, excl, seg_total);
    k_seg_chain<<<1, 32, 0, s>>>(st, na, chunk, nchunks, maps, seg_total, cst, seq, direct, seg_c);
    k_seg_fill<<<static_cast<unsigned>((nchunks + kThreads - 1) / kThreads), kThreads, 0, s>>>(nchunks, maps, excl,
                                                                                                direct, seg_c, cst,
                                                                                                seq);
    if (int rc = launch_status(); rc != MB2_OK) return rc;
    if (cudaMemcpyAsync(host_total, cst + nchunks, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return record_cuda_error(static_cast<int>(cudaGetLastError()));
    return MB2_OK;
}

int launch_exact_norm(const void* amps, uint32_t n, void* scratch, double* host_total, void* stream, int precision) {
    note_launches(6);
    return precision == MB2_C64 ? launch_exact_norm_t<float2>(amps, n, scratch, host_total, stream)
                                : launch_exact_norm_t<double2>(amps, n, scratch, host_total, stream);
}

int launch_sample(const void* amps, uint32_t n, const double* dev_uniforms_sorted, uint64_t shots, void* scratch,
                  uint64_t* dev_basis, void* stream, int precision) {
    note_launches(9);
    return precision == MB2_C64
               ? launch_sample_t<float2>(amps, n, dev_uniforms_sorted, shots, scratch, dev_basis, stream)
               : launch_sample_t<double2>(amps, n, dev_uniforms_sorted, shots, scratch, dev_basis, stream);
}

}  // namespace mb2
