// The serving loop: continuous batching of circuit requests on one GPU.
//
// Requests (any qubit count and depth, counts or <H>) arrive through
// mb2_server_submit at any time.  `slots` worker threads each own a CUDA
// stream; a worker takes the oldest pending request whose device memory
// (state + staging) fits what is left of the admission budget, runs it on
// its stream -- init, the tiled sweep, then the device sampler or the Pauli
// reduction -- and posts a completion.  Requests that arrive while others run
// are admitted as soon as a slot and memory free up, and their kernels run
// concurrently on the device.  Every kernel's result is independent of what
// else runs (fixed grids, fixed reduction orders), so a request's result is
// the same alone and in the mix.
//
// Admission mirrors the reference's two-level budget check: the job's own
// budget (the state must fit, else MB2_ERR_RESOURCE, src/engines/dense/
// state_vector.cpp:16-28) and a ledger of bytes currently held
// (src/common/memory_ledger.h:37-117), here the device budget of the server.
// An oldest request that has waited longer than the starvation limit stops
// smaller ones from being admitted ahead of it until it fits.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

#include "mb2_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    std::vector<mb2_op> ops;
    std::vector<std::vector<double>> matrices;
    uint32_t n = 0;
    double global_phase = 0.0;
    int32_t fuse = 1;
    int32_t output = MB2_OUT_EXPECTATION;
    int32_t precision = MB2_C128;
    uint64_t shots = 0, seed = 0;
    std::vector<uint32_t> targets;
    std::vector<uint64_t> xs, zs;
    std::vector<double> coefs;
    uint64_t bytes = 0;  // admission charge
    Clock::time_point submitted;
};

struct Done {
    mb2_completion c{};
    std::vector<uint64_t> outcomes, counts;
};

// What a request holds on the device while it runs: its state and the
// state's staging buffer at its largest (the same layout and rounding the
// engine's calls use), each allocation rounded up to the stream-ordered
// pool's 2 MiB granularity.
// Requests of 4..16 qubits run as part of a batch (run_small_batch) in
// complex128, whatever precision they ask for: their states are a few CTAs'
// work, so their cost is the launches and calls around them, which a batch
// shares; complex128 costs them nothing more and is the reference's result.
constexpr uint32_t kSmallMinQubits = 4, kSmallMaxQubits = 16, kSmallBatchMax = 64;
bool small_request(const Request& r) { return r.n >= kSmallMinQubits && r.n <= kSmallMaxQubits; }

uint64_t admission_bytes(const Request& r) {
    auto pool = [](uint64_t v) { return (v + (2ull << 20) - 1) & ~((2ull << 20) - 1); };
    const uint64_t state = (uint64_t{1} << r.n) * (r.precision == MB2_C64 && !small_request(r) ? 8 : 16);
    const uint64_t staging =
        mb2::scratch_bound(r.n, r.ops.data(), static_cast<uint32_t>(r.ops.size()),
                           r.output == MB2_OUT_COUNTS ? r.shots : 0,
                           r.output == MB2_OUT_EXPECTATION ? static_cast<uint32_t>(r.xs.size()) + 1 : 1);
    return pool(state) + pool(staging);
}

}  // namespace

struct mb2_server {
    mb2_context* ctx = nullptr;
    uint64_t budget = 0;
    uint64_t held = 0;
    double starvation_s = 0.5;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> pending;
    std::deque<Done> done;
    std::map<uint64_t, Done> released_wait;  // completions handed out, their arrays alive until release
    uint64_t next_ticket = 1;
    bool stop = false;
    uint32_t in_flight = 0;
    std::vector<std::thread> workers;
    std::vector<cudaStream_t> streams;
    // The caller's memory ledger (mb2_server_set_ledger), or none.
    mb2_ledger_charge_fn ledger_charge = nullptr;
    mb2_ledger_release_fn ledger_release = nullptr;
    void* ledger_user = nullptr;
};

namespace {

// Whether a request of `bytes` can be admitted now: it fits what is left of
// the budget and the caller's ledger (if any) takes the bytes -- a charge
// that succeeds is kept, so call this only for a request about to be admitted.
bool admit(mb2_server* s, uint64_t bytes) {
    if (s->held + bytes > s->budget) return false;
    return s->ledger_charge == nullptr || s->ledger_charge(s->ledger_user, bytes) != 0;
}

// The oldest pending request that can be admitted; none if the oldest has
// waited past the starvation limit and cannot be.
bool pick(mb2_server* s, Request& out) {
    if (s->pending.empty()) return false;
    auto take = [&](std::deque<Request>::iterator it) {
        out = std::move(*it);
        s->pending.erase(it);
        s->held += out.bytes;
        return true;
    };
    if (admit(s, s->pending.front().bytes)) return take(s->pending.begin());
    const double head_wait = std::chrono::duration<double>(Clock::now() - s->pending.front().submitted).count();
    if (head_wait > s->starvation_s) return false;
    for (auto it = s->pending.begin() + 1; it != s->pending.end(); ++it)
        if (admit(s, it->bytes)) return take(it);
    return false;
}

void run_request(mb2_server* s, cudaStream_t stream, Request& r, Done& d) {
    mb2_state* st = nullptr;
    int rc = mb2::state_on_stream(s->ctx, r.n, ~uint64_t{0}, stream, &st, r.precision);
    if (rc == MB2_OK) rc = mb2_init(st, r.global_phase);
    if (rc == MB2_OK) {
        mb2_sweep_options o{r.fuse, 0, 0, 0, 0, 0};
        rc = mb2_apply_program(st, r.ops.data(), static_cast<uint32_t>(r.ops.size()), &o);
    }
    // A complex64 state is renormalised in FP64 (its norm drifts by FP32
    // roundings over a deep circuit): <H> is divided by the norm, read in the
    // same grouped pass as the terms (the identity term); counts are drawn
    // from the rescaled state.  complex128 results stay the reference's.
    const bool c64 = r.precision == MB2_C64;
    if (rc == MB2_OK && r.output == MB2_OUT_EXPECTATION) {
        std::vector<uint64_t> xs(r.xs), zs(r.zs);
        if (c64) {
            xs.push_back(0);
            zs.push_back(0);
        }
        std::vector<double> terms(2 * xs.size());
        rc = mb2_expectation(st, xs.data(), zs.data(), static_cast<uint32_t>(xs.size()), terms.data());
        double total = 0.0;
        for (size_t t = 0; t < r.xs.size() && rc == MB2_OK; ++t) total += r.coefs[t] * terms[2 * t];
        if (c64 && rc == MB2_OK) total /= terms[2 * r.xs.size()];
        d.c.value = total;
    } else if (rc == MB2_OK && r.output == MB2_OUT_COUNTS) {
        if (c64) rc = mb2_normalize(st, nullptr);
        d.outcomes.resize(std::max<uint64_t>(1, r.shots));
        d.counts.resize(std::max<uint64_t>(1, r.shots));
        uint64_t distinct = d.outcomes.size();
        if (rc == MB2_OK)
            rc = mb2_sample(st, r.shots, r.seed, r.targets.data(), static_cast<uint32_t>(r.targets.size() / 2),
                            d.outcomes.data(), d.counts.data(), &distinct);
        d.outcomes.resize(rc == MB2_OK ? distinct : 0);
        d.counts.resize(rc == MB2_OK ? distinct : 0);
        d.c.num_outcomes = rc == MB2_OK ? distinct : 0;
    }
    if (st != nullptr) mb2_state_free(st);
    d.c.status = rc;
}

// Another pending small request that can be admitted now (no starvation
// rule: the batch only gathers what is already waiting).
bool pick_small(mb2_server* s, Request& out) {
    for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
        if (!small_request(*it)) continue;
        if (!admit(s, it->bytes)) continue;
        out = std::move(*it);
        s->pending.erase(it);
        s->held += out.bytes;
        return true;
    }
    return false;
}

// Small requests together, each step one launch for all of them: the states
// (complex128) in one allocation, zeroed with one memset and given their
// initial phase by one launch; pass p of every request's tiled program in
// one launch per tile width (k_tile_pass_jobs, a CTA per tile); every Pauli
// term of every expectation request in one launch; every counts request's
// exact walk in one launch; one upload and one download.  Each state's
// arithmetic is that of mb2_apply_program (bitwise), its counts the same
// walk over the same sorted uniforms as mb2_sample (identical), its terms a
// fixed-order reduction (within 1e-12 of the reference).
void run_small_batch(mb2_server* s, cudaStream_t stream, std::vector<Request>& batch, std::vector<Done>& dones) {
    const size_t B = batch.size();
    dones.assign(B, Done{});
    for (size_t i = 0; i < B; ++i) dones[i].c.ticket = batch[i].ticket;
    std::vector<mb2::TileProgram> progs(B);
    std::vector<uint32_t> tile(B, 0);
    std::vector<bool> ok(B, true);
    for (size_t i = 0; i < B; ++i) {
        const Request& r = batch[i];
        try {
            const std::vector<mb2::Block> blocks =
                mb2::build_blocks(r.ops.data(), static_cast<uint32_t>(r.ops.size()), r.fuse != 0);
            uint32_t m = std::min<uint32_t>(mb2::kMaxTileQubits, r.n);
            for (const mb2::Block& b : blocks) m = std::max(m, b.k);
            if (m > r.n) throw std::invalid_argument("a block wider than the state");
            progs[i] = mb2::plan_tile_program(blocks, r.n, m, mb2::kDefaultFixedLow, nullptr, false);
            mb2::encode_compact(progs[i]);
            tile[i] = std::min(m, r.n);
        } catch (const std::exception&) {
            ok[i] = false;
            dones[i].c.status = MB2_ERR_INVALID;
        }
    }
    // Device layout: [uploaded: programs, job tables, init table, uniforms]
    // [states] [written: terms, basis].
    auto up = [](size_t v) { return (v + 255) & ~size_t{255}; };
    size_t off = 0;
    std::vector<size_t> w_off(B), d_off(B), g_off(B), u_off(B, 0), st_off(B), b_off(B, 0);
    for (size_t i = 0; i < B; ++i) {
        if (!ok[i]) continue;
        w_off[i] = off;
        off = up(off + progs[i].words.size() * 4);
        d_off[i] = off;
        off = up(off + progs[i].data.size() * 8);
        g_off[i] = off;
        off = up(off + progs[i].gdata.size() * 8);
    }
    // Tile jobs, grouped by (pass index, tile width).
    struct Launch {
        uint32_t m, count, ctas;
        size_t off, smem;
    };
    std::vector<Launch> launches;
    std::vector<mb2::TileJob> jobs;  // device pointers filled in after allocation
    std::vector<size_t> job_req;     // job -> request
    std::vector<uint32_t> job_pass;  // job -> pass index
    size_t max_passes = 0;
    for (size_t i = 0; i < B; ++i)
        if (ok[i]) max_passes = std::max(max_passes, progs[i].passes.size());
    for (size_t p = 0; p < max_passes; ++p) {
        for (uint32_t m = mb2::kMinTileQubits; m <= mb2::kMaxTileQubits; ++m) {
            Launch L{m, 0, 0, 0, 0};
            const size_t first = jobs.size();
            for (size_t i = 0; i < B; ++i) {
                if (!ok[i] || tile[i] != m || p >= progs[i].passes.size()) continue;
                const mb2::TilePass& tp = progs[i].passes[p];
                mb2::TileJob J{};
                J.smask = tp.smask;
                J.gmask = tp.gmask;
                J.ntiles = uint64_t{1} << (batch[i].n - tp.m);
                J.n = batch[i].n;
                J.nwords = tp.word_count;
                J.nsdata = tp.sdata_count;
                J.cta_begin = L.ctas;
                J.nctas = static_cast<uint32_t>(J.ntiles);
                L.ctas += J.nctas;
                L.smem = std::max(L.smem, 2 * (size_t{1} << m) * 16 + size_t{tp.word_count} * 4 + size_t{tp.sdata_count} * 8);
                jobs.push_back(J);
                job_req.push_back(i);
                job_pass.push_back(static_cast<uint32_t>(p));
                ++L.count;
            }
            if (L.count == 0) continue;
            L.off = first;  // job index for now
            launches.push_back(L);
        }
    }
    const size_t jobs_off = off;
    off = up(off + jobs.size() * sizeof(mb2::TileJob));
    const size_t init_off = off;
    off = up(off + B * 8);
    const size_t initv_off = off;
    off = up(off + B * 16);
    std::vector<mb2::ExpectJob> ejobs;
    std::vector<size_t> e_first(B, 0);
    std::vector<mb2::WalkJob> wjobs;
    std::vector<std::vector<double>> uniforms(B);
    for (size_t i = 0; i < B; ++i) {
        if (!ok[i]) continue;
        const Request& r = batch[i];
        if (r.output == MB2_OUT_EXPECTATION) {
            e_first[i] = ejobs.size();
            for (size_t t = 0; t < r.xs.size(); ++t) ejobs.push_back(mb2::ExpectJob{nullptr, r.xs[t], r.zs[t], r.n, 0});
        } else if (r.shots > 0) {
            uniforms[i] = mb2::sorted_reference_uniforms(r.shots, r.seed);
            u_off[i] = off;
            off = up(off + r.shots * 8);
        }
    }
    const size_t ejobs_off = off;
    off = up(off + ejobs.size() * sizeof(mb2::ExpectJob));
    size_t nwalk = 0;
    for (size_t i = 0; i < B; ++i)
        if (ok[i] && batch[i].output == MB2_OUT_COUNTS && batch[i].shots > 0) ++nwalk;
    const size_t wjobs_off = off;
    off = up(off + nwalk * sizeof(mb2::WalkJob));
    const size_t upload_bytes = off;
    const size_t states_off = off;
    for (size_t i = 0; i < B; ++i) {
        st_off[i] = off;
        off = up(off + (ok[i] ? (size_t{16} << batch[i].n) : 0));
    }
    const size_t states_bytes = off - states_off;
    const size_t eout_off = off;
    off = up(off + ejobs.size() * 16);
    const size_t basis_off = off;
    for (size_t i = 0; i < B; ++i)
        if (u_off[i] != 0 || (ok[i] && batch[i].output == MB2_OUT_COUNTS && batch[i].shots > 0)) {
            b_off[i] = off;
            off = up(off + batch[i].shots * 8);
        }
    const size_t total = off;
    auto fail_all = [&](int rc) {
        for (size_t i = 0; i < B; ++i)
            if (dones[i].c.status == MB2_OK) dones[i].c.status = rc;
    };
    unsigned char* dev = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&dev), total, stream) != cudaSuccess) {
        cudaGetLastError();
        fail_all(MB2_ERR_RESOURCE);
        return;
    }
    std::vector<unsigned char> host(upload_bytes, 0);
    for (size_t i = 0; i < B; ++i) {
        if (!ok[i]) continue;
        std::memcpy(host.data() + w_off[i], progs[i].words.data(), progs[i].words.size() * 4);
        if (!progs[i].data.empty()) std::memcpy(host.data() + d_off[i], progs[i].data.data(), progs[i].data.size() * 8);
        if (!progs[i].gdata.empty())
            std::memcpy(host.data() + g_off[i], progs[i].gdata.data(), progs[i].gdata.size() * 8);
        if (!uniforms[i].empty()) std::memcpy(host.data() + u_off[i], uniforms[i].data(), uniforms[i].size() * 8);
    }
    for (size_t j = 0; j < jobs.size(); ++j) {
        const size_t i = job_req[j];
        const mb2::TilePass& tp = progs[i].passes[job_pass[j]];
        jobs[j].st = dev + st_off[i];
        jobs[j].words = reinterpret_cast<const uint32_t*>(dev + w_off[i]) + tp.word_begin;
        jobs[j].sdata = reinterpret_cast<const double*>(dev + d_off[i]) + tp.sdata_begin;
        jobs[j].gdata = reinterpret_cast<const double*>(dev + g_off[i]);
    }
    if (!jobs.empty()) std::memcpy(host.data() + jobs_off, jobs.data(), jobs.size() * sizeof(mb2::TileJob));
    auto* init_offsets = reinterpret_cast<uint64_t*>(host.data() + init_off);
    auto* init_vals = reinterpret_cast<double*>(host.data() + initv_off);
    uint32_t ninit = 0;
    for (size_t i = 0; i < B; ++i) {
        if (!ok[i]) continue;
        const mb2::Cd ph = mb2::initial_phase(batch[i].global_phase);
        init_offsets[ninit] = (st_off[i] - states_off) / 16;
        init_vals[2 * ninit] = ph.real();
        init_vals[2 * ninit + 1] = ph.imag();
        ++ninit;
    }
    for (size_t i = 0; i < B; ++i)
        if (ok[i] && batch[i].output == MB2_OUT_EXPECTATION)
            for (size_t t = 0; t < batch[i].xs.size(); ++t) ejobs[e_first[i] + t].st = dev + st_off[i];
    if (!ejobs.empty()) std::memcpy(host.data() + ejobs_off, ejobs.data(), ejobs.size() * sizeof(mb2::ExpectJob));
    for (size_t i = 0; i < B; ++i)
        if (ok[i] && batch[i].output == MB2_OUT_COUNTS && batch[i].shots > 0)
            wjobs.push_back(mb2::WalkJob{dev + st_off[i], reinterpret_cast<const double*>(dev + u_off[i]),
                                         reinterpret_cast<uint64_t*>(dev + b_off[i]), batch[i].shots, batch[i].n, 0});
    if (!wjobs.empty()) std::memcpy(host.data() + wjobs_off, wjobs.data(), wjobs.size() * sizeof(mb2::WalkJob));
    int rc = MB2_OK;
    if (cudaMemcpyAsync(dev, host.data(), upload_bytes, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
        cudaMemsetAsync(dev + states_off, 0, states_bytes, stream) != cudaSuccess)
        rc = mb2::record_cuda_error(static_cast<int>(cudaGetLastError()));
    if (rc == MB2_OK)
        rc = mb2::launch_init_jobs(dev + states_off, reinterpret_cast<const uint64_t*>(dev + init_off),
                                   reinterpret_cast<const double*>(dev + initv_off), ninit, stream);
    for (const Launch& L : launches) {
        if (rc != MB2_OK) break;
        rc = mb2::launch_tile_jobs(reinterpret_cast<const mb2::TileJob*>(dev + jobs_off) + L.off, L.count, L.ctas,
                                   L.m, L.smem, stream);
    }
    if (rc == MB2_OK)
        rc = mb2::launch_expect_jobs(reinterpret_cast<const mb2::ExpectJob*>(dev + ejobs_off),
                                     static_cast<uint32_t>(ejobs.size()), reinterpret_cast<double*>(dev + eout_off),
                                     stream);
    if (rc == MB2_OK)
        rc = mb2::launch_walk_jobs(reinterpret_cast<const mb2::WalkJob*>(dev + wjobs_off),
                                   static_cast<uint32_t>(wjobs.size()), stream);
    std::vector<double> eout(2 * ejobs.size());
    std::vector<uint64_t> basis((total - basis_off) / 8);
    if (rc == MB2_OK) {
        if ((!eout.empty() && cudaMemcpyAsync(eout.data(), dev + eout_off, eout.size() * 8, cudaMemcpyDeviceToHost,
                                              stream) != cudaSuccess) ||
            (!basis.empty() && cudaMemcpyAsync(basis.data(), dev + basis_off, basis.size() * 8,
                                               cudaMemcpyDeviceToHost, stream) != cudaSuccess) ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            rc = mb2::record_cuda_error(static_cast<int>(cudaGetLastError()));
    }
    cudaFreeAsync(dev, stream);
    if (rc != MB2_OK) {
        fail_all(rc);
        return;
    }
    for (size_t i = 0; i < B; ++i) {
        if (!ok[i]) continue;
        const Request& r = batch[i];
        Done& d = dones[i];
        if (r.output == MB2_OUT_EXPECTATION) {
            double total_h = 0.0;
            for (size_t t = 0; t < r.xs.size(); ++t) total_h += r.coefs[t] * eout[2 * (e_first[i] + t)];
            d.c.value = total_h;
        } else if (r.shots > 0) {
            const size_t first = (b_off[i] - basis_off) / 8;
            const std::vector<uint64_t> bs(basis.begin() + static_cast<long>(first),
                                           basis.begin() + static_cast<long>(first + r.shots));
            d.outcomes.resize(r.shots);
            d.counts.resize(r.shots);
            uint64_t distinct = r.shots;
            const int hr = mb2::counts_of(s->ctx, r.n, bs, r.targets.data(), static_cast<uint32_t>(r.targets.size() / 2),
                                          d.outcomes.data(), d.counts.data(), &distinct);
            d.outcomes.resize(hr == MB2_OK ? distinct : 0);
            d.counts.resize(hr == MB2_OK ? distinct : 0);
            d.c.num_outcomes = hr == MB2_OK ? distinct : 0;
            d.c.status = hr;
        }
    }
}

void worker(mb2_server* s, uint32_t slot) {
    cudaSetDevice(mb2::context_device(s->ctx));
    for (;;) {
        Request r;
        Clock::time_point admitted;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // With a ledger, memory can free up outside the server: look again
            // every few milliseconds as well as on submits and completions.
            auto ready = [&] { return s->stop || pick(s, r); };
            if (s->ledger_charge == nullptr) s->cv_work.wait(lk, ready);
            else
                while (!s->cv_work.wait_for(lk, std::chrono::milliseconds(4), ready)) {
                }
            if (r.ticket == 0) return;  // stopped with nothing picked
            admitted = Clock::now();
            ++s->in_flight;
        }
        std::vector<Request> batch;
        batch.push_back(std::move(r));
        if (small_request(batch[0])) {  // gather the small requests already waiting
            std::lock_guard<std::mutex> lk(s->mu);
            Request more;
            while (batch.size() < kSmallBatchMax && pick_small(s, more)) {
                batch.push_back(std::move(more));
                ++s->in_flight;
            }
        }
        std::vector<Done> dones;
        if (small_request(batch[0])) {
            run_small_batch(s, s->streams[slot], batch, dones);
        } else {
            dones.resize(1);
            dones[0].c.ticket = batch[0].ticket;
            run_request(s, s->streams[slot], batch[0], dones[0]);
        }
        const auto finished = Clock::now();
        for (size_t i = 0; i < batch.size(); ++i) {
            dones[i].c.queue_seconds = std::chrono::duration<double>(admitted - batch[i].submitted).count();
            dones[i].c.latency_seconds = std::chrono::duration<double>(finished - batch[i].submitted).count();
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t i = 0; i < batch.size(); ++i) {
                s->held -= batch[i].bytes;
                if (s->ledger_release != nullptr) s->ledger_release(s->ledger_user, batch[i].bytes);
                --s->in_flight;
                s->done.push_back(std::move(dones[i]));
            }
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();  // memory freed: others may fit now
    }
}

}  // namespace

extern "C" {

int mb2_server_create(mb2_context* ctx, const mb2_server_options* opts, mb2_server** out) {
    if (ctx == nullptr || out == nullptr) return MB2_ERR_INVALID;
    *out = nullptr;
    mb2_server_options o{0, 0, 0};
    if (opts != nullptr) o = *opts;
    uint64_t free_b = 0, total_b = 0;
    if (mb2_device_info(ctx, nullptr, &total_b, &free_b) != MB2_OK) return MB2_ERR_CUDA;
    cudaSetDevice(mb2::context_device(ctx));
    auto* s = new mb2_server;
    s->ctx = ctx;
    s->budget = o.device_budget_bytes != 0 ? std::min<uint64_t>(o.device_budget_bytes, free_b) : (free_b / 10) * 9;
    const uint32_t slots = o.slots != 0 ? std::min<uint32_t>(o.slots, 64) : 16;
    for (uint32_t i = 0; i < slots; ++i) {
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
            delete s;
            return MB2_ERR_CUDA;
        }
        s->streams.push_back(st);
    }
    // The admission budget is mapped into the device's stream-ordered pool
    // once, up front (the pool keeps freed memory, and the server gives it
    // back when it is destroyed): requests then take memory that is already
    // mapped, instead of the first ones mapping fresh memory while others
    // run.  A budget the pool cannot map at once is simply not warmed.
    {
        void* p = nullptr;
        if (cudaMallocAsync(&p, s->budget, s->streams[0]) == cudaSuccess) cudaFreeAsync(p, s->streams[0]);
        else cudaGetLastError();
        cudaStreamSynchronize(s->streams[0]);
    }
    for (uint32_t i = 0; i < slots; ++i) s->workers.emplace_back(worker, s, i);
    *out = s;
    return MB2_OK;
}

int mb2_server_submit(mb2_server* s, const mb2_request* q, uint64_t* ticket) {
    if (s == nullptr || q == nullptr || ticket == nullptr || (q->ops == nullptr && q->num_ops != 0))
        return MB2_ERR_INVALID;
    if (q->num_qubits < 1 || q->num_qubits > 34) return MB2_ERR_INVALID;
    if (q->output != MB2_OUT_COUNTS && q->output != MB2_OUT_EXPECTATION) return MB2_ERR_INVALID;
    Request r;
    r.n = q->num_qubits;
    r.global_phase = q->global_phase;
    r.fuse = q->fuse_gates;
    r.output = q->output;
    if (q->precision != MB2_C128 && q->precision != MB2_C64) return MB2_ERR_INVALID;
    r.precision = q->precision;
    r.shots = q->shots;
    r.seed = q->seed;
    r.ops.assign(q->ops, q->ops + q->num_ops);
    for (mb2_op& o : r.ops) {  // own the unitary matrices
        if (o.opcode != MB2_UNITARY || o.matrix == nullptr) continue;
        const size_t len = 2ull << (2 * o.num_qubits);
        r.matrices.emplace_back(o.matrix, o.matrix + len);
        o.matrix = r.matrices.back().data();
    }
    if (q->output == MB2_OUT_COUNTS) {
        if (q->num_targets > 0 && q->targets == nullptr) return MB2_ERR_INVALID;
        r.targets.assign(q->targets, q->targets + 2 * q->num_targets);
    } else {
        if (q->num_terms > 0 && (!q->x_masks || !q->z_masks || !q->coefs)) return MB2_ERR_INVALID;
        r.xs.assign(q->x_masks, q->x_masks + q->num_terms);
        r.zs.assign(q->z_masks, q->z_masks + q->num_terms);
        r.coefs.assign(q->coefs, q->coefs + q->num_terms);
    }
    r.bytes = admission_bytes(r);
    r.submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (r.bytes > s->budget) return MB2_ERR_RESOURCE;  // can never be admitted
        if (s->stop) return MB2_ERR_INVALID;
        r.ticket = s->next_ticket++;
        *ticket = r.ticket;
        s->pending.push_back(std::move(r));
    }
    s->cv_work.notify_one();
    return MB2_OK;
}

int mb2_server_poll(mb2_server* s, mb2_completion* out, uint32_t capacity, uint32_t* count, uint32_t timeout_ms) {
    if (s == nullptr || count == nullptr || (capacity > 0 && out == nullptr)) return MB2_ERR_INVALID;
    *count = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && timeout_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !s->done.empty(); });
    while (!s->done.empty() && *count < capacity) {
        Done d = std::move(s->done.front());
        s->done.pop_front();
        auto& kept = s->released_wait[d.c.ticket];
        kept = std::move(d);
        kept.c.outcomes = kept.outcomes.empty() ? nullptr : kept.outcomes.data();
        kept.c.counts = kept.counts.empty() ? nullptr : kept.counts.data();
        out[(*count)++] = kept.c;
    }
    return *count > 0 ? MB2_OK : MB2_ERR_TIMEOUT;
}

int mb2_server_set_ledger(mb2_server* s, mb2_ledger_charge_fn charge, mb2_ledger_release_fn release, void* user) {
    if (s == nullptr || (charge == nullptr) != (release == nullptr)) return MB2_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->in_flight != 0) return MB2_ERR_INVALID;  // charges already taken would be released elsewhere
    s->ledger_charge = charge;
    s->ledger_release = release;
    s->ledger_user = user;
    return MB2_OK;
}

int mb2_server_release(mb2_server* s, uint64_t ticket) {
    if (s == nullptr) return MB2_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    return s->released_wait.erase(ticket) ? MB2_OK : MB2_ERR_INVALID;
}

int mb2_server_stats(mb2_server* s, uint64_t* pending, uint64_t* in_flight, uint64_t* held_bytes,
                     uint64_t* budget_bytes) {
    if (s == nullptr) return MB2_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (pending) *pending = s->pending.size();
    if (in_flight) *in_flight = s->in_flight;
    if (held_bytes) *held_bytes = s->held;
    if (budget_bytes) *budget_bytes = s->budget;
    return MB2_OK;
}

int mb2_server_destroy(mb2_server* s) {
    if (s == nullptr) return MB2_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->pending.clear();
    }
    s->cv_work.notify_all();
    for (auto& w : s->workers) w.join();
    for (cudaStream_t st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    // Return the pool's unused memory (the warmed budget) to the device.
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, mb2::context_device(s->ctx)) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    delete s;
    return MB2_OK;
}

}  // extern "C"
