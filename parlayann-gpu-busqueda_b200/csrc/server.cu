// server.cu -- pgb_server_*: a continuous-batching request loop over a flat-graph or an
// HNSW index. (HNSW: each context holds an HNSW searcher state prepared for max_beam, and a
// batch runs as one HNSW launch with each query at its own (Ls, k).)
//
// Host side: submit() admits a request into a bounded slot pool (busy when full) and
// wakes the dispatcher thread. The dispatcher completes finished launches (event query),
// then packs the pending requests into batches -- longest beam first -- and launches each
// on a free stream context: one upload of the packed queries and per-request (Ls, k) and
// one work-queue launch of the batched kernel (the grid shrinks to the batch), which
// writes each query's outputs into the context's page-locked host buffers and then sets
// the query's completion flag there. The dispatcher publishes a request as soon as its
// flag is set, so a short query does not wait for the longest one of its batch; the
// launch's event frees the context. New arrivals start while earlier launches are still
// on the GPU, and their work overlaps on the device. Every request runs the same
// per-query code as the plain searcher, so its answer does not depend on the mix.
//
// Locking: one mutex guards the pending queue, the free-slot list, the counters and the
// contexts' busy state, and is held only for those short updates. Packing, launching and
// copying results run outside it. A ticket names its slot (generation << 32 | slot);
// a slot's results are published through its atomic `done` flag and collected by
// whichever poll retires the ticket (compare-and-swap to 0), so polls take the lock only
// to return freed slots. Under overload the GPU keeps running at its own rate while the
// excess requests are refused (PGB_ERR_BUSY).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "errors.h"
#include "index.h"
#include "search_hnsw.h"
#include "search_plan.h"
#include "searcher.h"

namespace pgb {
namespace {

using Clock = std::chrono::steady_clock;

struct Slot {
    std::atomic<uint64_t> ticket{0};  // the live ticket, 0 when free or collected
    std::atomic<bool> done{false};    // results below are complete
    uint32_t gen = 0;                 // generation of the last ticket issued here
    uint32_t Ls = 0, k = 0;
    Clock::time_point t_submit;
    std::vector<uint8_t> query;
    std::vector<uint32_t> ids;
    std::vector<int32_t> dists;
    pgb_query_stats stats{};
};

// one launch on its own stream
struct Context {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;            // written by the dispatcher under the lock
    std::vector<uint32_t> slots;  // pool slots, batch-local order
    uint8_t* h_in = nullptr;      // pinned: queries | ls | k | order
    // pinned outputs, written by the kernel through their device addresses (d_*), and the
    // per-query completion flags (h_done[j] == seq: batch position j is finished)
    uint32_t* h_ids = nullptr;
    int32_t* h_dists = nullptr;
    pgb_query_stats* h_stats = nullptr;
    uint32_t* h_done = nullptr;
    uint32_t seq = 0;                   // this context's launch count
    std::vector<uint32_t> unpublished;  // batch positions not yet handed to their slots
    uint8_t* d_in = nullptr;
    uint32_t* d_ids = nullptr;
    int32_t* d_dists = nullptr;
    pgb_query_stats* d_stats = nullptr;
    uint32_t* d_done = nullptr;
    uint32_t* d_queue = nullptr;
    uint32_t* gfilter = nullptr;
    uint32_t* gvisited = nullptr;
    HnswState hnsw;  // HNSW index: this context's searcher state, prepared for max_beam
};

constexpr size_t kLatencyRing = 65536;

}  // namespace
}  // namespace pgb

struct pgb_server {
    pgb_index* index = nullptr;
    pgb_server_options opt{};
    pgb::FlatPlan plan{};
    bool hnsw = false;            // HNSW index: per-(Ls, k) launches of the HNSW kernel
    size_t hnsw_scratch = 0;      // device bytes of one context's HNSW state
    uint32_t deg_lim = 0;
    size_t in_q_bytes = 0, in_bytes = 0;  // staging layout
    std::vector<pgb::Context> ctx;
    std::unique_ptr<pgb::Slot[]> pool;
    uint32_t pool_n = 0;
    std::vector<uint32_t> free_slots;
    std::deque<uint32_t> pending;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread dispatcher;
    bool stop = false;
    pgb_status failed = PGB_OK;
    std::string fail_msg;
    uint64_t submitted = 0, completed = 0, rejected = 0, launches = 0, launched_requests = 0;
    std::vector<float> lat_us;
    size_t lat_pos = 0;
    bool lat_full = false;
};

namespace pgb {
namespace {

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

void free_context(Context& c) {
    if (c.stream) cudaStreamDestroy(c.stream);
    if (c.done) cudaEventDestroy(c.done);
    cudaFreeHost(c.h_in);
    cudaFreeHost(c.h_ids);
    cudaFreeHost(c.h_dists);
    cudaFreeHost(c.h_stats);
    cudaFreeHost(c.h_done);
    cudaFree(c.d_in);
    cudaFree(c.d_queue);
    cudaFree(c.gfilter);
    cudaFree(c.gvisited);
    hnsw_release(c.hnsw);
    c = Context{};
}

// the searcher parameters an HNSW context is prepared with (the largest request)
pgb_query_params hnsw_params(const pgb_server* S) {
    pgb_query_params p{};
    p.k = S->opt.max_k;
    p.beam_size = S->opt.max_beam;
    p.cut = S->opt.cut;
    p.limit = S->opt.limit;
    return p;
}

pgb_status alloc_context(pgb_server* S, Context& c) {
    const size_t mb = S->opt.max_batch, mk = S->opt.max_k;
    pgb_status s;
    if ((s = cuda_status(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "stream")) != PGB_OK ||
        (s = cuda_status(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming), "event")) != PGB_OK ||
        (s = cuda_status(cudaMallocHost(&c.h_in, S->in_bytes), "pinned staging")) != PGB_OK ||
        (s = cuda_status(cudaMallocHost(&c.h_ids, 4 * mb * mk), "pinned staging")) != PGB_OK ||
        (s = cuda_status(cudaMallocHost(&c.h_dists, 4 * mb * mk), "pinned staging")) != PGB_OK ||
        (s = cuda_status(cudaMallocHost(&c.h_stats, sizeof(pgb_query_stats) * mb), "pinned staging")) != PGB_OK ||
        (s = cuda_status(cudaMallocHost(&c.h_done, 4 * mb), "pinned flags")) != PGB_OK ||
        (s = cuda_status(cudaHostGetDevicePointer((void**)&c.d_ids, c.h_ids, 0), "mapped outputs")) != PGB_OK ||
        (s = cuda_status(cudaHostGetDevicePointer((void**)&c.d_dists, c.h_dists, 0), "mapped outputs")) != PGB_OK ||
        (s = cuda_status(cudaHostGetDevicePointer((void**)&c.d_stats, c.h_stats, 0), "mapped outputs")) != PGB_OK ||
        (s = cuda_status(cudaHostGetDevicePointer((void**)&c.d_done, c.h_done, 0), "mapped flags")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&c.d_in, S->in_bytes), "device staging")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&c.d_queue, 4), "queue counter")) != PGB_OK)
        return s;
    memset(c.h_done, 0, 4 * mb);
    if (S->hnsw) {
        const pgb_query_params p = hnsw_params(S);
        return hnsw_prepare(S->index, p, c.hnsw);
    }
    const uint64_t tw = S->plan.total_warps;
    if (S->plan.gfilter_words &&
        (s = cuda_status(cudaMalloc(&c.gfilter, 4ull * S->plan.gfilter_words * tw), "filter scratch")) != PGB_OK)
        return s;
    if (S->plan.gvisited_words &&
        (s = cuda_status(cudaMalloc(&c.gvisited, 4ull * S->plan.gvisited_words * tw), "visited scratch")) != PGB_OK)
        return s;
    return PGB_OK;
}

size_t context_device_bytes(const pgb_server* S) {
    const size_t tw = S->plan.total_warps;
    const size_t staging = S->in_bytes + 4;  // the outputs live in page-locked host memory
    if (S->hnsw) return staging + S->hnsw_scratch;
    return staging + 4ull * (S->plan.gfilter_words + S->plan.gvisited_words) * tw;
}

// called with the lock held
void set_failed(pgb_server* S, pgb_status s, const std::string& m) {
    if (S->failed == PGB_OK) {
        S->failed = s;
        S->fail_msg = m;
    }
    S->cv_done.notify_all();
}

void fail_unlocked(pgb_server* S, pgb_status s, const std::string& m) {
    std::lock_guard<std::mutex> lk(S->mu);
    set_failed(S, s, m);
}

// records a launched batch's completion event (its outputs reach host memory from the
// kernel itself) and lists its positions as unpublished
bool track_completion(pgb_server* S, Context& c, uint32_t b) {
    c.unpublished.resize(b);
    std::iota(c.unpublished.begin(), c.unpublished.end(), 0u);
    cudaError_t e = cudaEventRecord(c.done, c.stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail_unlocked(S, PGB_ERR_CUDA, std::string("server launch: ") + cudaGetErrorString(e));
        return false;
    }
    return true;
}

// packs c.slots (taken from the pending queue under the lock) and launches them; runs
// without the lock: pending slots are not touched by anyone else until they are done
bool launch(pgb_server* S, Context& c) {
    const pgb_index* ix = S->index;
    const size_t mb = S->opt.max_batch;
    const uint32_t b = (uint32_t)c.slots.size();
    uint32_t* ls = reinterpret_cast<uint32_t*>(c.h_in + S->in_q_bytes);
    uint32_t* ks = ls + mb;
    uint32_t* order = ks + mb;
    for (uint32_t j = 0; j < b; j++) {
        const Slot& sl = S->pool[c.slots[j]];
        memcpy(c.h_in + (size_t)j * ix->dim, sl.query.data(), ix->dim);
        ls[j] = sl.Ls;
        ks[j] = sl.k;
        order[j] = j;
    }
    std::stable_sort(order, order + b, [&](uint32_t a, uint32_t d) { return ls[a] > ls[d]; });
    cudaError_t e = cudaMemcpyAsync(c.d_in, c.h_in, S->in_bytes, cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_queue, 0, 4, c.stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail_unlocked(S, PGB_ERR_CUDA, std::string("server upload: ") + cudaGetErrorString(e));
        return false;
    }
    const uint32_t* d_ls = reinterpret_cast<const uint32_t*>(c.d_in + S->in_q_bytes);
    if (++c.seq == 0) {  // flags of earlier launches hold older values; 0 is never one
        memset(c.h_done, 0, 4 * mb);
        c.seq = 1;
    }
    if (S->hnsw) {
        // one launch of the HNSW kernel: each query at its own (Ls, k), longest beam first
        if (hnsw_launch_at(ix, c.hnsw, S->opt.max_beam, S->opt.max_k, S->opt.limit, c.d_in, b, ix->dim,
                           c.d_ids, c.d_dists, c.d_stats, S->opt.max_k, c.stream, d_ls, d_ls + mb,
                           d_ls + 2 * mb, c.d_done, c.seq) != PGB_OK) {
            fail_unlocked(S, PGB_ERR_CUDA, pgb_last_error());
            return false;
        }
        return track_completion(S, c, b);
    }
    FlatArgs A{};
    A.rows = ix->rows;
    A.adj = ix->adj;
    A.n = ix->n;
    A.gs = ix->gs;
    A.deg_lim = S->deg_lim;
    A.dim = ix->dim;
    A.start = 0;
    A.queries = c.d_in;
    A.nq = b;
    A.qstride = ix->dim;
    A.cut = S->opt.cut;
    A.limit = S->opt.limit <= 0 ? (int64_t)ix->n : S->opt.limit;
    A.excl = 0;
    A.qbase = 0;
    A.norm_in_row = ix->norm_in_row ? 1u : 0u;
    A.ls_arr = reinterpret_cast<const uint32_t*>(c.d_in + S->in_q_bytes);
    A.k_arr = A.ls_arr + mb;
    A.order = A.k_arr + mb;
    A.out_stride = S->opt.max_k;
    A.ids = c.d_ids;
    A.dists = c.d_dists;
    A.stats = c.d_stats;
    A.gfilter = c.gfilter;
    A.gvisited = c.gvisited;
    A.queue = c.d_queue;
    A.done = c.d_done;
    A.done_seq = c.seq;
    if (launch_flat(S->plan, A, c.stream, ix) != PGB_OK) {
        fail_unlocked(S, PGB_ERR_CUDA, pgb_last_error());
        return false;
    }
    return track_completion(S, c, b);
}

// hands batch position j's results to its slot (no lock: the slot is this launch's)
void publish(pgb_server* S, Context& c, uint32_t j, Clock::time_point now, std::vector<float>& lat) {
    const size_t mk = S->opt.max_k;
    Slot& sl = S->pool[c.slots[j]];
    std::copy(c.h_ids + j * mk, c.h_ids + j * mk + sl.k, sl.ids.begin());
    std::copy(c.h_dists + j * mk, c.h_dists + j * mk + sl.k, sl.dists.begin());
    sl.stats = c.h_stats[j];
    lat.push_back(std::chrono::duration<float, std::micro>(now - sl.t_submit).count());
    sl.done.store(true, std::memory_order_release);
}

void record_latencies(pgb_server* S, const std::vector<float>& lat) {
    for (float us : lat) {
        S->lat_us[S->lat_pos] = us;
        S->lat_pos = (S->lat_pos + 1) % kLatencyRing;
        if (S->lat_pos == 0) S->lat_full = true;
    }
    S->completed += lat.size();
}

// publishes the positions of a running launch whose completion flags are set; returns
// whether any was
bool publish_ready(pgb_server* S, Context& c, std::vector<float>& lat) {
    lat.clear();
    const auto now = Clock::now();
    size_t keep = 0;
    for (size_t i = 0; i < c.unpublished.size(); i++) {
        const uint32_t j = c.unpublished[i];
        if (reinterpret_cast<volatile uint32_t*>(c.h_done)[j] == c.seq) {
            std::atomic_thread_fence(std::memory_order_acquire);  // flag, then its outputs
            publish(S, c, j, now, lat);
        } else {
            c.unpublished[keep++] = j;
        }
    }
    c.unpublished.resize(keep);
    if (lat.empty()) return false;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        record_latencies(S, lat);
    }
    S->cv_done.notify_all();
    return true;
}

// a finished launch: the positions not published yet, then the context is free again
void finish(pgb_server* S, Context& c, std::vector<float>& lat) {
    const auto now = Clock::now();
    lat.clear();
    for (const uint32_t j : c.unpublished) publish(S, c, j, now, lat);
    c.unpublished.clear();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        record_latencies(S, lat);
        c.slots.clear();
        c.busy = false;
    }
    S->cv_done.notify_all();
}

void dispatch_loop(pgb_server* S) {
    cudaSetDevice(S->index->device);
    std::vector<float> lat;
    for (;;) {
        bool progressed = false;
        int inflight = 0;
        for (Context& c : S->ctx) {
            if (!c.busy) continue;  // only this thread changes busy
            if (publish_ready(S, c, lat)) progressed = true;
            const cudaError_t q = cudaEventQuery(c.done);
            if (q == cudaSuccess) {
                finish(S, c, lat);
                progressed = true;
            } else if (q != cudaErrorNotReady) {
                cudaGetLastError();
                std::lock_guard<std::mutex> lk(S->mu);
                set_failed(S, PGB_ERR_CUDA, std::string("server kernel: ") + cudaGetErrorString(q));
                c.busy = false;
            } else {
                inflight++;
            }
        }
        for (Context& c : S->ctx) {
            if (c.busy) continue;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                if (S->failed != PGB_OK || S->pending.empty()) break;
                // while other launches run, a partial batch may wait a little to grow
                if (inflight > 0 && S->opt.max_wait_us > 0 && S->pending.size() < S->opt.max_batch) {
                    const auto age = Clock::now() - S->pool[S->pending.front()].t_submit;
                    if (age < std::chrono::microseconds(S->opt.max_wait_us)) break;
                }
                const size_t b = std::min<size_t>(S->opt.max_batch, S->pending.size());
                c.slots.assign(S->pending.begin(), S->pending.begin() + b);
                S->pending.erase(S->pending.begin(), S->pending.begin() + b);
                c.busy = true;
                S->launches++;
                S->launched_requests += b;
            }
            if (!launch(S, c)) {
                std::lock_guard<std::mutex> lk(S->mu);
                c.busy = false;
                break;
            }
            inflight++;
            progressed = true;
        }
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->stop && (S->pending.empty() || S->failed != PGB_OK) && inflight == 0) break;
            if (!progressed && inflight == 0) S->cv_work.wait_for(lk, std::chrono::milliseconds(2));
        }
        if (!progressed && inflight > 0) std::this_thread::yield();
    }
}

void destroy_server(pgb_server* S) {
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->dispatcher.joinable()) S->dispatcher.join();
    DeviceGuard g(S->index->device);
    for (Context& c : S->ctx) {
        if (c.stream) cudaStreamSynchronize(c.stream);
        free_context(c);
    }
    delete S;
}

// called with the lock held; the pool has a free slot
uint64_t admit(pgb_server* S, const uint8_t* query, uint32_t beam_size, uint32_t k,
               Clock::time_point now) {
    const uint32_t slot = S->free_slots.back();
    S->free_slots.pop_back();
    Slot& sl = S->pool[slot];
    memcpy(sl.query.data(), query, S->index->dim);
    sl.Ls = beam_size;
    sl.k = k;
    sl.t_submit = now;
    sl.gen++;
    if (sl.gen == 0) sl.gen = 1;  // tickets are never 0
    const uint64_t ticket = ((uint64_t)sl.gen << 32) | slot;
    sl.done.store(false, std::memory_order_relaxed);
    sl.ticket.store(ticket, std::memory_order_release);
    S->pending.push_back(slot);
    return ticket;
}

// the slot of a live ticket, or nullptr
Slot* slot_of(pgb_server* S, uint64_t ticket) {
    const uint32_t slot = (uint32_t)ticket;
    if (ticket == 0 || slot >= S->pool_n) return nullptr;
    Slot& sl = S->pool[slot];
    return sl.ticket.load(std::memory_order_acquire) == ticket ? &sl : nullptr;
}

// retires a done ticket (one caller wins) and copies its results out
bool collect(Slot& sl, uint64_t ticket, uint32_t* ids, int32_t* dists, pgb_query_stats* stats) {
    uint64_t expect = ticket;
    if (!sl.ticket.compare_exchange_strong(expect, 0, std::memory_order_acq_rel)) return false;
    std::copy(sl.ids.begin(), sl.ids.begin() + sl.k, ids);
    std::copy(sl.dists.begin(), sl.dists.begin() + sl.k, dists);
    if (stats) *stats = sl.stats;
    return true;
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" {

pgb_status pgb_server_create(pgb_index* ix, const pgb_server_options* opt, pgb_server** out) {
    if (!out) return fail(PGB_ERR_BAD_ARG, "null output handle");
    *out = nullptr;
    if (!ix || !opt) return fail(PGB_ERR_BAD_ARG, "null index or options");
    if (opt->max_beam == 0 || opt->max_beam > PGB_MAX_BEAM || opt->max_k == 0 ||
        opt->max_k > PGB_MAX_K || !(opt->cut > 0))
        return fail(PGB_ERR_BAD_ARG, "bad max_beam / max_k / cut");
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    pgb_server* S = new pgb_server();
    S->index = ix;
    S->opt = *opt;
    if (S->opt.max_batch == 0) S->opt.max_batch = 1024;
    if (S->opt.max_inflight == 0) S->opt.max_inflight = 4;
    pgb_status s;
    S->hnsw = ix->is_hnsw;
    if (S->hnsw) {
        // one context's HNSW tables, measured on a probe state
        HnswState probe;
        const pgb_query_params p = hnsw_params(S);
        if ((s = hnsw_prepare(ix, p, probe)) != PGB_OK) {
            hnsw_release(probe);
            delete S;
            return s;
        }
        S->hnsw_scratch = hnsw_scratch_bytes(probe);
        hnsw_release(probe);
    } else {
        S->deg_lim = opt->degree_limit ? std::min(opt->degree_limit, ix->G) : ix->G;
        FlatPlanRequest rq;
        rq.max_ls = S->opt.max_beam;
        rq.deg_lim = S->deg_lim;
        rq.is_signed = ix->elem == PGB_INT8;
        rq.batched = true;
        s = plan_flat(rq, S->plan);
        if (s != PGB_OK) {
            delete S;
            return s;
        }
    }
    const size_t mb = S->opt.max_batch;
    S->in_q_bytes = align16(mb * ix->dim);
    S->in_bytes = S->in_q_bytes + 12 * mb;
    // admission by free memory: as many stream contexts as the budget holds
    size_t free_b = 0, total_b = 0;
    if ((s = cuda_status(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo")) != PGB_OK) {
        delete S;
        return s;
    }
    const size_t budget = S->opt.memory_budget ? S->opt.memory_budget : free_b / 2;
    const size_t per = context_device_bytes(S);
    const size_t fit = per ? budget / per : 0;
    if (fit == 0) {
        delete S;
        return fail(PGB_ERR_OOM, "memory budget below one launch context");
    }
    S->ctx.resize(std::min<size_t>(S->opt.max_inflight, fit));
    for (Context& c : S->ctx)
        if ((s = alloc_context(S, c)) != PGB_OK) {
            for (Context& d : S->ctx) free_context(d);
            delete S;
            return s;
        }
    // pool: every context's batch in flight plus as many waiting
    S->pool_n = (uint32_t)(2 * S->ctx.size() * mb);
    S->pool.reset(new Slot[S->pool_n]);
    for (uint32_t i = 0; i < S->pool_n; i++) {
        S->pool[i].query.resize(ix->dim);
        S->pool[i].ids.resize(S->opt.max_k);
        S->pool[i].dists.resize(S->opt.max_k);
    }
    S->free_slots.resize(S->pool_n);
    std::iota(S->free_slots.rbegin(), S->free_slots.rend(), 0u);
    S->lat_us.assign(kLatencyRing, 0.f);
    S->dispatcher = std::thread(dispatch_loop, S);
    *out = S;
    return PGB_OK;
}

pgb_status pgb_server_submit(pgb_server* S, const void* query, uint32_t beam_size, uint32_t k,
                             uint64_t* ticket) {
    if (!S || !query || !ticket) return fail(PGB_ERR_BAD_ARG, "null argument");
    if (beam_size == 0 || beam_size > S->opt.max_beam) return fail(PGB_ERR_BAD_ARG, "beam size outside 1..max_beam");
    if (k == 0 || k > S->opt.max_k) return fail(PGB_ERR_BAD_ARG, "k outside 1..max_k");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->failed != PGB_OK) return fail(S->failed, S->fail_msg);
        if (S->stop) return fail(PGB_ERR_BAD_ARG, "server is shutting down");
        if (S->free_slots.empty()) {
            S->rejected++;
            return fail(PGB_ERR_BUSY, "request pool full");
        }
        *ticket = admit(S, static_cast<const uint8_t*>(query), beam_size, k, Clock::now());
        S->submitted++;
    }
    S->cv_work.notify_one();
    return PGB_OK;
}

pgb_status pgb_server_poll(pgb_server* S, uint64_t ticket, uint32_t timeout_us, uint32_t* ids,
                           int32_t* dists, pgb_query_stats* stats) {
    if (!S || !ids || !dists) return fail(PGB_ERR_BAD_ARG, "null argument");
    Slot* sl = slot_of(S, ticket);
    if (!sl) return fail(PGB_ERR_NOT_FOUND, "unknown ticket");
    if (!sl->done.load(std::memory_order_acquire)) {
        std::unique_lock<std::mutex> lk(S->mu);
        S->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), [&] {
            return sl->done.load(std::memory_order_acquire) || S->failed != PGB_OK ||
                   sl->ticket.load(std::memory_order_acquire) != ticket;
        });
        if (sl->ticket.load(std::memory_order_acquire) != ticket)
            return fail(PGB_ERR_NOT_FOUND, "unknown ticket");
        if (!sl->done.load(std::memory_order_acquire)) {
            if (S->failed != PGB_OK) return fail(S->failed, S->fail_msg);
            return fail(PGB_ERR_TIMEOUT, "request not finished");
        }
    }
    if (!collect(*sl, ticket, ids, dists, stats)) return fail(PGB_ERR_NOT_FOUND, "unknown ticket");
    std::lock_guard<std::mutex> lk(S->mu);
    S->free_slots.push_back((uint32_t)ticket);
    return PGB_OK;
}

pgb_status pgb_server_submit_many(pgb_server* S, const void* queries, uint32_t n,
                                  uint32_t query_stride, const uint32_t* beam_sizes,
                                  const uint32_t* ks, uint64_t* tickets, uint32_t* admitted) {
    if (!S || !queries || !beam_sizes || !ks || !tickets || !admitted)
        return fail(PGB_ERR_BAD_ARG, "null argument");
    *admitted = 0;
    if (query_stride < S->index->dim) return fail(PGB_ERR_BAD_ARG, "query_stride below dim");
    for (uint32_t i = 0; i < n; i++) {
        if (beam_sizes[i] == 0 || beam_sizes[i] > S->opt.max_beam)
            return fail(PGB_ERR_BAD_ARG, "beam size outside 1..max_beam");
        if (ks[i] == 0 || ks[i] > S->opt.max_k) return fail(PGB_ERR_BAD_ARG, "k outside 1..max_k");
    }
    uint32_t got = 0;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->failed != PGB_OK) return fail(S->failed, S->fail_msg);
        if (S->stop) return fail(PGB_ERR_BAD_ARG, "server is shutting down");
        const auto now = Clock::now();
        const uint8_t* q = static_cast<const uint8_t*>(queries);
        for (; got < n && !S->free_slots.empty(); got++)
            tickets[got] = admit(S, q + (size_t)got * query_stride, beam_sizes[got], ks[got], now);
        S->submitted += got;
        S->rejected += n - got;
    }
    *admitted = got;
    if (got) S->cv_work.notify_one();
    if (got == 0 && n > 0) return fail(PGB_ERR_BUSY, "request pool full");
    return PGB_OK;
}

pgb_status pgb_server_poll_many(pgb_server* S, const uint64_t* tickets, uint32_t n,
                                uint32_t* ids, int32_t* dists, pgb_query_stats* stats,
                                uint8_t* done, uint32_t* n_done) {
    if (!S || !tickets || !ids || !dists || !done || !n_done)
        return fail(PGB_ERR_BAD_ARG, "null argument");
    const size_t mk = S->opt.max_k;
    std::vector<uint32_t> freed;
    for (uint32_t i = 0; i < n; i++) {
        done[i] = 0;
        Slot* sl = slot_of(S, tickets[i]);
        if (!sl || !sl->done.load(std::memory_order_acquire)) continue;
        if (!collect(*sl, tickets[i], ids + i * mk, dists + i * mk, stats ? stats + i : nullptr))
            continue;
        freed.push_back((uint32_t)tickets[i]);
        done[i] = 1;
    }
    *n_done = (uint32_t)freed.size();
    std::lock_guard<std::mutex> lk(S->mu);
    S->free_slots.insert(S->free_slots.end(), freed.begin(), freed.end());
    if (S->failed != PGB_OK && freed.empty()) return fail(S->failed, S->fail_msg);
    return PGB_OK;
}

pgb_status pgb_server_get_stats(pgb_server* S, pgb_server_stats* out) {
    if (!S || !out) return fail(PGB_ERR_BAD_ARG, "null argument");
    std::vector<float> lat;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        out->submitted = S->submitted;
        out->completed = S->completed;
        out->rejected = S->rejected;
        out->launches = S->launches;
        out->pending = (uint32_t)S->pending.size();
        uint32_t inflight = 0;
        for (const Context& c : S->ctx) inflight += c.busy ? (uint32_t)c.slots.size() : 0u;
        out->in_flight = inflight;
        out->pool_slots = S->pool_n;
        out->streams = (uint32_t)S->ctx.size();
        out->mean_batch = S->launches ? (double)S->launched_requests / S->launches : 0.0;
        const size_t nl = S->lat_full ? kLatencyRing : S->lat_pos;
        lat.assign(S->lat_us.begin(), S->lat_us.begin() + nl);
    }
    out->p50_us = out->p99_us = 0;
    if (!lat.empty()) {
        const size_t i50 = lat.size() / 2, i99 = std::min(lat.size() - 1, lat.size() * 99 / 100);
        std::nth_element(lat.begin(), lat.begin() + i50, lat.end());
        out->p50_us = lat[i50];
        std::nth_element(lat.begin(), lat.begin() + i99, lat.end());
        out->p99_us = lat[i99];
    }
    return PGB_OK;
}

pgb_status pgb_server_destroy(pgb_server* S) {
    if (!S) return PGB_OK;
    destroy_server(S);
    return PGB_OK;
}

}  // extern "C"
