// batch.cu -- pgb_batch_*: the batched persistent form of the flat-graph and HNSW search.
//
// plan   : host step, per-query (Ls, k) -> longest-beam-first work order on the device
// search : cudaMemsetAsync(counter) + one persistent launch (capturable); a plan whose
//          queries all share one (Ls, k) runs the uniform-batch kernel
// tune   : times candidate (warps per block, filter / visited placement, resident blocks
//          per SM) on the planned queries and keeps the fastest; every candidate returns
//          identical neighbours, because all of them run the same per-query code
//          (flat_query). Fewer resident warps than fit can win on a batch of a few queries
//          per warp: the launch ends when its last query does, and with fewer warps each
//          takes more queries, so the tail in which SMs idle is a smaller share.
// An HNSW index runs the HNSW kernel with each query at its own (Ls, k), its tables sized
// for max_beam; its one kernel shape is tuned over resident blocks only. Every beam can be
// captured: the (epoch, id) filter of beams above 256 takes its epochs from a device word.
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "errors.h"
#include "index.h"
#include "search_hnsw.h"
#include "search_plan.h"
#include "searcher.h"

struct pgb_batch {
    pgb_index* index = nullptr;
    pgb_batch_options opt{};
    pgb::FlatPlan plan{};
    bool hnsw = false;
    pgb::HnswState hs{};  // HNSW index: the searcher state, prepared for max_beam
    float tuned_ms = 0.f;
    uint32_t* gfilter = nullptr;
    uint64_t gfilter_words = 0;   // allocated words
    uint32_t* gvisited = nullptr;
    uint64_t gvisited_words = 0;
    uint32_t* d_ls = nullptr;
    uint32_t* d_k = nullptr;
    uint32_t* d_order = nullptr;
    uint32_t* d_queue = nullptr;
    uint32_t nq = 0;
    uint32_t max_ls_planned = 0;
    uint32_t uniform_ls = 0, uniform_k = 0;  // the plan's (Ls, k) when all queries share it
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int64_t graph_launches = 0;  // search kernels in the captured graph
    uint64_t graph_epochs = 0;   // HNSW (epoch, id) filter: epochs one replay uses
    // host-memory path staging
    uint8_t* q_dev = nullptr;
    uint32_t* ids_dev = nullptr;
    int32_t* dists_dev = nullptr;
    pgb_query_stats* stats_dev = nullptr;
    cudaStream_t stream = nullptr;
};

namespace pgb {
namespace {

// max_bps: a cap on resident blocks per SM (0: as many as fit)
pgb_status make_plan(pgb_batch* b, int wpb, int filter_pl, int visited_pl, FlatPlan& P,
                     int max_bps = 0) {
    const pgb_index* ix = b->index;
    FlatPlanRequest rq;
    rq.max_ls = b->opt.max_beam;
    rq.deg_lim = b->opt.degree_limit ? std::min(b->opt.degree_limit, ix->G) : ix->G;
    rq.is_signed = ix->elem == PGB_INT8;
    rq.batched = true;
    rq.warps_per_block = wpb;
    rq.max_blocks_per_sm = max_bps;
    if (filter_pl) {
        rq.force_filter_placement = true;
        rq.filter_in_shared = filter_pl == 1;
    }
    if (visited_pl) {
        rq.force_visited_placement = true;
        rq.visited_in_shared = visited_pl == 1;
    }
    return plan_flat(rq, P);
}

// scratch for the plan's global tables (grown, never shrunk)
pgb_status ensure_scratch(pgb_batch* b, const FlatPlan& P) {
    const uint64_t fw = (uint64_t)P.gfilter_words * P.total_warps;
    const uint64_t vw = (uint64_t)P.gvisited_words * P.total_warps;
    pgb_status s;
    if (fw > b->gfilter_words) {
        cudaFree(b->gfilter);
        b->gfilter = nullptr;
        b->gfilter_words = 0;
        if ((s = cuda_status(cudaMalloc(&b->gfilter, 4 * fw), "batch filter scratch")) != PGB_OK) return s;
        b->gfilter_words = fw;
    }
    if (vw > b->gvisited_words) {
        cudaFree(b->gvisited);
        b->gvisited = nullptr;
        b->gvisited_words = 0;
        if ((s = cuda_status(cudaMalloc(&b->gvisited, 4 * vw), "batch visited scratch")) != PGB_OK) return s;
        b->gvisited_words = vw;
    }
    return PGB_OK;
}

// an HNSW batch launches at most max_bps blocks per SM (its tables stay sized for all)
pgb_status cap_hnsw_blocks(pgb_batch* b, int max_bps) {
    int sms = 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->index->device) != cudaSuccess)
        return cuda_status(cudaGetLastError(), "device attribute");
    b->hs.blocks = std::min(b->hs.blocks, max_bps * sms);
    return PGB_OK;
}

void drop_graph(pgb_batch* b) {
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
}

pgb_status enqueue(pgb_batch* b, const FlatPlan& P, const void* queries, uint32_t qstride,
                   uint32_t* ids, int32_t* dists, pgb_query_stats* stats, cudaStream_t st) {
    const pgb_index* ix = b->index;
    if (b->hnsw) {
        if (b->uniform_ls)
            return hnsw_launch_at(ix, b->hs, b->uniform_ls, b->uniform_k, b->opt.limit, queries, b->nq,
                                  qstride, ids, dists, stats, b->opt.max_k, st);
        return hnsw_launch_at(ix, b->hs, b->opt.max_beam, b->opt.max_k, b->opt.limit, queries, b->nq,
                              qstride, ids, dists, stats, b->opt.max_k, st, b->d_ls, b->d_k, b->d_order);
    }
    pgb_status s = cuda_status(cudaMemsetAsync(b->d_queue, 0, sizeof(uint32_t), st), "queue reset");
    if (s != PGB_OK) return s;
    FlatArgs A{};
    A.rows = ix->rows;
    A.adj = ix->adj;
    A.n = ix->n;
    A.gs = ix->gs;
    A.deg_lim = b->opt.degree_limit ? std::min(b->opt.degree_limit, ix->G) : ix->G;
    A.dim = ix->dim;
    A.start = 0;
    A.queries = (const uint8_t*)queries;
    A.nq = b->nq;
    A.qstride = qstride;
    A.cut = b->opt.cut;
    A.limit = b->opt.limit <= 0 ? (int64_t)ix->n : b->opt.limit;
    A.excl = b->opt.exclude_query_id ? 1u : 0u;
    A.qbase = b->opt.query_id_base;
    A.norm_in_row = ix->norm_in_row ? 1u : 0u;
    if (b->uniform_ls) {
        // one (Ls, k) for the whole plan: the uniform kernel reads it from A.Ls / A.k
        A.Ls = b->uniform_ls;
        A.k = b->uniform_k;
    } else {
        A.ls_arr = b->d_ls;
        A.k_arr = b->d_k;
    }
    A.order = b->d_order;
    A.out_stride = b->opt.max_k;
    A.ids = ids;
    A.dists = dists;
    A.stats = stats;
    A.gfilter = P.gfilter_words ? b->gfilter : nullptr;
    A.gvisited = P.gvisited_words ? b->gvisited : nullptr;
    A.queue = b->d_queue;
    return launch_flat(P, A, st, ix);
}

pgb_status check_call(pgb_batch* b, const void* queries, uint32_t qstride, uint32_t* ids,
                      int32_t* dists) {
    if (!b) return fail(PGB_ERR_BAD_ARG, "null batch");
    if (b->nq == 0) return fail(PGB_ERR_BAD_ARG, "batch has no planned queries");
    if (!queries || !ids || !dists) return fail(PGB_ERR_BAD_ARG, "null queries or outputs");
    if (qstride < b->index->dim) return fail(PGB_ERR_BAD_ARG, "query_stride below dim");
    return PGB_OK;
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" {

pgb_status pgb_batch_create(pgb_index* ix, const pgb_batch_options* opt, pgb_batch** out) {
    if (!out) return fail(PGB_ERR_BAD_ARG, "null output handle");
    *out = nullptr;
    if (!ix || !opt) return fail(PGB_ERR_BAD_ARG, "null index or options");
    if (opt->max_queries == 0 || opt->max_beam == 0 || opt->max_beam > PGB_MAX_BEAM ||
        opt->max_k == 0 || opt->max_k > PGB_MAX_K || !(opt->cut > 0))
        return fail(PGB_ERR_BAD_ARG, "bad max_queries / max_beam / max_k / cut");
    if (opt->warps_per_block > 4 || opt->filter_placement > 2 || opt->visited_placement > 2)
        return fail(PGB_ERR_BAD_ARG, "bad launch shape or placement option");
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    pgb_batch* b = new pgb_batch();
    b->index = ix;
    b->opt = *opt;
    b->hnsw = ix->is_hnsw;
    pgb_status s;
    const size_t nq = opt->max_queries;
    pgb_query_params hp{};
    hp.k = opt->max_k;
    hp.beam_size = opt->max_beam;
    hp.cut = opt->cut;
    hp.limit = opt->limit;
    if ((s = b->hnsw ? hnsw_prepare(ix, hp, b->hs)
                     : make_plan(b, (int)opt->warps_per_block, (int)opt->filter_placement,
                                 (int)opt->visited_placement, b->plan, (int)opt->blocks_per_sm)) != PGB_OK ||
        (!b->hnsw && (s = ensure_scratch(b, b->plan)) != PGB_OK) ||
        (b->hnsw && opt->blocks_per_sm && (s = cap_hnsw_blocks(b, (int)opt->blocks_per_sm)) != PGB_OK) ||
        (s = cuda_status(cudaMalloc(&b->d_ls, 4 * nq), "batch arrays")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&b->d_k, 4 * nq), "batch arrays")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&b->d_order, 4 * nq), "batch arrays")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&b->d_queue, 4), "batch counter")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&b->q_dev, nq * ix->dim), "query staging")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&b->ids_dev, 4 * nq * opt->max_k), "ids staging")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&b->dists_dev, 4 * nq * opt->max_k), "dists staging")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&b->stats_dev, sizeof(pgb_query_stats) * nq), "stats staging")) != PGB_OK ||
        (s = cuda_status(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream")) != PGB_OK) {
        pgb_batch_destroy(b);
        return s;
    }
    *out = b;
    return PGB_OK;
}

pgb_status pgb_batch_plan(pgb_batch* b, const uint32_t* beam_sizes, const uint32_t* ks,
                          uint32_t nq) {
    if (!b || !beam_sizes || !ks) return fail(PGB_ERR_BAD_ARG, "null argument");
    if (nq == 0 || nq > b->opt.max_queries) return fail(PGB_ERR_BAD_ARG, "nq outside 1..max_queries");
    uint32_t mx = 0;
    for (uint32_t i = 0; i < nq; i++) {
        if (beam_sizes[i] == 0 || beam_sizes[i] > b->opt.max_beam)
            return fail(PGB_ERR_BAD_ARG, "beam size outside 1..max_beam");
        if (ks[i] == 0 || ks[i] > b->opt.max_k) return fail(PGB_ERR_BAD_ARG, "k outside 1..max_k");
        mx = std::max(mx, beam_sizes[i]);
    }
    DeviceGuard guard(b->index->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    // longest beam first (stable), so the longest queries start before the short ones
    std::vector<uint32_t> order(nq);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t c) { return beam_sizes[a] > beam_sizes[c]; });
    pgb_status s;
    if ((s = cuda_status(cudaMemcpy(b->d_ls, beam_sizes, 4ull * nq, cudaMemcpyHostToDevice), "plan upload")) != PGB_OK ||
        (s = cuda_status(cudaMemcpy(b->d_k, ks, 4ull * nq, cudaMemcpyHostToDevice), "plan upload")) != PGB_OK ||
        (s = cuda_status(cudaMemcpy(b->d_order, order.data(), 4ull * nq, cudaMemcpyHostToDevice), "plan upload")) != PGB_OK)
        return s;
    b->nq = nq;
    b->max_ls_planned = mx;
    const bool uniform = std::all_of(beam_sizes, beam_sizes + nq, [&](uint32_t v) { return v == beam_sizes[0]; }) &&
                         std::all_of(ks, ks + nq, [&](uint32_t v) { return v == ks[0]; });
    b->uniform_ls = uniform ? beam_sizes[0] : 0u;
    b->uniform_k = uniform ? ks[0] : 0u;
    drop_graph(b);
    return PGB_OK;
}

pgb_status pgb_batch_search(pgb_batch* b, const void* queries, uint32_t qstride, uint32_t* ids,
                            int32_t* dists, pgb_query_stats* stats, void* stream) {
    pgb_status s = check_call(b, queries, qstride, ids, dists);
    if (s != PGB_OK) return s;
    DeviceGuard guard(b->index->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    return enqueue(b, b->plan, queries, qstride, ids, dists, stats, (cudaStream_t)stream);
}

pgb_status pgb_batch_search_host(pgb_batch* b, const void* queries, uint32_t qstride,
                                 uint32_t* ids, int32_t* dists, pgb_query_stats* stats) {
    pgb_status s = check_call(b, queries, qstride, ids, dists);
    if (s != PGB_OK) return s;
    DeviceGuard guard(b->index->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    const pgb_index* ix = b->index;
    const size_t nq = b->nq, row = 4ull * b->opt.max_k;
    cudaStream_t st = b->stream;
    // page-locked host buffers: one launch reads the queries and writes the results
    // through them, so the transfers overlap the search instead of bracketing it
    void* pq = pinned_device_ptr(queries);
    void* pi = pinned_device_ptr(ids);
    void* pd = pinned_device_ptr(dists);
    void* ps = stats ? pinned_device_ptr(stats) : nullptr;
    if (pq && pi && pd && (!stats || ps)) {
        if ((s = enqueue(b, b->plan, pq, qstride, static_cast<uint32_t*>(pi), static_cast<int32_t*>(pd),
                         static_cast<pgb_query_stats*>(ps), st)) != PGB_OK)
            return s;
        return cuda_status(cudaStreamSynchronize(st), "batch search");
    }
    cudaError_t ce = (qstride == ix->dim)
                         ? cudaMemcpyAsync(b->q_dev, queries, nq * ix->dim, cudaMemcpyHostToDevice, st)
                         : cudaMemcpy2DAsync(b->q_dev, ix->dim, queries, qstride, ix->dim, nq,
                                             cudaMemcpyHostToDevice, st);
    if ((s = cuda_status(ce, "query upload")) != PGB_OK) return s;
    if ((s = enqueue(b, b->plan, b->q_dev, ix->dim, b->ids_dev, b->dists_dev,
                     stats ? b->stats_dev : nullptr, st)) != PGB_OK)
        return s;
    if ((s = cuda_status(cudaMemcpyAsync(ids, b->ids_dev, nq * row, cudaMemcpyDeviceToHost, st),
                         "ids download")) != PGB_OK ||
        (s = cuda_status(cudaMemcpyAsync(dists, b->dists_dev, nq * row, cudaMemcpyDeviceToHost, st),
                         "dists download")) != PGB_OK)
        return s;
    if (stats && (s = cuda_status(cudaMemcpyAsync(stats, b->stats_dev, sizeof(pgb_query_stats) * nq,
                                                  cudaMemcpyDeviceToHost, st),
                                  "stats download")) != PGB_OK)
        return s;
    return cuda_status(cudaStreamSynchronize(st), "batch search");
}

pgb_status pgb_batch_tune(pgb_batch* b, const void* queries, uint32_t qstride, uint32_t* ids,
                          int32_t* dists, pgb_query_stats* stats) {
    pgb_status s = check_call(b, queries, qstride, ids, dists);
    if (s != PGB_OK) return s;
    DeviceGuard guard(b->index->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st;
    if ((s = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "tune stream")) != PGB_OK)
        return s;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (b->hnsw) {
        // one kernel shape; the resident blocks are all that fit, three quarters or five
        // eighths of them (fewer warps also hold fewer global filter tables in L2). The
        // tables stay allocated for every warp of the prepared shape, so an epoch
        // wrap-around still clears all of them.
        int sms = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->index->device);
        const int full = b->hs.blocks, bps = std::max(1, full / std::max(1, sms));
        const bool fixed = b->opt.blocks_per_sm != 0;
        const int cands[] = {full, fixed ? 0 : (3 * bps / 4) * sms, fixed ? 0 : (5 * bps / 8) * sms};
        float best = 1e30f;
        int best_blocks = full, last = full + 1;
        for (int c = 0; c < 3 && s == PGB_OK; c++) {
            const int blocks = cands[c];
            if (blocks < sms || blocks >= last) continue;
            last = blocks;
            b->hs.blocks = blocks;
            float ms = 0.f, t = 0.f;
            s = enqueue(b, b->plan, queries, qstride, ids, dists, stats, st);  // warm
            for (int r = 0; r < 2 && s == PGB_OK; r++) {
                cudaEventRecord(e0, st);
                s = enqueue(b, b->plan, queries, qstride, ids, dists, stats, st);
                cudaEventRecord(e1, st);
                if (s == PGB_OK && cudaEventSynchronize(e1) == cudaSuccess) {
                    cudaEventElapsedTime(&t, e0, e1);
                    ms += t;
                }
            }
            if (s == PGB_OK && ms / 2 < best) {
                best = ms / 2;
                best_blocks = blocks;
            }
        }
        b->hs.blocks = best_blocks;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        const cudaError_t e = cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        if (s != PGB_OK) return s;
        if (e != cudaSuccess) return cuda_status(e, "tune");
        b->tuned_ms = best;
        drop_graph(b);
        return PGB_OK;
    }
    const int wpbs[] = {1, 2, 4};
    const int fpls[] = {1, 2};
    const int vpls[] = {1, 2};
    float best = 1e30f;
    FlatPlan best_plan = b->plan;
    for (int wpb : wpbs)
        for (int fp : fpls)
            for (int vp : vpls) {
                if (b->opt.warps_per_block && (int)b->opt.warps_per_block != wpb) continue;
                if (b->opt.filter_placement && (int)b->opt.filter_placement != fp) continue;
                if (b->opt.visited_placement && (int)b->opt.visited_placement != vp) continue;
                FlatPlan full;
                const int fixed = (int)b->opt.blocks_per_sm;  // the caller's cap, if any
                if (make_plan(b, wpb, fp, vp, full, fixed) != PGB_OK) continue;  // does not fit
                if (full.warps_per_block != wpb) continue;
                // every block that fits, then three quarters and five eighths of them
                const int caps[] = {0, fixed ? 0 : (3 * full.blocks_per_sm) / 4,
                                    fixed ? 0 : (5 * full.blocks_per_sm) / 8};
                int last = full.blocks_per_sm;
                for (int c = 0; c < 3; c++) {
                    const int cap = caps[c];
                    // a reduced cap is tried only when it keeps a block and drops one
                    if (c > 0 && (cap < 1 || cap >= last)) continue;
                    FlatPlan P = full;
                    if (c > 0 && make_plan(b, wpb, fp, vp, P, cap) != PGB_OK) continue;
                    last = P.blocks_per_sm;
                    if (ensure_scratch(b, P) != PGB_OK) continue;
                    float ms = 0.f, t = 0.f;
                    bool ok = enqueue(b, P, queries, qstride, ids, dists, stats, st) == PGB_OK;  // warm
                    for (int r = 0; r < 2 && ok; r++) {
                        cudaEventRecord(e0, st);
                        ok = enqueue(b, P, queries, qstride, ids, dists, stats, st) == PGB_OK;
                        cudaEventRecord(e1, st);
                        ok = ok && cudaEventSynchronize(e1) == cudaSuccess;
                        cudaEventElapsedTime(&t, e0, e1);
                        ms += t;
                    }
                    if (ok && ms / 2 < best) {
                        best = ms / 2;
                        best_plan = P;
                    }
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return cuda_status(e, "tune");
    if (best >= 1e30f) return fail(PGB_ERR_CUDA, "no candidate configuration ran");
    b->plan = best_plan;
    b->tuned_ms = best;
    drop_graph(b);
    return PGB_OK;
}

pgb_status pgb_batch_get_config(const pgb_batch* b, pgb_batch_config* out) {
    if (!b || !out) return fail(PGB_ERR_BAD_ARG, "null argument");
    if (b->hnsw) {
        out->warps_per_block = (uint32_t)b->hs.warps_per_block;
        out->blocks = (uint32_t)b->hs.blocks;
        out->filter_in_shared = b->hs.fmode == 0 ? 1u : 0u;
        out->visited_in_shared = 1u;  // is_inw is the workset, in shared memory
        out->shared_bytes_per_warp = b->hs.warp_bytes;
        out->tuned_ms = b->tuned_ms;
        return PGB_OK;
    }
    out->warps_per_block = (uint32_t)b->plan.warps_per_block;
    out->blocks = (uint32_t)b->plan.blocks;
    out->filter_in_shared = b->plan.sfilt ? 1u : 0u;
    out->visited_in_shared = b->plan.svis ? 1u : 0u;
    out->shared_bytes_per_warp = b->plan.L.bytes;
    out->tuned_ms = b->tuned_ms;
    return PGB_OK;
}

pgb_status pgb_batch_capture(pgb_batch* b, const void* queries, uint32_t qstride, uint32_t* ids,
                             int32_t* dists, pgb_query_stats* stats) {
    pgb_status s = check_call(b, queries, qstride, ids, dists);
    if (s != PGB_OK) return s;
    DeviceGuard guard(b->index->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    drop_graph(b);
    cudaStream_t st;
    if ((s = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "capture stream")) != PGB_OK)
        return s;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        // launches made during the capture only record graph nodes: they count once per
        // replay instead
        const int64_t before = (int64_t)pgb_search_launches();
        // an HNSW (epoch, id) filter (beams above 256): the captured launch reads its first
        // epoch from the device word that the graph's last node advances, so every replay
        // searches with fresh epochs; the host mirror is reserved per replay instead
        const uint64_t epochs_before = b->hs.epoch_base;
        pgb_status ls = enqueue(b, b->plan, queries, qstride, ids, dists, stats, st);
        b->graph_launches = (int64_t)pgb_search_launches() - before;
        count_launches(-b->graph_launches);
        b->graph_epochs = (b->hnsw && b->hs.d_epoch) ? hnsw_epoch_need(b->index, b->nq) : 0;
        b->hs.epoch_base = epochs_before;
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(st, &g);
        if (ls != PGB_OK) {
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(st);
            cudaGetLastError();  // the invalidated capture must not leak into later calls
            return ls;
        }
        if (e == cudaSuccess) {
            b->graph = g;
            e = cudaGraphInstantiate(&b->graph_exec, g, 0);
        }
    }
    cudaStreamDestroy(st);
    if (e != cudaSuccess) {
        drop_graph(b);
        return cuda_status(e, "graph capture");  // cuda_status clears the error state
    }
    return PGB_OK;
}

pgb_status pgb_batch_replay(pgb_batch* b, void* stream) {
    if (!b || !b->graph_exec) return fail(PGB_ERR_BAD_ARG, "no captured graph");
    DeviceGuard guard(b->index->device);
    if (b->graph_epochs) {
        const pgb_status r = hnsw_epoch_reserve(b->hs, b->graph_epochs, (cudaStream_t)stream);
        if (r != PGB_OK) return r;
    }
    const pgb_status s = cuda_status(cudaGraphLaunch(b->graph_exec, (cudaStream_t)stream), "graph launch");
    if (s == PGB_OK) count_launches(b->graph_launches);
    return s;
}

pgb_status pgb_batch_destroy(pgb_batch* b) {
    if (!b) return PGB_OK;
    DeviceGuard guard(b->index ? b->index->device : 0);
    drop_graph(b);
    hnsw_release(b->hs);
    cudaFree(b->gfilter);
    cudaFree(b->gvisited);
    cudaFree(b->d_ls);
    cudaFree(b->d_k);
    cudaFree(b->d_order);
    cudaFree(b->d_queue);
    cudaFree(b->q_dev);
    cudaFree(b->ids_dev);
    cudaFree(b->dists_dev);
    cudaFree(b->stats_dev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return PGB_OK;
}

}  // extern "C"
