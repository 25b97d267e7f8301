// searcher.cu -- pgb_searcher_*: the drop-in for BuscadorGPU / BuscadorHnsw
// (preparar = create, lanzar = search, liberar = destroy; reference
// cuda/busqueda.cu:525-594, cuda/busqueda_hnsw.cu:551-645).
#include <algorithm>
#include <string>

#include "codes.h"
#include "errors.h"
#include "index.h"
#include "search_hnsw.h"
#include "search_plan.h"
#include "searcher.h"

namespace pgb {

pgb_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PGB_OK;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(PGB_ERR_OOM, std::string(what) + ": out of memory");
    return fail(PGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

pgb_status check_params(const pgb_index* ix, const pgb_query_params* p) {
    if (!p) return fail(PGB_ERR_BAD_ARG, "null params");
    if (p->k == 0 || p->k > PGB_MAX_K) return fail(PGB_ERR_BAD_ARG, "k outside 1..1024");
    if (p->beam_size == 0 || p->beam_size > PGB_MAX_BEAM)
        return fail(PGB_ERR_BAD_ARG, "beam_size outside 1..1024");
    if (!ix->is_hnsw && !(p->cut > 0)) return fail(PGB_ERR_BAD_ARG, "cut must be > 0");
    return PGB_OK;
}

void* pinned_device_ptr(const void* p) {
    if (!p) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

namespace {

// rerank > 0: a search over the index's code rows keeping `rerank` candidates per query
pgb_status create_searcher(pgb_index* ix, uint32_t max_queries, const pgb_query_params* params,
                           uint32_t rerank, pgb_searcher** out) {
    if (!out) return fail(PGB_ERR_BAD_ARG, "null output handle");
    *out = nullptr;
    if (!ix || max_queries == 0) return fail(PGB_ERR_BAD_ARG, "null index or max_queries == 0");
    pgb_status s = check_params(ix, params);
    if (s != PGB_OK) return s;
    if (rerank) {
        if (ix->is_hnsw || !ix->codes) return fail(PGB_ERR_BAD_ARG, "index has no code rows (pgb_index_compress)");
        if (rerank < params->k || rerank > params->beam_size)
            return fail(PGB_ERR_BAD_ARG, "rerank outside k..beam_size");
    }
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    pgb_searcher* S = new pgb_searcher();
    S->index = ix;
    S->params = *params;
    S->max_queries = max_queries;
    S->codes = rerank > 0;
    S->rerank = rerank;
    if (!ix->is_hnsw) {
        FlatPlanRequest rq;
        rq.max_ls = params->beam_size;
        rq.deg_lim = params->degree_limit ? std::min(params->degree_limit, ix->G) : ix->G;
        rq.is_signed = ix->elem == PGB_INT8;
        rq.batched = false;
        rq.codes = S->codes;
        if ((s = plan_flat(rq, S->flat)) != PGB_OK) {
            delete S;
            return s;
        }
        if (S->codes &&
            ((s = cuda_status(cudaMalloc(&S->cand, 4ull * max_queries * rerank), "candidate ids")) != PGB_OK ||
             (s = cuda_status(cudaMalloc(&S->cand_d, 4ull * max_queries * rerank), "candidate distances")) !=
                 PGB_OK)) {
            pgb_searcher_destroy(S);
            return s;
        }
        if (S->flat.gfilter_words &&
            (s = cuda_status(cudaMalloc(&S->gfilter, 4ull * S->flat.gfilter_words * S->flat.total_warps),
                             "filter scratch")) != PGB_OK) {
            pgb_searcher_destroy(S);
            return s;
        }
        if (S->flat.gvisited_words &&
            (s = cuda_status(cudaMalloc(&S->gvisited, 4ull * S->flat.gvisited_words * S->flat.total_warps),
                             "visited scratch")) != PGB_OK) {
            pgb_searcher_destroy(S);
            return s;
        }
    } else {
        if ((s = hnsw_prepare(ix, *params, S->hnsw)) != PGB_OK) {
            pgb_searcher_destroy(S);
            return s;
        }
    }
    // staging for the host-memory path
    const size_t k = params->k;
    if ((s = cuda_status(cudaMalloc(&S->q_dev, (size_t)max_queries * ix->dim), "query staging")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&S->ids_dev, 4ull * max_queries * k), "ids staging")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&S->dists_dev, 4ull * max_queries * k), "dists staging")) != PGB_OK ||
        (s = cuda_status(cudaMalloc(&S->stats_dev, sizeof(pgb_query_stats) * max_queries),
                         "stats staging")) != PGB_OK ||
        (s = cuda_status(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking), "stream")) != PGB_OK) {
        pgb_searcher_destroy(S);
        return s;
    }
    *out = S;
    return PGB_OK;
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" {

pgb_status pgb_searcher_create(pgb_index* ix, uint32_t max_queries,
                               const pgb_query_params* params, pgb_searcher** out) {
    return create_searcher(ix, max_queries, params, 0, out);
}

pgb_status pgb_searcher_create_compressed(pgb_index* ix, uint32_t max_queries,
                                          const pgb_query_params* params, uint32_t rerank,
                                          pgb_searcher** out) {
    if (rerank == 0) return fail(PGB_ERR_BAD_ARG, "rerank == 0");
    return create_searcher(ix, max_queries, params, rerank, out);
}

pgb_status pgb_searcher_search(pgb_searcher* S, const void* queries, uint32_t nq,
                               uint32_t query_stride, uint32_t* ids, int32_t* dists,
                               pgb_query_stats* stats, void* stream) {
    if (!S) return fail(PGB_ERR_BAD_ARG, "null searcher");
    if (nq == 0) return PGB_OK;
    if (!queries || !ids || !dists) return fail(PGB_ERR_BAD_ARG, "null queries or outputs");
    const pgb_index* ix = S->index;
    if (nq > S->max_queries) return fail(PGB_ERR_BAD_ARG, "nq above the searcher's max_queries");
    if (query_stride < ix->dim) return fail(PGB_ERR_BAD_ARG, "query_stride below dim");
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    const pgb_query_params& p = S->params;
    cudaStream_t st = (cudaStream_t)stream;
    if (ix->is_hnsw) return hnsw_launch(ix, S->hnsw, p, queries, nq, query_stride, ids, dists, stats, st);
    FlatArgs A{};
    A.rows = ix->rows;
    A.adj = ix->adj;
    A.n = ix->n;
    A.gs = ix->gs;
    A.deg_lim = p.degree_limit ? std::min(p.degree_limit, ix->G) : ix->G;
    A.dim = ix->dim;
    A.start = 0;  // ParlayANN's wrapper always starts at point 0 (busqueda.cu:166-167)
    A.queries = (const uint8_t*)queries;
    A.nq = nq;
    A.qstride = query_stride;
    A.cut = p.cut;
    A.limit = (p.limit <= 0) ? (int64_t)ix->n : p.limit;
    A.excl = p.exclude_query_id ? 1u : 0u;
    A.qbase = p.query_id_base;
    A.norm_in_row = ix->norm_in_row ? 1u : 0u;
    A.Ls = p.beam_size;
    A.k = p.k;
    A.out_stride = p.k;
    A.ids = ids;
    A.dists = dists;
    A.stats = stats;
    A.gfilter = S->gfilter;
    A.gvisited = S->gvisited;
    if (!S->codes) return launch_flat(S->flat, A, st, ix);
    // code rows: the search keeps the first `rerank` entries of each frontier, then the
    // exact re-rank writes the caller's k
    A.rows = ix->codes;
    A.code_step = ix->code_step;
    A.code_off = ix->code_off;
    A.k = S->rerank;
    A.out_stride = S->rerank;
    A.ids = S->cand;
    A.dists = S->cand_d;
    pgb_status s = launch_flat(S->flat, A, st, ix);
    if (s != PGB_OK) return s;
    return rerank_launch(ix, queries, nq, query_stride, S->cand, S->rerank, p.k, ids, dists, st);
}

pgb_status pgb_searcher_search_host(pgb_searcher* S, const void* queries, uint32_t nq,
                                    uint32_t query_stride, uint32_t* ids, int32_t* dists,
                                    pgb_query_stats* stats) {
    if (!S) return fail(PGB_ERR_BAD_ARG, "null searcher");
    if (nq == 0) return PGB_OK;
    if (!queries || !ids || !dists) return fail(PGB_ERR_BAD_ARG, "null queries or outputs");
    const pgb_index* ix = S->index;
    if (nq > S->max_queries) return fail(PGB_ERR_BAD_ARG, "nq above the searcher's max_queries");
    if (query_stride < ix->dim) return fail(PGB_ERR_BAD_ARG, "query_stride below dim");
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    const size_t k = S->params.k;
    cudaStream_t st = S->stream;
    pgb_status s;
    // page-locked host buffers: the launch reads the queries (at their stride) and writes
    // the results through them, so the transfers overlap the search
    void* pq = pinned_device_ptr(queries);
    void* pi = pinned_device_ptr(ids);
    void* pd = pinned_device_ptr(dists);
    void* ps = stats ? pinned_device_ptr(stats) : nullptr;
    if (pq && pi && pd && (!stats || ps)) {
        if ((s = pgb_searcher_search(S, pq, nq, query_stride, static_cast<uint32_t*>(pi),
                                     static_cast<int32_t*>(pd), static_cast<pgb_query_stats*>(ps),
                                     st)) != PGB_OK)
            return s;
        return cuda_status(cudaStreamSynchronize(st), "search");
    }
    // queries packed to dim bytes on the way in (one linear copy when already packed)
    cudaError_t ce =
        (query_stride == ix->dim)
            ? cudaMemcpyAsync(S->q_dev, queries, (size_t)nq * ix->dim, cudaMemcpyHostToDevice, st)
            : cudaMemcpy2DAsync(S->q_dev, ix->dim, queries, query_stride, ix->dim, nq,
                                cudaMemcpyHostToDevice, st);
    if ((s = cuda_status(ce, "query upload")) != PGB_OK) return s;
    if ((s = pgb_searcher_search(S, S->q_dev, nq, ix->dim, S->ids_dev, S->dists_dev,
                                 stats ? S->stats_dev : nullptr, st)) != PGB_OK)
        return s;
    if ((s = cuda_status(cudaMemcpyAsync(ids, S->ids_dev, 4ull * nq * k, cudaMemcpyDeviceToHost, st),
                         "ids download")) != PGB_OK ||
        (s = cuda_status(cudaMemcpyAsync(dists, S->dists_dev, 4ull * nq * k, cudaMemcpyDeviceToHost, st),
                         "dists download")) != PGB_OK)
        return s;
    if (stats &&
        (s = cuda_status(cudaMemcpyAsync(stats, S->stats_dev, sizeof(pgb_query_stats) * nq,
                                         cudaMemcpyDeviceToHost, st),
                         "stats download")) != PGB_OK)
        return s;
    return cuda_status(cudaStreamSynchronize(st), "search");
}

pgb_status pgb_searcher_destroy(pgb_searcher* S) {
    if (!S) return PGB_OK;
    DeviceGuard guard(S->index ? S->index->device : 0);
    if (S->stream) cudaStreamDestroy(S->stream);
    cudaFree(S->gfilter);
    cudaFree(S->gvisited);
    cudaFree(S->cand);
    cudaFree(S->cand_d);
    cudaFree(S->q_dev);
    cudaFree(S->ids_dev);
    cudaFree(S->dists_dev);
    cudaFree(S->stats_dev);
    hnsw_release(S->hnsw);
    delete S;
    return PGB_OK;
}

}  // extern "C"
