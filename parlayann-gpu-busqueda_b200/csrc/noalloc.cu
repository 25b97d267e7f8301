// noalloc.cu -- pgb_search_flat_noalloc: the plain flat-graph search for callers that
// may not allocate device memory at query time (cudaMalloc / cudaFree can synchronise
// the device and stall a serving process's other streams, and a host framework's caching
// allocator may already hold the free memory). The kernel is flat_plain_kernel, the same
// one pgb_searcher_search launches; only where its per-warp visited tables live differs:
// in the fixed array below instead of a searcher's cudaMalloc'd scratch.
#include <algorithm>
#include <mutex>
#include <string>

#include "errors.h"
#include "index.h"
#include "search_plan.h"
#include "searcher.h"

namespace {

constexpr size_t kScratchWords = PGB_NOALLOC_SCRATCH_BYTES / 4;

// The visited tables of every pgb_search_flat_noalloc call on a device (16 MiB). Each
// query clears its own table before use, so no part of it has to start at zero. All calls
// share it: two calls whose kernels overlap on the GPU corrupt each other's tables.
// Host code must not hand this name to a kernel (on the host it is only a stand-in for
// the symbol); the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;

// per device: the array's device address (looked up once, with that device current) and
// the last launch plan, reused while (beam, degree limit, element type) stay the same
struct DeviceSlot {
    uint32_t* scratch = nullptr;
    bool have_plan = false;
    uint32_t ls = 0, deg_lim = 0;
    bool is_signed = false;
    pgb::FlatPlan plan{};
};
std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];

}  // namespace

using namespace pgb;

extern "C" pgb_status pgb_search_flat_noalloc(const pgb_index* ix, const pgb_query_params* params,
                                              const void* queries, uint32_t nq,
                                              uint32_t query_stride, uint32_t* ids,
                                              int32_t* dists, pgb_query_stats* stats,
                                              void* stream) {
    if (!ix) return fail(PGB_ERR_BAD_ARG, "null index");
    if (ix->is_hnsw)
        return fail(PGB_ERR_BAD_ARG, "pgb_search_flat_noalloc serves flat-graph indexes only");
    pgb_status s = check_params(ix, params);
    if (s != PGB_OK) return s;
    if (params->beam_size > PGB_NOALLOC_MAX_BEAM)
        return fail(PGB_ERR_BAD_ARG, "beam_size " + std::to_string(params->beam_size) +
                                         " above the no-allocation maximum of " +
                                         std::to_string(PGB_NOALLOC_MAX_BEAM));
    if (nq == 0) return PGB_OK;
    if (!queries || !ids || !dists) return fail(PGB_ERR_BAD_ARG, "null queries or outputs");
    if (query_stride < ix->dim) return fail(PGB_ERR_BAD_ARG, "query_stride below dim");
    if (ix->device < 0 || ix->device >= kMaxDevices)
        return fail(PGB_ERR_BAD_ARG, "device ordinal above the no-allocation table");
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");

    const pgb_query_params& p = *params;
    const uint32_t deg_lim = p.degree_limit ? std::min(p.degree_limit, ix->G) : ix->G;
    const bool is_signed = ix->elem == PGB_INT8;
    FlatPlan P;
    uint32_t* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        DeviceSlot& d = g_slots[ix->device];
        if (!d.scratch) {
            // set-up, once per device, with that device current (the guard above)
            uint32_t* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_status(e, "no-allocation scratch address");
            d.scratch = ptr;
        }
        scratch = d.scratch;
        if (!d.have_plan || d.ls != p.beam_size || d.deg_lim != deg_lim || d.is_signed != is_signed) {
            FlatPlanRequest rq;
            rq.max_ls = p.beam_size;
            rq.deg_lim = deg_lim;
            rq.is_signed = is_signed;
            rq.batched = false;
            rq.force_filter_placement = true;  // the filter never takes scratch
            rq.filter_in_shared = true;
            rq.visited_smem_limit = 0;         // the visited tables live in the array
            FlatPlan np;
            if ((s = plan_flat(rq, np)) != PGB_OK) return s;
            // run no more warps than the array holds visited tables for
            const uint64_t fit_blocks =
                (kScratchWords / np.gvisited_words) / (uint64_t)np.warps_per_block;
            if (fit_blocks == 0) return fail(PGB_ERR_BAD_ARG, "beam too wide for the no-allocation scratch");
            if ((uint64_t)np.blocks > fit_blocks) {
                np.blocks = (int)fit_blocks;
                np.total_warps = fit_blocks * (uint64_t)np.warps_per_block;
            }
            d.plan = np;
            d.ls = p.beam_size;
            d.deg_lim = deg_lim;
            d.is_signed = is_signed;
            d.have_plan = true;
        }
        P = d.plan;
    }

    FlatArgs A{};
    A.rows = ix->rows;
    A.adj = ix->adj;
    A.n = ix->n;
    A.gs = ix->gs;
    A.deg_lim = deg_lim;
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
    A.gfilter = nullptr;
    A.gvisited = scratch;
    return launch_flat(P, A, (cudaStream_t)stream);
}
