// capi_host.cpp -- host-only C ABI entry points: errors, recall, builders, graph writer.
#include <algorithm>
#include <cmath>
#include <vector>

#include "builders.h"
#include "errors.h"
#include "formats.h"
#include "host_common.h"

namespace pgb {

static thread_local std::string g_last_error;
void set_error(const std::string& m) { g_last_error = m; }

static pgb_status check_vectors(const void* v, uint32_t n, uint32_t dim, pgb_elem elem,
                                HostVectors& hv) {
    if (!v || n == 0 || dim == 0 || dim > PGB_MAX_DIM)
        return fail(PGB_ERR_BAD_ARG, "vectors: null pointer, n == 0 or dim outside 1..128");
    if (elem != PGB_INT8 && elem != PGB_UINT8) return fail(PGB_ERR_BAD_ARG, "unknown element type");
    hv.data = static_cast<const uint8_t*>(v);
    hv.n = n;
    hv.dim = dim;
    hv.stride = dim;
    hv.is_signed = elem == PGB_INT8;
    return PGB_OK;
}

}  // namespace pgb

using namespace pgb;

extern "C" {

const char* pgb_status_string(pgb_status s) {
    switch (s) {
        case PGB_OK: return "ok";
        case PGB_ERR_BAD_ARG: return "bad argument";
        case PGB_ERR_OOM: return "out of memory";
        case PGB_ERR_CUDA: return "CUDA error";
        case PGB_ERR_OVERFLOW: return "capacity overflow";
        case PGB_ERR_IO: return "I/O error";
        case PGB_ERR_FORMAT: return "format error";
        case PGB_ERR_BUSY: return "busy";
        case PGB_ERR_TIMEOUT: return "timeout";
        case PGB_ERR_NOT_FOUND: return "not found";
    }
    return "unknown status";
}

const char* pgb_last_error(void) { return g_last_error.c_str(); }

double pgb_recall(const uint32_t* gt_ids, const float* gt_dists, uint32_t nq, uint32_t gt_k,
                  const uint32_t* ids, uint32_t k) {
    if (!gt_ids || !gt_dists || !ids || nq == 0 || k == 0 || k > gt_k) return -1.0;
    long long total = 0;
    std::vector<uint32_t> mine;
    for (uint32_t q = 0; q < nq; q++) {
        const uint32_t* truth = gt_ids + (size_t)q * gt_k;
        const float* dt = gt_dists + (size_t)q * gt_k;
        // ground-truth prefix extended over distance ties with the k-th
        uint32_t end = gt_k;
        if (gt_k != k) {
            const float ref = dt[k - 1];
            for (uint32_t i = k; i < gt_k; i++)
                if (!(std::fabs(ref - dt[i]) < 1e-6f)) {
                    end = i;
                    break;
                }
        }
        mine.assign(ids + (size_t)q * k, ids + (size_t)(q + 1) * k);
        std::sort(mine.begin(), mine.end());
        mine.erase(std::unique(mine.begin(), mine.end()), mine.end());
        for (uint32_t x : mine)
            if (std::find(truth, truth + end, x) != truth + end) total++;
    }
    return (double)total / nq / k;
}

pgb_status pgb_build_vamana(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                            uint32_t R, uint32_t L, float alpha, int passes, uint64_t seed,
                            int nthreads, uint32_t* degrees, uint32_t* adjacency) {
    HostVectors hv;
    pgb_status s = check_vectors(vectors, n, dim, elem, hv);
    if (s != PGB_OK) return s;
    if (!degrees || !adjacency || R == 0 || R > PGB_MAX_DEGREE || L == 0 || passes < 1 ||
        !(alpha > 0))
        return fail(PGB_ERR_BAD_ARG, "vamana: bad R / L / alpha / passes or null output");
    build_vamana(hv, R, L, alpha, passes, seed, nthreads, degrees, adjacency);
    return PGB_OK;
}

pgb_status pgb_build_hcnng(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                           uint32_t trees, uint32_t leaf, uint32_t mst_deg, uint64_t seed,
                           int nthreads, uint32_t* degrees, uint32_t* adjacency) {
    HostVectors hv;
    pgb_status s = check_vectors(vectors, n, dim, elem, hv);
    if (s != PGB_OK) return s;
    if (!degrees || !adjacency || trees == 0 || mst_deg == 0 || leaf < 2 ||
        (uint64_t)trees * mst_deg > PGB_MAX_DEGREE)
        return fail(PGB_ERR_BAD_ARG, "hcnng: bad trees / leaf / mst_deg or null output");
    build_hcnng(hv, trees, leaf, mst_deg, seed, nthreads, degrees, adjacency);
    return PGB_OK;
}

pgb_status pgb_build_nndescent(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                               uint32_t K, uint32_t init_trees, uint32_t leaf, float alpha,
                               float delta, uint32_t max_iters, uint64_t seed, int nthreads,
                               uint32_t* degrees, uint32_t* adjacency) {
    HostVectors hv;
    pgb_status s = check_vectors(vectors, n, dim, elem, hv);
    if (s != PGB_OK) return s;
    if (!degrees || !adjacency || K == 0 || K > PGB_MAX_DEGREE || init_trees == 0 ||
        !(alpha > 0))
        return fail(PGB_ERR_BAD_ARG, "nndescent: bad K / init_trees / alpha or null output");
    build_nndescent(hv, K, init_trees, leaf, alpha, delta, max_iters, seed, nthreads, degrees,
                    adjacency);
    return PGB_OK;
}

pgb_status pgb_build_hnsw(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                          uint32_t M, uint32_t ef_construction, float ml, float alpha,
                          uint64_t seed, int nthreads, const char* path) {
    HostVectors hv;
    pgb_status s = check_vectors(vectors, n, dim, elem, hv);
    if (s != PGB_OK) return s;
    if (!path || M == 0 || 2 * M > PGB_MAX_DEGREE || ef_construction == 0 || !(ml > 0))
        return fail(PGB_ERR_BAD_ARG, "hnsw: bad M / ef_construction / ml or null path");
    HnswBuilt B;
    build_hnsw(hv, M, ef_construction, ml, alpha, seed, nthreads, B);
    HnswFile h;
    h.n = n;
    h.dim = dim;
    h.m = M;
    h.efc = ef_construction;
    h.ml = ml;
    h.alpha = alpha;
    h.levels = B.level;
    h.node_point.resize(n);
    for (uint32_t i = 0; i < n; i++) h.node_point[i] = i;
    h.list_sizes = B.sizes;
    for (size_t li = 0; li < B.sizes.size(); li++)
        h.ids.insert(h.ids.end(), B.rows.begin() + B.row_off[li],
                     B.rows.begin() + B.row_off[li] + B.sizes[li]);
    h.entries = {B.entry};
    std::string e = write_hnsw(path, h);
    if (!e.empty()) return fail(PGB_ERR_IO, e);
    return PGB_OK;
}

pgb_status pgb_file_check(const char* path, int kind, uint64_t info[4]) {
    if (!path) return fail(PGB_ERR_BAD_ARG, "null path");
    bool io = false;
    std::string e;
    uint64_t out[4] = {0, 0, 0, 0};
    if (kind == 0) {
        VectorFile v;
        e = read_vectors(path, v, &io);
        out[0] = v.n, out[1] = v.dim, out[2] = v.data.size();
    } else if (kind == 1) {
        GraphFile g;
        e = read_graph(path, g, &io);
        out[0] = g.n, out[1] = g.max_degree, out[2] = g.edges.size();
    } else if (kind == 2) {
        HnswFile h;
        e = read_hnsw(path, h, &io);
        out[0] = h.n, out[1] = h.dim, out[2] = h.list_sizes.size(), out[3] = h.entries.size();
    } else {
        return fail(PGB_ERR_BAD_ARG, "kind must be 0 (vectors), 1 (graph) or 2 (HNSW)");
    }
    if (!e.empty()) return fail(io ? PGB_ERR_IO : PGB_ERR_FORMAT, e);
    if (info)
        for (int i = 0; i < 4; i++) info[i] = out[i];
    return PGB_OK;
}

pgb_status pgb_write_graph(const char* path, uint32_t n, uint32_t slots,
                           const uint32_t* degrees, const uint32_t* adjacency) {
    if (!path || !degrees || !adjacency || n == 0 || slots == 0)
        return fail(PGB_ERR_BAD_ARG, "write_graph: null argument or empty graph");
    for (uint32_t i = 0; i < n; i++)
        if (degrees[i] > slots) return fail(PGB_ERR_BAD_ARG, "write_graph: degree above slots");
    std::string e = write_graph(path, n, slots, degrees, adjacency);
    if (!e.empty()) return fail(PGB_ERR_IO, e);
    return PGB_OK;
}

}  // extern "C"
