// index.cu -- index creation: uploads and device-side re-layout of vectors and graphs.
// Replaces subirVectores / subirGrafo / subirHnsw (reference cuda/datos_gpu.cu:8-81,
// cuda/busqueda_hnsw.cu:462-530). Padding happens on the device, so no padded host
// copy (the reference builds up to 600 MB on the host, cuda/datos_gpu.cu:68-72).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "errors.h"
#include "formats.h"
#include "index.h"

namespace pgb {
namespace {

// packed rows of `dim` bytes -> 128-byte zero-padded rows, one thread per 16-byte word
__global__ void pad_rows_kernel(const uint8_t* __restrict__ packed, uint32_t n, uint32_t dim,
                                const uint32_t* __restrict__ gather, uint8_t* __restrict__ rows) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t r = t >> 3;
    const uint32_t w = (uint32_t)(t & 7);
    if (r >= n) return;
    const uint64_t src_row = gather ? gather[r] : r;
    const uint8_t* src = packed + src_row * dim;
    uint8_t b[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t c = w * 16 + i;
        b[i] = (c < dim) ? src[c] : 0;
    }
    int4 v;
    memcpy(&v, b, 16);
    reinterpret_cast<int4*>(rows + r * 128)[w] = v;
}

// squared norm of each row into bytes 124..127 (rows of at most 124 meaningful bytes)
template <bool Signed>
__global__ void norm_rows_kernel(uint8_t* __restrict__ rows, uint32_t n) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int4* row = reinterpret_cast<int4*>(rows + r * 128);
    int32_t s = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        int4 v = row[w];
        if (w == 7) v.w = 0;
        s += partial_sq<Signed>(v);
    }
    reinterpret_cast<int32_t*>(rows + r * 128)[31] = s;
}

// CSR rows -> fixed-stride rows padded with 0xFFFFFFFF, one thread per slot
__global__ void expand_rows_kernel(const uint64_t* __restrict__ offsets,
                                   const uint32_t* __restrict__ sizes,
                                   const uint32_t* __restrict__ edges, uint64_t nrows,
                                   uint32_t stride, uint32_t* __restrict__ out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t r = t / stride;
    const uint32_t j = (uint32_t)(t % stride);
    if (r >= nrows) return;
    out[t] = (j < sizes[r]) ? edges[offsets[r] + j] : 0xFFFFFFFFu;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

pgb_status cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(PGB_ERR_OOM, std::string(what) + ": out of device memory");
    return fail(PGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

pgb_status dev_alloc(void** p, size_t bytes, const char* what) {
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_fail(e, what);
    }
    return PGB_OK;
}

pgb_status upload(void* dst, const void* src, size_t bytes, const char* what) {
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? PGB_OK : cuda_fail(e, what);
}

// packed host vectors -> padded device rows (optionally gathered by node); rows of at
// most 124 bytes get their squared norm in bytes 124..127
pgb_status make_rows(const void* vectors, uint32_t n_src, uint32_t dim, bool is_signed,
                     const uint32_t* gather, uint32_t n_out, uint8_t** rows) {
    DevBuf packed, g;
    pgb_status s = dev_alloc(&packed.p, (size_t)n_src * dim, "vectors");
    if (s != PGB_OK) return s;
    if ((s = upload(packed.p, vectors, (size_t)n_src * dim, "vectors")) != PGB_OK) return s;
    if (gather) {
        if ((s = dev_alloc(&g.p, 4ull * n_out, "node map")) != PGB_OK) return s;
        if ((s = upload(g.p, gather, 4ull * n_out, "node map")) != PGB_OK) return s;
    }
    if ((s = dev_alloc((void**)rows, 128ull * n_out, "vector rows")) != PGB_OK) return s;
    const uint64_t threads = 8ull * n_out;
    pad_rows_kernel<<<(unsigned)((threads + 255) / 256), 256>>>(
        (const uint8_t*)packed.p, n_out, dim, (const uint32_t*)g.p, *rows);
    if (dim <= kNormInRowMaxDim) {
        const unsigned nb = (unsigned)((n_out + 255ull) / 256);
        if (is_signed) norm_rows_kernel<true><<<nb, 256>>>(*rows, n_out);
        else norm_rows_kernel<false><<<nb, 256>>>(*rows, n_out);
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? PGB_OK : cuda_fail(e, "pad rows");
}

// CSR (sizes + concatenated ids) -> padded matrix nrows x stride on the device
pgb_status make_matrix(const std::vector<uint32_t>& sizes, const uint32_t* ids, uint64_t nids,
                       uint32_t stride, uint32_t** out) {
    const uint64_t nrows = sizes.size();
    std::vector<uint64_t> off(nrows + 1, 0);
    for (uint64_t i = 0; i < nrows; i++) off[i + 1] = off[i] + sizes[i];
    DevBuf doff, dsz, de;
    pgb_status s;
    if ((s = dev_alloc(&doff.p, 8 * nrows, "row offsets")) != PGB_OK) return s;
    if ((s = dev_alloc(&dsz.p, 4 * nrows, "row sizes")) != PGB_OK) return s;
    if ((s = dev_alloc(&de.p, 4 * nids, "edges")) != PGB_OK) return s;
    if ((s = upload(doff.p, off.data(), 8 * nrows, "row offsets")) != PGB_OK) return s;
    if ((s = upload(dsz.p, sizes.data(), 4 * nrows, "row sizes")) != PGB_OK) return s;
    if (nids && (s = upload(de.p, ids, 4 * nids, "edges")) != PGB_OK) return s;
    if ((s = dev_alloc((void**)out, 4ull * nrows * stride, "adjacency")) != PGB_OK) return s;
    const uint64_t threads = nrows * stride;
    expand_rows_kernel<<<(unsigned)((threads + 255) / 256), 256>>>(
        (const uint64_t*)doff.p, (const uint32_t*)dsz.p, (const uint32_t*)de.p, nrows, stride,
        *out);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? PGB_OK : cuda_fail(e, "expand rows");
}

uint32_t round32(uint32_t x) { return std::max<uint32_t>(32, (x + 31u) & ~31u); }

void free_index(pgb_index* ix) {
    if (!ix) return;
    DeviceGuard g(ix->device);
    cudaFree(ix->rows);
    cudaFree(ix->adj);
    cudaFree(ix->adj0);
    cudaFree(ix->adju);
    cudaFree(ix->upper_start);
    cudaFree(ix->node_point);
    if (ix->node_rows && ix->node_rows != ix->rows) cudaFree(ix->node_rows);
    cudaFree(ix->codes);
    cudaFree(ix->code_off);
    delete ix;
}

pgb_status check_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(PGB_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(PGB_ERR_BAD_ARG, "device index out of range");
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess)
        return fail(PGB_ERR_CUDA, "cudaGetDeviceProperties failed");
    if (p.major != 10)
        return fail(PGB_ERR_CUDA, "device is not compute capability 10.x (this build is sm_100a)");
    return PGB_OK;
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" {

int pgb_device_available(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    for (int d = 0; d < count; d++) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) return 1;
    }
    return 0;
}

pgb_status pgb_index_create_flat(int device, const void* vectors, uint32_t n, uint32_t dim,
                                 pgb_elem elem, const uint32_t* degrees, const uint32_t* edges,
                                 pgb_index** out) {
    if (!out) return fail(PGB_ERR_BAD_ARG, "null output handle");
    *out = nullptr;
    if (!vectors || !degrees || n == 0 || dim == 0 || dim > PGB_MAX_DIM)
        return fail(PGB_ERR_BAD_ARG, "null arrays, n == 0 or dim outside 1..128");
    if (elem != PGB_INT8 && elem != PGB_UINT8) return fail(PGB_ERR_BAD_ARG, "unknown element type");
    uint64_t total = 0;
    uint32_t G = 0;
    for (uint32_t i = 0; i < n; i++) {
        if (degrees[i] > PGB_MAX_DEGREE) return fail(PGB_ERR_BAD_ARG, "degree above 256");
        G = std::max(G, degrees[i]);
        total += degrees[i];
    }
    if (total && !edges) return fail(PGB_ERR_BAD_ARG, "null edges");
    for (uint64_t e = 0; e < total; e++)
        if (edges[e] >= n) return fail(PGB_ERR_FORMAT, "edge id out of range");
    pgb_status s = check_device(device);
    if (s != PGB_OK) return s;
    DeviceGuard guard(device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    pgb_index* ix = new pgb_index();
    ix->device = device;
    ix->n = n;
    ix->dim = dim;
    ix->elem = elem;
    ix->G = std::max<uint32_t>(G, 1);
    ix->gs = round32(ix->G);
    std::vector<uint32_t> sizes(degrees, degrees + n);
    ix->norm_in_row = dim <= kNormInRowMaxDim;
    if ((s = make_rows(vectors, n, dim, elem == PGB_INT8, nullptr, n, &ix->rows)) != PGB_OK ||
        (s = make_matrix(sizes, edges, total, ix->gs, &ix->adj)) != PGB_OK) {
        free_index(ix);
        return s;
    }
    ix->device_bytes = 128ull * n + 4ull * n * ix->gs;
    *out = ix;
    return PGB_OK;
}

pgb_status pgb_index_create_hnsw(int device, const void* vectors, uint32_t n_points,
                                 uint32_t dim, pgb_elem elem, uint32_t n_nodes,
                                 const uint32_t* levels, const uint32_t* node_point,
                                 const uint32_t* list_sizes, const uint32_t* ids,
                                 const uint32_t* entries, uint32_t n_entries, pgb_index** out) {
    if (!out) return fail(PGB_ERR_BAD_ARG, "null output handle");
    *out = nullptr;
    if (!vectors || !levels || !node_point || !list_sizes || !entries || n_points == 0 ||
        n_nodes == 0 || dim == 0 || dim > PGB_MAX_DIM)
        return fail(PGB_ERR_BAD_ARG, "null arrays, empty index or dim outside 1..128");
    if (elem != PGB_INT8 && elem != PGB_UINT8) return fail(PGB_ERR_BAD_ARG, "unknown element type");
    if (n_entries == 0 || n_entries > PGB_MAX_HNSW_ENTRIES)
        return fail(PGB_ERR_FORMAT, "HNSW needs 1..8 entry points");
    // list index of each node's level-0 list
    std::vector<uint64_t> first(n_nodes);
    uint64_t nl = 0;
    for (uint32_t i = 0; i < n_nodes; i++) {
        if (levels[i] > 64) return fail(PGB_ERR_FORMAT, "node level above 64");
        if (node_point[i] >= n_points) return fail(PGB_ERR_FORMAT, "node maps to a missing point");
        first[i] = nl;
        nl += (uint64_t)levels[i] + 1;
    }
    uint64_t total = 0;
    uint32_t G0 = 0, GA = 0;
    for (uint32_t i = 0; i < n_nodes; i++)
        for (uint32_t l = 0; l <= levels[i]; l++) {
            const uint32_t sz = list_sizes[first[i] + l];
            if (sz > PGB_MAX_DEGREE) return fail(PGB_ERR_BAD_ARG, "HNSW degree above 256");
            if (l == 0) G0 = std::max(G0, sz);
            else GA = std::max(GA, sz);
            total += sz;
        }
    if (total && !ids) return fail(PGB_ERR_BAD_ARG, "null ids");
    // neighbours at level l must exist at level l (their rows are read there)
    {
        uint64_t off = 0;
        for (uint32_t i = 0; i < n_nodes; i++)
            for (uint32_t l = 0; l <= levels[i]; l++) {
                const uint32_t sz = list_sizes[first[i] + l];
                for (uint32_t j = 0; j < sz; j++) {
                    const uint32_t v = ids[off + j];
                    if (v >= n_nodes) return fail(PGB_ERR_FORMAT, "HNSW neighbour out of range");
                    if (levels[v] < l) return fail(PGB_ERR_FORMAT, "HNSW neighbour below its level");
                }
                off += sz;
            }
    }
    const uint32_t top = levels[entries[0] < n_nodes ? entries[0] : 0];
    for (uint32_t e = 0; e < n_entries; e++) {
        if (entries[e] >= n_nodes) return fail(PGB_ERR_FORMAT, "entry point out of range");
        if (levels[entries[e]] < top) return fail(PGB_ERR_FORMAT, "entry point below the top level");
    }
    pgb_status s = check_device(device);
    if (s != PGB_OK) return s;
    DeviceGuard guard(device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");

    pgb_index* ix = new pgb_index();
    ix->device = device;
    ix->is_hnsw = true;
    ix->n = n_points;
    ix->n_nodes = n_nodes;
    ix->dim = dim;
    ix->elem = elem;
    ix->G0 = std::max<uint32_t>(G0, 1);
    ix->g0s = round32(ix->G0);
    ix->GA = std::max<uint32_t>(GA, 1);
    ix->gas = round32(ix->GA);
    ix->top_level = top;
    ix->n_entries = n_entries;
    for (uint32_t e = 0; e < n_entries; e++) ix->entries[e] = entries[e];

    // split the lists into level 0 and upper-level blocks
    std::vector<uint32_t> sz0(n_nodes), ids0, szu, idsu, ustart(n_nodes, 0xFFFFFFFFu);
    ids0.reserve(total);
    {
        uint64_t off = 0;
        uint32_t blocks = 0;
        for (uint32_t i = 0; i < n_nodes; i++)
            for (uint32_t l = 0; l <= levels[i]; l++) {
                const uint32_t sz = list_sizes[first[i] + l];
                if (l == 0) {
                    sz0[i] = sz;
                    ids0.insert(ids0.end(), ids + off, ids + off + sz);
                } else {
                    if (l == 1) ustart[i] = blocks;
                    blocks++;
                    szu.push_back(sz);
                    idsu.insert(idsu.end(), ids + off, ids + off + sz);
                }
                off += sz;
            }
        if (szu.empty()) szu.push_back(0);  // keep a valid (empty) upper matrix
    }
    bool identity = n_nodes == n_points;
    for (uint32_t i = 0; i < n_nodes && identity; i++) identity = node_point[i] == i;
    ix->norm_in_row = dim <= kNormInRowMaxDim;
    if ((s = make_rows(vectors, n_points, dim, elem == PGB_INT8, nullptr, n_points, &ix->rows)) !=
        PGB_OK) {
        free_index(ix);
        return s;
    }
    if (identity) {
        ix->node_rows = ix->rows;
    } else if ((s = make_rows(vectors, n_points, dim, elem == PGB_INT8, node_point, n_nodes,
                              &ix->node_rows)) != PGB_OK) {
        free_index(ix);
        return s;
    }
    if ((s = make_matrix(sz0, ids0.data(), ids0.size(), ix->g0s, &ix->adj0)) != PGB_OK ||
        (s = make_matrix(szu, idsu.data(), idsu.size(), ix->gas, &ix->adju)) != PGB_OK ||
        (s = dev_alloc((void**)&ix->upper_start, 4ull * n_nodes, "upper starts")) != PGB_OK ||
        (s = upload(ix->upper_start, ustart.data(), 4ull * n_nodes, "upper starts")) != PGB_OK ||
        (s = dev_alloc((void**)&ix->node_point, 4ull * n_nodes, "node map")) != PGB_OK ||
        (s = upload(ix->node_point, node_point, 4ull * n_nodes, "node map")) != PGB_OK) {
        free_index(ix);
        return s;
    }
    ix->device_bytes = 128ull * n_points + (identity ? 0 : 128ull * n_nodes) +
                       4ull * n_nodes * ix->g0s + 4ull * szu.size() * ix->gas + 8ull * n_nodes;
    *out = ix;
    return PGB_OK;
}

pgb_status pgb_index_load_flat(int device, const char* vectors_path, pgb_elem elem,
                               const char* graph_path, pgb_index** out) {
    if (!out || !vectors_path || !graph_path) return fail(PGB_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    VectorFile v;
    GraphFile g;
    bool io = false;
    std::string e = read_vectors(vectors_path, v, &io);
    if (!e.empty()) return fail(io ? PGB_ERR_IO : PGB_ERR_FORMAT, e);
    e = read_graph(graph_path, g, &io);
    if (!e.empty()) return fail(io ? PGB_ERR_IO : PGB_ERR_FORMAT, e);
    if (g.n != v.n) return fail(PGB_ERR_FORMAT, "graph and vectors disagree on n");
    return pgb_index_create_flat(device, v.data.data(), v.n, v.dim, elem, g.degrees.data(),
                                 g.edges.data(), out);
}

pgb_status pgb_index_load_hnsw(int device, const char* vectors_path, pgb_elem elem,
                               const char* hnsw_path, pgb_index** out) {
    if (!out || !vectors_path || !hnsw_path) return fail(PGB_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    VectorFile v;
    HnswFile h;
    bool io = false;
    std::string e = read_vectors(vectors_path, v, &io);
    if (!e.empty()) return fail(io ? PGB_ERR_IO : PGB_ERR_FORMAT, e);
    e = read_hnsw(hnsw_path, h, &io);
    if (!e.empty()) return fail(io ? PGB_ERR_IO : PGB_ERR_FORMAT, e);
    return pgb_index_create_hnsw(device, v.data.data(), v.n, v.dim, elem, h.n, h.levels.data(),
                                 h.node_point.data(), h.list_sizes.data(), h.ids.data(),
                                 h.entries.data(), (uint32_t)h.entries.size(), out);
}

pgb_status pgb_index_get_info(const pgb_index* ix, pgb_index_info* out) {
    if (!ix || !out) return fail(PGB_ERR_BAD_ARG, "null argument");
    out->n_points = ix->n;
    out->dim = ix->dim;
    out->elem = (uint32_t)ix->elem;
    out->is_hnsw = ix->is_hnsw ? 1u : 0u;
    out->max_degree = ix->is_hnsw ? ix->G0 : ix->G;
    out->upper_degree = ix->is_hnsw ? ix->GA : 0u;
    out->top_level = ix->top_level;
    out->n_entries = ix->n_entries;
    out->device_bytes = ix->device_bytes;
    return PGB_OK;
}

pgb_status pgb_index_set_l2_window(pgb_index* ix, uint32_t region, uint64_t max_bytes,
                                   uint64_t* window_bytes, float* hit_ratio) {
    if (!ix) return fail(PGB_ERR_BAD_ARG, "null index");
    if (ix->is_hnsw) return fail(PGB_ERR_BAD_ARG, "the L2 window applies to flat-graph searches");
    const uint8_t* base = nullptr;
    size_t size = 0;
    switch (region) {
        case PGB_L2_NONE: break;
        case PGB_L2_ROWS: base = ix->rows; size = (size_t)kRowBytes * ix->n; break;
        case PGB_L2_CODES:
            if (!ix->codes) return fail(PGB_ERR_BAD_ARG, "index has no code rows (pgb_index_compress)");
            base = ix->codes;
            size = (size_t)kCodeRowBytes * ix->n;
            break;
        case PGB_L2_GRAPH: base = reinterpret_cast<const uint8_t*>(ix->adj); size = 4ull * ix->gs * ix->n; break;
        default: return fail(PGB_ERR_BAD_ARG, "unknown L2 window region");
    }
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e;
    if (region == PGB_L2_NONE) {
        // this process's set-aside back to none; persisting lines become normal lines
        ix->l2_base = nullptr;
        ix->l2_bytes = 0;
        ix->l2_hit = 0.f;
        e = cudaCtxResetPersistingL2Cache();
        if (e == cudaSuccess) e = cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
        if (e != cudaSuccess) return cuda_fail(e, "L2 set-aside");
        if (window_bytes) *window_bytes = 0;
        if (hit_ratio) *hit_ratio = 0.f;
        return PGB_OK;
    }
    int max_win = 0, max_persist = 0;
    if ((e = cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, ix->device)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ix->device)) != cudaSuccess)
        return cuda_fail(e, "L2 attributes");
    if (max_win <= 0 || max_persist <= 0) return fail(PGB_ERR_BAD_ARG, "device has no persisting L2 lines");
    size_t win = std::min(size, (size_t)max_win);
    if (max_bytes) win = std::min(win, (size_t)max_bytes);
    const size_t set_aside = std::min(win, (size_t)max_persist);
    // the set-aside belongs to this process's context and ends with it
    if ((e = cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, set_aside)) != cudaSuccess)
        return cuda_fail(e, "L2 set-aside");
    ix->l2_base = const_cast<uint8_t*>(base);
    ix->l2_bytes = win;
    ix->l2_hit = win ? std::min(1.f, (float)((double)set_aside / (double)win)) : 0.f;
    if (window_bytes) *window_bytes = win;
    if (hit_ratio) *hit_ratio = ix->l2_hit;
    return PGB_OK;
}

pgb_status pgb_index_destroy(pgb_index* ix) {
    if (ix && ix->l2_bytes) pgb_index_set_l2_window(ix, PGB_L2_NONE, 0, nullptr, nullptr);
    free_index(ix);
    return PGB_OK;
}

}  // extern "C"
