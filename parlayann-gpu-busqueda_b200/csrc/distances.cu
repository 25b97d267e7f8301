// distances.cu -- pgb_index_distances: exact squared L2 of (query, point) pairs, computed
// by the search kernels' own row code (row_round: 4 lanes per 128-byte row, dp4a, the norm
// folded into the row padding). It is the library's form of the reference's load-and-
// verify step, which compares the GPU distance of random and ground-truth pairs with the
// CPU one (cuda/paso1_carga.cu:33-123, cuda/lectores.cpp:172-179), and a building block
// for callers that re-rank candidates exactly.
#include <algorithm>
#include <string>

#include "errors.h"
#include "index.h"
#include "search_flat.cuh"
#include "search_plan.h"
#include "searcher.h"

namespace pgb {
namespace {

constexpr int kPairWarps = 4;  // warps per block; each warp takes 8 pairs per round

// One 4-lane group per pair: the group stages its query as a zero-padded 128-byte row in
// shared memory, computes ||q||^2, and row_round adds the row's part. Pairs naming a
// query or point out of range write INT32_MIN and raise *bad.
template <bool Signed>
__global__ void __launch_bounds__(kPairWarps * 32) pair_distance_kernel(
    const uint8_t* __restrict__ rows, uint32_t n, uint32_t dim, uint32_t norm_in_row,
    const uint8_t* __restrict__ queries, uint32_t nq, uint32_t qstride,
    const uint32_t* __restrict__ pairs, uint64_t npairs, int32_t* __restrict__ out,
    uint32_t* bad) {
    __shared__ __align__(16) uint32_t qrow[kPairWarps][8][32];
    __shared__ uint32_t pid[kPairWarps][8];
    __shared__ int32_t dout[kPairWarps][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int grp = lane >> 2, c = lane & 3;
    const bool nir = norm_in_row != 0;
    const bool need_a = (uint32_t)(c * 16) < dim;
    const bool need_b = (uint32_t)((c + 4) * 16) < dim || (nir && c == 3);
    const uint64_t stride = (uint64_t)gridDim.x * kPairWarps * 8u;
    for (uint64_t base = ((uint64_t)blockIdx.x * kPairWarps + w) * 8u; base < npairs; base += stride) {
        const uint64_t p = base + (uint64_t)grp;
        bool valid = p < npairs;
        uint32_t qi = 0, pi = 0;
        if (valid) {
            qi = __ldg(pairs + 2 * p);
            pi = __ldg(pairs + 2 * p + 1);
            if (qi >= nq || pi >= n) {
                if (c == 0) atomicOr(bad, 1u);
                valid = false;
                qi = 0;
                pi = 0;
            }
        }
        // the group's query row: lane c fills words c, c + 4, ..., zero past dim
        const uint8_t* src = queries + (size_t)qi * qstride;
        for (int wd = c; wd < 32; wd += 4) {
            uint32_t v = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const uint32_t i = 4u * wd + b;
                v |= (uint32_t)(i < dim ? src[i] : 0u) << (8 * b);
            }
            qrow[w][grp][wd] = v;
        }
        if (c == 0) pid[w][grp] = pi;
        __syncwarp();
        const int4* q4 = reinterpret_cast<const int4*>(qrow[w][grp]);
        const int4 qa = q4[c], qb = q4[c + 4];
        int32_t qq = partial_sq<Signed>(qa) + partial_sq<Signed>(qb);
        qq += __shfl_xor_sync(kFull, qq, 2, 4);
        qq += __shfl_xor_sync(kFull, qq, 1, 4);
        row_round<Signed, 1>(rows, pid[w], dout[w], 8, 0, qa, qb, qq, need_a, need_b, nir, grp, c);
        __syncwarp();
        if (c == 0 && p < npairs) out[p] = valid ? dout[w][grp] : INT32_MIN;
        __syncwarp();
    }
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" pgb_status pgb_index_distances(const pgb_index* ix, const void* queries, uint32_t nq,
                                          uint32_t query_stride, const uint32_t* pairs,
                                          uint64_t npairs, int32_t* out, void* stream) {
    if (!ix) return fail(PGB_ERR_BAD_ARG, "null index");
    if (npairs == 0) return PGB_OK;
    if (!queries || !pairs || !out || nq == 0) return fail(PGB_ERR_BAD_ARG, "null queries, pairs or output");
    if (query_stride < ix->dim) return fail(PGB_ERR_BAD_ARG, "query_stride below dim");
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st = (cudaStream_t)stream;
    // one device word for the range check, freed once the launch has completed
    uint32_t* bad = nullptr;
    pgb_status s = cuda_status(cudaMalloc(&bad, sizeof(uint32_t)), "distance check word");
    if (s != PGB_OK) return s;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t rounds = (npairs + 8u * kPairWarps - 1) / (8u * kPairWarps);
    const unsigned blocks = (unsigned)std::min<uint64_t>(rounds, (uint64_t)sms * 16u);
    // point rows: the index's point order (flat graphs; HNSW models store point i in row
    // i of `rows` as well)
    const uint8_t* rows = ix->rows;
    cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess) {
        if (ix->elem == PGB_INT8)
            pair_distance_kernel<true><<<blocks, kPairWarps * 32, 0, st>>>(
                rows, ix->n, ix->dim, ix->norm_in_row ? 1u : 0u, (const uint8_t*)queries, nq,
                query_stride, pairs, npairs, out, bad);
        else
            pair_distance_kernel<false><<<blocks, kPairWarps * 32, 0, st>>>(
                rows, ix->n, ix->dim, ix->norm_in_row ? 1u : 0u, (const uint8_t*)queries, nq,
                query_stride, pairs, npairs, out, bad);
        e = cudaGetLastError();
        if (e == cudaSuccess) count_launches(1);
    }
    uint32_t hbad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(bad);
    if (e != cudaSuccess) return cuda_status(e, "pair distances");
    if (hbad) return fail(PGB_ERR_BAD_ARG, "a pair names a query or point out of range (its output is INT32_MIN)");
    return PGB_OK;
}

// ---- gather calibration ----------------------------------------------------------------
// pgb_gather_probe: the distance of one query to n rows named by ids, with LANES threads
// per 128-byte row, to measure how fast this device gathers random rows (the reference
// measures the same, cuda/micro_distancias.cu:19-63). LANES 4 runs the search kernels' own
// row code (row_round, two slots: 16 rows in flight per warp, each load instruction
// covering whole 32-byte sectors of 8 rows); 1, 8 and 32 are the alternatives it was
// chosen over. Ids >= n give INT32_MIN (the row read is row 0's).
namespace pgb {
namespace {

constexpr int kProbeWarps = 4;

template <bool Signed, int LANES>
__global__ void __launch_bounds__(kProbeWarps * 32) gather_probe_kernel(
    const uint8_t* __restrict__ rows, uint32_t n, uint32_t dim, uint32_t norm_in_row,
    const uint8_t* __restrict__ query, const uint32_t* __restrict__ ids, uint64_t count,
    int32_t* __restrict__ out) {
    __shared__ __align__(16) uint32_t qrow[32];
    __shared__ uint32_t sid[kProbeWarps][16];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x < 32) {
        uint32_t v = 0;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const uint32_t i = 4u * threadIdx.x + b;
            v |= (uint32_t)(i < dim ? query[i] : 0u) << (8 * b);
        }
        qrow[threadIdx.x] = v;
    }
    __syncthreads();
    const int4* q4 = reinterpret_cast<const int4*>(qrow);
    const bool nir = norm_in_row != 0;
    const uint64_t warp = (uint64_t)blockIdx.x * kProbeWarps + w;
    const uint64_t warps = (uint64_t)gridDim.x * kProbeWarps;
    if constexpr (LANES == 4) {
        // the search's layout: 16 rows per warp per round, ids staged in shared memory
        const int grp = lane >> 2, c = lane & 3;
        const int4 qa = q4[c], qb = q4[c + 4];
        int32_t qq = partial_sq<Signed>(qa) + partial_sq<Signed>(qb);
        qq += __shfl_xor_sync(kFull, qq, 2, 4);
        qq += __shfl_xor_sync(kFull, qq, 1, 4);
        const bool need_a = (uint32_t)(c * 16) < dim;
        const bool need_b = (uint32_t)((c + 4) * 16) < dim || (nir && c == 3);
        for (uint64_t base = warp * 16u; base < count; base += warps * 16u) {
            const int np = count - base < 16u ? (int)(count - base) : 16;
            if (lane < np) {
                const uint32_t id = __ldg(ids + base + lane);
                sid[w][lane] = id < n ? id : 0u;
            }
            __syncwarp();
            row_round<Signed, 2>(rows, sid[w], out + base, np, 0, qa, qb, qq, need_a, need_b, nir, grp, c);
            __syncwarp();
            if (lane < np && __ldg(ids + base + lane) >= n) out[base + lane] = INT32_MIN;
            __syncwarp();
        }
    } else {
        // LANES threads per row, each reading 128 / LANES bytes; rows per warp per round:
        // 32 / LANES, times SLOTS rows in flight per group
        constexpr int GROUPS = 32 / LANES;
        constexpr int SLOTS = LANES == 1 ? 1 : (LANES == 8 ? 2 : 4);
        constexpr int BYTES = 128 / LANES;
        const int grp = lane / LANES, c = lane % LANES;
        int32_t qq = partial_sq<Signed>(q4[lane & 7]);
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) qq += __shfl_xor_sync(kFull, qq, off, 8);
        for (uint64_t base = warp * (GROUPS * SLOTS); base < count; base += warps * (GROUPS * SLOTS)) {
            int32_t t[SLOTS];
            uint32_t rid[SLOTS];
#pragma unroll
            for (int r = 0; r < SLOTS; r++) {
                const uint64_t i = base + (uint64_t)r * GROUPS + grp;
                const uint32_t id = i < count ? __ldg(ids + i) : 0u;
                rid[r] = id;
                const uint8_t* row = rows + (size_t)(id < n ? id : 0u) * kRowBytes + c * BYTES;
                int32_t acc = 0;
                if constexpr (BYTES >= 16) {
#pragma unroll
                    for (int j = 0; j < BYTES / 16; j++) {
                        const int wd = c * (BYTES / 16) + j;  // 16-byte word of the row
                        const int4 v = ldg16(row + 16 * j);
                        acc += (nir ? (wd == 7 ? v.w : 0) - 2 * partial_dot<Signed>(v, q4[wd])
                                    : partial_l2<Signed>(v, q4[wd]));
                    }
                } else {
                    const int32_t v = __ldg(reinterpret_cast<const int32_t*>(row));
                    const int32_t qw = (int32_t)qrow[c];
                    int32_t d;
                    if (Signed) d = __dp4a(v, qw, 0);
                    else d = (int32_t)__dp4a((uint32_t)v, (uint32_t)qw, 0u);
                    int32_t pp;
                    if (Signed) pp = __dp4a(v, v, 0);
                    else pp = (int32_t)__dp4a((uint32_t)v, (uint32_t)v, 0u);
                    acc = nir ? (c == 31 ? v : 0) - 2 * d : pp - 2 * d;
                }
                t[r] = acc;
            }
#pragma unroll
            for (int off = LANES / 2; off > 0; off >>= 1)
#pragma unroll
                for (int r = 0; r < SLOTS; r++) t[r] += __shfl_xor_sync(kFull, t[r], off, LANES);
            if (c == 0) {
#pragma unroll
                for (int r = 0; r < SLOTS; r++) {
                    const uint64_t i = base + (uint64_t)r * GROUPS + grp;
                    if (i < count) out[i] = rid[r] < n ? qq + t[r] : INT32_MIN;
                }
            }
        }
    }
}

template <int LANES>
void* probe_kernel(bool is_signed) {
    return is_signed ? (void*)gather_probe_kernel<true, LANES> : (void*)gather_probe_kernel<false, LANES>;
}

}  // namespace
}  // namespace pgb

extern "C" pgb_status pgb_gather_probe(const pgb_index* ix, const void* query, const uint32_t* ids,
                                       uint64_t count, int32_t* out, uint32_t lanes_per_row,
                                       void* stream) {
    if (!ix) return fail(PGB_ERR_BAD_ARG, "null index");
    if (count == 0) return PGB_OK;
    if (!query || !ids || !out) return fail(PGB_ERR_BAD_ARG, "null query, ids or output");
    void* kern = nullptr;
    const bool sg = ix->elem == PGB_INT8;
    switch (lanes_per_row) {
        case 1: kern = probe_kernel<1>(sg); break;
        case 4: kern = probe_kernel<4>(sg); break;
        case 8: kern = probe_kernel<8>(sg); break;
        case 32: kern = probe_kernel<32>(sg); break;
        default: return fail(PGB_ERR_BAD_ARG, "lanes_per_row must be 1, 4, 8 or 32");
    }
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    int dev = 0, sms = 148, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kProbeWarps * 32, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const uint8_t* rows = ix->rows;
    uint32_t n = ix->n, dim = ix->dim, nir = ix->norm_in_row ? 1u : 0u;
    const uint8_t* q = (const uint8_t*)query;
    void* args[] = {&rows, &n, &dim, &nir, &q, &ids, &count, &out};
    const cudaError_t e = cudaLaunchKernel(kern, dim3((unsigned)(sms * per_sm)), dim3(kProbeWarps * 32),
                                           args, 0, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_status(e, "gather probe");
    count_launches(1);
    return PGB_OK;
}
