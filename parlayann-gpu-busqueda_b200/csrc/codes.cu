// codes.cu -- compressed rows for the flat-graph search: 4-bit codes (64 bytes per row,
// half a vector row) searched by the plain kernel, then an exact re-rank of each query's
// first R candidates on the full rows. The reference has no compressed format; this is
// the "compressed vectors" direction its paper names (BANG's PQ, paper/paper.tex:134-136),
// in a form whose distances are exact integers: a code c of dimension d stands for
// v = step * c + offset[d], so the search over codes equals the exact search over the
// reconstructed vectors, and the oracle checks it bit for bit on those.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "codes.h"
#include "device_common.cuh"
#include "errors.h"
#include "index.h"
#include "search_flat.cuh"
#include "search_plan.h"

namespace pgb {
namespace {

constexpr int kHistDims = 8;  // dimensions per histogram block

// per-dimension 256-bin histograms of the vector rows; block (g, s) counts dimensions
// 8g..8g+7 over the rows s, s + gridDim.y, ... into shared memory, then into hist
template <bool Signed>
__global__ void code_hist_kernel(const uint8_t* __restrict__ rows, uint32_t n, uint32_t dim,
                                 unsigned long long* __restrict__ hist) {
    __shared__ uint32_t h[kHistDims][256];
    for (uint32_t i = threadIdx.x; i < kHistDims * 256u; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    const uint32_t d0 = blockIdx.x * kHistDims;
    const uint32_t nd = min((uint32_t)kHistDims, dim - d0);
    for (uint64_t r = (uint64_t)blockIdx.y * blockDim.x + threadIdx.x; r < n;
         r += (uint64_t)gridDim.y * blockDim.x) {
        const uint2 w = __ldg(reinterpret_cast<const uint2*>(rows + r * kRowBytes + d0));
        for (uint32_t j = 0; j < nd; j++) {
            const uint32_t b = ((j < 4 ? w.x : w.y) >> (8 * (j & 3))) & 0xFFu;
            atomicAdd(&h[j][Signed ? (b ^ 0x80u) : b], 1u);  // int8 value + 128
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nd * 256u; i += blockDim.x)
        if ((&h[0][0])[i]) atomicAdd(&hist[(size_t)d0 * 256 + i], (unsigned long long)(&h[0][0])[i]);
}

// one thread per row: 4-bit codes (nibble layout of kCodeRowBytes rows) and ||v||^2
template <bool Signed>
__global__ void code_encode_kernel(const uint8_t* __restrict__ rows, uint32_t n, uint32_t dim,
                                   int32_t step, const uint8_t* __restrict__ off_row,
                                   uint8_t* __restrict__ codes) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint8_t* x = rows + r * kRowBytes;
    uint32_t out[16] = {0};
    int32_t norm = 0;
    for (uint32_t d = 0; d < dim; d++) {
        const int32_t xv = Signed ? (int32_t)(int8_t)x[d] : (int32_t)x[d];
        const int32_t o = Signed ? (int32_t)(int8_t)off_row[d] : (int32_t)off_row[d];
        const int32_t num = 2 * (xv - o) + step;  // round half up of (x - o) / step
        const int32_t c = num < 0 ? 0 : min(15, num / (2 * step));
        const int32_t v = step * c + o;
        norm += v * v;
        const uint32_t cw = d >> 5, j = (d >> 3) & 3, b = d & 3, hi = (d >> 2) & 1;
        out[cw * 4 + j] |= (uint32_t)c << (8 * b + 4 * hi);
    }
    out[15] = (uint32_t)norm;  // bytes 60..63 (dimensions 120..127 never hold codes)
    uint4* dst = reinterpret_cast<uint4*>(codes + r * kCodeRowBytes);
#pragma unroll
    for (int w = 0; w < 4; w++) dst[w] = make_uint4(out[4 * w], out[4 * w + 1], out[4 * w + 2], out[4 * w + 3]);
}

struct RerankArgs {
    const uint8_t* rows;
    uint32_t dim, norm_in_row;
    const uint8_t* queries;
    uint32_t nq, qstride;
    const uint32_t* cand;
    uint32_t R, P, k;  // candidates per query, keys per warp (power of two >= R), outputs
    uint32_t off_ids, off_d, off_keys, warp_bytes;
    uint32_t* ids;
    int32_t* dists;
};

// one warp per query: exact distances of the candidates, bitonic sort of (dist, id) keys
// in shared memory, the first k written out
template <bool Signed>
__global__ void __launch_bounds__(128) rerank_kernel(RerankArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const uint32_t w = threadIdx.x >> 5;
    unsigned char* wmem = smem + (size_t)w * A.warp_bytes;
    uint32_t* qwords = reinterpret_cast<uint32_t*>(wmem);
    uint32_t* sid = reinterpret_cast<uint32_t*>(wmem + A.off_ids);
    int32_t* sd = reinterpret_cast<int32_t*>(wmem + A.off_d);
    uint64_t* keys = reinterpret_cast<uint64_t*>(wmem + A.off_keys);
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t total = gridDim.x * wpb;
    const int4* q4 = reinterpret_cast<const int4*>(qwords);
    for (uint32_t q = blockIdx.x * wpb + w; q < A.nq; q += total) {
        load_query_row(A.queries + (size_t)q * A.qstride, A.dim, lane, qwords);
        // the candidates that are ids (padding dropped), in the search's order
        const uint32_t* cq = A.cand + (size_t)q * A.R;
        uint32_t nv = 0;
        for (uint32_t b = 0; b < A.R; b += 32) {
            const uint32_t i = b + lane;
            const uint32_t id = i < A.R ? cq[i] : kEmptyId;
            const bool ok = id != kEmptyId;
            const uint32_t m = __ballot_sync(kFull, ok);
            if (ok) sid[nv + __popc(m & lanemask_lt())] = id;
            nv += __popc(m);
        }
        __syncwarp();
        const int32_t qq = query_sq_norm<Signed>(q4, lane);
        if (nv) row_distances<Signed>(A.rows, sid, sd, (int)nv, q4, qq, A.dim, A.norm_in_row != 0, lane);
        for (uint32_t i = lane; i < A.P; i += 32) keys[i] = i < nv ? pack_key(sd[i], sid[i]) : kEmptyKey;
        __syncwarp();
        for (uint32_t kk = 2; kk <= A.P; kk <<= 1) {
            for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
                for (uint32_t i = lane; i < A.P; i += 32) {
                    const uint32_t l = i ^ j;
                    if (l > i) {
                        const uint64_t a = keys[i], b = keys[l];
                        if ((a > b) == ((i & kk) == 0)) {
                            keys[i] = b;
                            keys[l] = a;
                        }
                    }
                }
                __syncwarp();
            }
        }
        for (uint32_t i = lane; i < A.k; i += 32) {
            const bool ok = i < nv;
            A.ids[(size_t)q * A.k + i] = ok ? key_id(keys[i]) : PGB_NO_NEIGHBOR;
            A.dists[(size_t)q * A.k + i] = ok ? key_dist(keys[i]) : INT32_MAX;
        }
        __syncwarp();
    }
}

uint32_t round16u(uint32_t x) { return (x + 15u) & ~15u; }

pgb_status cuda_error(cudaError_t e, const char* what) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(PGB_ERR_OOM, std::string(what) + ": out of device memory");
    return fail(PGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

void choose_codes(const uint64_t* hist, uint32_t dim, bool is_signed, int32_t* step,
                  int32_t* offsets) {
    const int lo = is_signed ? -128 : 0, hi = is_signed ? 127 : 255;
    // the values present in each dimension with their counts
    std::vector<std::vector<std::pair<int, uint64_t>>> vals(dim);
    for (uint32_t d = 0; d < dim; d++)
        for (int b = 0; b < 256; b++)
            if (hist[(size_t)d * 256 + b]) vals[d].push_back({lo + b, hist[(size_t)d * 256 + b]});
    uint64_t best_total = UINT64_MAX;
    std::vector<int32_t> off(dim), best_off(dim);
    int32_t best_step = 1;
    for (int s = 1; 15 * s <= hi - lo; s++) {
        uint64_t total = 0;
        for (uint32_t d = 0; d < dim && total < best_total; d++) {
            uint64_t best = UINT64_MAX;
            int bo = lo;
            for (int o = lo; o + 15 * s <= hi; o++) {
                uint64_t e = 0;
                for (const auto& vc : vals[d]) {
                    const int num = 2 * (vc.first - o) + s;
                    const int c = num < 0 ? 0 : std::min(15, num / (2 * s));
                    const int64_t diff = vc.first - (s * c + o);
                    e += (uint64_t)(diff * diff) * vc.second;
                    if (e >= best) break;
                }
                if (e < best) {
                    best = e;
                    bo = o;
                }
            }
            off[d] = bo;
            total += best;
        }
        if (total < best_total) {
            best_total = total;
            best_step = s;
            best_off = off;
        }
    }
    *step = best_step;
    for (uint32_t d = 0; d < dim; d++) offsets[d] = best_off[d];
}

pgb_status rerank_launch(const pgb_index* ix, const void* queries, uint32_t nq,
                         uint32_t query_stride, const uint32_t* cand, uint32_t R, uint32_t k,
                         uint32_t* ids, int32_t* dists, cudaStream_t stream) {
    if (nq == 0) return PGB_OK;
    RerankArgs A{};
    A.rows = ix->rows;
    A.dim = ix->dim;
    A.norm_in_row = ix->norm_in_row ? 1u : 0u;
    A.queries = static_cast<const uint8_t*>(queries);
    A.nq = nq;
    A.qstride = query_stride;
    A.cand = cand;
    A.R = R;
    A.P = 1;
    while (A.P < R) A.P <<= 1;
    A.k = k;
    A.off_ids = kRowBytes;
    A.off_d = A.off_ids + round16u(4u * R);
    A.off_keys = A.off_d + round16u(4u * R);
    A.warp_bytes = round16u(A.off_keys + 8u * A.P);  // each warp's query row 16-byte aligned
    A.ids = ids;
    A.dists = dists;
    const int wpb = 4;
    const size_t smem = (size_t)wpb * A.warp_bytes;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* kern = ix->elem == PGB_INT8 ? (const void*)rerank_kernel<true> : (const void*)rerank_kernel<false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_error(e, "re-rank shared memory");
    const unsigned blocks = (unsigned)std::min<uint64_t>((nq + wpb - 1) / wpb, (uint64_t)sms * 8);
    void* args[] = {&A};
    e = cudaLaunchKernel(kern, dim3(blocks), dim3(wpb * 32), args, smem, stream);
    if (e == cudaSuccess) count_launches(1);
    return e == cudaSuccess ? PGB_OK : cuda_error(e, "re-rank launch");
}

}  // namespace pgb

using namespace pgb;

extern "C" {

pgb_status pgb_index_compress(pgb_index* ix, int32_t step, const int32_t* offsets) {
    if (!ix) return fail(PGB_ERR_BAD_ARG, "null index");
    if (ix->is_hnsw) return fail(PGB_ERR_BAD_ARG, "code rows are built for flat-graph indexes");
    if (ix->dim > kCodeMaxDim) return fail(PGB_ERR_BAD_ARG, "code rows hold at most 120 dimensions");
    const bool sg = ix->elem == PGB_INT8;
    const int lo = sg ? -128 : 0, hi = sg ? 127 : 255;
    int32_t s = step;
    int32_t off[PGB_MAX_DIM] = {0};
    DeviceGuard guard(ix->device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e;
    if (step == 0) {
        // histograms on the device, the choice on the host
        unsigned long long* dh = nullptr;
        const size_t hb = sizeof(unsigned long long) * 256 * ix->dim;
        if ((e = cudaMalloc(&dh, hb)) != cudaSuccess) return cuda_error(e, "code histograms");
        e = cudaMemset(dh, 0, hb);
        const unsigned groups = (ix->dim + kHistDims - 1) / kHistDims;
        const unsigned slices = (unsigned)std::min<uint64_t>((ix->n + 255) / 256, 256);
        if (e == cudaSuccess) {
            if (sg) code_hist_kernel<true><<<dim3(groups, slices), 256>>>(ix->rows, ix->n, ix->dim, dh);
            else code_hist_kernel<false><<<dim3(groups, slices), 256>>>(ix->rows, ix->n, ix->dim, dh);
            e = cudaGetLastError();
        }
        std::vector<uint64_t> h(256ull * ix->dim);
        if (e == cudaSuccess) e = cudaMemcpy(h.data(), dh, hb, cudaMemcpyDeviceToHost);
        cudaFree(dh);
        if (e != cudaSuccess) return cuda_error(e, "code histograms");
        choose_codes(h.data(), ix->dim, sg, &s, off);
    } else {
        if (!offsets) return fail(PGB_ERR_BAD_ARG, "null offsets with an explicit step");
        if (step < 1 || 15 * step > hi - lo) return fail(PGB_ERR_BAD_ARG, "step outside 1..17");
        for (uint32_t d = 0; d < ix->dim; d++) {
            if (offsets[d] < lo || offsets[d] + 15 * step > hi)
                return fail(PGB_ERR_BAD_ARG, "offset leaves the element's range");
            off[d] = offsets[d];
        }
    }
    uint8_t off_row[kRowBytes] = {0};
    for (uint32_t d = 0; d < ix->dim; d++) off_row[d] = (uint8_t)(off[d] & 0xFF);
    uint8_t *codes = nullptr, *doff = nullptr;
    if ((e = cudaMalloc(&codes, (size_t)kCodeRowBytes * ix->n)) != cudaSuccess)
        return cuda_error(e, "code rows");
    if ((e = cudaMalloc(&doff, kRowBytes)) != cudaSuccess ||
        (e = cudaMemcpy(doff, off_row, kRowBytes, cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFree(codes);
        cudaFree(doff);
        return cuda_error(e, "code offsets");
    }
    const unsigned nb = (unsigned)((ix->n + 255ull) / 256);
    if (sg) code_encode_kernel<true><<<nb, 256>>>(ix->rows, ix->n, ix->dim, s, doff, codes);
    else code_encode_kernel<false><<<nb, 256>>>(ix->rows, ix->n, ix->dim, s, doff, codes);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(codes);
        cudaFree(doff);
        return cuda_error(e, "code encode");
    }
    if (ix->codes) ix->device_bytes -= (uint64_t)kCodeRowBytes * ix->n + kRowBytes;
    cudaFree(ix->codes);
    cudaFree(ix->code_off);
    ix->codes = codes;
    ix->code_off = doff;
    ix->code_step = s;
    std::memcpy(ix->code_off_host, off, sizeof(off));
    ix->device_bytes += (uint64_t)kCodeRowBytes * ix->n + kRowBytes;
    return PGB_OK;
}

pgb_status pgb_index_get_codes(const pgb_index* ix, int32_t* step, int32_t* offsets,
                               uint8_t* codes) {
    if (!ix || !step) return fail(PGB_ERR_BAD_ARG, "null argument");
    if (!ix->codes) return fail(PGB_ERR_BAD_ARG, "index has no code rows (pgb_index_compress)");
    *step = ix->code_step;
    if (offsets) std::memcpy(offsets, ix->code_off_host, sizeof(int32_t) * ix->dim);
    if (codes) {
        DeviceGuard guard(ix->device);
        if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
        cudaError_t e = cudaMemcpy(codes, ix->codes, (size_t)kCodeRowBytes * ix->n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_error(e, "code rows download");
    }
    return PGB_OK;
}

}  // extern "C"
