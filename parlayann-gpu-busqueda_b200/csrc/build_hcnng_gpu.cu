// build_hcnng_gpu.cu -- HCNNG graph construction on the GPU (pgb_build_hcnng_gpu).
//
// The algorithm is the CPU builder's (builders.cpp: build_hcnng, cluster_leaves,
// leaf_knn), step for step, so the two produce the same graph for the same seed:
//   tree t draws from SplitMix64(seed * 1000003 + t). Its partition tree is walked depth
//   first from the range of all points, the second piece of a split first; a range of at
//   most `leaf` points is a leaf; otherwise two pivots a, c are drawn (a first), each
//   uniform over the range's current positions, and the points with d(x, a) <= d(x, c)
//   go left, both pieces keeping their order; when a == c or one piece is empty the range
//   is halved at its middle instead, in place.
//   Per leaf of m >= 2 points: the exact min(10, m - 1) nearest points of each point
//   within the leaf by (distance, id); every such pair gives the edge (d, a, c) with a < c
//   the positions in the leaf; the edges in ascending (d, a, c) order go through Kruskal
//   with node degree <= mst_deg. A repeated edge always meets the same outcome as its
//   first copy, so the CPU's de-duplication does not change the result and is skipped.
//   Each point's row is the concatenation, tree after tree, of the edges accepted for it
//   in acceptance order.
// GPU form (per group of trees that fits the memory budget):
//   partition: one 1,024-thread block per tree; the pivots of every range come from the
//   tree's sequential stream, so a tree cannot be split level by level; each split is a
//   block-wide pass (flags, count) and a stable scatter (block scans) into the other of
//   two id buffers; the buffer holding a range travels with it on the stack.
//   k-NN + edge sort: one 512-thread block per leaf, the leaf's rows in shared memory,
//   one point per thread (two passes), the top 10 in registers; then the edges are sorted
//   by a bitonic sort in the same shared memory.
//   Kruskal: one warp per leaf, union-find and degrees in shared memory.
//   append: one thread per point, trees of the group in order.
#include <algorithm>
#include <string>
#include <vector>

#include "builders.h"
#include "errors.h"
#include "index.h"
#include "search_flat.cuh"

namespace pgb {
namespace {

constexpr int kPartThreads = 1024;
constexpr int kKnnThreads = 512;
constexpr int kKnnPasses = 2;              // kKnnThreads * kKnnPasses >= kMaxGpuLeaf
constexpr uint32_t kLeafK = 10;            // the CPU builder's leaf k-NN size
constexpr uint32_t kMaxGpuLeaf = 1024;     // leaf positions fit 10 bits of an edge key
constexpr uint32_t kBufBit = 0x80000000u;  // range end: bit 31 = which id buffer
constexpr int kKruskalWarps = 4;

struct HcnngArgs {
    const uint8_t* rows;    // n x 128, zero padded
    uint32_t n, leaf, mst_deg;
    const uint64_t* seeds;  // per tree of the group
    uint32_t* ids;          // per tree: n (the two id buffers)
    uint32_t* alt;
    uint8_t* flags;         // per tree: n
    uint2* stack;           // per tree: n + 2 ranges (b, e | buffer << 31)
    uint2* leaves;          // per tree: n ranges
    uint32_t* n_leaves;     // per tree
    uint64_t* edges;        // per tree: 10 n sorted edge keys, leaf [b, e) at 10 b
    uint32_t* out;          // per tree: n x mst_deg accepted neighbours
    uint32_t* out_n;        // per tree: n
    uint32_t* error;        // set if a partition stack would overflow (cannot happen)
};

__device__ __forceinline__ uint64_t splitmix_next(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

template <bool Signed>
__device__ __forceinline__ int32_t dot4(uint32_t a, uint32_t b) {
    if (Signed) return __dp4a((int)a, (int)b, 0);
    return (int32_t)__dp4a(a, b, 0u);
}

template <bool Signed>
__device__ __forceinline__ int32_t dot16(const uint4& a, const uint4& b) {
    return dot4<Signed>(a.x, b.x) + dot4<Signed>(a.y, b.y) + dot4<Signed>(a.z, b.z) +
           dot4<Signed>(a.w, b.w);
}

// ---------------------------------------------------------------------------
// Partition trees: block t walks tree t of the group.
template <bool Signed, int NQ>
__global__ void __launch_bounds__(kPartThreads, 1) hcnng_partition_kernel(HcnngArgs A) {
    const uint32_t t = blockIdx.x, tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const size_t n = A.n;
    uint32_t* const buf0 = A.ids + t * n;
    uint32_t* const buf1 = A.alt + t * n;
    uint8_t* const fl = A.flags + t * n;
    uint2* const stack = A.stack + t * (n + 2);
    uint2* const leaves = A.leaves + t * n;
    __shared__ __align__(16) uint32_t prow[2][32];
    __shared__ int32_t pnorm[2];
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t s_b, s_e, s_buf, s_mode, s_a, s_c, s_total;
    uint64_t rng = A.seeds[t];  // thread 0's
    uint32_t top = 0, nleaf = 0;
    for (uint32_t i = tid; i < n; i += kPartThreads) buf0[i] = i;
    if (tid == 0) {
        stack[0] = make_uint2(0u, (uint32_t)n);
        top = 1;
    }
    for (;;) {
        __syncthreads();  // the last range's readers are done with the shared state
        if (tid == 0) {
            uint32_t mode = 0;  // 0 done, 1 leaf, 2 split by pivots, 3 halve in place
            if (top > 0) {
                const uint2 r = stack[--top];
                const uint32_t b = r.x, e = r.y & ~kBufBit, m = e - b;
                s_b = b;
                s_e = e;
                s_buf = r.y >> 31;
                if (m <= A.leaf) {
                    mode = 1;
                    leaves[nleaf++] = r;
                } else {
                    const uint32_t* src = s_buf ? buf1 : buf0;
                    const uint32_t a = src[b + splitmix_next(rng) % m];
                    const uint32_t c = src[b + splitmix_next(rng) % m];
                    s_a = a;
                    s_c = c;
                    mode = a != c ? 2u : 3u;
                }
            }
            s_mode = mode;
        }
        __syncthreads();
        const uint32_t mode = s_mode;
        if (mode == 0) break;
        if (mode == 1) continue;
        const uint32_t b = s_b, e = s_e, m = e - b, bsel = s_buf;
        uint32_t mid = b + m / 2u, nbuf = bsel;
        if (mode == 2) {
            const uint32_t* src = bsel ? buf1 : buf0;
            uint32_t* dst = bsel ? buf0 : buf1;
            if (tid < 64) {
                const uint32_t p = tid < 32 ? s_a : s_c;
                prow[tid >> 5][lane] = __ldg(reinterpret_cast<const uint32_t*>(A.rows) + (size_t)p * 32u + lane);
            }
            __syncthreads();
            if (warp < 2) {
                int32_t v = dot4<Signed>(prow[warp][lane], prow[warp][lane]);
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
                if (lane == 0) pnorm[warp] = v;
            }
            __syncthreads();
            const uint4* pa = reinterpret_cast<const uint4*>(prow[0]);
            const uint4* pc = reinterpret_cast<const uint4*>(prow[1]);
            // pass 1: side of every point (d(x, a) <= d(x, c) <=> |a|^2 - 2 x.a <= |c|^2 - 2 x.c)
            uint32_t lc = 0;
            for (uint32_t base = b; base < e; base += kPartThreads) {
                const uint32_t i = base + tid;
                bool left = false;
                if (i < e) {
                    const uint4* xr = reinterpret_cast<const uint4*>(A.rows + (size_t)src[i] * kRowBytes);
                    uint4 x[NQ];
#pragma unroll
                    for (int c = 0; c < NQ; c++) x[c] = __ldg(xr + c);
                    int32_t da = 0, dc = 0;
#pragma unroll
                    for (int c = 0; c < NQ; c++) {
                        da += dot16<Signed>(x[c], pa[c]);
                        dc += dot16<Signed>(x[c], pc[c]);
                    }
                    left = pnorm[0] - 2 * da <= pnorm[1] - 2 * dc;
                    fl[i] = left ? 1 : 0;
                }
                lc += (uint32_t)__syncthreads_count(left);
            }
            if (lc != 0 && lc != m) {
                // pass 2: stable scatter into the other buffer
                uint32_t lbase = 0, rbase = 0;
                for (uint32_t base = b; base < e; base += kPartThreads) {
                    const uint32_t i = base + tid;
                    const bool in = i < e;
                    const bool f = in && fl[i];
                    const uint32_t x = in ? src[i] : 0u;
                    const unsigned bal = __ballot_sync(kFull, f);
                    if (lane == 0) wsum[warp] = (uint32_t)__popc(bal);
                    __syncthreads();
                    if (warp == 0) {
                        const uint32_t v = wsum[lane];
                        uint32_t incl = v;
#pragma unroll
                        for (int off = 1; off < 32; off <<= 1) {
                            const uint32_t u = __shfl_up_sync(kFull, incl, off);
                            if (lane >= (uint32_t)off) incl += u;
                        }
                        wsum[lane] = incl - v;
                        if (lane == 31) s_total = incl;
                    }
                    __syncthreads();
                    const uint32_t before = wsum[warp] + (uint32_t)__popc(bal & lanemask_lt());
                    const uint32_t tot = s_total;
                    if (in) {
                        const uint32_t k = i - base;
                        dst[f ? b + lbase + before : b + lc + rbase + (k - before)] = x;
                    }
                    lbase += tot;
                    rbase += min((uint32_t)kPartThreads, e - base) - tot;
                    __syncthreads();  // wsum and s_total are rewritten by the next chunk
                }
                mid = b + lc;
                nbuf = bsel ^ 1u;
            }
        }
        if (tid == 0) {
            if (top + 2 > n + 2) {
                atomicExch(A.error, 1u);
            } else {
                stack[top++] = make_uint2(b, mid | (nbuf << 31));
                stack[top++] = make_uint2(mid, e | (nbuf << 31));
            }
        }
    }
    if (tid == 0) A.n_leaves[t] = nleaf;
}

// ---------------------------------------------------------------------------
// Leaf k-NN and the leaf's sorted edge list: block (leaf, tree).
template <bool Signed, int NQ>
__global__ void __launch_bounds__(kKnnThreads, 1) hcnng_leaf_knn_kernel(HcnngArgs A) {
    const uint32_t t = blockIdx.y, li = blockIdx.x, tid = threadIdx.x;
    if (li >= A.n_leaves[t]) return;
    const size_t n = A.n;
    const uint2 L = A.leaves[t * n + li];
    const uint32_t b = L.x, e = L.y & ~kBufBit, m = e - b;
    if (m < 2) return;
    const uint32_t* pts = ((L.y & kBufBit) ? A.alt : A.ids) + t * n + b;
    const uint32_t kk = min(kLeafK, m - 1u);
    extern __shared__ __align__(16) unsigned char smem[];
    uint4* srow = reinterpret_cast<uint4*>(smem);                                // m x NQ
    int32_t* snorm = reinterpret_cast<int32_t*>(smem + (size_t)m * NQ * 16u);    // m
    uint32_t* sgid = reinterpret_cast<uint32_t*>(snorm + m);                     // m
    for (uint32_t idx = tid; idx < m * NQ; idx += kKnnThreads) {
        const uint32_t r = idx / NQ, c = idx - r * NQ;
        srow[idx] = __ldg(reinterpret_cast<const uint4*>(A.rows + (size_t)pts[r] * kRowBytes) + c);
    }
    for (uint32_t r = tid; r < m; r += kKnnThreads) sgid[r] = pts[r];
    __syncthreads();
    for (uint32_t r = tid; r < m; r += kKnnThreads) {
        int32_t v = 0;
#pragma unroll
        for (int c = 0; c < NQ; c++) v += dot16<Signed>(srow[r * NQ + c], srow[r * NQ + c]);
        snorm[r] = v;
    }
    __syncthreads();
    // key (d, id, position): d < 2^23 for 8-bit data of at most 128 dimensions, id < 2^31
    uint64_t top[kKnnPasses][kLeafK];
#pragma unroll
    for (int p = 0; p < kKnnPasses; p++) {
#pragma unroll
        for (int r = 0; r < (int)kLeafK; r++) top[p][r] = ~0ull;
        const uint32_t i = tid + (uint32_t)p * kKnnThreads;
        if (i < m) {
            uint4 q[NQ];
#pragma unroll
            for (int c = 0; c < NQ; c++) q[c] = srow[i * NQ + c];
            const int32_t qn = snorm[i];
            for (uint32_t j = 0; j < m; j++) {
                int32_t dot = 0;
#pragma unroll
                for (int c = 0; c < NQ; c++) dot += dot16<Signed>(q[c], srow[j * NQ + c]);
                const uint32_t d = (uint32_t)(qn + snorm[j] - 2 * dot);
                const uint64_t key = ((uint64_t)d << 41) | ((uint64_t)sgid[j] << 10) | j;
                if (j != i && key < top[p][kLeafK - 1]) {
                    top[p][kLeafK - 1] = key;
#pragma unroll
                    for (int s = (int)kLeafK - 1; s > 0; s--) {
                        if (top[p][s] < top[p][s - 1]) {
                            const uint64_t w = top[p][s];
                            top[p][s] = top[p][s - 1];
                            top[p][s - 1] = w;
                        }
                    }
                }
            }
        }
    }
    __syncthreads();  // the rows are dead: the edge keys take their place
    uint64_t* se = reinterpret_cast<uint64_t*>(smem);
    const uint32_t E = m * kk, P = next_pow2_u32(E);
#pragma unroll
    for (int p = 0; p < kKnnPasses; p++) {
        const uint32_t i = tid + (uint32_t)p * kKnnThreads;
        if (i < m) {
#pragma unroll
            for (int r = 0; r < (int)kLeafK; r++) {
                if ((uint32_t)r < kk) {
                    const uint64_t key = top[p][r];
                    const uint32_t j = (uint32_t)key & 1023u, d = (uint32_t)(key >> 41);
                    se[i * kk + r] = ((uint64_t)d << 20) | ((uint64_t)min(i, j) << 10) | max(i, j);
                }
            }
        }
    }
    for (uint32_t idx = E + tid; idx < P; idx += kKnnThreads) se[idx] = ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
            for (uint32_t idx = tid; idx < P; idx += kKnnThreads) {
                const uint32_t o = idx ^ jj;
                if (o > idx) {
                    const uint64_t x = se[idx], y = se[o];
                    if ((x > y) == ((idx & k) == 0)) {
                        se[idx] = y;
                        se[o] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    uint64_t* out = A.edges + t * n * kLeafK + (size_t)b * kLeafK;
    for (uint32_t idx = tid; idx < E; idx += kKnnThreads) out[idx] = se[idx];
}

// ---------------------------------------------------------------------------
// Degree-bounded Kruskal over a leaf's sorted edges: warp (leaf, tree).
__device__ __forceinline__ uint32_t uf_find(uint16_t* par, uint32_t x) {
    while (par[x] != x) {
        const uint32_t g = par[par[x]];
        par[x] = (uint16_t)g;
        x = g;
    }
    return x;
}

__global__ void __launch_bounds__(kKruskalWarps * 32) hcnng_kruskal_kernel(HcnngArgs A) {
    const uint32_t t = blockIdx.y, w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t li = blockIdx.x * kKruskalWarps + w;
    __shared__ uint16_t par[kKruskalWarps][kMaxGpuLeaf];
    __shared__ uint16_t dg[kKruskalWarps][kMaxGpuLeaf];
    __shared__ uint32_t gid[kKruskalWarps][kMaxGpuLeaf];
    __shared__ uint64_t stage[kKruskalWarps][32];
    if (li >= A.n_leaves[t]) return;  // the whole warp
    const size_t n = A.n;
    const uint2 L = A.leaves[t * n + li];
    const uint32_t b = L.x, e = L.y & ~kBufBit, m = e - b;
    if (m < 2) return;
    const uint32_t* pts = ((L.y & kBufBit) ? A.alt : A.ids) + t * n + b;
    const uint32_t E = m * min(kLeafK, m - 1u), D = A.mst_deg;
    for (uint32_t r = lane; r < m; r += 32) {
        par[w][r] = (uint16_t)r;
        dg[w][r] = 0;
        gid[w][r] = pts[r];
    }
    __syncwarp();
    const uint64_t* ed = A.edges + t * n * kLeafK + (size_t)b * kLeafK;
    uint32_t* out = A.out + t * n * D;
    for (uint32_t base = 0; base < E; base += 32) {
        stage[w][lane] = base + lane < E ? ed[base + lane] : ~0ull;
        __syncwarp();
        if (lane == 0) {
            const uint32_t cnt = min(32u, E - base);
            for (uint32_t r = 0; r < cnt; r++) {
                const uint64_t key = stage[w][r];
                const uint32_t a = (uint32_t)(key >> 10) & 1023u, c = (uint32_t)key & 1023u;
                if (dg[w][a] >= D || dg[w][c] >= D) continue;
                const uint32_t ra = uf_find(par[w], a), rc = uf_find(par[w], c);
                if (ra == rc) continue;
                par[w][ra] = (uint16_t)rc;
                const uint32_t pa = gid[w][a], pc = gid[w][c];
                out[(size_t)pa * D + dg[w][a]] = pc;
                out[(size_t)pc * D + dg[w][c]] = pa;
                dg[w][a]++;
                dg[w][c]++;
            }
        }
        __syncwarp();
    }
    for (uint32_t r = lane; r < m; r += 32) A.out_n[t * n + gid[w][r]] = dg[w][r];
}

// rows: the group's trees in order after what earlier groups appended
__global__ void hcnng_append_kernel(HcnngArgs A, uint32_t g, uint32_t slots, uint32_t* adj,
                                    uint32_t* deg) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n) return;
    const size_t n = A.n, D = A.mst_deg;
    uint32_t d = deg[p];
    uint32_t* row = adj + (size_t)p * slots;
    for (uint32_t tl = 0; tl < g; tl++) {
        const uint32_t c = A.out_n[tl * n + p];
        const uint32_t* src = A.out + (tl * n + p) * D;
        for (uint32_t k = 0; k < c; k++) row[d++] = src[k];
    }
    deg[p] = d;
}

template <bool Signed>
void hcnng_kernels(int nq, void*& part, void*& knn) {
    switch (nq) {
        case 4:
            part = (void*)hcnng_partition_kernel<Signed, 4>;
            knn = (void*)hcnng_leaf_knn_kernel<Signed, 4>;
            break;
        case 7:
            part = (void*)hcnng_partition_kernel<Signed, 7>;
            knn = (void*)hcnng_leaf_knn_kernel<Signed, 7>;
            break;
        default:
            part = (void*)hcnng_partition_kernel<Signed, 8>;
            knn = (void*)hcnng_leaf_knn_kernel<Signed, 8>;
            break;
    }
}

struct Buffers {
    std::vector<void*> ptrs;
    ~Buffers() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    pgb_status alloc(T** p, size_t count, const char* what) {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? PGB_ERR_OOM : PGB_ERR_CUDA,
                        std::string("hcnng (GPU): ") + what + ": " + cudaGetErrorString(e));
        }
        ptrs.push_back(*p);
        return PGB_OK;
    }
};

pgb_status ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PGB_OK;
    cudaGetLastError();
    return fail(PGB_ERR_CUDA, std::string("hcnng (GPU): ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" pgb_status pgb_build_hcnng_gpu(int device, const void* vectors, uint32_t n,
                                          uint32_t dim, pgb_elem elem, uint32_t trees,
                                          uint32_t leaf, uint32_t mst_deg, uint64_t seed,
                                          uint32_t* degrees, uint32_t* adjacency) {
    if (!vectors || !degrees || !adjacency) return fail(PGB_ERR_BAD_ARG, "hcnng (GPU): null argument");
    if (n == 0 || dim == 0 || dim > PGB_MAX_DIM) return fail(PGB_ERR_BAD_ARG, "hcnng (GPU): n == 0 or dim outside 1..128");
    if (elem != PGB_INT8 && elem != PGB_UINT8) return fail(PGB_ERR_BAD_ARG, "hcnng (GPU): element type");
    if (trees == 0 || mst_deg == 0 || leaf < 2 || (uint64_t)trees * mst_deg > PGB_MAX_DEGREE)
        return fail(PGB_ERR_BAD_ARG, "hcnng (GPU): bad trees / leaf / mst_deg");
    if (leaf > kMaxGpuLeaf) return fail(PGB_ERR_BAD_ARG, "hcnng (GPU): leaves of at most 1,024 points");
    if (n >= kBufBit) return fail(PGB_ERR_BAD_ARG, "hcnng (GPU): n must be below 2^31");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    const uint32_t slots = trees * mst_deg;
    std::fill(degrees, degrees + n, 0u);
    std::fill(adjacency, adjacency + (size_t)n * slots, kNoNeighbor);
    if (n <= 1) return PGB_OK;
    const bool sgn = elem == PGB_INT8;
    const int nq = dim <= 64 ? 4 : dim <= 112 ? 7 : 8;
    void *part = nullptr, *knn = nullptr;
    if (sgn) hcnng_kernels<true>(nq, part, knn);
    else hcnng_kernels<false>(nq, part, knn);

    // trees per group: the per-tree buffers within half the free memory (at most 16 GB)
    size_t free_b = 0, total_b = 0;
    pgb_status s;
    if ((s = ck(cudaMemGetInfo(&free_b, &total_b), "memory info")) != PGB_OK) return s;
    const size_t per_tree = (size_t)n * (4 + 4 + 1 + 8 + 8 + 8 * kLeafK + 4 * (size_t)mst_deg + 4) + 16;
    const size_t budget = std::min<size_t>(free_b / 2, (size_t)16 << 30);
    const uint32_t g = (uint32_t)std::max<size_t>(1, std::min<size_t>(trees, budget / per_tree));

    Buffers bb;
    uint8_t* rows;
    uint32_t *adj, *deg, *ids, *alt, *n_leaves, *out, *out_n, *error;
    uint8_t* flags;
    uint2 *stack, *leaves;
    uint64_t *edges, *seeds;
    const size_t gn = (size_t)g * n;
    if ((s = bb.alloc(&rows, (size_t)n * kRowBytes, "rows")) != PGB_OK ||
        (s = bb.alloc(&adj, (size_t)n * slots, "adjacency")) != PGB_OK ||
        (s = bb.alloc(&deg, n, "degrees")) != PGB_OK ||
        (s = bb.alloc(&ids, gn, "ids")) != PGB_OK ||
        (s = bb.alloc(&alt, gn, "ids")) != PGB_OK ||
        (s = bb.alloc(&flags, gn, "flags")) != PGB_OK ||
        (s = bb.alloc(&stack, (size_t)g * (n + 2), "stacks")) != PGB_OK ||
        (s = bb.alloc(&leaves, gn, "leaves")) != PGB_OK ||
        (s = bb.alloc(&n_leaves, g, "leaf counts")) != PGB_OK ||
        (s = bb.alloc(&edges, gn * kLeafK, "edges")) != PGB_OK ||
        (s = bb.alloc(&out, gn * mst_deg, "tree edges")) != PGB_OK ||
        (s = bb.alloc(&out_n, gn, "tree degrees")) != PGB_OK ||
        (s = bb.alloc(&seeds, g, "seeds")) != PGB_OK ||
        (s = bb.alloc(&error, 1, "error flag")) != PGB_OK)
        return s;
    if ((s = ck(cudaMemset(rows, 0, (size_t)n * kRowBytes), "rows")) != PGB_OK ||
        (s = ck(cudaMemcpy2D(rows, kRowBytes, vectors, dim, dim, n, cudaMemcpyHostToDevice), "rows")) != PGB_OK ||
        (s = ck(cudaMemset(adj, 0xFF, (size_t)n * slots * 4), "adjacency")) != PGB_OK ||
        (s = ck(cudaMemset(deg, 0, (size_t)n * 4), "degrees")) != PGB_OK ||
        (s = ck(cudaMemset(error, 0, 4), "error flag")) != PGB_OK)
        return s;

    // leaf k-NN shared memory: the rows (with norms and ids), later the padded edge keys
    const uint32_t lmax = std::min(std::max(leaf, 2u), n);
    const size_t knn_smem = std::max<size_t>((size_t)lmax * (16u * nq + 8u),
                                             (size_t)next_pow2_u32(lmax * std::min(kLeafK, lmax - 1u)) * 8u);
    if ((s = ck(cudaFuncSetAttribute(knn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)knn_smem),
                "kernel attribute")) != PGB_OK)
        return s;

    HcnngArgs A{};
    A.rows = rows;
    A.n = n;
    A.leaf = std::max(leaf, 2u);
    A.mst_deg = mst_deg;
    A.seeds = seeds;
    A.ids = ids;
    A.alt = alt;
    A.flags = flags;
    A.stack = stack;
    A.leaves = leaves;
    A.n_leaves = n_leaves;
    A.edges = edges;
    A.out = out;
    A.out_n = out_n;
    A.error = error;
    std::vector<uint64_t> hseeds(g);
    std::vector<uint32_t> hleaves(g);
    for (uint32_t t0 = 0; t0 < trees; t0 += g) {
        const uint32_t gg = std::min(g, trees - t0);
        for (uint32_t k = 0; k < gg; k++) hseeds[k] = seed * 1000003ull + (t0 + k);
        if ((s = ck(cudaMemcpy(seeds, hseeds.data(), gg * 8u, cudaMemcpyHostToDevice), "seeds")) != PGB_OK)
            return s;
        {
            void* args[] = {&A};
            if ((s = ck(cudaLaunchKernel(part, dim3(gg), dim3(kPartThreads), args, 0, nullptr), "partition launch")) != PGB_OK)
                return s;
        }
        if ((s = ck(cudaMemcpy(hleaves.data(), n_leaves, gg * 4u, cudaMemcpyDeviceToHost), "partition")) != PGB_OK)
            return s;
        uint32_t err = 0;
        if ((s = ck(cudaMemcpy(&err, error, 4, cudaMemcpyDeviceToHost), "error flag")) != PGB_OK) return s;
        if (err) return fail(PGB_ERR_OVERFLOW, "hcnng (GPU): partition stack overflow");
        const uint32_t max_leaves = *std::max_element(hleaves.begin(), hleaves.begin() + gg);
        {
            void* args[] = {&A};
            if ((s = ck(cudaLaunchKernel(knn, dim3(max_leaves, gg), dim3(kKnnThreads), args, knn_smem, nullptr),
                        "leaf k-NN launch")) != PGB_OK)
                return s;
        }
        if ((s = ck(cudaMemsetAsync(out_n, 0, (size_t)gg * n * 4), "tree degrees")) != PGB_OK) return s;
        hcnng_kruskal_kernel<<<dim3((max_leaves + kKruskalWarps - 1) / kKruskalWarps, gg), kKruskalWarps * 32>>>(A);
        if ((s = ck(cudaGetLastError(), "Kruskal launch")) != PGB_OK) return s;
        hcnng_append_kernel<<<(n + 255) / 256, 256>>>(A, gg, slots, adj, deg);
        if ((s = ck(cudaGetLastError(), "append launch")) != PGB_OK) return s;
    }
    if ((s = ck(cudaMemcpy(adjacency, adj, (size_t)n * slots * 4, cudaMemcpyDeviceToHost), "adjacency")) != PGB_OK ||
        (s = ck(cudaMemcpy(degrees, deg, (size_t)n * 4, cudaMemcpyDeviceToHost), "degrees")) != PGB_OK)
        return s;
    return PGB_OK;
}
