// build_gpu.cu -- Vamana graph construction on the GPU (pgb_build_vamana_gpu).
//
// The algorithm is the CPU builder's (builders.cpp: build_vamana), step for step, so the
// two produce the same graph for the same seed:
//   insertion order: vamana_insertion_order(n, seed), prefix-doubling batches of 1, 2,
//   4, ... up to 2 % of n points; each batch searches the graph as it stood before it;
//   per point: greedy beam search of width L from point 0 with an exact "seen" set,
//   every expanded node a candidate, then RobustPrune (alpha) to at most R out-edges;
//   per batch: the reverse of every new edge p -> q is merged into q's row: appended in
//   ascending p when the row has room, else q's row is re-pruned.
// GPU form: one warp per point for search + prune; the batch's new edges become 64-bit
// (q, p) keys sorted by a radix sort (deterministic, no atomics in the order), grouped by
// q, one warp per group for the merge.
//
// Beam search acceptance. The CPU inserts the neighbours of an expanded node one by one,
// skipping one whose distance is not below the last entry of a full list. Equivalently
// (the rule the HNSW kernel uses): neighbour j enters iff fewer than L elements of the
// list plus the earlier new neighbours of this row have distance <= d_j, and the list
// becomes the first L of its union with the entering ones. The next node expanded is the
// first unexpanded entry of the list, as on the CPU.
//
// Capacity: a point whose seen set or candidate list would outgrow its per-warp tables is
// flagged and searched again with tables four times larger, so the result never depends
// on the table sizes.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <string>
#include <vector>

#include "builders.h"
#include "errors.h"
#include "formats.h"
#include "index.h"
#include "search_flat.cuh"
#include "search_plan.h"

namespace pgb {
namespace {

constexpr uint32_t kKeptStride = 33;  // words per kept row in shared memory (bank-conflict free)

struct BuildLayout {
    uint32_t lcap, gs, seen_cap, R;
    uint32_t off_f0, off_f1, off_v0, off_v1, off_pend, off_pdist, off_akey, off_x, off_knorm,
        off_crow, off_out, bytes;
};

__host__ __device__ inline BuildLayout make_build_layout(uint32_t L, uint32_t gs, uint32_t seen_cap,
                                                         uint32_t R) {
    BuildLayout B{};
    B.lcap = (L + 7u) & ~7u;
    B.gs = gs;
    B.seen_cap = seen_cap;
    B.R = R;
    uint32_t o = kRowBytes;  // the point's own row (the query)
    B.off_f0 = o;
    o += 8u * B.lcap;
    B.off_f1 = o;
    o += 8u * B.lcap;
    B.off_v0 = o;
    o += B.lcap;
    B.off_v1 = o;
    o = round16(o + B.lcap);
    B.off_pend = o;
    o += 4u * gs;
    B.off_pdist = o;
    o += 4u * gs;
    B.off_akey = o;
    o += 8u * gs;
    // search: seen-slot occupancy bitmap; prune: kept rows -- never both at once
    B.off_x = o;
    o += round16(std::max(seen_cap / 8u, 4u * kKeptStride * R));
    B.off_knorm = o;
    o += round16(4u * R);
    B.off_crow = o;
    o += kRowBytes;
    B.off_out = o;
    o += round16(4u * R);
    B.bytes = round16(o);
    return B;
}

struct SearchPruneArgs {
    const uint8_t* rows;      // n x 128, zero padded
    const uint32_t* adj;      // n x R, kNoNeighbor padded (the graph before this batch)
    const uint32_t* deg;      // n
    uint32_t n, dim, R, L;
    float alpha;
    const uint32_t* points;   // this launch's points
    const uint32_t* slots;    // their batch slots (null: slot = index)
    uint32_t np;
    uint32_t* out;            // batch slots x R
    uint32_t* out_n;          // batch slots
    uint32_t* seen_tab;       // per warp: seen_cap ids
    uint64_t* cand;           // per warp: 2 x cand_cap keys (candidates, sorted)
    uint32_t cand_cap;
    BuildLayout B;
    uint32_t* flagged;        // slots to search again with larger tables
    uint32_t* n_flagged;
    uint32_t* queue;
};

// home slot of an id in a warp's seen set (only membership matters)
__device__ __forceinline__ uint32_t seen_home(uint32_t id, uint32_t shift) {
    return (id * 0x9E3779B1u) >> shift;
}

__device__ bool seen_contains(const uint32_t* tab, const uint32_t* occ, uint32_t mask,
                              uint32_t shift, uint32_t id) {
    uint32_t h = seen_home(id, shift);
    for (uint32_t i = 0; i <= mask; i++) {
        if (!((occ[h >> 5] >> (h & 31u)) & 1u)) return false;
        if (__ldcg(tab + h) == id) return true;
        h = (h + 1) & mask;
    }
    return false;
}

// insert of an absent id; several lanes at once with distinct ids (slot claimed with a
// shared-memory atomic, then written; lookups run after a __syncwarp)
__device__ void seen_insert(uint32_t* tab, uint32_t* occ, uint32_t mask, uint32_t shift,
                            uint32_t id) {
    uint32_t h = seen_home(id, shift);
    for (uint32_t i = 0; i <= mask; i++) {
        const uint32_t bit = 1u << (h & 31u);
        if (!(occ[h >> 5] & bit) && !(atomicOr(&occ[h >> 5], bit) & bit)) {
            tab[h] = id;
            return;
        }
        h = (h + 1) & mask;
    }
}

template <bool Signed>
__device__ __forceinline__ int32_t dot4(uint32_t a, uint32_t b) {
    if (Signed) return __dp4a((int)a, (int)b, 0);
    return (int32_t)__dp4a(a, b, 0u);
}

// sorts keys[0, m) into out[0, m) by rank (equal keys keep their order); global memory
__device__ void rank_sort(const uint64_t* keys, int m, uint64_t* out, int lane) {
    for (int i = lane; i < m; i += 32) {
        const uint64_t k = keys[i];
        int r = 0;
        for (int j = 0; j < m; j++) {
            const uint64_t o = keys[j];
            r += (o < k || (o == k && j < i)) ? 1 : 0;
        }
        out[r] = k;
    }
    __syncwarp();
}

// Neighbour selection over the sorted candidate keys (dist to `self`, id): drops repeats of
// an id and `self`, stops at R kept, and keeps c unless a kept o dominates it -- Vamana's
// RobustPrune: alpha * d(o, c) <= d(self, c); HNSW's heuristic (HnswRule): d(o, c) <
// alpha * d(self, c); both with the CPU builders' float arithmetic. Kept rows are staged
// in shared memory. Returns the count; out_ids[0, count) in shared memory.
template <bool Signed, bool HnswRule = false>
__device__ int warp_prune(const uint32_t* rows32, const uint64_t* sorted, int m, uint32_t self,
                          float alpha, int R, uint32_t* kept_rows, int32_t* kept_norm,
                          uint32_t* crow, uint32_t* out_ids, int lane) {
    int kept = 0;
    uint64_t prev = ~0ull;
    for (int i = 0; i < m && kept < R; i++) {
        const uint64_t key = sorted[i];
        const bool repeat = key == prev;
        prev = key;
        const uint32_t cid = key_id(key);
        if (repeat || cid == self) continue;
        const int32_t cd = key_dist(key);
        const uint32_t cw = __ldg(rows32 + (size_t)cid * 32u + lane);
        int32_t cn = dot4<Signed>(cw, cw);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cn += __shfl_xor_sync(kFull, cn, off);
        crow[lane] = cw;
        __syncwarp();
        bool dominated = false;
        for (int kk = lane; kk < kept; kk += 32) {
            const uint32_t* kr = kept_rows + kk * kKeptStride;
            int32_t dot = 0;
#pragma unroll 8
            for (int w = 0; w < 32; w++) dot += dot4<Signed>(kr[w], crow[w]);
            const int32_t d = kept_norm[kk] + cn - 2 * dot;
            if (HnswRule ? ((float)d < __fmul_rn(alpha, (float)cd)) : (__fmul_rn(alpha, (float)d) <= (float)cd))
                dominated = true;
        }
        const bool any = __any_sync(kFull, dominated);
        if (!any) {
            kept_rows[kept * kKeptStride + lane] = cw;
            if (lane == 0) {
                kept_norm[kept] = cn;
                out_ids[kept] = cid;
            }
            kept++;
        }
        __syncwarp();
    }
    return kept;
}

// Neighbour rows of one graph level: node u's row is `start[u] + sub` when `start` is set
// (HNSW levels above 0: one block per (node, level)), else u.
struct LevelRows {
    uint32_t* adj;         // rows of `stride` ids, kNoNeighbor padded (searches only read)
    uint32_t* size;        // entries of each row
    const uint32_t* start;
    uint32_t stride, sub;
    __device__ uint32_t row_of(uint32_t u) const { return start ? start[u] + sub : u; }
};

// A warp's search state: frontier buffers and scratch in shared memory, seen ids and
// expanded keys in its global slices.
struct WarpSearch {
    unsigned char* wm;
    uint32_t off_f0, off_f1, off_v0, off_v1;
    uint32_t* pend;
    int32_t* pdist;
    uint64_t* akey;
    uint32_t* occ;
    uint32_t* tab;
    uint32_t mask, shift, seen_cap;
    uint64_t* cand;     // expanded keys (when kept)
    int cand_limit;     // expansions allowed before the list would overflow
};

// Greedy beam search of width ef over one level (the CPU builders' build search). On entry
// the frontier, sorted and unexpanded, holds fsize keys in buffer `cur`, and their ids are
// in the seen set (nseen ids). Expands the first unexpanded entry until none is left; with
// KeepExpanded every expanded key is appended to cand[nvis++]. Returns the final frontier
// size (in buffer `cur`), or -1 when the seen set or the expanded list would overflow.
template <int CH, bool Signed, bool KeepExpanded>
__device__ int level_search(const uint8_t* rows, uint32_t dim, const LevelRows& G, int ef,
                            const WarpSearch& S, const int4* q4, int32_t qq, int fsize, int& cur,
                            int& nvis, int& nseen, int lane) {
    const uint32_t lt = lanemask_lt();
    uint64_t* const f0 = reinterpret_cast<uint64_t*>(S.wm + S.off_f0);
    uint64_t* const f1 = reinterpret_cast<uint64_t*>(S.wm + S.off_f1);
    for (;;) {
        // the frontier and its expanded flags alternate between two buffers
        uint64_t* F = cur ? f1 : f0;
        uint8_t* V = S.wm + (cur ? S.off_v1 : S.off_v0);
        int u = -1;
        for (int base = 0; base < fsize; base += 32) {
            const int i = base + lane;
            const uint32_t m = __ballot_sync(kFull, i < fsize && !V[i]);
            if (m) {
                u = base + __ffs(m) - 1;
                break;
            }
        }
        if (u < 0) return fsize;
        if (KeepExpanded && nvis >= S.cand_limit) return -1;
        const uint64_t ukey = F[u];
        if (lane == 0) {
            V[u] = 1;
            if (KeepExpanded) S.cand[nvis] = ukey;
        }
        if (KeepExpanded) nvis++;
        const uint32_t ri = G.row_of(key_id(ukey));
        const uint32_t du = G.size[ri];
        const uint32_t* row = G.adj + (size_t)ri * G.stride;
        // unseen neighbours, in row order
        int np = 0;
#pragma unroll
        for (int t = 0; t < CH; t++) {
            const uint32_t j = (uint32_t)(t * 32 + lane);
            const uint32_t x = j < du ? __ldg(row + j) : kEmptyId;
            const bool valid = x != kEmptyId;
            const uint32_t peers = __match_any_sync(kFull, valid ? x : (0x80000000u | j));
            const bool first = valid && (peers & lt) == 0;
            const bool fresh = first && !seen_contains(S.tab, S.occ, S.mask, S.shift, x);
            __syncwarp();
            if (fresh) seen_insert(S.tab, S.occ, S.mask, S.shift, x);
            const uint32_t m = __ballot_sync(kFull, fresh);
            if (fresh) S.pend[np + __popc(m & lt)] = x;
            np += __popc(m);
            __syncwarp();
        }
        nseen += np;
        if (nseen > (int)(S.seen_cap / 2u)) return -1;
        row_distances<Signed>(rows, S.pend, S.pdist, np, q4, qq, dim, false, lane);
        // acceptance: fewer than ef of (list + earlier new neighbours) at distance <= d
        int na = 0;
        for (int base = 0; base < np; base += 32) {
            const int j = base + lane;
            bool acc = false;
            int32_t d = 0;
            if (j < np) {
                d = S.pdist[j];
                int c = upper_bound_key(F, fsize, pack_key(d, 0xFFFFFFFFu));
                for (int i = 0; i < j && c < ef; i++) c += S.pdist[i] <= d ? 1 : 0;
                acc = c < ef;
            }
            const uint32_t m = __ballot_sync(kFull, acc);
            if (acc) S.akey[na + __popc(m & lt)] = pack_key(d, S.pend[j]);
            na += __popc(m);
        }
        __syncwarp();
        if (na > 0) {
            sort_keys<CH>(S.akey, na, lane);
            uint64_t* Fn = cur ? f0 : f1;
            uint8_t* Vn = S.wm + (cur ? S.off_v0 : S.off_v1);
            for (int k = lane; k < fsize; k += 32) {
                const int pos = k + lower_bound_key(S.akey, na, F[k]);
                if (pos < ef) {
                    Fn[pos] = F[k];
                    Vn[pos] = V[k];
                }
            }
            for (int i = lane; i < na; i += 32) {
                const int pos = i + lower_bound_key(F, fsize, S.akey[i]);
                if (pos < ef) {
                    Fn[pos] = S.akey[i];
                    Vn[pos] = 0;
                }
            }
            __syncwarp();
            fsize = min(ef, fsize + na);
            cur ^= 1;
        }
    }
}

// One warp per point: beam search over the graph before this batch, then prune.
template <int CH, bool Signed>
__global__ void __launch_bounds__(128, 4) search_prune_kernel(SearchPruneArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + w;
    const BuildLayout& B = A.B;
    unsigned char* wm = smem + (size_t)w * B.bytes;
    uint32_t* qwords = reinterpret_cast<uint32_t*>(wm);
    uint64_t* const fbuf0 = reinterpret_cast<uint64_t*>(wm + B.off_f0);
    uint32_t* pend = reinterpret_cast<uint32_t*>(wm + B.off_pend);
    int32_t* pdist = reinterpret_cast<int32_t*>(wm + B.off_pdist);
    uint64_t* akey = reinterpret_cast<uint64_t*>(wm + B.off_akey);
    uint32_t* occ = reinterpret_cast<uint32_t*>(wm + B.off_x);
    uint32_t* kept_rows = reinterpret_cast<uint32_t*>(wm + B.off_x);
    int32_t* kept_norm = reinterpret_cast<int32_t*>(wm + B.off_knorm);
    uint32_t* crow = reinterpret_cast<uint32_t*>(wm + B.off_crow);
    uint32_t* out_ids = reinterpret_cast<uint32_t*>(wm + B.off_out);
    uint32_t* tab = A.seen_tab + (size_t)gw * B.seen_cap;
    uint64_t* cand = A.cand + (size_t)gw * 2u * A.cand_cap;
    uint64_t* sorted = cand + A.cand_cap;
    const uint32_t mask = B.seen_cap - 1u;
    const uint32_t shift = 32u - (uint32_t)ceil_log2_u64(B.seen_cap);
    const int L = (int)A.L, R = (int)A.R;
    const uint32_t* rows32 = reinterpret_cast<const uint32_t*>(A.rows);
    WarpSearch S;
    S.wm = wm;
    S.off_f0 = B.off_f0;
    S.off_f1 = B.off_f1;
    S.off_v0 = B.off_v0;
    S.off_v1 = B.off_v1;
    S.pend = pend;
    S.pdist = pdist;
    S.akey = akey;
    S.occ = occ;
    S.tab = tab;
    S.mask = mask;
    S.shift = shift;
    S.seen_cap = B.seen_cap;
    S.cand = cand;
    S.cand_limit = (int)A.cand_cap - R;  // room left for the point's own row

    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(kFull, it, 0);
        if (it >= A.np) break;
        const uint32_t p = A.points[it];
        const uint32_t slot = A.slots ? A.slots[it] : it;
        qwords[lane] = __ldg(rows32 + (size_t)p * 32u + lane);
        for (uint32_t i = lane; i < B.seen_cap / 32u; i += 32) occ[i] = 0u;
        __syncwarp();
        const int4* q4 = reinterpret_cast<const int4*>(qwords);
        const int32_t qq = query_sq_norm<Signed>(q4, lane);
        // start point 0: seen, one entry
        if (lane == 0) {
            pend[0] = 0u;
            seen_insert(tab, occ, mask, shift, 0u);
        }
        __syncwarp();
        row_distances<Signed>(A.rows, pend, pdist, 1, q4, qq, A.dim, false, lane);
        int cur = 0;
        if (lane == 0) {
            fbuf0[0] = pack_key(pdist[0], 0u);
            wm[B.off_v0] = 0;
        }
        __syncwarp();
        int nvis = 0, nseen = 1;
        // the search only reads the rows
        const LevelRows G{const_cast<uint32_t*>(A.adj), const_cast<uint32_t*>(A.deg), nullptr, A.R, 0u};
        const int fsize = level_search<CH, Signed, true>(A.rows, A.dim, G, L, S, q4, qq, 1, cur, nvis,
                                                         nseen, lane);
        if (fsize < 0) {
            if (lane == 0) A.flagged[atomicAdd(A.n_flagged, 1u)] = slot;
            __syncwarp();
            continue;
        }
        // the point's current out-neighbours stay candidates
        const uint32_t dp = A.deg[p];
        const uint32_t* prow = A.adj + (size_t)p * A.R;
        for (uint32_t base = 0; base < dp; base += 32u * CH) {
            const uint32_t cnt = min(dp - base, 32u * CH);
            for (uint32_t j = lane; j < cnt; j += 32) pend[j] = __ldg(prow + base + j);
            __syncwarp();
            row_distances<Signed>(A.rows, pend, pdist, (int)cnt, q4, qq, A.dim, false, lane);
            for (uint32_t j = lane; j < cnt; j += 32) cand[nvis + base + j] = pack_key(pdist[j], pend[j]);
            __syncwarp();
        }
        const int m = nvis + (int)dp;
        __syncwarp();
        rank_sort(cand, m, sorted, lane);
        const int kept = warp_prune<Signed>(rows32, sorted, m, p, A.alpha, R, kept_rows, kept_norm,
                                            crow, out_ids, lane);
        for (int j = lane; j < R; j += 32) A.out[(size_t)slot * A.R + j] = j < kept ? out_ids[j] : kEmptyId;
        if (lane == 0) A.out_n[slot] = (uint32_t)kept;
        __syncwarp();
    }
}

// the batch's new rows replace the old ones
__global__ void write_rows_kernel(const uint32_t* points, uint32_t nb, const uint32_t* out,
                                  const uint32_t* out_n, uint32_t R, uint32_t* adj, uint32_t* deg) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)nb * R) return;
    const uint32_t b = (uint32_t)(t / R), j = (uint32_t)(t % R);
    const uint32_t p = points[b];
    adj[(size_t)p * R + j] = out[t];
    if (j == 0) deg[p] = out_n[b];
}

// (q, p) keys of the batch's new edges p -> q; unused slots sort last
__global__ void pair_keys_kernel(const uint32_t* points, uint32_t nb, const uint32_t* out,
                                 const uint32_t* out_n, uint32_t R, uint64_t* keys) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)nb * R) return;
    const uint32_t b = (uint32_t)(t / R), j = (uint32_t)(t % R);
    keys[t] = j < out_n[b] ? (((uint64_t)out[t] << 32) | points[b]) : ~0ull;
}

__global__ void key_targets_kernel(const uint64_t* keys, uint32_t n, uint32_t* q) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) q[t] = (uint32_t)(keys[t] >> 32);
}

struct MergeArgs {
    const uint8_t* rows;
    LevelRows G;                // the level whose rows receive the reverse edges
    uint32_t dim, cap;          // cap: entries a row may hold
    float alpha;
    const uint64_t* keys;       // sorted (q, p)
    const uint32_t* run_q;      // per group: q (kEmptyId: unused pair slots)
    const uint32_t* run_cnt;
    const uint32_t* run_off;
    const uint32_t* n_runs;
    const uint32_t* groups;     // null: every group; else these group indices
    uint32_t n_groups;
    uint32_t* gid;              // per warp: wcap candidate ids
    int32_t* gdist;             //           their distances to q
    uint64_t* gkey;             //           2 x wcap keys (candidates, sorted)
    uint32_t wcap;
    uint32_t* big;              // groups whose candidates exceed wcap, merged again later
    uint32_t* n_big;
    BuildLayout B;
    uint32_t* queue;
};

// One warp per target q: new sources not yet in q's row are appended in ascending order
// when the row has room, else q's row is re-selected (RobustPrune, or HNSW's heuristic)
// from its entries and the new sources.
template <int CH, bool Signed, bool HnswRule>
__global__ void __launch_bounds__(128, 4) merge_reverse_kernel(MergeArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const BuildLayout& B = A.B;
    unsigned char* wm = smem + (size_t)w * B.bytes;
    uint32_t* qwords = reinterpret_cast<uint32_t*>(wm);
    uint32_t* kept_rows = reinterpret_cast<uint32_t*>(wm + B.off_x);
    int32_t* kept_norm = reinterpret_cast<int32_t*>(wm + B.off_knorm);
    uint32_t* crow = reinterpret_cast<uint32_t*>(wm + B.off_crow);
    uint32_t* out_ids = reinterpret_cast<uint32_t*>(wm + B.off_out);
    uint32_t* rowbuf = reinterpret_cast<uint32_t*>(wm + B.off_pend);  // q's row (<= gs ids)
    const uint32_t lt = lanemask_lt();
    const uint32_t* rows32 = reinterpret_cast<const uint32_t*>(A.rows);
    const uint32_t total = A.groups ? A.n_groups : *A.n_runs;
    const int R = (int)A.cap;
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + w;
    uint32_t* ids = A.gid + (size_t)gw * A.wcap;
    int32_t* dists = A.gdist + (size_t)gw * A.wcap;
    uint64_t* keys = A.gkey + (size_t)gw * 2u * A.wcap;
    uint64_t* sorted = keys + A.wcap;
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(kFull, it, 0);
        if (it >= total) break;
        const uint32_t g = A.groups ? A.groups[it] : it;
        const uint32_t q = A.run_q[g];
        if (q == kEmptyId) continue;
        const uint32_t cnt = A.run_cnt[g], off = A.run_off[g];
        const uint32_t ri = A.G.row_of(q);
        const uint32_t dq = A.G.size[ri];
        uint32_t* qrow = A.G.adj + (size_t)ri * A.G.stride;
        for (uint32_t j = lane; j < dq; j += 32) rowbuf[j] = qrow[j];
        __syncwarp();
        // new sources: not in q's row and not q itself, ascending (keys are sorted)
        uint32_t added = 0;
        for (uint32_t b0 = 0; b0 < cnt; b0 += 32) {
            const uint32_t i = b0 + lane;
            bool fresh = false;
            uint32_t p = 0;
            if (i < cnt) {
                p = (uint32_t)A.keys[off + i];
                fresh = p != q;
                for (uint32_t j = 0; j < dq && fresh; j++)
                    if (rowbuf[j] == p) fresh = false;
            }
            const uint32_t m = __ballot_sync(kFull, fresh);
            const uint32_t at = dq + added + __popc(m & lt);
            if (fresh && at < A.wcap) ids[at] = p;
            added += __popc(m);
        }
        __syncwarp();
        if (added == 0) continue;
        if (dq + added > A.wcap) {  // a hub: merged again with larger scratch
            if (lane == 0) A.big[atomicAdd(A.n_big, 1u)] = g;
            __syncwarp();
            continue;
        }
        if (dq + added <= A.cap) {
            for (uint32_t j = lane; j < added; j += 32) qrow[dq + j] = ids[dq + j];
            if (lane == 0) A.G.size[ri] = dq + added;
            __syncwarp();
            continue;
        }
        // re-prune q's row: candidates are its entries and the new sources
        for (uint32_t j = lane; j < dq; j += 32) ids[j] = rowbuf[j];
        qwords[lane] = __ldg(rows32 + (size_t)q * 32u + lane);
        __syncwarp();
        const int4* q4 = reinterpret_cast<const int4*>(qwords);
        const int32_t qq = query_sq_norm<Signed>(q4, lane);
        const int m = (int)(dq + added);
        row_distances<Signed>(A.rows, ids, dists, m, q4, qq, A.dim, false, lane);
        for (int j = lane; j < m; j += 32) keys[j] = pack_key(dists[j], ids[j]);
        __syncwarp();
        rank_sort(keys, m, sorted, lane);
        const int kept = warp_prune<Signed, HnswRule>(rows32, sorted, m, q, A.alpha, R, kept_rows,
                                                      kept_norm, crow, out_ids, lane);
        for (int j = lane; j < R; j += 32) qrow[j] = j < kept ? out_ids[j] : kEmptyId;
        if (lane == 0) A.G.size[ri] = (uint32_t)kept;
        __syncwarp();
    }
}

template <bool Signed>
void* search_prune_for(int ch) {
    switch (ch) {
        case 1: return (void*)search_prune_kernel<1, Signed>;
        case 2: return (void*)search_prune_kernel<2, Signed>;
        case 3: return (void*)search_prune_kernel<3, Signed>;
        case 4: return (void*)search_prune_kernel<4, Signed>;
        default: return (void*)search_prune_kernel<8, Signed>;
    }
}

template <bool Signed, bool HnswRule>
void* merge_for(int ch) {
    switch (ch) {
        case 1: return (void*)merge_reverse_kernel<1, Signed, HnswRule>;
        case 2: return (void*)merge_reverse_kernel<2, Signed, HnswRule>;
        case 3: return (void*)merge_reverse_kernel<3, Signed, HnswRule>;
        case 4: return (void*)merge_reverse_kernel<4, Signed, HnswRule>;
        default: return (void*)merge_reverse_kernel<8, Signed, HnswRule>;
    }
}

// ---- HNSW -----------------------------------------------------------------------------
// The CPU builder's (builders.cpp: build_hnsw) insertion, per point: greedy descent
// from the entry through the levels above the point's own (move to the smallest (d, id)
// of the current node's row until none is smaller), then from the lower of its level and
// the top level down to 0 a beam search of width efc starting from the previous level's
// final list, whose final list gives the level's neighbours by HNSW's heuristic (at most
// 2M at level 0, M above). Rows at level 0 are n x 2M; a node's rows at levels 1..l are
// blocks of M at ustart[node] + level - 1.

struct HnswInsertArgs {
    const uint8_t* rows;
    uint32_t n, dim, M, efc;
    float alpha;
    LevelRows L0;             // level 0 rows
    uint32_t* adju;           // levels >= 1
    uint32_t* sizeu;
    const uint32_t* ustart;
    const uint32_t* level;
    uint32_t entry, top;      // the graph's entry point and top level before this batch
    const uint32_t* points;
    const uint32_t* slots;    // batch slots (null: slot = index)
    uint32_t np;
    uint32_t* out;            // per slot: level 0 (2M ids), then M ids per level >= 1
    const uint64_t* out_off;
    uint32_t* out_n;          // per slot: selected count per level
    const uint32_t* outn_off;
    uint32_t* seen_tab;
    BuildLayout B;
    uint32_t* flagged;
    uint32_t* n_flagged;
    uint32_t* queue;
};

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const uint64_t o = __shfl_xor_sync(kFull, v, off);
        v = o < v ? o : v;
    }
    return v;
}

template <int CH, bool Signed>
__global__ void __launch_bounds__(128, 4) hnsw_insert_kernel(HnswInsertArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + w;
    const BuildLayout& B = A.B;
    unsigned char* wm = smem + (size_t)w * B.bytes;
    uint32_t* qwords = reinterpret_cast<uint32_t*>(wm);
    uint32_t* pend = reinterpret_cast<uint32_t*>(wm + B.off_pend);
    int32_t* pdist = reinterpret_cast<int32_t*>(wm + B.off_pdist);
    uint32_t* occ = reinterpret_cast<uint32_t*>(wm + B.off_x);
    uint32_t* kept_rows = reinterpret_cast<uint32_t*>(wm + B.off_x);
    int32_t* kept_norm = reinterpret_cast<int32_t*>(wm + B.off_knorm);
    uint32_t* crow = reinterpret_cast<uint32_t*>(wm + B.off_crow);
    uint32_t* out_ids = reinterpret_cast<uint32_t*>(wm + B.off_out);
    const uint32_t* rows32 = reinterpret_cast<const uint32_t*>(A.rows);
    WarpSearch S;
    S.wm = wm;
    S.off_f0 = B.off_f0;
    S.off_f1 = B.off_f1;
    S.off_v0 = B.off_v0;
    S.off_v1 = B.off_v1;
    S.pend = pend;
    S.pdist = pdist;
    S.akey = reinterpret_cast<uint64_t*>(wm + B.off_akey);
    S.occ = occ;
    S.tab = A.seen_tab + (size_t)gw * B.seen_cap;
    S.mask = B.seen_cap - 1u;
    S.shift = 32u - (uint32_t)ceil_log2_u64(B.seen_cap);
    S.seen_cap = B.seen_cap;
    S.cand = nullptr;
    S.cand_limit = 0;
    uint64_t* const f0 = reinterpret_cast<uint64_t*>(wm + B.off_f0);
    uint64_t* const f1 = reinterpret_cast<uint64_t*>(wm + B.off_f1);
    const int M = (int)A.M;
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(A.queue, 1u);
        it = __shfl_sync(kFull, it, 0);
        if (it >= A.np) break;
        const uint32_t p = A.points[it];
        const uint32_t slot = A.slots ? A.slots[it] : it;
        const uint32_t lvl = A.level[p];
        qwords[lane] = __ldg(rows32 + (size_t)p * 32u + lane);
        if (lane == 0) pend[0] = A.entry;
        __syncwarp();
        const int4* q4 = reinterpret_cast<const int4*>(qwords);
        const int32_t qq = query_sq_norm<Signed>(q4, lane);
        row_distances<Signed>(A.rows, pend, pdist, 1, q4, qq, A.dim, false, lane);
        uint64_t best = pack_key(pdist[0], A.entry);
        __syncwarp();
        // greedy descent through the levels above the point's own; each move lowers (d, id)
        for (int l = (int)A.top; l > (int)lvl; l--) {
            for (uint32_t guard = 0; guard < A.n; guard++) {
                const uint32_t ri = A.ustart[key_id(best)] + (uint32_t)(l - 1);
                const uint32_t sz = A.sizeu[ri];
                const uint32_t* row = A.adju + (size_t)ri * A.M;
                for (uint32_t j = lane; j < sz; j += 32) pend[j] = row[j];
                __syncwarp();
                row_distances<Signed>(A.rows, pend, pdist, (int)sz, q4, qq, A.dim, false, lane);
                uint64_t m = ~0ull;
                for (uint32_t j = lane; j < sz; j += 32) m = min(m, pack_key(pdist[j], pend[j]));
                m = warp_min_u64(m);
                __syncwarp();
                if (m >= best) break;
                best = m;
            }
        }
        // levels above the graph's top get no neighbours (the point becomes the new top)
        for (int l = (int)lvl; l > (int)min(A.top, lvl); l--) {
            uint32_t* o = A.out + A.out_off[slot] + 2u * A.M + (uint32_t)(l - 1) * A.M;
            for (int j = lane; j < M; j += 32) o[j] = kEmptyId;
            if (lane == 0) A.out_n[A.outn_off[slot] + l] = 0u;
        }
        // per level: a fresh seen set holding the list, every entry unexpanded
        int cur = 0, fsize = 1;
        if (lane == 0) f0[0] = best;
        __syncwarp();
        bool over = false;
        for (int l = (int)min(A.top, lvl); l >= 0; l--) {
            uint64_t* F = cur ? f1 : f0;
            uint8_t* V = wm + (cur ? B.off_v1 : B.off_v0);
            for (uint32_t i = lane; i < B.seen_cap / 32u; i += 32) occ[i] = 0u;
            __syncwarp();
            for (int i = lane; i < fsize; i += 32) {
                V[i] = 0;
                seen_insert(S.tab, occ, S.mask, S.shift, key_id(F[i]));
            }
            __syncwarp();
            int nseen = fsize, nvis = 0;
            const LevelRows G = l == 0 ? A.L0 : LevelRows{A.adju, A.sizeu, A.ustart, A.M, (uint32_t)(l - 1)};
            fsize = level_search<CH, Signed, false>(A.rows, A.dim, G, (int)A.efc, S, q4, qq, fsize, cur,
                                                    nvis, nseen, lane);
            if (fsize < 0) {
                over = true;
                break;
            }
            F = cur ? f1 : f0;
            const int capl = l == 0 ? 2 * M : M;
            const int kept = warp_prune<Signed, true>(rows32, F, fsize, p, A.alpha, capl, kept_rows,
                                                      kept_norm, crow, out_ids, lane);
            uint32_t* o = A.out + A.out_off[slot] + (l == 0 ? 0u : 2u * A.M + (uint32_t)(l - 1) * A.M);
            for (int j = lane; j < capl; j += 32) o[j] = j < kept ? out_ids[j] : kEmptyId;
            if (lane == 0) A.out_n[A.outn_off[slot] + l] = (uint32_t)kept;
            __syncwarp();
        }
        if (over) {
            if (lane == 0) A.flagged[atomicAdd(A.n_flagged, 1u)] = slot;
            __syncwarp();
        }
    }
}

// the batch's selected rows replace the old ones, at every level of each point; one warp
// per batch point
__global__ void hnsw_write_rows_kernel(const uint32_t* points, uint32_t nb, const uint32_t* level,
                                       const uint32_t* out, const uint64_t* out_off,
                                       const uint32_t* out_n, const uint32_t* outn_off, uint32_t M,
                                       LevelRows L0, uint32_t* adju, uint32_t* sizeu,
                                       const uint32_t* ustart) {
    const uint32_t b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nb) return;
    const uint32_t p = points[b], lvl = level[p];
    for (uint32_t l = 0; l <= lvl; l++) {
        const uint32_t capl = l == 0 ? 2u * M : M;
        const uint32_t* src = out + out_off[b] + (l == 0 ? 0u : 2u * M + (l - 1) * M);
        const uint32_t ri = l == 0 ? p : ustart[p] + l - 1;
        uint32_t* dst = l == 0 ? L0.adj + (size_t)p * L0.stride : adju + (size_t)ri * M;
        for (uint32_t j = lane; j < capl; j += 32) dst[j] = src[j];
        if (lane == 0) (l == 0 ? L0.size : sizeu)[ri] = out_n[outn_off[b] + l];
    }
}

// (q, p) keys of the batch's new level-l edges p -> q; other slots sort last
__global__ void hnsw_pair_keys_kernel(const uint32_t* points, uint32_t nb, const uint32_t* level,
                                      const uint32_t* out, const uint64_t* out_off,
                                      const uint32_t* out_n, const uint32_t* outn_off, uint32_t M,
                                      uint32_t l, uint32_t capl, uint64_t* keys) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)nb * capl) return;
    const uint32_t b = (uint32_t)(t / capl), j = (uint32_t)(t % capl);
    const uint32_t p = points[b];
    const bool ok = level[p] >= l && j < out_n[outn_off[b] + l];
    keys[t] = ok ? (((uint64_t)out[out_off[b] + (l == 0 ? 0u : 2u * M + (l - 1) * M) + j] << 32) | p)
                 : ~0ull;
}

template <bool Signed>
void* hnsw_insert_for(int ch) {
    switch (ch) {
        case 1: return (void*)hnsw_insert_kernel<1, Signed>;
        case 2: return (void*)hnsw_insert_kernel<2, Signed>;
        case 3: return (void*)hnsw_insert_kernel<3, Signed>;
        case 4: return (void*)hnsw_insert_kernel<4, Signed>;
        default: return (void*)hnsw_insert_kernel<8, Signed>;
    }
}

// device buffers of one build, freed on every exit path
struct BuildBuffers {
    std::vector<void*> ptrs;
    ~BuildBuffers() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    pgb_status alloc(T** p, size_t count, const char* what) {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? PGB_ERR_OOM : PGB_ERR_CUDA,
                        std::string("GPU build: ") + what + ": " + cudaGetErrorString(e));
        }
        ptrs.push_back(*p);
        return PGB_OK;
    }
};

pgb_status ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PGB_OK;
    cudaGetLastError();
    return fail(PGB_ERR_CUDA, std::string("GPU build: ") + what + ": " + cudaGetErrorString(e));
}

// Reverse edges of one batch (and level): radix sort of the (q, p) keys, runs of equal q,
// their offsets, then the merge kernel, with a second launch for hub targets.
struct ReverseMerger {
    uint64_t* keys_out = nullptr;
    uint32_t *tq = nullptr, *run_q = nullptr, *run_cnt = nullptr, *run_off = nullptr;
    uint32_t *n_runs = nullptr, *big = nullptr, *n_big = nullptr, *queue = nullptr;
    uint32_t* gid = nullptr;
    int32_t* gdist = nullptr;
    uint64_t* gkey = nullptr;
    uint32_t* hgid = nullptr;
    int32_t* hgdist = nullptr;
    uint64_t* hgkey = nullptr;
    void* cub_tmp = nullptr;
    size_t t_cub = 0;
    void* kernel = nullptr;
    BuildLayout BM{};
    int wpb = 4, blocks = 1;
    uint32_t wcap = 0, hub_cap = 0, hub_warps = 0;
    BuildBuffers* bb = nullptr;

    pgb_status init(BuildBuffers& b, size_t max_pairs, void* kern, const BuildLayout& layout, int wpbm,
                    int blocksm, uint32_t warp_cap, uint32_t hubcap, uint32_t hubwarps, uint32_t* q) {
        bb = &b;
        kernel = kern;
        BM = layout;
        wpb = wpbm;
        blocks = blocksm;
        wcap = warp_cap;
        hub_cap = hubcap;
        hub_warps = hubwarps;
        queue = q;
        const size_t warps = (size_t)wpb * blocks;
        pgb_status s;
        if ((s = b.alloc(&keys_out, max_pairs, "pair keys")) != PGB_OK ||
            (s = b.alloc(&tq, max_pairs, "targets")) != PGB_OK ||
            (s = b.alloc(&run_q, max_pairs, "runs")) != PGB_OK ||
            (s = b.alloc(&run_cnt, max_pairs, "runs")) != PGB_OK ||
            (s = b.alloc(&run_off, max_pairs, "runs")) != PGB_OK ||
            (s = b.alloc(&n_runs, 1, "runs")) != PGB_OK ||
            (s = b.alloc(&big, max_pairs, "hub groups")) != PGB_OK ||
            (s = b.alloc(&n_big, 1, "hub groups")) != PGB_OK ||
            (s = b.alloc(&gid, warps * wcap, "merge scratch")) != PGB_OK ||
            (s = b.alloc(&gdist, warps * wcap, "merge scratch")) != PGB_OK ||
            (s = b.alloc(&gkey, warps * 2 * wcap, "merge scratch")) != PGB_OK)
            return s;
        size_t t_sort = 0, t_rle = 0, t_scan = 0;
        if ((s = ck(cub::DeviceRadixSort::SortKeys(nullptr, t_sort, keys_out, keys_out, (int)max_pairs), "sort size")) != PGB_OK ||
            (s = ck(cub::DeviceRunLengthEncode::Encode(nullptr, t_rle, tq, run_q, run_cnt, n_runs, (int)max_pairs), "rle size")) != PGB_OK ||
            (s = ck(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, run_cnt, run_off, (int)max_pairs), "scan size")) != PGB_OK)
            return s;
        t_cub = std::max(t_sort, std::max(t_rle, t_scan));
        return b.alloc(reinterpret_cast<uint8_t**>(&cub_tmp), t_cub, "sort scratch");
    }

    // merges the nt keys in keys_in (unused slots ~0) into the rows of G (at most cap each)
    pgb_status run(const uint64_t* keys_in, uint64_t nt, const LevelRows& G, uint32_t cap,
                   const uint8_t* rows, uint32_t dim, float alpha, cudaStream_t st) {
        pgb_status s;
        const unsigned tb = 256, gb = (unsigned)((nt + tb - 1) / tb);
        size_t tmp = t_cub;
        if ((s = ck(cub::DeviceRadixSort::SortKeys(cub_tmp, tmp, keys_in, keys_out, (int)nt, 0, 64, st), "sort")) != PGB_OK)
            return s;
        key_targets_kernel<<<gb, tb, 0, st>>>(keys_out, (uint32_t)nt, tq);
        tmp = t_cub;
        if ((s = ck(cub::DeviceRunLengthEncode::Encode(cub_tmp, tmp, tq, run_q, run_cnt, n_runs, (int)nt, st), "rle")) != PGB_OK)
            return s;
        tmp = t_cub;
        if ((s = ck(cub::DeviceScan::ExclusiveSum(cub_tmp, tmp, run_cnt, run_off, (int)nt, st), "scan")) != PGB_OK)
            return s;
        MergeArgs M{};
        M.rows = rows;
        M.G = G;
        M.dim = dim;
        M.cap = cap;
        M.alpha = alpha;
        M.keys = keys_out;
        M.run_q = run_q;
        M.run_cnt = run_cnt;
        M.run_off = run_off;
        M.n_runs = n_runs;
        M.groups = nullptr;
        M.n_groups = 0;
        M.gid = gid;
        M.gdist = gdist;
        M.gkey = gkey;
        M.wcap = wcap;
        M.big = big;
        M.n_big = n_big;
        M.B = BM;
        M.queue = queue;
        if ((s = ck(cudaMemsetAsync(queue, 0, 4, st), "counter")) != PGB_OK ||
            (s = ck(cudaMemsetAsync(n_big, 0, 4, st), "counter")) != PGB_OK)
            return s;
        {
            void* args[] = {&M};
            if ((s = ck(cudaLaunchKernel(kernel, dim3(blocks), dim3(wpb * 32), args, (size_t)wpb * BM.bytes, st),
                        "merge launch")) != PGB_OK)
                return s;
        }
        uint32_t nbig = 0;
        if ((s = ck(cudaMemcpy(&nbig, n_big, 4, cudaMemcpyDeviceToHost), "hub count")) != PGB_OK) return s;
        if (nbig == 0) return PGB_OK;
        if (!hgid && ((s = bb->alloc(&hgid, (size_t)hub_warps * hub_cap, "hub scratch")) != PGB_OK ||
                      (s = bb->alloc(&hgdist, (size_t)hub_warps * hub_cap, "hub scratch")) != PGB_OK ||
                      (s = bb->alloc(&hgkey, (size_t)hub_warps * 2 * hub_cap, "hub scratch")) != PGB_OK))
            return s;
        MergeArgs H = M;
        H.groups = big;
        H.n_groups = nbig;
        H.gid = hgid;
        H.gdist = hgdist;
        H.gkey = hgkey;
        H.wcap = hub_cap;  // every new source of a batch fits: no further deferral
        if ((s = ck(cudaMemsetAsync(queue, 0, 4, st), "counter")) != PGB_OK) return s;
        void* args[] = {&H};
        return ck(cudaLaunchKernel(kernel, dim3(std::min(nbig, hub_warps)), dim3(32), args, BM.bytes, st),
                  "hub merge launch");
    }
};

// tables of a first search (seen set, candidate list) sized from L and R, and the merge
// scratch per warp (q's row plus up to 2,048 new sources); a test hook
// (PGB_BUILD_SMALL_TABLES=1) starts from the smallest sizes to exercise the retried
// searches and the hub merges
void first_caps(uint32_t L, uint32_t R, uint32_t& seen_cap, uint32_t& cand_cap, uint32_t& wcap) {
    const char* small = std::getenv("PGB_BUILD_SMALL_TABLES");
    if (small && small[0] == '1') {
        seen_cap = 256;
        cand_cap = R + 8u;
        wcap = R + 8u;
        return;
    }
    seen_cap = next_pow2_u32(std::max<uint32_t>(4096u, 4u * L * R));
    cand_cap = 4u * L + 2u * R;
    wcap = R + 2048u;
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" pgb_status pgb_build_vamana_gpu(int device, const void* vectors, uint32_t n,
                                           uint32_t dim, pgb_elem elem, uint32_t R, uint32_t L,
                                           float alpha, int passes, uint64_t seed,
                                           uint32_t* degrees, uint32_t* adjacency) {
    if (!vectors || !degrees || !adjacency) return fail(PGB_ERR_BAD_ARG, "vamana (GPU): null argument");
    if (n == 0 || dim == 0 || dim > PGB_MAX_DIM) return fail(PGB_ERR_BAD_ARG, "vamana (GPU): n == 0 or dim outside 1..128");
    if (elem != PGB_INT8 && elem != PGB_UINT8) return fail(PGB_ERR_BAD_ARG, "vamana (GPU): element type");
    if (R == 0 || R > PGB_MAX_DEGREE || L == 0 || L > PGB_MAX_BEAM || passes < 1 || !(alpha > 0))
        return fail(PGB_ERR_BAD_ARG, "vamana (GPU): bad R / L / alpha / passes");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    std::fill(degrees, degrees + n, 0u);
    std::fill(adjacency, adjacency + (size_t)n * R, kNoNeighbor);
    if (n <= 1) return PGB_OK;
    const bool sgn = elem == PGB_INT8;
    const int ch = flat_chunks_for(R);
    const uint32_t gs = 32u * (uint32_t)ch;
    const std::vector<uint32_t> order = vamana_insertion_order(n, seed);
    const size_t max_batch = vamana_max_batch(n);
    const size_t max_pairs = max_batch * R;

    cudaDeviceProp prop;
    pgb_status s;
    if ((s = ck(cudaGetDeviceProperties(&prop, device), "device properties")) != PGB_OK) return s;
    BuildBuffers bb;
    uint8_t* rows;
    uint32_t *adj, *deg, *d_order, *out, *out_n, *flagged, *n_flagged, *queue;
    if ((s = bb.alloc(&rows, (size_t)n * kRowBytes, "rows")) != PGB_OK ||
        (s = bb.alloc(&adj, (size_t)n * R, "adjacency")) != PGB_OK ||
        (s = bb.alloc(&deg, n, "degrees")) != PGB_OK ||
        (s = bb.alloc(&d_order, n, "insertion order")) != PGB_OK ||
        (s = bb.alloc(&out, max_pairs, "batch rows")) != PGB_OK ||
        (s = bb.alloc(&out_n, max_batch, "batch degrees")) != PGB_OK ||
        (s = bb.alloc(&flagged, max_batch, "flags")) != PGB_OK ||
        (s = bb.alloc(&n_flagged, 1, "flags")) != PGB_OK ||
        (s = bb.alloc(&queue, 1, "work counter")) != PGB_OK)
        return s;
    if ((s = ck(cudaMemset(rows, 0, (size_t)n * kRowBytes), "rows")) != PGB_OK ||
        (s = ck(cudaMemcpy2D(rows, kRowBytes, vectors, dim, dim, n, cudaMemcpyHostToDevice), "rows")) != PGB_OK ||
        (s = ck(cudaMemset(adj, 0xFF, (size_t)n * R * 4), "adjacency")) != PGB_OK ||
        (s = ck(cudaMemset(deg, 0, (size_t)n * 4), "degrees")) != PGB_OK ||
        (s = ck(cudaMemcpy(d_order, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice), "order")) != PGB_OK)
        return s;

    // search + prune launch shape: persistent grid, 4 warps per block
    uint32_t seen_cap, cand_cap, wcap;
    first_caps(L, R, seen_cap, cand_cap, wcap);
    void* sp_kernel = sgn ? search_prune_for<true>(ch) : search_prune_for<false>(ch);
    void* mg_kernel = sgn ? merge_for<true, false>(ch) : merge_for<false, false>(ch);
    const size_t smem_cap = prop.sharedMemPerBlockOptin;
    for (void* k : {sp_kernel, mg_kernel})
        if ((s = ck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap),
                    "kernel attribute")) != PGB_OK)
            return s;
    auto shape = [&](void* kern, const BuildLayout& Bl, int& wpb, int& blocks) -> pgb_status {
        wpb = 4;
        while (wpb > 1 && (size_t)wpb * Bl.bytes > smem_cap) wpb >>= 1;
        if ((size_t)wpb * Bl.bytes > smem_cap) return fail(PGB_ERR_BAD_ARG, "vamana (GPU): L or R too large for shared memory");
        int bps = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, wpb * 32, (size_t)wpb * Bl.bytes) != cudaSuccess || bps < 1)
            return fail(PGB_ERR_CUDA, "vamana (GPU): kernel does not fit");
        blocks = bps * prop.multiProcessorCount;
        return PGB_OK;
    };
    BuildLayout B1 = make_build_layout(L, gs, seen_cap, R);
    int wpb1 = 4, blocks1 = 1;
    if ((s = shape(sp_kernel, B1, wpb1, blocks1)) != PGB_OK) return s;
    const size_t warps1 = (size_t)wpb1 * blocks1;
    uint32_t* seen_tab;
    uint64_t* cand;
    if ((s = bb.alloc(&seen_tab, warps1 * seen_cap, "seen tables")) != PGB_OK ||
        (s = bb.alloc(&cand, warps1 * 2 * cand_cap, "candidate lists")) != PGB_OK)
        return s;

    // reverse-edge merge: per-warp scratch of wcap candidates; a target with more (a hub)
    // is merged again by one warp per SM whose scratch holds a whole batch
    uint64_t* keys_in;
    if ((s = bb.alloc(&keys_in, max_pairs, "pair keys")) != PGB_OK) return s;
    BuildLayout BM = make_build_layout(L, gs, 0u, R);
    int wpbm = 4, blocksm = 1;
    if ((s = shape(mg_kernel, BM, wpbm, blocksm)) != PGB_OK) return s;
    ReverseMerger rm;
    if ((s = rm.init(bb, max_pairs, mg_kernel, BM, wpbm, blocksm, wcap, R + (uint32_t)max_batch,
                     (uint32_t)prop.multiProcessorCount, queue)) != PGB_OK)
        return s;

    cudaStream_t st = 0;
    for (int pass = 0; pass < passes; pass++) {
        const float a = (passes > 1 && pass == 0) ? 1.0f : alpha;
        size_t pos = (pass == 0) ? 1 : 0;
        size_t batch = 1;
        while (pos < n) {
            const size_t end = std::min<size_t>(n, pos + batch);
            const uint32_t nb = (uint32_t)(end - pos);
            const uint32_t* pts = d_order + pos;
            // search + prune, then again with larger tables for the points that outgrew them
            SearchPruneArgs A{};
            A.rows = rows;
            A.adj = adj;
            A.deg = deg;
            A.n = n;
            A.dim = dim;
            A.R = R;
            A.L = L;
            A.alpha = a;
            A.points = pts;
            A.slots = nullptr;
            A.np = nb;
            A.out = out;
            A.out_n = out_n;
            A.seen_tab = seen_tab;
            A.cand = cand;
            A.cand_cap = cand_cap;
            A.B = B1;
            A.flagged = flagged;
            A.n_flagged = n_flagged;
            A.queue = queue;
            if ((s = ck(cudaMemsetAsync(queue, 0, 4, st), "counter")) != PGB_OK ||
                (s = ck(cudaMemsetAsync(n_flagged, 0, 4, st), "counter")) != PGB_OK)
                return s;
            {
                void* args[] = {&A};
                const int blocks = (int)std::min<size_t>(blocks1, (nb + wpb1 - 1) / wpb1);
                if ((s = ck(cudaLaunchKernel(sp_kernel, dim3(blocks), dim3(wpb1 * 32), args,
                                             (size_t)wpb1 * B1.bytes, st), "search launch")) != PGB_OK)
                    return s;
            }
            uint32_t nf = 0;
            if ((s = ck(cudaMemcpy(&nf, n_flagged, 4, cudaMemcpyDeviceToHost), "flag count")) != PGB_OK) return s;
            uint32_t rseen = seen_cap, rcand = cand_cap;
            while (nf > 0) {
                // the flagged points again, one warp per block, tables four times larger
                rseen *= 4u;
                rcand *= 4u;
                BuildLayout BR = make_build_layout(L, gs, rseen, R);
                if (BR.bytes > smem_cap)
                    return fail(PGB_ERR_BAD_ARG, "vamana (GPU): seen set beyond shared-memory bitmap limit");
                std::vector<uint32_t> fl(nf), fpts(nf);
                if ((s = ck(cudaMemcpy(fl.data(), flagged, 4ull * nf, cudaMemcpyDeviceToHost), "flags")) != PGB_OK)
                    return s;
                for (uint32_t i = 0; i < nf; i++) fpts[i] = order[pos + fl[i]];
                BuildBuffers rb;
                uint32_t *r_pts, *r_slots, *r_seen;
                uint64_t* r_cand;
                const uint32_t rw = std::min<uint32_t>(nf, (uint32_t)prop.multiProcessorCount);
                if ((s = rb.alloc(&r_pts, nf, "retry")) != PGB_OK || (s = rb.alloc(&r_slots, nf, "retry")) != PGB_OK ||
                    (s = rb.alloc(&r_seen, (size_t)rw * rseen, "retry")) != PGB_OK ||
                    (s = rb.alloc(&r_cand, (size_t)rw * 2 * rcand, "retry")) != PGB_OK)
                    return s;
                if ((s = ck(cudaMemcpy(r_pts, fpts.data(), 4ull * nf, cudaMemcpyHostToDevice), "retry")) != PGB_OK ||
                    (s = ck(cudaMemcpy(r_slots, fl.data(), 4ull * nf, cudaMemcpyHostToDevice), "retry")) != PGB_OK ||
                    (s = ck(cudaMemset(queue, 0, 4), "counter")) != PGB_OK ||
                    (s = ck(cudaMemset(n_flagged, 0, 4), "counter")) != PGB_OK)
                    return s;
                SearchPruneArgs RA = A;
                RA.points = r_pts;
                RA.slots = r_slots;
                RA.np = nf;
                RA.seen_tab = r_seen;
                RA.cand = r_cand;
                RA.cand_cap = rcand;
                RA.B = BR;
                void* args[] = {&RA};
                if ((s = ck(cudaLaunchKernel(sp_kernel, dim3(rw), dim3(32), args, BR.bytes, st), "retry launch")) != PGB_OK ||
                    (s = ck(cudaMemcpy(&nf, n_flagged, 4, cudaMemcpyDeviceToHost), "flag count")) != PGB_OK)
                    return s;
            }
            // new rows, then the reverse edges
            const uint64_t nt = (uint64_t)nb * R;
            const unsigned tb = 256, gb = (unsigned)((nt + tb - 1) / tb);
            write_rows_kernel<<<gb, tb, 0, st>>>(pts, nb, out, out_n, R, adj, deg);
            pair_keys_kernel<<<gb, tb, 0, st>>>(pts, nb, out, out_n, R, keys_in);
            if ((s = ck(cudaGetLastError(), "row kernels")) != PGB_OK) return s;
            if ((s = rm.run(keys_in, nt, LevelRows{adj, deg, nullptr, R, 0u}, R, rows, dim, a, st)) != PGB_OK)
                return s;
            pos = end;
            batch = std::min(batch * 2, max_batch);
        }
    }
    if ((s = ck(cudaMemcpy(degrees, deg, (size_t)n * 4, cudaMemcpyDeviceToHost), "degrees download")) != PGB_OK ||
        (s = ck(cudaMemcpy(adjacency, adj, (size_t)n * R * 4, cudaMemcpyDeviceToHost), "adjacency download")) != PGB_OK)
        return s;
    return PGB_OK;
}

extern "C" pgb_status pgb_build_hnsw_gpu(int device, const void* vectors, uint32_t n, uint32_t dim,
                                         pgb_elem elem, uint32_t M, uint32_t ef_construction,
                                         float ml, float alpha, uint64_t seed, const char* path) {
    if (!vectors || !path) return fail(PGB_ERR_BAD_ARG, "hnsw (GPU): null argument");
    if (n == 0 || dim == 0 || dim > PGB_MAX_DIM) return fail(PGB_ERR_BAD_ARG, "hnsw (GPU): n == 0 or dim outside 1..128");
    if (elem != PGB_INT8 && elem != PGB_UINT8) return fail(PGB_ERR_BAD_ARG, "hnsw (GPU): element type");
    if (M == 0 || 2 * M > PGB_MAX_DEGREE || ef_construction == 0 || ef_construction > PGB_MAX_BEAM || !(ml > 0))
        return fail(PGB_ERR_BAD_ARG, "hnsw (GPU): bad M / ef_construction / ml");
    DeviceGuard guard(device);
    if (!guard.ok) return fail(PGB_ERR_CUDA, "cudaSetDevice failed");
    const bool sgn = elem == PGB_INT8;
    const uint32_t cap0 = 2 * M;
    const int ch = flat_chunks_for(cap0);
    const uint32_t gs = 32u * (uint32_t)ch;
    const std::vector<uint32_t> level = hnsw_levels(n, ml, seed);
    const std::vector<uint32_t> order = hnsw_insertion_order(n, seed);
    std::vector<uint32_t> ustart(n);
    uint64_t n_up = 0;
    uint32_t max_level = 0;
    for (uint32_t i = 0; i < n; i++) {
        ustart[i] = (uint32_t)n_up;
        n_up += level[i];
        max_level = std::max(max_level, level[i]);
    }
    if (n_up >= 0xFFFFFFFFull) return fail(PGB_ERR_BAD_ARG, "hnsw (GPU): too many upper-level rows");
    const size_t max_batch = vamana_max_batch(n);

    cudaDeviceProp prop;
    pgb_status s;
    if ((s = ck(cudaGetDeviceProperties(&prop, device), "device properties")) != PGB_OK) return s;
    BuildBuffers bb;
    uint8_t* rows;
    uint32_t *adj0, *size0, *adju, *sizeu, *d_ustart, *d_level, *d_order;
    if ((s = bb.alloc(&rows, (size_t)n * kRowBytes, "rows")) != PGB_OK ||
        (s = bb.alloc(&adj0, (size_t)n * cap0, "level-0 rows")) != PGB_OK ||
        (s = bb.alloc(&size0, n, "level-0 sizes")) != PGB_OK ||
        (s = bb.alloc(&adju, (size_t)std::max<uint64_t>(n_up, 1) * M, "upper rows")) != PGB_OK ||
        (s = bb.alloc(&sizeu, (size_t)std::max<uint64_t>(n_up, 1), "upper sizes")) != PGB_OK ||
        (s = bb.alloc(&d_ustart, n, "upper starts")) != PGB_OK ||
        (s = bb.alloc(&d_level, n, "levels")) != PGB_OK ||
        (s = bb.alloc(&d_order, n, "insertion order")) != PGB_OK)
        return s;
    if ((s = ck(cudaMemset(rows, 0, (size_t)n * kRowBytes), "rows")) != PGB_OK ||
        (s = ck(cudaMemcpy2D(rows, kRowBytes, vectors, dim, dim, n, cudaMemcpyHostToDevice), "rows")) != PGB_OK ||
        (s = ck(cudaMemset(adj0, 0xFF, (size_t)n * cap0 * 4), "rows")) != PGB_OK ||
        (s = ck(cudaMemset(size0, 0, (size_t)n * 4), "sizes")) != PGB_OK ||
        (s = ck(cudaMemset(adju, 0xFF, (size_t)std::max<uint64_t>(n_up, 1) * M * 4), "rows")) != PGB_OK ||
        (s = ck(cudaMemset(sizeu, 0, (size_t)std::max<uint64_t>(n_up, 1) * 4), "sizes")) != PGB_OK ||
        (s = ck(cudaMemcpy(d_ustart, ustart.data(), (size_t)n * 4, cudaMemcpyHostToDevice), "starts")) != PGB_OK ||
        (s = ck(cudaMemcpy(d_level, level.data(), (size_t)n * 4, cudaMemcpyHostToDevice), "levels")) != PGB_OK ||
        (s = ck(cudaMemcpy(d_order, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice), "order")) != PGB_OK)
        return s;
    const LevelRows L0{adj0, size0, nullptr, cap0, 0u};

    // per batch: selected rows (level 0 then M per upper level), their counts, offsets
    const size_t out_cap = max_batch * ((size_t)cap0 + (size_t)max_level * M);
    const size_t outn_cap = max_batch * ((size_t)max_level + 1);
    const size_t max_pairs = max_batch * cap0;
    uint32_t *out, *out_n, *outn_off, *flagged, *n_flagged, *queue;
    uint64_t *out_off, *keys_in;
    if ((s = bb.alloc(&out, out_cap, "batch rows")) != PGB_OK ||
        (s = bb.alloc(&out_n, outn_cap, "batch counts")) != PGB_OK ||
        (s = bb.alloc(&out_off, max_batch, "batch offsets")) != PGB_OK ||
        (s = bb.alloc(&outn_off, max_batch, "batch offsets")) != PGB_OK ||
        (s = bb.alloc(&flagged, max_batch, "flags")) != PGB_OK ||
        (s = bb.alloc(&n_flagged, 1, "flags")) != PGB_OK ||
        (s = bb.alloc(&queue, 1, "work counter")) != PGB_OK ||
        (s = bb.alloc(&keys_in, max_pairs, "pair keys")) != PGB_OK)
        return s;

    uint32_t seen_cap, cand_cap, wcap;
    first_caps(ef_construction, cap0, seen_cap, cand_cap, wcap);
    void* ins_kernel = sgn ? hnsw_insert_for<true>(ch) : hnsw_insert_for<false>(ch);
    void* mg_kernel = sgn ? merge_for<true, true>(ch) : merge_for<false, true>(ch);
    const size_t smem_cap = prop.sharedMemPerBlockOptin;
    for (void* k : {ins_kernel, mg_kernel})
        if ((s = ck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap),
                    "kernel attribute")) != PGB_OK)
            return s;
    auto shape = [&](void* kern, const BuildLayout& Bl, int& wpb, int& blocks) -> pgb_status {
        wpb = 4;
        while (wpb > 1 && (size_t)wpb * Bl.bytes > smem_cap) wpb >>= 1;
        if ((size_t)wpb * Bl.bytes > smem_cap) return fail(PGB_ERR_BAD_ARG, "hnsw (GPU): ef_construction or M too large for shared memory");
        int bps = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, wpb * 32, (size_t)wpb * Bl.bytes) != cudaSuccess || bps < 1)
            return fail(PGB_ERR_CUDA, "hnsw (GPU): kernel does not fit");
        blocks = bps * prop.multiProcessorCount;
        return PGB_OK;
    };
    const BuildLayout B1 = make_build_layout(ef_construction, gs, seen_cap, cap0);
    int wpb1 = 4, blocks1 = 1;
    if ((s = shape(ins_kernel, B1, wpb1, blocks1)) != PGB_OK) return s;
    uint32_t* seen_tab;
    if ((s = bb.alloc(&seen_tab, (size_t)wpb1 * blocks1 * seen_cap, "seen tables")) != PGB_OK) return s;
    const BuildLayout BM = make_build_layout(8u, gs, 0u, cap0);
    int wpbm = 4, blocksm = 1;
    if ((s = shape(mg_kernel, BM, wpbm, blocksm)) != PGB_OK) return s;
    ReverseMerger rm;
    if ((s = rm.init(bb, max_pairs, mg_kernel, BM, wpbm, blocksm, wcap, cap0 + (uint32_t)max_batch,
                     (uint32_t)prop.multiProcessorCount, queue)) != PGB_OK)
        return s;

    cudaStream_t st = 0;
    uint32_t entry = order[0], top = level[entry];
    size_t pos = 1, batch = 1;
    std::vector<uint64_t> h_out_off(max_batch);
    std::vector<uint32_t> h_outn_off(max_batch);
    while (pos < n) {
        const size_t end = std::min<size_t>(n, pos + batch);
        const uint32_t nb = (uint32_t)(end - pos);
        const uint32_t* pts = d_order + pos;
        uint64_t o = 0;
        uint32_t on = 0, batch_top = 0;
        for (uint32_t b = 0; b < nb; b++) {
            const uint32_t lv = level[order[pos + b]];
            h_out_off[b] = o;
            h_outn_off[b] = on;
            o += cap0 + (uint64_t)lv * M;
            on += lv + 1;
            batch_top = std::max(batch_top, lv);
        }
        if ((s = ck(cudaMemcpy(out_off, h_out_off.data(), 8ull * nb, cudaMemcpyHostToDevice), "offsets")) != PGB_OK ||
            (s = ck(cudaMemcpy(outn_off, h_outn_off.data(), 4ull * nb, cudaMemcpyHostToDevice), "offsets")) != PGB_OK)
            return s;
        HnswInsertArgs A{};
        A.rows = rows;
        A.n = n;
        A.dim = dim;
        A.M = M;
        A.efc = ef_construction;
        A.alpha = alpha;
        A.L0 = L0;
        A.adju = adju;
        A.sizeu = sizeu;
        A.ustart = d_ustart;
        A.level = d_level;
        A.entry = entry;
        A.top = top;
        A.points = pts;
        A.slots = nullptr;
        A.np = nb;
        A.out = out;
        A.out_off = out_off;
        A.out_n = out_n;
        A.outn_off = outn_off;
        A.seen_tab = seen_tab;
        A.B = B1;
        A.flagged = flagged;
        A.n_flagged = n_flagged;
        A.queue = queue;
        if ((s = ck(cudaMemsetAsync(queue, 0, 4, st), "counter")) != PGB_OK ||
            (s = ck(cudaMemsetAsync(n_flagged, 0, 4, st), "counter")) != PGB_OK)
            return s;
        {
            void* args[] = {&A};
            const int blocks = (int)std::min<size_t>(blocks1, (nb + wpb1 - 1) / wpb1);
            if ((s = ck(cudaLaunchKernel(ins_kernel, dim3(blocks), dim3(wpb1 * 32), args, (size_t)wpb1 * B1.bytes, st),
                        "insert launch")) != PGB_OK)
                return s;
        }
        uint32_t nf = 0;
        if ((s = ck(cudaMemcpy(&nf, n_flagged, 4, cudaMemcpyDeviceToHost), "flag count")) != PGB_OK) return s;
        uint32_t rseen = seen_cap;
        while (nf > 0) {
            // the flagged points again, one warp per block, a seen set four times larger
            rseen *= 4u;
            const BuildLayout BR = make_build_layout(ef_construction, gs, rseen, cap0);
            if (BR.bytes > smem_cap) return fail(PGB_ERR_BAD_ARG, "hnsw (GPU): seen set beyond shared-memory bitmap limit");
            std::vector<uint32_t> fl(nf), fpts(nf);
            if ((s = ck(cudaMemcpy(fl.data(), flagged, 4ull * nf, cudaMemcpyDeviceToHost), "flags")) != PGB_OK) return s;
            for (uint32_t i = 0; i < nf; i++) fpts[i] = order[pos + fl[i]];
            BuildBuffers rb;
            uint32_t *r_pts, *r_slots, *r_seen;
            const uint32_t rw = std::min<uint32_t>(nf, (uint32_t)prop.multiProcessorCount);
            if ((s = rb.alloc(&r_pts, nf, "retry")) != PGB_OK || (s = rb.alloc(&r_slots, nf, "retry")) != PGB_OK ||
                (s = rb.alloc(&r_seen, (size_t)rw * rseen, "retry")) != PGB_OK)
                return s;
            if ((s = ck(cudaMemcpy(r_pts, fpts.data(), 4ull * nf, cudaMemcpyHostToDevice), "retry")) != PGB_OK ||
                (s = ck(cudaMemcpy(r_slots, fl.data(), 4ull * nf, cudaMemcpyHostToDevice), "retry")) != PGB_OK ||
                (s = ck(cudaMemset(queue, 0, 4), "counter")) != PGB_OK ||
                (s = ck(cudaMemset(n_flagged, 0, 4), "counter")) != PGB_OK)
                return s;
            HnswInsertArgs RA = A;
            RA.points = r_pts;
            RA.slots = r_slots;
            RA.np = nf;
            RA.seen_tab = r_seen;
            RA.B = BR;
            void* args[] = {&RA};
            if ((s = ck(cudaLaunchKernel(ins_kernel, dim3(rw), dim3(32), args, BR.bytes, st), "retry launch")) != PGB_OK ||
                (s = ck(cudaMemcpy(&nf, n_flagged, 4, cudaMemcpyDeviceToHost), "flag count")) != PGB_OK)
                return s;
        }
        // new rows at every level, then each level's reverse edges
        hnsw_write_rows_kernel<<<(nb + 3) / 4, 128, 0, st>>>(pts, nb, d_level, out, out_off, out_n, outn_off, M,
                                                             L0, adju, sizeu, d_ustart);
        if ((s = ck(cudaGetLastError(), "row kernel")) != PGB_OK) return s;
        for (uint32_t l = 0; l <= std::min(batch_top, top); l++) {
            const uint32_t capl = l == 0 ? cap0 : M;
            const uint64_t nt = (uint64_t)nb * capl;
            const unsigned tb = 256, gb = (unsigned)((nt + tb - 1) / tb);
            hnsw_pair_keys_kernel<<<gb, tb, 0, st>>>(pts, nb, d_level, out, out_off, out_n, outn_off, M, l, capl,
                                                     keys_in);
            if ((s = ck(cudaGetLastError(), "pair keys")) != PGB_OK) return s;
            const LevelRows G = l == 0 ? L0 : LevelRows{adju, sizeu, d_ustart, M, l - 1};
            if ((s = rm.run(keys_in, nt, G, capl, rows, dim, alpha, st)) != PGB_OK) return s;
        }
        for (size_t b = pos; b < end; b++)
            if (level[order[b]] > top) {
                top = level[order[b]];
                entry = order[b];
            }
        pos = end;
        batch = std::min(batch * 2, max_batch);
    }

    // the CPU builder's file: rows of every (node, level), node-major
    std::vector<uint32_t> h_adj0((size_t)n * cap0), h_size0(n), h_adju((size_t)n_up * M), h_sizeu(n_up);
    if ((s = ck(cudaMemcpy(h_adj0.data(), adj0, h_adj0.size() * 4, cudaMemcpyDeviceToHost), "rows download")) != PGB_OK ||
        (s = ck(cudaMemcpy(h_size0.data(), size0, (size_t)n * 4, cudaMemcpyDeviceToHost), "sizes download")) != PGB_OK ||
        (n_up && (s = ck(cudaMemcpy(h_adju.data(), adju, h_adju.size() * 4, cudaMemcpyDeviceToHost), "rows download")) != PGB_OK) ||
        (n_up && (s = ck(cudaMemcpy(h_sizeu.data(), sizeu, (size_t)n_up * 4, cudaMemcpyDeviceToHost), "sizes download")) != PGB_OK))
        return s;
    HnswFile h;
    h.n = n;
    h.dim = dim;
    h.m = M;
    h.efc = ef_construction;
    h.ml = ml;
    h.alpha = alpha;
    h.levels = level;
    h.node_point.resize(n);
    for (uint32_t i = 0; i < n; i++) h.node_point[i] = i;
    for (uint32_t i = 0; i < n; i++) {
        h.list_sizes.push_back(h_size0[i]);
        h.ids.insert(h.ids.end(), h_adj0.begin() + (size_t)i * cap0, h_adj0.begin() + (size_t)i * cap0 + h_size0[i]);
        for (uint32_t l = 1; l <= level[i]; l++) {
            const size_t ri = (size_t)ustart[i] + l - 1;
            h.list_sizes.push_back(h_sizeu[ri]);
            h.ids.insert(h.ids.end(), h_adju.begin() + ri * M, h_adju.begin() + ri * M + h_sizeu[ri]);
        }
    }
    h.entries = {entry};
    const std::string e = write_hnsw(path, h);
    if (!e.empty()) return fail(PGB_ERR_IO, e);
    return PGB_OK;
}
