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

// RobustPrune of the sorted candidate keys (dist to `self`, id): drops repeats of an id
// and `self`, keeps c unless a kept o has alpha * d(o, c) <= d(self, c) (the CPU's float
// comparison), stops at R kept. Kept rows are staged in shared memory. Returns the count;
// out_ids[0, count) in shared memory.
template <bool Signed>
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
            if (__fmul_rn(alpha, (float)d) <= (float)cd) dominated = true;
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
    uint64_t* const fbuf1 = reinterpret_cast<uint64_t*>(wm + B.off_f1);
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
    const uint32_t lt = lanemask_lt();
    const int L = (int)A.L, R = (int)A.R;
    const uint32_t* rows32 = reinterpret_cast<const uint32_t*>(A.rows);

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
        int fsize = 1, nvis = 0, nseen = 1;
        bool over = false;
        for (;;) {
            // the frontier and its expanded flags alternate between two buffers
            uint64_t* F = cur ? fbuf1 : fbuf0;
            uint8_t* V = wm + (cur ? B.off_v1 : B.off_v0);
            // first unexpanded entry
            int u = -1;
            for (int base = 0; base < fsize; base += 32) {
                const int i = base + lane;
                const uint32_t m = __ballot_sync(kFull, i < fsize && !V[i]);
                if (m) {
                    u = base + __ffs(m) - 1;
                    break;
                }
            }
            if (u < 0) break;
            if (nvis + R + 1 > (int)A.cand_cap) {
                over = true;
                break;
            }
            const uint64_t ukey = F[u];
            if (lane == 0) {
                V[u] = 1;
                cand[nvis] = ukey;
            }
            nvis++;
            const uint32_t uid = key_id(ukey);
            const uint32_t du = A.deg[uid];
            const uint32_t* row = A.adj + (size_t)uid * A.R;
            // unseen neighbours, in row order
            int np = 0;
#pragma unroll
            for (int t = 0; t < CH; t++) {
                const uint32_t j = (uint32_t)(t * 32 + lane);
                const uint32_t x = j < du ? __ldg(row + j) : kEmptyId;
                const bool valid = x != kEmptyId;
                const uint32_t peers = __match_any_sync(kFull, valid ? x : (0x80000000u | j));
                const bool first = valid && (peers & lt) == 0;
                const bool fresh = first && !seen_contains(tab, occ, mask, shift, x);
                __syncwarp();
                if (fresh) seen_insert(tab, occ, mask, shift, x);
                const uint32_t m = __ballot_sync(kFull, fresh);
                if (fresh) pend[np + __popc(m & lt)] = x;
                np += __popc(m);
                __syncwarp();
            }
            nseen += np;
            if (nseen > (int)(B.seen_cap / 2u)) {
                over = true;
                break;
            }
            row_distances<Signed>(A.rows, pend, pdist, np, q4, qq, A.dim, false, lane);
            // acceptance: fewer than L of (list + earlier new neighbours) at distance <= d
            int na = 0;
            for (int base = 0; base < np; base += 32) {
                const int j = base + lane;
                bool acc = false;
                int32_t d = 0;
                if (j < np) {
                    d = pdist[j];
                    int c = upper_bound_key(F, fsize, pack_key(d, 0xFFFFFFFFu));
                    for (int i = 0; i < j && c < L; i++) c += pdist[i] <= d ? 1 : 0;
                    acc = c < L;
                }
                const uint32_t m = __ballot_sync(kFull, acc);
                if (acc) akey[na + __popc(m & lt)] = pack_key(d, pend[j]);
                na += __popc(m);
            }
            __syncwarp();
            if (na > 0) {
                sort_keys<CH>(akey, na, lane);
                uint64_t* Fn = cur ? fbuf0 : fbuf1;
                uint8_t* Vn = wm + (cur ? B.off_v0 : B.off_v1);
                for (int k = lane; k < fsize; k += 32) {
                    const int pos = k + lower_bound_key(akey, na, F[k]);
                    if (pos < L) {
                        Fn[pos] = F[k];
                        Vn[pos] = V[k];
                    }
                }
                for (int i = lane; i < na; i += 32) {
                    const int pos = i + lower_bound_key(F, fsize, akey[i]);
                    if (pos < L) {
                        Fn[pos] = akey[i];
                        Vn[pos] = 0;
                    }
                }
                __syncwarp();
                fsize = min(L, fsize + na);
                cur ^= 1;
            }
        }
        if (over) {
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
    uint32_t* adj;
    uint32_t* deg;
    uint32_t dim, R;
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
// when the row has room, else q's row is re-pruned from its entries and the new sources.
template <int CH, bool Signed>
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
    const int R = (int)A.R;
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
        const uint32_t dq = A.deg[q];
        uint32_t* qrow = A.adj + (size_t)q * A.R;
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
        if (dq + added <= A.R) {
            for (uint32_t j = lane; j < added; j += 32) qrow[dq + j] = ids[dq + j];
            if (lane == 0) A.deg[q] = dq + added;
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
        const int kept = warp_prune<Signed>(rows32, sorted, m, q, A.alpha, R, kept_rows, kept_norm,
                                            crow, out_ids, lane);
        for (int j = lane; j < R; j += 32) qrow[j] = j < kept ? out_ids[j] : kEmptyId;
        if (lane == 0) A.deg[q] = (uint32_t)kept;
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

template <bool Signed>
void* merge_for(int ch) {
    switch (ch) {
        case 1: return (void*)merge_reverse_kernel<1, Signed>;
        case 2: return (void*)merge_reverse_kernel<2, Signed>;
        case 3: return (void*)merge_reverse_kernel<3, Signed>;
        case 4: return (void*)merge_reverse_kernel<4, Signed>;
        default: return (void*)merge_reverse_kernel<8, Signed>;
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
    void* mg_kernel = sgn ? merge_for<true>(ch) : merge_for<false>(ch);
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

    // reverse-edge merge buffers and radix-sort / run-length / scan scratch
    uint64_t *keys_in, *keys_out;
    uint32_t *tq, *run_q, *run_cnt, *run_off, *n_runs, *big, *n_big;
    if ((s = bb.alloc(&keys_in, max_pairs, "pair keys")) != PGB_OK ||
        (s = bb.alloc(&keys_out, max_pairs, "pair keys")) != PGB_OK ||
        (s = bb.alloc(&tq, max_pairs, "targets")) != PGB_OK ||
        (s = bb.alloc(&run_q, max_pairs, "runs")) != PGB_OK ||
        (s = bb.alloc(&run_cnt, max_pairs, "runs")) != PGB_OK ||
        (s = bb.alloc(&run_off, max_pairs, "runs")) != PGB_OK ||
        (s = bb.alloc(&n_runs, 1, "runs")) != PGB_OK ||
        (s = bb.alloc(&big, max_pairs, "hub groups")) != PGB_OK ||
        (s = bb.alloc(&n_big, 1, "hub groups")) != PGB_OK)
        return s;
    size_t t_sort = 0, t_rle = 0, t_scan = 0;
    if ((s = ck(cub::DeviceRadixSort::SortKeys(nullptr, t_sort, keys_in, keys_out, (int)max_pairs), "sort size")) != PGB_OK ||
        (s = ck(cub::DeviceRunLengthEncode::Encode(nullptr, t_rle, tq, run_q, run_cnt, n_runs, (int)max_pairs), "rle size")) != PGB_OK ||
        (s = ck(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, run_cnt, run_off, (int)max_pairs), "scan size")) != PGB_OK)
        return s;
    void* cub_tmp;
    size_t t_cub = std::max(t_sort, std::max(t_rle, t_scan));
    if ((s = bb.alloc((uint8_t**)&cub_tmp, t_cub, "sort scratch")) != PGB_OK) return s;
    BuildLayout BM = make_build_layout(L, gs, 0u, R);
    int wpbm = 4, blocksm = 1;
    if ((s = shape(mg_kernel, BM, wpbm, blocksm)) != PGB_OK) return s;
    // merge scratch per warp (wcap); a target with more candidates (a hub) is merged
    // again by a few warps whose scratch holds a whole batch
    const size_t warpsm = (size_t)wpbm * blocksm;
    uint32_t* gid;
    int32_t* gdist;
    uint64_t* gkey;
    if ((s = bb.alloc(&gid, warpsm * wcap, "merge scratch")) != PGB_OK ||
        (s = bb.alloc(&gdist, warpsm * wcap, "merge scratch")) != PGB_OK ||
        (s = bb.alloc(&gkey, warpsm * 2 * wcap, "merge scratch")) != PGB_OK)
        return s;
    const uint32_t hub_warps = (uint32_t)prop.multiProcessorCount;
    const uint32_t hub_cap = R + (uint32_t)max_batch;
    uint32_t* hgid = nullptr;
    int32_t* hgdist = nullptr;
    uint64_t* hgkey = nullptr;  // allocated when the first hub appears

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
            M.adj = adj;
            M.deg = deg;
            M.dim = dim;
            M.R = R;
            M.alpha = a;
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
                if ((s = ck(cudaLaunchKernel(mg_kernel, dim3(blocksm), dim3(wpbm * 32), args,
                                             (size_t)wpbm * BM.bytes, st), "merge launch")) != PGB_OK)
                    return s;
            }
            uint32_t nbig = 0;
            if ((s = ck(cudaMemcpy(&nbig, n_big, 4, cudaMemcpyDeviceToHost), "hub count")) != PGB_OK) return s;
            if (nbig > 0) {
                if (!hgid && ((s = bb.alloc(&hgid, (size_t)hub_warps * hub_cap, "hub scratch")) != PGB_OK ||
                              (s = bb.alloc(&hgdist, (size_t)hub_warps * hub_cap, "hub scratch")) != PGB_OK ||
                              (s = bb.alloc(&hgkey, (size_t)hub_warps * 2 * hub_cap, "hub scratch")) != PGB_OK))
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
                if ((s = ck(cudaLaunchKernel(mg_kernel, dim3(std::min(nbig, hub_warps)), dim3(32), args,
                                             BM.bytes, st), "hub merge launch")) != PGB_OK)
                    return s;
            }
            pos = end;
            batch = std::min(batch * 2, max_batch);
        }
    }
    if ((s = ck(cudaMemcpy(degrees, deg, (size_t)n * 4, cudaMemcpyDeviceToHost), "degrees download")) != PGB_OK ||
        (s = ck(cudaMemcpy(adjacency, adj, (size_t)n * R * 4, cudaMemcpyDeviceToHost), "adjacency download")) != PGB_OK)
        return s;
    return PGB_OK;
}
