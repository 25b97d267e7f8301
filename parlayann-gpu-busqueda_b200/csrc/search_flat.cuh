// search_flat.cuh -- one query of ParlayANN beam_search over a fixed-degree graph,
// executed by one warp. Shared by the plain kernel and the batched persistent kernel,
// so both return bit-identical neighbours.
//
// Semantics (same integers, same order as the reference kernel, cuda/busqueda.cu:151-499):
//   F = {(d(q, start), start)}, comps = 1; lossy filter H[2^bits] cleared per query
//   while an unvisited entry of F exists and expansions < limit:
//     u = first unvisited entry; mark visited; expansions++ (overflow rule :205-208)
//     for the first degree_limit row entries a, in row order: skip a == query index
//       (when requested) and a seen by the lossy filter (slot hash64_2(a) & mask);
//       every survivor costs one distance (comps++)
//     candidates: d < cutoff (INT_MAX while |F| < Ls, else F.back().d), sorted by (d, id)
//     F = first Ls of multiset set_union(F, candidates); cut at
//       upper_bound(F, (id 0, float(cut * F[k].d))) under (float dist, id) order
//   output: first k entries of F (padded), comps, expansions, flags
//
// Layout per warp (shared memory): query row, frontier keys + visited bytes, candidate
// scratch, and -- when they fit -- the lossy filter and the exact visited table.
#pragma once

#include <climits>

#include "../../include/pgb.h"
#include "device_common.cuh"

namespace pgb {

__host__ __device__ inline int ceil_log2_u64(uint64_t x) {
    int b = 0;
    while ((1ull << b) < x) b++;
    return b;
}
__host__ __device__ inline uint32_t next_pow2_u32(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
// lossy filter size, a semantic parameter (reference cuda/busqueda.cu:536-538)
__host__ __device__ inline int flat_filter_bits(uint32_t Ls) {
    int b = ceil_log2_u64((uint64_t)Ls * Ls) - 2;
    return b > 10 ? b : 10;
}
// exact visited-table capacity and the expansion count that raises the overflow flag
// (reference cuda/busqueda.cu:540 and :205-208)
__host__ __device__ inline uint32_t flat_visited_cap(uint32_t Ls) {
    return next_pow2_u32(8u * Ls + 128u);
}

// Compile-time section profiler (build with -DPGB_SECTION_PROFILE, as the reference's
// -DPERFIL build): each warp adds the clock64() cycles of every phase of the search to
// counters in its shared memory and folds them into device totals when it exits.
enum FlatSection {
    SEC_SETUP = 0,   // query load, table clears, start point, output
    SEC_VISIT,       // row fetch, visited marking
    SEC_FILTER,      // lossy filter pass
    SEC_DIST,        // distances
    SEC_SORT,        // candidates under the cutoff, sort
    SEC_UNION,       // multiset union decisions, visited lookups, next-row request
    SEC_SHIFT,       // frontier shift and inserts
    SEC_CUT_NEXT,    // cut, next unvisited, insert completion, prefetch
    SEC_ITERATIONS,  // (count) expansions
    SEC_QUERIES,     // (count) queries
    SEC_N_PENDING,   // (count) rows past the lossy filter (distances computed)
    SEC_N_CAND,      // (count) candidates under the cutoff
    SEC_N_ENTER,     // (count) candidates entering the frontier
    SEC_NO_CAND,     // (count) expansions with no candidate under the cutoff
    SEC_PRED_HIT,    // (count) expansions whose row was predicted
    NUM_SECTIONS
};
#ifdef PGB_SECTION_PROFILE
constexpr uint32_t kProfileBytes = 8u * NUM_SECTIONS;
#define PGB_PROF_BEGIN(t) long long t = clock64()
#define PGB_PROF_ADD(sec, t)                                                  \
    do {                                                                      \
        const long long now_ = clock64();                                     \
        if (lane == 0) prof[sec] += (unsigned long long)(now_ - t);           \
        t = now_;                                                             \
    } while (0)
#define PGB_PROF_COUNT(sec) \
    do {                    \
        if (lane == 0) prof[sec] += 1ull; \
    } while (0)
#define PGB_PROF_COUNT_N(sec, n)                                  \
    do {                                                          \
        if (lane == 0) prof[sec] += (unsigned long long)(n);      \
    } while (0)
#else
constexpr uint32_t kProfileBytes = 0;
#define PGB_PROF_BEGIN(t)
#define PGB_PROF_ADD(sec, t)
#define PGB_PROF_COUNT(sec)
#define PGB_PROF_COUNT_N(sec, n)
#endif

// Per-warp shared memory. Everything before the frontier keys is sized by the kernel's
// template parameters alone (adjacency chunks, shared-filter size), so the kernel
// addresses it with compile-time offsets; the frontier and the optional shared visited
// table follow, sized by the plan's beam capacity.
struct FlatLayout {
    uint32_t ls_cap;         // frontier capacity (>= largest Ls served)
    uint32_t gs;             // adjacency entries per chunked row, 32 * chunks (>= degree limit)
    uint32_t filter_words;   // lossy filter words kept in shared memory (0: global)
    uint32_t visited_words;  // visited-table words in shared memory (0: global)
    uint32_t off_a, off_b, off_c, off_vbits, off_filter, off_fkey, off_fvis, off_visited,
        off_prof, bytes;
};

// "maybe visited" bitmap per warp: a node's bit is set when it is expanded, so a
// candidate whose bit is clear has never been expanded and needs no table lookup
constexpr uint32_t kVisitedBits = 1024;  // visited_bit() yields 10 bits

// shared-memory lossy filters come in these sizes (words): beams up to 64, 90 and 128
constexpr uint32_t kSharedFilterMaxWords = 4096;

// capacity of the frontier's visited bytes: the largest beam a kernel serves (128 with a
// shared filter, PGB_MAX_BEAM otherwise), so that the region has a fixed size
__host__ __device__ constexpr uint32_t flat_fvis_cap(uint32_t filter_words) {
    return filter_words ? 128u : (uint32_t)PGB_MAX_BEAM;
}

__host__ __device__ constexpr uint32_t round16(uint32_t x) { return (x + 15u) & ~15u; }

__host__ __device__ constexpr FlatLayout make_flat_layout(uint32_t ls_cap, uint32_t gs,
                                                          uint32_t filter_words,
                                                          uint32_t visited_words) {
    FlatLayout L{};
    L.ls_cap = ls_cap;
    L.gs = gs;
    L.filter_words = filter_words;
    L.visited_words = visited_words;
    uint32_t o = kRowBytes;  // query row at offset 0
    L.off_a = o;  // pending ids + distances, later entering keys
    o += 8u * gs;
    L.off_b = o;  // candidate keys
    o += 8u * gs;
    L.off_c = o;  // entering positions + visited bytes
    o = round16(o + 5u * gs);
    L.off_vbits = o;
    o += kVisitedBits / 8u;
    L.off_fvis = o;
    o += flat_fvis_cap(filter_words);
    L.off_filter = o;  // 16-byte aligned; its size is a multiple of 16
    o += 4u * filter_words;
    L.off_fkey = o;  // offsets up to here depend on (gs, filter_words) only
    o = round16(o + 8u * ls_cap);
    L.off_visited = o;
    o += 4u * visited_words;
    L.off_prof = o;
    o += kProfileBytes;
    L.bytes = round16(o);
    return L;
}

// plain: static query striding; batched: device work queue with per-query (Ls, k);
// batched uniform: work queue, one (Ls, k) for the whole launch; plain codes: the plain
// schedule over 4-bit code rows
enum class FlatSchedule { kPlain, kBatched, kBatchedUniform, kPlainCodes };

struct FlatArgs {
    const uint8_t* rows;   // n x 128-byte vector rows
    const uint32_t* adj;   // n x gs neighbour ids, padded with kEmptyId
    uint32_t n, gs, deg_lim, dim, start;
    const uint8_t* queries;
    uint32_t nq, qstride;
    double cut;
    int64_t limit;         // resolved: > 0
    uint32_t excl, qbase;
    uint32_t norm_in_row;           // rows carry their squared norm in bytes 124..127
    uint32_t Ls, k;                 // uniform values (plain kernel)
    const uint32_t* ls_arr;         // per-query Ls (batched), indexed by query
    const uint32_t* k_arr;          // per-query k (batched)
    const uint32_t* order;          // batched: processing order of the queries
    uint32_t out_stride;            // output row stride (>= k)
    uint32_t* ids;
    int32_t* dists;
    pgb_query_stats* stats;
    FlatLayout L;
    uint32_t* gfilter;              // per-warp global filters when not in shared memory
    uint32_t gfilter_words;
    uint32_t* gvisited;             // per-warp global visited tables when not in shared
    uint32_t gvisited_words;
    uint32_t* queue;                // batched: next-query counter
    // batched, optional: per-query completion flags in host-mapped memory. When query q's
    // outputs are written (system-visible), done[q] = done_seq, so a host thread can take
    // the query's results before the launch ends (the serving loop does)
    uint32_t* done;
    uint32_t done_seq;
    // code rows (kPlainCodes): rows holds n x 64-byte code rows, a dimension's value is
    // code_step * code + its offset (code_off: one 128-byte row of element values)
    int32_t code_step;
    const uint8_t* code_off;
};

// ---- exact visited multiset (keys only; duplicates occupy several slots) ----------
// Slot positions in this table and in the bitmap are private (only the counts matter),
// so they use 32-bit multiplicative hashes (Knuth's golden-ratio constant for the home
// slot's top bits, a second odd constant for the bitmap bit) instead of hash64_2.
__device__ __forceinline__ uint32_t visited_home(uint32_t id, uint32_t shift) {
    return (id * 0x9E3779B1u) >> shift;
}
__device__ __forceinline__ uint32_t visited_bit(uint32_t id) {
    return (id * 0x85EBCA6Bu) >> (32 - 10);  // 1,024-bit bitmap
}

// continues an insert whose first 32 probe slots were all taken
static __device__ __noinline__ void visited_insert_from(uint32_t* tab, uint32_t mask, uint32_t id,
                                                 uint32_t h, int lane) {
    for (uint32_t probe = 32; probe <= mask; probe += 32) {
        const uint32_t s = (h + probe + (uint32_t)lane) & mask;
        const uint32_t empty = __ballot_sync(kFull, tab[s] == kEmptyId);
        if (empty) {
            if (lane == __ffs(empty) - 1) tab[s] = id;
            break;
        }
    }
}

// number of copies of id whose home slot is h (single lane)
__device__ __forceinline__ int visited_count(const uint32_t* tab, uint32_t mask, uint32_t id,
                                             uint32_t h) {
    int c = 0;
    for (uint32_t i = 0; i <= mask; i++) {
        const uint32_t v = tab[(h + i) & mask];
        if (v == kEmptyId) break;
        c += (v == id);
    }
    return c;
}

// ---- sorted-key searches over shared memory ----------------------------------------
__device__ __forceinline__ int lower_bound_key(const uint64_t* a, int n, uint64_t key) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int upper_bound_key(const uint64_t* a, int n, uint64_t key) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] <= key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ---- warp bitonic sort of 32*E keys held E per lane (element e = t*32 + lane) -------
template <int E>
__device__ __forceinline__ void bitonic_sort(uint64_t (&v)[E], int lane) {
#pragma unroll
    for (int kk = 2; kk <= 32 * E; kk <<= 1) {
#pragma unroll
        for (int j = kk >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
#pragma unroll
                for (int t = 0; t < E; t++) {
                    const int tp = t ^ (j >> 5);
                    if (tp > t) {
                        const bool asc = (((t * 32 + lane) & kk) == 0);
                        const uint64_t a = v[t], b = v[tp];
                        const bool sw = asc ? (a > b) : (a < b);
                        v[t] = sw ? b : a;
                        v[tp] = sw ? a : b;
                    }
                }
            } else {
#pragma unroll
                for (int t = 0; t < E; t++) {
                    const uint64_t o = __shfl_xor_sync(kFull, v[t], j);
                    const bool asc = (((t * 32 + lane) & kk) == 0);
                    const bool lower = (lane & j) == 0;
                    const uint64_t mn = v[t] < o ? v[t] : o;
                    const uint64_t mx = v[t] < o ? o : v[t];
                    v[t] = (lower == asc) ? mn : mx;
                }
            }
        }
    }
}

template <int E>
__device__ __forceinline__ void sort_keys_e(uint64_t* keys, int nc, int lane) {
    uint64_t v[E];
#pragma unroll
    for (int t = 0; t < E; t++) {
        const int e = t * 32 + lane;
        v[t] = (e < nc) ? keys[e] : kEmptyKey;
    }
    bitonic_sort<E>(v, lane);
    __syncwarp();
#pragma unroll
    for (int t = 0; t < E; t++) {
        const int e = t * 32 + lane;
        if (e < nc) keys[e] = v[t];
    }
    __syncwarp();
}

// sorts keys[0..nc) ascending; nc <= 32 * CH. Few keys: each lane counts the keys below
// its own and scatters it to that rank (equal keys are identical, so their order is moot).
template <int CH>
__device__ __forceinline__ void sort_keys(uint64_t* keys, int nc, int lane) {
    if (nc <= 1) return;
    if (nc <= 20) {
        const uint64_t mine = lane < nc ? keys[lane] : 0;
        int rank = 0;
        for (int j = 0; j < nc; j++) {
            const uint64_t o = keys[j];
            rank += (o < mine || (o == mine && j < lane)) ? 1 : 0;
        }
        __syncwarp();
        if (lane < nc) keys[rank] = mine;
        __syncwarp();
    } else if (nc <= 32) {
        sort_keys_e<1>(keys, nc, lane);
    } else if (CH >= 2 && nc <= 64) {
        sort_keys_e<(CH >= 2 ? 2 : 1)>(keys, nc, lane);
    } else if (CH >= 3 && nc <= 128) {
        sort_keys_e<(CH >= 3 ? 4 : 1)>(keys, nc, lane);
    } else {
        sort_keys_e<(CH >= 5 ? 8 : 1)>(keys, nc, lane);
    }
}

// ---- distances of pending rows: 4 lanes per 128-byte row, 8*SLOTS rows in flight ---
// Lane c of a row reads its 16-byte words c and c+4, so each load instruction covers two
// whole 32-byte sectors of 8 rows. q4: the query row (128 bytes, shared memory).
// norm_in_row: the row's squared norm sits in bytes 124..127 (word 7, held by lane 3).
#ifndef PGB_DIST_SLOTS
#define PGB_DIST_SLOTS 2
#endif
// one round: rows base .. base + 8*SLOTS - 1 (those past np are not stored)
template <bool Signed, int SLOTS>
__device__ __forceinline__ void row_round(const uint8_t* __restrict__ rows, const uint32_t* ids,
                                          int32_t* out, int np, int base, const int4 qa,
                                          const int4 qb, const int32_t qq, bool need_a,
                                          bool need_b, bool norm_in_row, int grp, int c) {
    {
        int4 va[SLOTS], vb[SLOTS];
#pragma unroll
        for (int r = 0; r < SLOTS; r++) {
            const int i = base + r * 8 + grp;
            // slots past np re-read row ids[0] (valid and cached): every lane loads
            // unconditionally, and those slots' sums are never stored
            const uint8_t* row = rows + (size_t)ids[i < np ? i : 0] * kRowBytes + c * 16;
            va[r] = need_a ? ldg16(row) : make_int4(0, 0, 0, 0);
            vb[r] = need_b ? ldg16(row + 64) : make_int4(0, 0, 0, 0);
        }
        int32_t t[SLOTS];
        if (norm_in_row) {
#pragma unroll
            for (int r = 0; r < SLOTS; r++)
                t[r] = (c == 3 ? vb[r].w : 0) -
                       2 * (partial_dot<Signed>(va[r], qa) + partial_dot<Signed>(vb[r], qb));
        } else {
#pragma unroll
            for (int r = 0; r < SLOTS; r++)
                t[r] = partial_l2<Signed>(va[r], qa) + partial_l2<Signed>(vb[r], qb);
        }
#pragma unroll
        for (int off = 2; off > 0; off >>= 1)
#pragma unroll
            for (int r = 0; r < SLOTS; r++) t[r] += __shfl_xor_sync(kFull, t[r], off, 4);
        if (c == 0) {
#pragma unroll
            for (int r = 0; r < SLOTS; r++) {
                const int i = base + r * 8 + grp;
                if (i < np) out[i] = qq + t[r];
            }
        }
    }
}

// TAIL: a tail of at most 8 rows takes a one-slot round (fewer instructions per
// expansion; the batched kernels use it: +1 % there, while the plain kernel's register
// budget spills more with it and loses 3 %)
template <bool Signed, int SLOTS = PGB_DIST_SLOTS, bool TAIL = false>
__device__ __forceinline__ void row_distances(const uint8_t* __restrict__ rows,
                                              const uint32_t* ids, int32_t* out, int np,
                                              const int4* q4, const int32_t qq, uint32_t dim,
                                              bool norm_in_row, int lane) {
    const int grp = lane >> 2, c = lane & 3;
    const int4 qa = q4[c], qb = q4[c + 4];
    // bytes past dim are zero in every row; lane 3 also loads word 7 when it holds the norm
    const bool need_a = (uint32_t)(c * 16) < dim;
    const bool need_b = (uint32_t)((c + 4) * 16) < dim || (norm_in_row && c == 3);
    for (int base = 0; base < np; base += 8 * SLOTS) {
        if (TAIL && SLOTS > 1 && np - base <= 8) {
            row_round<Signed, 1>(rows, ids, out, np, base, qa, qb, qq, need_a, need_b, norm_in_row, grp, c);
            break;
        }
        row_round<Signed, SLOTS>(rows, ids, out, np, base, qa, qb, qq, need_a, need_b, norm_in_row, grp, c);
    }
    __syncwarp();
}

// ---- distances over 4-bit code rows: 4 lanes per 64-byte row, 8*SLOTS rows in flight --
// Lane c reads the row's 16-byte word c (dimensions 32c..32c+31) and pairs it with query
// words 2c and 2c+1. With v = step * code + offset per dimension,
//   ||q - v||^2 = (||q||^2 - 2 q.offset) - 2 step (q.code) + ||v||^2,
// where qq carries the first term and ||v||^2 sits in bytes 60..63 (word 3's last int,
// held by lane 3; the query is zero over those dimensions, so its codes add nothing).
// One round: code rows base .. base + 8*SLOTS - 1 (those past np are not stored).
template <bool Signed, int SLOTS>
__device__ __forceinline__ void code_round(const uint8_t* __restrict__ codes, const uint32_t* ids,
                                           int32_t* out, int np, int base, const int4 qa,
                                           const int4 qb, const int32_t qq, int32_t step,
                                           int grp, int c) {
    int4 v[SLOTS];
#pragma unroll
    for (int r = 0; r < SLOTS; r++) {
        const int i = base + r * 8 + grp;
        // slots past np re-read row ids[0], as in row_distances
        v[r] = ldg16(codes + (size_t)ids[i < np ? i : 0] * kCodeRowBytes + c * 16);
    }
    int32_t t[SLOTS];
#pragma unroll
    for (int r = 0; r < SLOTS; r++)
        t[r] = (c == 3 ? v[r].w : 0) - 2 * step * code_dot<Signed>(v[r], qa, qb);
#pragma unroll
    for (int off = 2; off > 0; off >>= 1)
#pragma unroll
        for (int r = 0; r < SLOTS; r++) t[r] += __shfl_xor_sync(kFull, t[r], off, 4);
    if (c == 0) {
#pragma unroll
        for (int r = 0; r < SLOTS; r++) {
            const int i = base + r * 8 + grp;
            if (i < np) out[i] = qq + t[r];
        }
    }
}

template <bool Signed, int SLOTS = PGB_DIST_SLOTS>
__device__ __forceinline__ void code_row_distances(const uint8_t* __restrict__ codes,
                                                   const uint32_t* ids, int32_t* out, int np,
                                                   const int4* q4, const int32_t qq,
                                                   int32_t step, int lane) {
    const int grp = lane >> 2, c = lane & 3;
    const int4 qa = q4[2 * c], qb = q4[2 * c + 1];
    for (int base = 0; base < np; base += 8 * SLOTS) {
        // a tail of at most 8 rows takes a one-slot round (the code-row kernel has the
        // registers for both loop bodies)
        if (SLOTS > 1 && np - base <= 8) {
            code_round<Signed, 1>(codes, ids, out, np, base, qa, qb, qq, step, grp, c);
            break;
        }
        code_round<Signed, SLOTS>(codes, ids, out, np, base, qa, qb, qq, step, grp, c);
    }
    __syncwarp();
}

// dot(q, o) of a zero-padded 128-byte query row with a 128-byte row o, on every lane
template <bool Signed>
__device__ __forceinline__ int32_t query_row_dot(const int4* q4, const uint8_t* o, int lane) {
    int32_t s = partial_dot<Signed>(ldg16(o + 16 * (lane & 7)), q4[lane & 7]);
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) s += __shfl_xor_sync(kFull, s, off, 8);
    return s;
}

// ||q||^2 of a zero-padded 128-byte query row, on every lane
template <bool Signed>
__device__ __forceinline__ int32_t query_sq_norm(const int4* q4, int lane) {
    int32_t s = partial_sq<Signed>(q4[lane & 7]);
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) s += __shfl_xor_sync(kFull, s, off, 8);
    return s;
}

// ---- one query -----------------------------------------------------------------------
// CH: adjacency chunks of 32. SFILT: lossy filter in shared memory (else gfilter).
// The visited table lives in gvisited when that is non-null, else in shared memory.
// FW: words of the lossy filter in shared memory (1024, 2048 or 4096), 0 when it lives in
// gfilter. Offsets up to the frontier keys are compile-time constants (K); a shared
// visited table sits after the frontier, at the plan's offset (A.L), which the host
// computes with the same make_flat_layout.
// C4: A.rows holds 4-bit code rows (kCodeRowBytes each) and distances are those of the
// reconstructed vectors (code_row_distances); otherwise 128-byte vector rows.
// TAIL: row_distances' one-slot tail round (the batched kernels).
template <bool Signed, bool C4, bool TAIL>
__device__ __forceinline__ void pending_distances(const FlatArgs& A, const uint32_t* ids,
                                                  int32_t* out, int np, const int4* q4,
                                                  int32_t qq, bool nir, int lane) {
    if constexpr (C4)
        code_row_distances<Signed>(A.rows, ids, out, np, q4, qq, A.code_step, lane);
    else
        row_distances<Signed, PGB_DIST_SLOTS, TAIL>(A.rows, ids, out, np, q4, qq, A.dim, nir, lane);
}

template <int CH, bool Signed, int FW, bool C4 = false, bool TAIL = false>
__device__ void flat_query(const FlatArgs& A, unsigned char* wmem, uint32_t* gfilter,
                           uint32_t* gvisited, uint32_t q, uint32_t Ls, uint32_t k, int lane) {
    constexpr bool SFILT = FW > 0;
    constexpr FlatLayout K = make_flat_layout(0u, 32u * CH, (uint32_t)FW, 0u);
    uint32_t* qwords = reinterpret_cast<uint32_t*>(wmem);
    uint64_t* fkey = reinterpret_cast<uint64_t*>(wmem + K.off_fkey);
    uint8_t* fvis = wmem + K.off_fvis;
    uint32_t* pend = reinterpret_cast<uint32_t*>(wmem + K.off_a);
    int32_t* pdist = reinterpret_cast<int32_t*>(wmem + K.off_a + 4u * K.gs);
    uint64_t* ekey = reinterpret_cast<uint64_t*>(wmem + K.off_a);  // reuses pend/pdist
    uint64_t* ckey = reinterpret_cast<uint64_t*>(wmem + K.off_b);
    int32_t* epos = reinterpret_cast<int32_t*>(wmem + K.off_c);
    uint8_t* evis = wmem + K.off_c + 4u * K.gs;
    uint32_t* filter = SFILT ? reinterpret_cast<uint32_t*>(wmem + K.off_filter) : gfilter;
    uint32_t* vtab = gvisited ? gvisited : reinterpret_cast<uint32_t*>(wmem + A.L.off_visited);
    uint32_t* vbits = reinterpret_cast<uint32_t*>(wmem + K.off_vbits);
#ifdef PGB_SECTION_PROFILE
    unsigned long long* prof = reinterpret_cast<unsigned long long*>(wmem + A.L.off_prof);
#endif
    PGB_PROF_BEGIN(tp);
    PGB_PROF_COUNT(SEC_QUERIES);

    const uint32_t qid = A.qbase + q;
    const uint32_t fmask = (1u << flat_filter_bits(Ls)) - 1u;
    const uint32_t vcap = flat_visited_cap(Ls);
    const uint32_t vmask = vcap - 1u;
    const uint32_t vshift = 32u - (uint32_t)ceil_log2_u64(vcap);
    const int max_visits = (int)(vcap / 2u);
    const int64_t limit = A.limit;
    const uint32_t lt = lanemask_lt(), gt = lanemask_gt();

    // query row (zero padded) and ||q||^2
    load_query_row(A.queries + (size_t)q * A.qstride, A.dim, lane, qwords);
    // clear this query's tables (both sizes are multiples of 128 words, 16-byte aligned)
    {
        const uint4 e4 = make_uint4(kEmptyId, kEmptyId, kEmptyId, kEmptyId);
        uint4* f4 = reinterpret_cast<uint4*>(filter);
        for (uint32_t i = lane; i < (fmask + 1u) / 4u; i += 32) f4[i] = e4;
        uint4* v4 = reinterpret_cast<uint4*>(vtab);
        for (uint32_t i = lane; i < vcap / 4u; i += 32) v4[i] = e4;
        if (lane < (int)(kVisitedBits / 128u)) reinterpret_cast<uint4*>(vbits)[lane] = make_uint4(0, 0, 0, 0);
    }
    __syncwarp();
    const int4* q4 = reinterpret_cast<const int4*>(qwords);
    int32_t qq = query_sq_norm<Signed>(q4, lane);
    if constexpr (C4) qq -= 2 * query_row_dot<Signed>(q4, A.code_off, lane);

    // start point: F = {(d(q, start), start)}, one distance
    if (lane == 0) pend[0] = A.start;
    __syncwarp();
    const bool nir = A.norm_in_row != 0;
    pending_distances<Signed, C4, TAIL>(A, pend, pdist, 1, q4, qq, nir, lane);
    if (lane == 0) {
        fkey[0] = pack_key(pdist[0], A.start);
        fvis[0] = 0;
    }
    __syncwarp();

    int fsize = 1, u = 0, flags = 0;
    int nvis = 0;
    int comps = 1;
    const int deg_lim = (int)A.deg_lim;
    // row of the predicted next expansion, loaded while the current one is merged
    uint32_t pred = kEmptyId;
    uint32_t apred[CH];
    int u2 = -1;  // second unvisited frontier entry when known

    PGB_PROF_ADD(SEC_SETUP, tp);
    while (u >= 0 && (int64_t)nvis < limit) {
        PGB_PROF_COUNT(SEC_ITERATIONS);
        const uint64_t cur_key = fkey[u];
        const uint32_t cur = key_id(cur_key);
        // whole neighbour row: the predicted one, or requested now
        uint32_t a[CH];
        if (cur == pred) {
            PGB_PROF_COUNT(SEC_PRED_HIT);
#pragma unroll
            for (int t = 0; t < CH; t++) a[t] = apred[t];
        } else {
            const uint32_t* row = A.adj + (size_t)cur * A.gs;
#pragma unroll
            for (int t = 0; t < CH; t++) {
                const int j = t * 32 + lane;
                a[t] = (j < deg_lim) ? __ldg(row + j) : kEmptyId;
            }
        }
        if (lane == 0) fvis[u] = 1;
        // visited insert of cur, in two halves: the 32 probe slots are read now and the
        // slot is claimed at the end of the iteration (only this warp writes the table);
        // lookups in between add the pending copy themselves
        const uint32_t vhome = visited_home(cur, vshift);
        const uint32_t vslot = (vhome + (uint32_t)lane) & vmask;
        const uint32_t vprobe = vtab[vslot];
        if (lane == 0) {
            const uint32_t b = visited_bit(cur);
            vbits[b >> 5] |= 1u << (b & 31u);
        }
        nvis++;
        if (nvis > max_visits) {
            flags |= PGB_FLAG_OVERFLOW;
            break;
        }
        const int32_t cutoff = (fsize < (int)Ls) ? INT_MAX : key_dist(fkey[fsize - 1]);
        PGB_PROF_ADD(SEC_VISIT, tp);

        // ---- lossy filter in row order -> pending ids ------------------------------
        int np = 0;
        if (SFILT) {
            // chunks in order: each chunk sees the writes of the previous ones
#pragma unroll
            for (int t = 0; t < CH; t++) {
                const uint32_t x = a[t];
                const bool part = x != kEmptyId && !(A.excl && x == qid);
                const uint32_t slot =
                    part ? (uint32_t)(hash64_2(x) & fmask) : (0x80000000u | (uint32_t)(t * 32 + lane));
                const uint32_t peers = __match_any_sync(kFull, slot);
                const uint32_t before = peers & lt;
                const int src = before ? 31 - __clz(before) : lane;
                const uint32_t prev = __shfl_sync(kFull, x, src);
                bool seen;
                if (before) seen = part && prev == x;
                else seen = part && filter[slot] == x;
                __syncwarp();
                if (part && (peers & gt) == 0) filter[slot] = x;
                const bool pass = part && !seen;
                const uint32_t m = __ballot_sync(kFull, pass);
                if (pass) pend[np + __popc(m & lt)] = x;
                np += __popc(m);
                __syncwarp();
            }
        } else {
            // global table: all slots read up front (one round trip); an entry with no
            // earlier same-slot entry in its chunk takes the value written by the last
            // earlier chunk entry of that slot, else the table value
            uint32_t slot[CH], mem[CH];
#pragma unroll
            for (int t = 0; t < CH; t++) {
                const uint32_t x = a[t];
                const bool part = x != kEmptyId && !(A.excl && x == qid);
                slot[t] = part ? (uint32_t)(hash64_2(x) & fmask)
                               : (0x80000000u | (uint32_t)(t * 32 + lane));
                mem[t] = part ? filter[slot[t]] : kEmptyId;
            }
            uint32_t* sslot = reinterpret_cast<uint32_t*>(ckey);  // scratch: slots of row
            uint32_t* sid = sslot + 32 * CH;                        // and ids
#pragma unroll
            for (int t = 0; t < CH; t++) {
                const uint32_t x = a[t];
                const bool part = x != kEmptyId && !(A.excl && x == qid);
                const uint32_t peers = __match_any_sync(kFull, slot[t]);
                const uint32_t before = peers & lt;
                const int src = before ? 31 - __clz(before) : lane;
                const uint32_t prev = __shfl_sync(kFull, x, src);
                bool seen;
                if (before) {
                    seen = part && prev == x;
                } else {
                    seen = part && mem[t] == x;
                    if (part)
                        for (int p = t * 32 - 1; p >= 0; p--)
                            if (sslot[p] == slot[t]) {
                                seen = sid[p] == x;
                                break;
                            }
                }
                __syncwarp();
                sslot[t * 32 + lane] = slot[t];
                sid[t * 32 + lane] = x;
                if (part && (peers & gt) == 0) filter[slot[t]] = x;
                const bool pass = part && !seen;
                const uint32_t m = __ballot_sync(kFull, pass);
                if (pass) pend[np + __popc(m & lt)] = x;
                np += __popc(m);
                __syncwarp();
            }
        }
        comps += np;
        PGB_PROF_COUNT_N(SEC_N_PENDING, np);
        PGB_PROF_ADD(SEC_FILTER, tp);

        // ---- distances ------------------------------------------------------------
        pending_distances<Signed, C4, TAIL>(A, pend, pdist, np, q4, qq, nir, lane);
        PGB_PROF_ADD(SEC_DIST, tp);

        // ---- candidates under the cutoff, in arrival order ------------------------
        int nc = 0;
        for (int base = 0; base < np; base += 32) {
            const int i = base + lane;
            const bool c = i < np && pdist[i] < cutoff;
            const uint32_t m = __ballot_sync(kFull, c);
            if (c) ckey[nc + __popc(m & lt)] = pack_key(pdist[i], pend[i]);
            nc += __popc(m);
        }
        __syncwarp();
        // the next expansion is the smaller of the second unvisited entry and the best
        // unvisited candidate that enters the frontier (unless the cut drops it); its row
        // is requested as soon as that is known, before the frontier is shifted
        uint64_t best = (u2 >= 0 && u2 < fsize) ? fkey[u2] : kEmptyKey;

        int unew = u;
        int ne = 0;
        PGB_PROF_COUNT_N(SEC_N_CAND, nc);
        if (nc == 0) PGB_PROF_COUNT(SEC_NO_CAND);
        if (nc > 0) {
            sort_keys<CH>(ckey, nc, lane);
            PGB_PROF_ADD(SEC_SORT, tp);
            // ---- multiset set_union: copy `rep` of a key enters iff rep >= copies in F
            bool found = false;  // best unvisited entering key seen (keys ascend)
            for (int base = 0; base < nc; base += 32) {
                const int i = base + lane;
                bool enter = false;
                int hi = 0;
                uint64_t key = 0;
                uint8_t vis = 0;
                if (i < nc) {
                    key = ckey[i];
                    hi = upper_bound_key(fkey, fsize, key);
                    int cf = 0;
                    if (hi > 0 && fkey[hi - 1] == key) cf = hi - lower_bound_key(fkey, fsize, key);
                    int rep = 0;
                    while (i - rep - 1 >= 0 && ckey[i - rep - 1] == key) rep++;
                    enter = rep >= cf;
                    if (enter) {
                        const uint32_t id = key_id(key);
                        const uint32_t b = visited_bit(id);
                        int cnt = 0;
                        if ((vbits[b >> 5] >> (b & 31u)) & 1u)
                            cnt = visited_count(vtab, vmask, id, visited_home(id, vshift)) +
                                  (id == cur ? 1 : 0);
                        vis = (uint8_t)(rep < cnt);
                    }
                }
                const uint32_t m = __ballot_sync(kFull, enter);
                // new copies follow the frontier copies of an equal key
                const int pos = hi + ne + __popc(m & lt);
                const bool keep = enter && pos < (int)Ls;
                const uint32_t mk = __ballot_sync(kFull, keep);
                const uint32_t mnv = __ballot_sync(kFull, keep && !vis);
                if (mnv && !found) {
                    const uint64_t k0 = __shfl_sync(kFull, key, __ffs(mnv) - 1);
                    best = k0 < best ? k0 : best;
                    found = true;
                }
                if (keep) {
                    const int jk = ne + __popc(mk & lt);
                    ekey[jk] = key;
                    epos[jk] = pos;
                    evis[jk] = vis;
                }
                ne += __popc(mk);
                if (mk != m) break;  // later keys land at or past Ls
            }
            __syncwarp();
        }
        PGB_PROF_COUNT_N(SEC_N_ENTER, ne);
        pred = (best != kEmptyKey) ? key_id(best) : kEmptyId;
        if (pred != kEmptyId) {
            const uint32_t* prow = A.adj + (size_t)pred * A.gs;
#pragma unroll
            for (int t = 0; t < CH; t++) {
                const int j = t * 32 + lane;
                apred[t] = (j < deg_lim) ? __ldg(prow + j) : kEmptyId;
            }
        }
        PGB_PROF_ADD(SEC_UNION, tp);

        int from;
        if (ne > 0) {
            // the expanded entry's new position, then shift the frontier tail
            unew = u + lower_bound_key(ekey, ne, cur_key);
            const int first = epos[0];
            for (int top = fsize - 1; top >= first; top -= 32) {
                const int i = top - lane;
                const bool act = i >= first;
                uint64_t key = 0;
                uint8_t vis = 0;
                int np2 = 0;
                if (act) {
                    key = fkey[i];
                    vis = fvis[i];
                    np2 = i + lower_bound_key(ekey, ne, key);
                }
                __syncwarp();
                if (act && np2 < (int)Ls) {
                    fkey[np2] = key;
                    fvis[np2] = vis;
                }
                __syncwarp();
            }
            int minpos = INT_MAX;
            for (int j = lane; j < ne; j += 32) {
                fkey[epos[j]] = ekey[j];
                fvis[epos[j]] = evis[j];
                if (!evis[j]) minpos = min(minpos, epos[j]);
            }
            __syncwarp();
            fsize = min((int)Ls, fsize + ne);
            PGB_PROF_ADD(SEC_SHIFT, tp);

            // ---- cut (only a changed frontier can need one) ---------------------------
            if (fsize > (int)k) {
                const float thr = (float)(A.cut * (double)key_dist(fkey[k]));
                // "after the threshold" is monotone along F: when the last entry is not
                // after it, nothing is cut (the common case once the beam has converged)
                const uint64_t last = fkey[fsize - 1];
                const float dl = (float)key_dist(last);
                const bool any_cut = thr < dl || (thr == dl && 0u < key_id(last));
                int newsize = fsize;
                for (int base = 0; any_cut && base < fsize; base += 32) {
                    const int i = base + lane;
                    bool after = false;
                    if (i < fsize) {
                        const uint64_t e = fkey[i];
                        const float de = (float)key_dist(e);
                        after = thr < de || (thr == de && 0u < key_id(e));
                    }
                    const uint32_t m = __ballot_sync(kFull, after);
                    if (m) {
                        newsize = base + __ffs(m) - 1;
                        break;
                    }
                }
                fsize = newsize;
            }
            minpos = (int)__reduce_min_sync(kFull, (unsigned)minpos);
            from = min(unew, minpos);
        } else {
            // unchanged frontier (already cut): the next unvisited entry is the second one
            from = (u2 >= 0) ? u2 : u + 1;
        }

        // ---- next unvisited ---------------------------------------------------------
        u = -1;
        u2 = -1;
        for (int base = from; base < fsize; base += 32) {
            const int i = base + lane;
            const bool un = i < fsize && !fvis[i];
            const uint32_t m = __ballot_sync(kFull, un);
            if (m) {
                u = base + __ffs(m) - 1;
                const uint32_t rest = m & (m - 1);
                u2 = rest ? base + __ffs(rest) - 1 : -1;
                break;
            }
        }
        // second half of the visited insert
        {
            const uint32_t empty = __ballot_sync(kFull, vprobe == kEmptyId);
            if (empty) {
                if (lane == __ffs(empty) - 1) vtab[vslot] = cur;
            } else {
                visited_insert_from(vtab, vmask, cur, vhome, lane);
            }
        }
        // the prediction held: pull the vector rows of its neighbours into L2 now, ahead
        // of the next distance phase (rows the filter will drop are fetched too)
        if (u >= 0 && key_id(fkey[u]) == pred) {
#pragma unroll
            for (int t = 0; t < CH; t++)
                if (apred[t] != kEmptyId)
                    prefetch_row_l2(A.rows + (size_t)apred[t] * (C4 ? kCodeRowBytes : kRowBytes));
        }
        __syncwarp();
        PGB_PROF_ADD(SEC_CUT_NEXT, tp);
    }

    // ---- output: first k of the frontier ----------------------------------------------
    if (fsize < (int)k) flags |= PGB_FLAG_SHORT;
    uint32_t* oid = A.ids + (size_t)q * A.out_stride;
    int32_t* od = A.dists + (size_t)q * A.out_stride;
    for (uint32_t j = lane; j < k; j += 32) {
        const bool have = (int)j < fsize;
        const uint64_t e = have ? fkey[j] : 0;
        oid[j] = have ? key_id(e) : kEmptyId;
        od[j] = have ? key_dist(e) : INT_MAX;
    }
    if (lane == 0 && A.stats) {
        pgb_query_stats s;
        s.dist_comps = comps;
        s.expansions = nvis;
        s.flags = flags;
        s.reserved = 0;
        A.stats[q] = s;
    }
    __syncwarp();
    PGB_PROF_ADD(SEC_SETUP, tp);
}

}  // namespace pgb
