// search_hnsw.cu -- HNSW layered search, one warp per query.
//
// Semantics follow the reference's HNSW kernel (cuda/busqueda_hnsw.cu:215-456), itself
// ParlayANN's HNSW::search: per layer from the top, ef = 1 and 2 filter bits above
// layer 0, ef = Ls and bits0 = 2*ceil(log2 Ls) - 2 on layer 0 with limit_eval; entry
// points marked with hash64, neighbours with hash64_2; cand ordered by distance only
// (equal distances rejected); workset W ordered by (dist, id); is_inw exact; next
// layer's entry = W's worst; output the first k of W mapped node -> point.
//
// The reference decides acceptance neighbour by neighbour (:400-418). Here the
// decisions are made lane-parallel from a closed form that yields the same set:
// with m = max(ef, |W|), neighbour j is accepted iff it is eligible (not in is_inw and
// the first copy of its id among this expansion's survivors) and fewer than m elements
// of W plus the eligible neighbours before j have distance <= d_j. (A rejected
// neighbour has d >= the current worst, so counting it never moves the threshold.)
// W then becomes the smallest m' = min(m, |W| + accepted) of W + accepted, and cand the
// ef smallest distinct distances of cand + accepted (first copy of each distance
// wins); when cand starts above ef (several entry points on the top layer) its
// per-neighbour trim rule is replayed sequentially instead.
//
// is_inw needs no table. Every id it receives on a layer also enters W, and once W is
// full its worst key never grows, so an id that has left W has a key above W's current
// worst. A neighbour that can be accepted has d < W's worst distance (or W is not full
// and has lost nothing), hence for such a neighbour "in is_inw" is "in W", a lookup in
// the sorted W already in shared memory; neighbours at or beyond the worst are never
// looked up. Only the count of is_inw inserts is kept, for the overflow flag
// (capInw / 2, busqueda_hnsw.cu:559).
#include <algorithm>
#include <climits>
#include <string>

#include "errors.h"
#include "index.h"
#include "search_flat.cuh"
#include "search_hnsw.h"
#include "search_plan.h"

// largest lossy filter kept in shared memory (bytes); larger ones live in global memory
#ifndef PGB_HNSW_SHARED_FILTER_BYTES
#define PGB_HNSW_SHARED_FILTER_BYTES 4096
#endif
// resident 128-thread blocks per SM the HNSW kernel is compiled for (8: 64 registers)
#ifndef PGB_HNSW_MIN_BLOCKS
#define PGB_HNSW_MIN_BLOCKS 8
#endif
// distance rounds of the HNSW kernel: 8 * slots rows in flight per warp; TAIL: a tail of
// at most 8 rows takes a one-slot round
#ifndef PGB_HNSW_DIST_SLOTS
#define PGB_HNSW_DIST_SLOTS 2
#endif
#ifndef PGB_HNSW_DIST_TAIL
#define PGB_HNSW_DIST_TAIL false
#endif

namespace pgb {

__host__ __device__ inline uint32_t hnsw_bits0(uint32_t Ls) {
    return Ls > 2 ? 2u * (uint32_t)ceil_log2_u64(Ls) - 2u : 2u;  // busqueda_hnsw.cu:556-557
}
__host__ __device__ inline uint32_t hnsw_cap_inw(uint32_t Ls) {
    return next_pow2_u32(32u * Ls + 2048u);  // busqueda_hnsw.cu:559
}

struct HnswLayout {
    uint32_t wcap, gs, filter_words, wbits_words;
    uint32_t off_w, off_c, off_pend, off_pd, off_ak, off_nk, off_pos, off_fl, off_eps, off_wbits,
        off_filter, off_prof, bytes;
};

// The candidate list is a window ckey[c0, c0 + nC) that slides up as the closest entry is
// popped; it is moved back to the start when an update would run past this capacity.
__host__ __device__ inline uint32_t hnsw_ccap(uint32_t wcap) { return 2u * wcap; }

// filter_words: shared-memory filter (FMODE 0); wbits_words: written-slot bitmap of a
// global id filter (FMODE 1)
__host__ __device__ inline HnswLayout make_hnsw_layout(uint32_t wcap, uint32_t gs,
                                                       uint32_t filter_words, uint32_t wbits_words) {
    HnswLayout L;
    L.wcap = wcap;
    L.gs = gs;
    L.filter_words = filter_words;
    L.wbits_words = wbits_words;
    uint32_t o = kRowBytes;
    L.off_w = o;
    o += 8u * wcap;
    L.off_c = o;
    o += 8u * hnsw_ccap(wcap);
    L.off_pend = o;
    o += 4u * gs;
    L.off_pd = o;
    o += 4u * gs;
    L.off_ak = o;
    o += 8u * gs;
    L.off_nk = o;
    o += 8u * gs;
    L.off_pos = o;
    o += 4u * gs;
    L.off_fl = o;
    o = round16(o + gs);
    L.off_eps = o;
    o += 4u * PGB_MAX_HNSW_ENTRIES;
    L.off_wbits = o;
    o = round16(o + 4u * wbits_words);
    L.off_filter = o;
    o += 4u * filter_words;
    L.off_prof = o;  // section counters of the profiling build (kProfileBytes = 0 otherwise)
    o += kProfileBytes;
    L.bytes = round16(o);
    return L;
}

struct HnswArgs {
    const uint8_t* rows;  // node order
    const uint32_t* adj0;
    uint32_t g0s, G0;
    const uint32_t* adju;
    uint32_t gas, GA;
    const uint32_t* upper_start;
    const uint32_t* node_point;
    uint32_t entries[PGB_MAX_HNSW_ENTRIES];
    uint32_t n_entries, top, dim, norm_in_row;
    const uint8_t* queries;
    uint32_t nq, qstride;
    uint32_t Ls, k;
    uint64_t limit0;
    uint32_t bits0, cap_inw, filter_slots;
    HnswLayout L;
    uint32_t* ids;
    int32_t* dists;
    pgb_query_stats* stats;
    unsigned long long* gfilter;
    uint64_t epoch_base;
    // (epoch, id) filter: the launch's first epoch read from device memory (a captured
    // graph replays one launch; hnsw_epoch_advance moves this word on after each launch);
    // null: epoch_base
    const uint64_t* epoch_ptr;
    uint32_t* queue;  // query work queue: each warp takes the next query when it is free
    uint32_t out_stride;  // query q's k outputs start at q * out_stride
    // batched launch (else null): query q's beam and k, and the order the queue hands the
    // queries out in (longest beam first)
    const uint32_t* ls_arr;
    const uint32_t* k_arr;
    const uint32_t* order;
    // optional per-query completion flags in host-mapped memory (done[q] = done_seq once
    // query q's outputs are system-visible)
    uint32_t* done;
    uint32_t done_seq;
};

__device__ __forceinline__ unsigned long long tag(uint32_t epoch, uint32_t id) {
    return ((unsigned long long)epoch << 32) | id;
}

// The number of W entries at distance <= d, and whether (d, id) is one of them: W is
// sorted by (dist, id), so the entries at distance d follow the lower bound of (d, 0)
__device__ __forceinline__ int w_count_le(const uint64_t* wkey, int nW, int32_t d, uint32_t id,
                                          bool& in_w) {
    int c = lower_bound_key(wkey, nW, pack_key(d, 0));
    in_w = false;
    while (c < nW) {
        const uint64_t k = wkey[c];
        if (key_dist(k) != d) break;
        in_w |= key_id(k) == id;
        c++;
    }
    return c;
}

// moves keys[from, from + n) to keys[0, n) (from >= 0; chunk reads precede chunk writes)
__device__ __forceinline__ void slide_to_start(uint64_t* keys, int from, int n, int lane) {
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        uint64_t v = 0;
        if (i < n) v = keys[from + i];
        __syncwarp();
        if (i < n) keys[i] = v;
        __syncwarp();
    }
}

#ifdef PGB_SECTION_PROFILE
// the HNSW kernel's section totals (this translation unit's own device variable)
static __device__ unsigned long long g_hnsw_section_cycles[NUM_SECTIONS];
#endif

// FMODE: where the lossy filter lives. 0: shared memory. 1: per-warp global table of ids
// plus a shared-memory bitmap of the slots written on this layer (cleared per layer, so
// unwritten slots need no load). 2: per-warp global table of (epoch, id) pairs, for
// filters whose written-bitmap would not fit in shared memory.
template <int CH, bool Signed, int FMODE>
__global__ void __launch_bounds__(128, PGB_HNSW_MIN_BLOCKS) hnsw_kernel(HnswArgs A) {
    constexpr bool SFILT = FMODE == 0;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t gw = blockIdx.x * wpb + w;
    const HnswLayout& L = A.L;
    unsigned char* wmem = smem + (size_t)w * L.bytes;
    uint32_t* qwords = reinterpret_cast<uint32_t*>(wmem);
    uint64_t* wkey = reinterpret_cast<uint64_t*>(wmem + L.off_w);
    uint64_t* ckey = reinterpret_cast<uint64_t*>(wmem + L.off_c);
    uint32_t* pend = reinterpret_cast<uint32_t*>(wmem + L.off_pend);
    int32_t* pd = reinterpret_cast<int32_t*>(wmem + L.off_pd);
    uint64_t* akey = reinterpret_cast<uint64_t*>(wmem + L.off_ak);
    uint64_t* nkey = reinterpret_cast<uint64_t*>(wmem + L.off_nk);
    int32_t* pos = reinterpret_cast<int32_t*>(wmem + L.off_pos);
    uint8_t* fl = wmem + L.off_fl;
    uint32_t* eps = reinterpret_cast<uint32_t*>(wmem + L.off_eps);
    uint32_t* sfilter = reinterpret_cast<uint32_t*>(wmem + L.off_filter);
    unsigned long long* gfil = FMODE == 2 ? A.gfilter + (size_t)gw * A.filter_slots : nullptr;
    uint32_t* gf32 = FMODE == 1 ? reinterpret_cast<uint32_t*>(A.gfilter) + (size_t)gw * A.filter_slots
                                : nullptr;
    uint32_t* wbits = reinterpret_cast<uint32_t*>(wmem + L.off_wbits);
    const int ccap = (int)hnsw_ccap(L.wcap);
    const uint32_t lt = lanemask_lt(), gt = lanemask_gt();
    const uint32_t layers = A.top + 1u;
    const uint64_t epoch_base = (FMODE == 2 && A.epoch_ptr) ? *A.epoch_ptr : A.epoch_base;
    // queries are taken from the work queue, so a warp that drew short searches takes more
    // of them and the launch does not wait on the warps with the longest share
    auto take = [&]() -> uint32_t {
        uint32_t v = 0;
        if (lane == 0) v = atomicAdd(A.queue, 1u);
        return __shfl_sync(kFull, v, 0);
    };

#ifdef PGB_SECTION_PROFILE
    unsigned long long* prof = reinterpret_cast<unsigned long long*>(wmem + L.off_prof);
    if (lane < NUM_SECTIONS) prof[lane] = 0ull;
    __syncwarp();
#endif

    for (uint32_t t = take(); t < A.nq; t = take()) {
        const uint32_t q = A.order ? A.order[t] : t;
        // this query's beam, k, layer-0 filter bits and is_inw overflow threshold
        uint32_t qLs = A.Ls, qk = A.k, qbits0 = A.bits0, qcap_half = A.cap_inw / 2;
        if (A.ls_arr) {
            qLs = A.ls_arr[q];
            qk = A.k_arr[q];
            qbits0 = hnsw_bits0(qLs);
            qcap_half = hnsw_cap_inw(qLs) / 2;
        }
        PGB_PROF_BEGIN(tp);
        PGB_PROF_COUNT(SEC_QUERIES);
        load_query_row(A.queries + (size_t)q * A.qstride, A.dim, lane, qwords);
        __syncwarp();
        const int4* q4 = reinterpret_cast<const int4*>(qwords);
        const int32_t qq = query_sq_norm<Signed>(q4, lane);

        int comps = 0, exps = 0, flags = 0;
        int neps = (int)A.n_entries;
        if (lane < neps) eps[lane] = A.entries[lane];
        __syncwarp();
        int nW = 0;

        for (int layer = (int)A.top; layer >= 0; layer--) {
            const int ef = (layer > 0) ? 1 : (int)qLs;
            const uint32_t bits = (layer > 0) ? 2u : qbits0;
            const uint32_t fmask = (1u << bits) - 1u;
            const uint64_t limit = (layer > 0) ? ~0ull : A.limit0;
            const uint32_t* mat = (layer > 0) ? A.adju : A.adj0;
            const uint32_t stride = (layer > 0) ? A.gas : A.g0s;
            const int G = (int)((layer > 0) ? A.GA : A.G0);
            const uint32_t epoch =
                (uint32_t)(epoch_base + (uint64_t)q * layers + (A.top - (uint32_t)layer) + 1u);
            if (SFILT) {
                for (uint32_t i = lane; i <= fmask; i += 32) sfilter[i] = kEmptyId;
            } else if (FMODE == 1) {
                for (uint32_t i = lane; i < (fmask + 32u) / 32u; i += 32) wbits[i] = 0u;
            }
            __syncwarp();
            // ---- entry points: distances, then the sequential inserts on lane 0 ----
            for (int e = lane; e < neps; e += 32) pend[e] = eps[e];
            __syncwarp();
            row_distances<Signed>(A.rows, pend, pd, neps, q4, qq, A.dim, A.norm_in_row != 0, lane);
            int nC = 0;
            nW = 0;
            if (lane == 0) {
                for (int e = 0; e < neps; e++) {
                    const uint32_t pe = pend[e];
                    const int32_t d = pd[e];
                    const uint32_t s = (uint32_t)(hash64(pe) & fmask);
                    if (SFILT) {
                        sfilter[s] = pe;
                    } else if (FMODE == 1) {
                        gf32[s] = pe;
                        wbits[s >> 5] |= 1u << (s & 31u);
                    } else {
                        gfil[s] = tag(epoch, pe);
                    }
                    // is_inw: W below holds every entry point (inserted without a
                    // membership test, so a repeated entry point appears twice)
                    // cand: by distance, equal distance rejected
                    const uint64_t key = pack_key(d, pe);
                    int pos = lower_bound_key(ckey, nC, pack_key(d, 0));
                    if (!(pos < nC && key_dist(ckey[pos]) == d)) {
                        for (int i = nC; i > pos; i--) ckey[i] = ckey[i - 1];
                        ckey[pos] = key;
                        nC++;
                    }
                    // W: (dist, id) order, no trim
                    pos = upper_bound_key(wkey, nW, key);
                    for (int i = nW; i > pos; i--) wkey[i] = wkey[i - 1];
                    wkey[pos] = key;
                    nW++;
                }
            }
            nC = __shfl_sync(kFull, nC, 0);
            nW = __shfl_sync(kFull, nW, 0);
            __syncwarp();
            int32_t wlast = key_dist(wkey[nW - 1]);  // W's worst distance, kept in a register
            comps += neps;
            uint32_t inserted = (uint32_t)neps;
            uint64_t cnt = 0;
            int c0 = 0;  // the candidate window is ckey[c0, c0 + nC)
            // neighbour row of the next expansion, requested as soon as cand is updated
            uint32_t unext = kEmptyId;
            uint32_t anext[CH];
            auto request_row = [&](uint32_t v) {
                const uint32_t* row =
                    (layer > 0) ? mat + ((size_t)A.upper_start[v] + (uint32_t)(layer - 1)) * stride
                                : mat + (size_t)v * stride;
#pragma unroll
                for (int t = 0; t < CH; t++) {
                    const int j = t * 32 + lane;
                    anext[t] = (j < G) ? __ldg(row + j) : kEmptyId;
                }
                unext = v;
            };

            PGB_PROF_ADD(SEC_SETUP, tp);
            while (nC > 0) {
                if (key_dist(ckey[c0]) > wlast) break;
                if (++cnt > limit) break;
                const uint32_t u = key_id(ckey[c0]);
                c0++;  // pop the closest candidate
                nC--;
                exps++;
                uint32_t a[CH];
                PGB_PROF_COUNT(SEC_ITERATIONS);
                if (u == unext) {
                    PGB_PROF_COUNT(SEC_PRED_HIT);
#pragma unroll
                    for (int t = 0; t < CH; t++) a[t] = anext[t];
                } else {
                    const uint32_t* row =
                        (layer > 0) ? mat + ((size_t)A.upper_start[u] + (uint32_t)(layer - 1)) * stride
                                    : mat + (size_t)u * stride;
#pragma unroll
                    for (int t = 0; t < CH; t++) {
                        const int j = t * 32 + lane;
                        a[t] = (j < G) ? __ldg(row + j) : kEmptyId;
                    }
                }
                PGB_PROF_ADD(SEC_VISIT, tp);
                // ---- lossy visited filter in row order ---------------------------------
                int np = 0;
                if (SFILT) {
#pragma unroll
                    for (int t = 0; t < CH; t++) {
                        const uint32_t x = a[t];
                        const bool part = x != kEmptyId;
                        const uint32_t slot = part ? (uint32_t)(hash64_2(x) & fmask)
                                                   : (0x80000000u | (uint32_t)(t * 32 + lane));
                        const uint32_t peers = __match_any_sync(kFull, slot);
                        const uint32_t before = peers & lt;
                        const int src = before ? 31 - __clz(before) : lane;
                        const uint32_t prev = __shfl_sync(kFull, x, src);
                        bool seen;
                        if (before) seen = part && prev == x;
                        else seen = part && sfilter[slot] == x;
                        __syncwarp();
                        if (part && (peers & gt) == 0) sfilter[slot] = x;
                        const bool pass = part && !seen;
                        const uint32_t m = __ballot_sync(kFull, pass);
                        if (pass) pend[np + __popc(m & lt)] = x;
                        np += __popc(m);
                        __syncwarp();
                    }
                } else {
                    // each slot's id at the start of the row: one round of loads, skipped
                    // (FMODE 1) for slots not written on this layer
                    uint32_t slot[CH], mem[CH];
#pragma unroll
                    for (int t = 0; t < CH; t++) {
                        const bool part = a[t] != kEmptyId;
                        slot[t] = part ? (uint32_t)(hash64_2(a[t]) & fmask)
                                       : (0x80000000u | (uint32_t)(t * 32 + lane));
                        mem[t] = kEmptyId;
                        if (FMODE == 1) {
                            if (part && ((wbits[slot[t] >> 5] >> (slot[t] & 31u)) & 1u))
                                mem[t] = __ldcg(gf32 + slot[t]);
                        } else if (part) {
                            const unsigned long long m = __ldcg(gfil + slot[t]);
                            if ((uint32_t)(m >> 32) == epoch) mem[t] = (uint32_t)m;
                        }
                    }
                    uint32_t* sslot = reinterpret_cast<uint32_t*>(akey);
                    uint32_t* sid = sslot + 32 * CH;
                    // slots of this row's earlier chunks, hashed into 2,048 bits (in nkey,
                    // unused until the cand update): a clear bit proves that no earlier
                    // chunk wrote the slot, so the backward scan runs only on a set bit
                    uint32_t* rbits = reinterpret_cast<uint32_t*>(nkey);
                    if (CH > 1) {
                        reinterpret_cast<uint2*>(rbits)[lane] = make_uint2(0u, 0u);
                        __syncwarp();
                    }
#pragma unroll
                    for (int t = 0; t < CH; t++) {
                        const uint32_t x = a[t];
                        const bool part = x != kEmptyId;
                        const uint32_t peers = __match_any_sync(kFull, slot[t]);
                        const uint32_t before = peers & lt;
                        const int src = before ? 31 - __clz(before) : lane;
                        const uint32_t prev = __shfl_sync(kFull, x, src);
                        const uint32_t rb = slot[t] & 2047u;
                        bool seen;
                        if (before) {
                            seen = part && prev == x;
                        } else {
                            seen = part && mem[t] == x;
                            if (t > 0 && part && ((rbits[rb >> 5] >> (rb & 31u)) & 1u))
                                for (int p = t * 32 - 1; p >= 0; p--)
                                    if (sslot[p] == slot[t]) {
                                        seen = sid[p] == x;
                                        break;
                                    }
                        }
                        __syncwarp();
                        sslot[t * 32 + lane] = slot[t];
                        sid[t * 32 + lane] = x;
                        if (CH > 1 && t + 1 < CH && part && (peers & gt) == 0)
                            atomicOr(&rbits[rb >> 5], 1u << (rb & 31u));
                        if (part && (peers & gt) == 0) {
                            if (FMODE == 1) {
                                gf32[slot[t]] = x;
                                atomicOr(&wbits[slot[t] >> 5], 1u << (slot[t] & 31u));
                            } else {
                                gfil[slot[t]] = tag(epoch, x);
                            }
                        }
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
                row_distances<Signed, PGB_HNSW_DIST_SLOTS, PGB_HNSW_DIST_TAIL>(A.rows, pend, pd, np, q4, qq, A.dim,
                                                                            A.norm_in_row != 0, lane);
                PGB_PROF_ADD(SEC_DIST, tp);

                // ---- eligibility (first copy in this expansion, not in is_inw) and
                // acceptance (fewer than m elements of W + earlier eligible at <= d). With
                // W full (nW >= ef, so m = nW) acceptance needs d < W's worst distance, and
                // a neighbour at or beyond it never counts for one below it: only these
                // "near" neighbours are checked at all. Copies of an id share a distance,
                // so the first copy of a near id is near too.
                const int m = max(ef, nW);
                const int32_t worst = nW >= ef ? wlast : INT_MAX;
                int na = 0;
                if (np <= 32) {
                    // one chunk: earlier copies are the lanes below with the same id, and
                    // the earlier eligible neighbours are a ballot mask. Only near lanes
                    // take part (copies of an id share a distance), and an expansion with
                    // none (most of them) skips the rest.
                    const uint32_t pv = lane < np ? pend[lane] : kEmptyId;
                    const int32_t dv = lane < np ? pd[lane] : INT_MAX;
                    const bool near = lane < np && dv < worst;
                    const uint32_t nm = __ballot_sync(kFull, near);
                    if (nm) {
                        bool elig = false;
                        int c = 0;
                        if (near && (__match_any_sync(nm, pv) & lt) == 0) {
                            bool in_w;
                            c = w_count_le(wkey, nW, dv, pv, in_w);
                            elig = !in_w;
                        }
                        const uint32_t em = __ballot_sync(kFull, elig);
                        bool acc = false;
                        if (elig) {
                            for (uint32_t mm = em & lt; mm != 0u && c < m; mm &= mm - 1u)
                                c += pd[__ffs(mm) - 1] <= dv ? 1 : 0;
                            acc = c < m;
                        }
                        const uint32_t mk = __ballot_sync(kFull, acc);
                        if (acc) akey[__popc(mk & lt)] = pack_key(dv, pv);
                        na = __popc(mk);
                    }
                } else {
                    for (int j = lane; j < np; j += 32) {
                        const uint32_t pv = pend[j];
                        bool elig = pd[j] < worst;
                        for (int i = 0; i < j && elig; i++)
                            if (pend[i] == pv) elig = false;
                        if (elig) {
                            bool in_w;
                            w_count_le(wkey, nW, pd[j], pv, in_w);
                            elig = !in_w;
                        }
                        fl[j] = elig ? 1 : 0;
                    }
                    __syncwarp();
                    for (int base = 0; base < np; base += 32) {
                        const int j = base + lane;
                        bool acc = false;
                        int32_t d = 0;
                        uint32_t pv = 0;
                        if (j < np && fl[j]) {
                            d = pd[j];
                            pv = pend[j];
                            int c = lower_bound_key(wkey, nW, pack_key(d + 1, 0));
                            for (int i = 0; i < j && c < m; i++) c += (fl[i] && pd[i] <= d) ? 1 : 0;
                            acc = c < m;
                        }
                        const uint32_t mk = __ballot_sync(kFull, acc);
                        if (acc) akey[na + __popc(mk & lt)] = pack_key(d, pv);
                        na += __popc(mk);
                    }
                }
                __syncwarp();
                PGB_PROF_COUNT_N(SEC_N_CAND, na);
                if (na == 0) PGB_PROF_COUNT(SEC_NO_CAND);
                PGB_PROF_ADD(SEC_SORT, tp);
                if (na > 0) {
                    inserted += (uint32_t)na;  // is_inw inserts (the set itself is W)
                    // ---- cand update (accepted keys still in arrival order) ---------------
                    const int nC0 = nC;
                    uint64_t* cq = ckey + c0;
                    if (nC0 <= ef) {
                        // new distances only, first copy of each distance
                        int nn = 0;
                        for (int base = 0; base < na; base += 32) {
                            const int j = base + lane;
                            bool nw = false;
                            uint64_t key = 0;
                            if (j < na) {
                                key = akey[j];
                                const int32_t d = key_dist(key);
                                const int p = lower_bound_key(cq, nC0, pack_key(d, 0));
                                nw = !(p < nC0 && key_dist(cq[p]) == d);
                                for (int i = 0; i < j && nw; i++)
                                    if (key_dist(akey[i]) == d) nw = false;
                            }
                            const uint32_t mk = __ballot_sync(kFull, nw);
                            if (nw) nkey[nn + __popc(mk & lt)] = key;
                            nn += __popc(mk);
                        }
                        __syncwarp();
                        if (nn > 0) {
                            sort_keys<CH>(nkey, nn, lane);
                            const int nCn = min(ef, nC0 + nn);
                            if (c0 + nCn > ccap) {
                                slide_to_start(ckey, c0, nC0, lane);
                                c0 = 0;
                                cq = ckey;
                            }
                            for (int j = lane; j < nn; j += 32)
                                pos[j] = lower_bound_key(cq, nC0, pack_key(key_dist(nkey[j]), 0)) + j;
                            __syncwarp();
                            const int first = pos[0];
                            for (int topi = nC0 - 1; topi >= first; topi -= 32) {
                                const int i = topi - lane;
                                const bool act = i >= first;
                                uint64_t key = 0;
                                int np2 = 0;
                                if (act) {
                                    key = cq[i];
                                    np2 = i + lower_bound_key(nkey, nn, pack_key(key_dist(key), 0));
                                }
                                __syncwarp();
                                if (act && np2 < nCn) cq[np2] = key;
                                __syncwarp();
                            }
                            for (int j = lane; j < nn; j += 32)
                                if (pos[j] < nCn) cq[pos[j]] = nkey[j];
                            __syncwarp();
                            nC = nCn;
                        }
                    } else {
                        // cand above ef (several top-layer entries): replay the rule, which
                        // holds cand at nC0 entries after each insert (one slot of headroom)
                        if (c0 + nC0 + 1 > ccap) {
                            slide_to_start(ckey, c0, nC0, lane);
                            c0 = 0;
                            cq = ckey;
                        }
                        if (lane == 0) {
                            for (int j = 0; j < na; j++) {
                                const uint64_t key = akey[j];
                                const int32_t d = key_dist(key);
                                const int p = lower_bound_key(cq, nC, pack_key(d, 0));
                                if (!(p < nC && key_dist(cq[p]) == d)) {
                                    for (int i = nC; i > p; i--) cq[i] = cq[i - 1];
                                    cq[p] = key;
                                    nC++;
                                }
                                if (nC > ef) nC--;
                            }
                        }
                    }
                    nC = __shfl_sync(kFull, nC, 0);
                    __syncwarp();
                    // the next expansion is cand's new closest entry: request its row now,
                    // while W is updated
                    if (nC > 0) request_row(key_id(ckey[c0]));
                    PGB_PROF_ADD(SEC_UNION, tp);
                    // ---- W update: the m' smallest of W + accepted -----------------------
                    sort_keys<CH>(akey, na, lane);
                    const int nWn = min(m, nW + na);
                    for (int j = lane; j < na; j += 32) pos[j] = upper_bound_key(wkey, nW, akey[j]) + j;
                    __syncwarp();
                    const int firstw = pos[0];
                    for (int topi = nW - 1; topi >= firstw; topi -= 32) {
                        const int i = topi - lane;
                        const bool act = i >= firstw;
                        uint64_t key = 0;
                        int np2 = 0;
                        if (act) {
                            key = wkey[i];
                            np2 = i + lower_bound_key(akey, na, key);
                        }
                        __syncwarp();
                        if (act && np2 < nWn) wkey[np2] = key;
                        __syncwarp();
                    }
                    for (int j = lane; j < na; j += 32)
                        if (pos[j] < nWn) wkey[pos[j]] = akey[j];
                    __syncwarp();
                    nW = nWn;
                    wlast = key_dist(wkey[nW - 1]);
                    PGB_PROF_ADD(SEC_SHIFT, tp);
                } else if (nC > 0) {
                    request_row(key_id(ckey[c0]));  // cand unchanged
                }
                if (inserted > qcap_half) {
                    flags |= PGB_FLAG_OVERFLOW;
                    break;
                }
                PGB_PROF_ADD(SEC_CUT_NEXT, tp);
            }
            if (layer > 0) {
                if (lane == 0) eps[0] = key_id(wkey[nW - 1]);
                neps = 1;
                __syncwarp();
            }
        }
        // ---- output: first k of W, node -> point ------------------------------------
        if (nW < (int)qk) flags |= PGB_FLAG_SHORT;
        uint32_t* oid = A.ids + (size_t)q * A.out_stride;
        int32_t* od = A.dists + (size_t)q * A.out_stride;
        for (uint32_t j = lane; j < qk; j += 32) {
            const bool have = (int)j < nW;
            const uint64_t e = have ? wkey[j] : 0;
            oid[j] = have ? A.node_point[key_id(e)] : kEmptyId;
            od[j] = have ? key_dist(e) : INT_MAX;
        }
        if (lane == 0 && A.stats) {
            pgb_query_stats s;
            s.dist_comps = comps;
            s.expansions = exps;
            s.flags = flags;
            s.reserved = 0;
            A.stats[q] = s;
        }
        __syncwarp();
        if (A.done) publish_query_done(A.done, q, A.done_seq, lane);
        PGB_PROF_ADD(SEC_SETUP, tp);
    }
#ifdef PGB_SECTION_PROFILE
    __syncwarp();
    if (lane < NUM_SECTIONS) atomicAdd(&g_hnsw_section_cycles[lane], prof[lane]);
#endif
}

}  // namespace pgb

namespace pgb {
namespace {

using HnswKernel = void (*)(HnswArgs);

template <int CH, bool Signed>
HnswKernel pick_hnsw_mode(int fmode) {
    return fmode == 0   ? hnsw_kernel<CH, Signed, 0>
           : fmode == 1 ? hnsw_kernel<CH, Signed, 1>
                        : hnsw_kernel<CH, Signed, 2>;
}

template <int CH>
HnswKernel pick_hnsw_ch(bool is_signed, int fmode) {
    return is_signed ? pick_hnsw_mode<CH, true>(fmode) : pick_hnsw_mode<CH, false>(fmode);
}

HnswKernel pick_hnsw(int ch, bool is_signed, int fmode) {
    switch (ch) {
        case 1: return pick_hnsw_ch<1>(is_signed, fmode);
        case 2: return pick_hnsw_ch<2>(is_signed, fmode);
        case 3: return pick_hnsw_ch<3>(is_signed, fmode);
        case 4: return pick_hnsw_ch<4>(is_signed, fmode);
        default: return pick_hnsw_ch<8>(is_signed, fmode);
    }
}

pgb_status hnsw_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PGB_OK;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(PGB_ERR_OOM, std::string(what) + ": out of memory");
    return fail(PGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

HnswLayout hnsw_layout_of(const HnswState& H) {
    return make_hnsw_layout(H.wcap, 32u * H.ch, H.fmode == 0 ? (1u << H.bits0) : 0u,
                            H.fmode == 1 ? H.filter_slots / 32u : 0u);
}

pgb_status hnsw_prepare(const pgb_index* ix, const pgb_query_params& p, HnswState& H) {
    H = HnswState{};
    const uint32_t Ls = p.beam_size;
    H.ch = flat_chunks_for(std::max(ix->G0, ix->GA));
    H.bits0 = hnsw_bits0(Ls);
    H.cap_inw = hnsw_cap_inw(Ls);
    const uint32_t fwords = 1u << H.bits0;
    // shared-memory filter only while small (Ls <= 64): a 16 KB filter would cap the
    // kernel at 8 resident warps per SM. Up to 16,384 slots (Ls <= 256) the global table
    // holds bare ids beside a written-slot bitmap in shared memory (2 KB at most); larger
    // filters use (epoch, id) pairs.
    H.fmode = 4ull * fwords <= PGB_HNSW_SHARED_FILTER_BYTES ? 0 : (fwords <= 16384 ? 1 : 2);
    H.filter_slots = H.fmode ? fwords : 0u;
    H.wcap = ((std::max<uint32_t>(Ls, PGB_MAX_HNSW_ENTRIES) + 8u) + 7u) & ~7u;
    const HnswLayout L = hnsw_layout_of(H);
    H.warp_bytes = L.bytes;
    H.kernel = (void*)pick_hnsw(H.ch, ix->elem == PGB_INT8, H.fmode);
    cudaDeviceProp prop;
    int dev = 0;
    pgb_status s;
    if ((s = hnsw_cuda(cudaGetDevice(&dev), "cudaGetDevice")) != PGB_OK) return s;
    if ((s = hnsw_cuda(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties")) != PGB_OK) return s;
    int wpb = 4;
    while (wpb > 1 && (size_t)wpb * L.bytes > prop.sharedMemPerBlockOptin) wpb >>= 1;
    if ((size_t)wpb * L.bytes > prop.sharedMemPerBlockOptin)
        return fail(PGB_ERR_BAD_ARG, "beam too wide for shared memory");
    H.warps_per_block = wpb;
    H.smem_bytes = (size_t)wpb * L.bytes;
    // per-kernel attribute shared by all searchers: the device maximum, never shrunk
    if ((s = hnsw_cuda(cudaFuncSetAttribute(H.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)prop.sharedMemPerBlockOptin),
                       "cudaFuncSetAttribute")) != PGB_OK ||
        (s = hnsw_cuda(cudaFuncSetAttribute(H.kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            (int)cudaSharedmemCarveoutMaxShared),
                       "cudaFuncSetAttribute")) != PGB_OK)
        return s;
    int bps = 0;
    if ((s = hnsw_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, H.kernel, wpb * 32, H.smem_bytes),
                       "occupancy")) != PGB_OK)
        return s;
    if (bps < 1) return fail(PGB_ERR_CUDA, "HNSW kernel does not fit on a multiprocessor");
    H.blocks = bps * prop.multiProcessorCount;
    H.total_warps = (uint64_t)H.blocks * wpb;
    if ((s = hnsw_cuda(cudaMalloc(&H.queue, sizeof(uint32_t)), "query queue")) != PGB_OK) return s;
    if (H.fmode == 1) {  // ids only; validity is the shared written-slot bitmap
        if ((s = hnsw_cuda(cudaMalloc(&H.gfilter, 4ull * H.filter_slots * H.total_warps),
                           "filter tables")) != PGB_OK)
            return s;
    } else if (H.fmode == 2) {
        const size_t fb = 8ull * H.filter_slots * H.total_warps;
        if ((s = hnsw_cuda(cudaMalloc(&H.gfilter, fb), "filter tables")) != PGB_OK) return s;
        if ((s = hnsw_cuda(cudaMemset(H.gfilter, 0, fb), "filter clear")) != PGB_OK) return s;
        if ((s = hnsw_cuda(cudaMalloc(&H.d_epoch, sizeof(uint64_t)), "epoch word")) != PGB_OK) return s;
        if ((s = hnsw_cuda(cudaMemset(H.d_epoch, 0, sizeof(uint64_t)), "epoch word")) != PGB_OK) return s;
    }
    H.epoch_base = 0;
    H.max_ls = Ls;
    H.ready = true;
    return PGB_OK;
}

// moves the device epoch word past the epochs the launch before it used (stream order:
// the search kernel has finished reading it)
__global__ void hnsw_epoch_advance(uint64_t* epoch, uint64_t need) { *epoch += need; }

pgb_status hnsw_launch(const pgb_index* ix, HnswState& H, const pgb_query_params& p,
                       const void* queries, uint32_t nq, uint32_t qstride, uint32_t* ids,
                       int32_t* dists, pgb_query_stats* stats, cudaStream_t stream) {
    return hnsw_launch_at(ix, H, p.beam_size, p.k, p.limit, queries, nq, qstride, ids, dists, stats,
                          p.k, stream);
}

size_t hnsw_scratch_bytes(const HnswState& H) {
    const size_t per_slot = H.fmode == 1 ? 4 : H.fmode == 2 ? 8 : 0;
    return per_slot * H.filter_slots * H.total_warps + sizeof(uint32_t);
}

pgb_status hnsw_launch_at(const pgb_index* ix, HnswState& H, uint32_t Ls, uint32_t k, int64_t limit,
                          const void* queries, uint32_t nq, uint32_t qstride, uint32_t* ids,
                          int32_t* dists, pgb_query_stats* stats, uint32_t out_stride,
                          cudaStream_t stream, const uint32_t* ls_arr, const uint32_t* k_arr,
                          const uint32_t* order, uint32_t* done, uint32_t done_seq) {
    if (!H.ready) return fail(PGB_ERR_BAD_ARG, "HNSW searcher not prepared");
    if (Ls == 0 || Ls > H.max_ls || k == 0 || out_stride < k || (ls_arr == nullptr) != (k_arr == nullptr))
        return fail(PGB_ERR_BAD_ARG, "HNSW launch: beam above the prepared one, or bad k / stride");
    HnswArgs A{};
    A.done = done;
    A.done_seq = done_seq;
    A.ls_arr = ls_arr;
    A.k_arr = k_arr;
    A.order = order;
    A.rows = ix->node_rows;
    A.adj0 = ix->adj0;
    A.g0s = ix->g0s;
    A.G0 = ix->G0;
    A.adju = ix->adju;
    A.gas = ix->gas;
    A.GA = ix->GA;
    A.upper_start = ix->upper_start;
    A.node_point = ix->node_point;
    for (uint32_t e = 0; e < ix->n_entries; e++) A.entries[e] = ix->entries[e];
    A.n_entries = ix->n_entries;
    A.top = ix->top_level;
    A.dim = ix->dim;
    A.norm_in_row = ix->norm_in_row ? 1u : 0u;
    A.queries = (const uint8_t*)queries;
    A.nq = nq;
    A.qstride = qstride;
    A.Ls = Ls;
    A.k = k;
    A.out_stride = out_stride;
    // limit_eval on layer 0: the visit limit when set below n, else n (busqueda_hnsw.cu:610)
    A.limit0 = (limit > 0 && (uint64_t)limit < ix->n_nodes) ? (uint64_t)limit : ix->n_nodes;
    // the filter and is_inw capacity of this beam; the tables (sized for H.max_ls, with
    // its filter placement) hold them
    A.bits0 = hnsw_bits0(Ls);
    A.cap_inw = hnsw_cap_inw(Ls);
    A.filter_slots = H.filter_slots;
    A.L = hnsw_layout_of(H);
    A.ids = ids;
    A.dists = dists;
    A.stats = stats;
    A.gfilter = H.gfilter;
    // every (query, layer) of every launch gets a fresh epoch for an (epoch, id) global
    // filter; the device word d_epoch holds the next unused one and H.epoch_base mirrors it
    // on the host (hnsw_epoch_reserve; wrap -> clear the tables)
    const uint64_t need = hnsw_epoch_need(ix, nq);
    {
        const pgb_status s = hnsw_epoch_reserve(H, need, stream);
        if (s != PGB_OK) return s;
    }
    A.epoch_base = H.epoch_base - need;
    A.epoch_ptr = H.d_epoch;
    A.queue = H.queue;
    {
        const pgb_status s = hnsw_cuda(cudaMemsetAsync(H.queue, 0, sizeof(uint32_t), stream), "query queue");
        if (s != PGB_OK) return s;
    }
    void* args[] = {&A};
    cudaError_t e = cudaLaunchKernel(H.kernel, dim3(H.blocks), dim3(H.warps_per_block * 32), args,
                                     H.smem_bytes, stream);
    if (e == cudaSuccess) count_launches(1);
    if (e == cudaSuccess && H.d_epoch) {
        hnsw_epoch_advance<<<1, 1, 0, stream>>>(H.d_epoch, need);
        e = cudaGetLastError();
    }
    return hnsw_cuda(e, "HNSW launch");
}

uint64_t hnsw_epoch_need(const pgb_index* ix, uint32_t nq) {
    return (uint64_t)nq * (ix->top_level + 1ull) + 1ull;
}

pgb_status hnsw_epoch_reserve(HnswState& H, uint64_t need, cudaStream_t stream) {
    if (H.epoch_base + need >= 0xFFFFFFFFull) {
        pgb_status s;
        if (H.fmode == 2 &&
            ((s = hnsw_cuda(cudaMemsetAsync(H.gfilter, 0, 8ull * H.filter_slots * H.total_warps, stream),
                            "filter clear")) != PGB_OK ||
             (s = hnsw_cuda(cudaMemsetAsync(H.d_epoch, 0, sizeof(uint64_t), stream), "epoch reset")) != PGB_OK))
            return s;
        H.epoch_base = 0;
    }
    H.epoch_base += need;
    return PGB_OK;
}

cudaError_t hnsw_section_totals(unsigned long long* acc, bool reset) {
#ifdef PGB_SECTION_PROFILE
    unsigned long long v[NUM_SECTIONS];
    cudaError_t e = cudaMemcpyFromSymbol(v, g_hnsw_section_cycles, sizeof(v));
    if (e != cudaSuccess) return e;
    for (int i = 0; i < NUM_SECTIONS; i++) acc[i] += v[i];
    if (reset) {
        unsigned long long zero[NUM_SECTIONS] = {0};
        e = cudaMemcpyToSymbol(g_hnsw_section_cycles, zero, sizeof(zero));
    }
    return e;
#else
    (void)acc;
    (void)reset;
    return cudaSuccess;
#endif
}

void hnsw_release(HnswState& H) {
    cudaFree(H.gfilter);
    cudaFree(H.queue);
    cudaFree(H.d_epoch);
    H = HnswState{};
}

}  // namespace pgb
