// search_flat_pair.cuh -- the batched form's paired schedule: two queries per warp, one on
// each 16-lane half.
//
// The per-query algorithm is flat_query's (search_flat.cuh), integer for integer and in the
// same order, so the neighbours, distances, counts and flags are identical. What changes
// is the execution: a 32-lane warp spends most of an expansion on work that is either
// per-query scalar (frontier bookkeeping, cut, next unvisited, loop control) or spread
// over a handful of lanes (sorting ~8 candidates, their union decisions, shifting a
// 40-entry frontier). Run by 16 lanes, the row-wide work (filter, distances) takes twice
// the instructions per query while everything else costs the same instructions as before
// and serves two queries at once. Each half runs its own query state machine: one
// expansion per loop trip, and a half whose query ends writes it out and pulls the next
// query from the work queue in the next trip, so a short query never waits for the
// longer one beside it. Every collective names only its half's lanes (mask, width 16),
// which keeps it defined when the halves diverge; when they agree they issue together.
//
// Per-query shared memory is flat_query's layout (make_flat_layout), one slice per half;
// the global filter / visited tables are per query slot (2 per warp).
#pragma once

#include "search_flat.cuh"

namespace pgb {

// the 16 lanes of one half-warp
struct HalfWarp {
    uint32_t mask;  // this half's lanes
    uint32_t lt;    // lanes of this half below this lane
    uint32_t gt;    // lanes of this half above this lane
    int base;       // first lane of the half (0 or 16)
    int sl;         // lane within the half
    __device__ __forceinline__ explicit HalfWarp(int lane) {
        base = lane & 16;
        sl = lane & 15;
        mask = 0xFFFFu << base;
        lt = lanemask_lt() & mask;
        gt = lanemask_gt() & mask;
    }
    // bits of this half's lanes only (absolute lane positions)
    __device__ __forceinline__ uint32_t ballot(bool p) const { return __ballot_sync(mask, p) & mask; }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    // position within the half of the lowest set bit of a nonzero ballot
    __device__ __forceinline__ int first(uint32_t m) const { return __ffs(m) - 1 - base; }
};

// ---- distances: 4 lanes per 128-byte row, 4 rows per slot over the half ---------------
template <bool Signed, int SLOTS>
__device__ __forceinline__ void half_row_round(const uint8_t* __restrict__ rows, const uint32_t* ids,
                                               int32_t* out, int np, int base, const int4 qa,
                                               const int4 qb, const int32_t qq, bool need_a,
                                               bool need_b, bool norm_in_row, int grp, int c,
                                               uint32_t hmask) {
    int4 va[SLOTS], vb[SLOTS];
#pragma unroll
    for (int r = 0; r < SLOTS; r++) {
        const int i = base + r * 4 + grp;
        // slots past np re-read row ids[0] (valid and cached); their sums are never stored
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
        for (int r = 0; r < SLOTS; r++) t[r] += __shfl_xor_sync(hmask, t[r], off, 4);
    if (c == 0) {
#pragma unroll
        for (int r = 0; r < SLOTS; r++) {
            const int i = base + r * 4 + grp;
            if (i < np) out[i] = qq + t[r];
        }
    }
}

// rounds of 16 rows while more than 8 remain, then one round of 8 or 4
template <bool Signed>
__device__ __forceinline__ void half_row_distances(const uint8_t* __restrict__ rows,
                                                   const uint32_t* ids, int32_t* out, int np,
                                                   const int4* q4, const int32_t qq, uint32_t dim,
                                                   bool norm_in_row, const HalfWarp& H) {
    const int grp = H.sl >> 2, c = H.sl & 3;
    const int4 qa = q4[c], qb = q4[c + 4];
    const bool need_a = (uint32_t)(c * 16) < dim;
    const bool need_b = (uint32_t)((c + 4) * 16) < dim || (norm_in_row && c == 3);
    int base = 0;
    for (; np - base > 8; base += 16)
        half_row_round<Signed, 4>(rows, ids, out, np, base, qa, qb, qq, need_a, need_b, norm_in_row, grp, c, H.mask);
    if (np - base > 4)
        half_row_round<Signed, 2>(rows, ids, out, np, base, qa, qb, qq, need_a, need_b, norm_in_row, grp, c, H.mask);
    else if (np - base > 0)
        half_row_round<Signed, 1>(rows, ids, out, np, base, qa, qb, qq, need_a, need_b, norm_in_row, grp, c, H.mask);
    H.sync();
}

// ---- half-warp bitonic sort of 16*E keys held E per lane (element e = t*16 + sl) ------
template <int E>
__device__ __forceinline__ void half_bitonic(uint64_t (&v)[E], const HalfWarp& H) {
#pragma unroll
    for (int kk = 2; kk <= 16 * E; kk <<= 1) {
#pragma unroll
        for (int j = kk >> 1; j > 0; j >>= 1) {
            if (j >= 16) {
#pragma unroll
                for (int t = 0; t < E; t++) {
                    const int tp = t ^ (j >> 4);
                    if (tp > t) {
                        const bool asc = (((t * 16 + H.sl) & kk) == 0);
                        const uint64_t a = v[t], b = v[tp];
                        const bool sw = asc ? (a > b) : (a < b);
                        v[t] = sw ? b : a;
                        v[tp] = sw ? a : b;
                    }
                }
            } else {
#pragma unroll
                for (int t = 0; t < E; t++) {
                    const uint64_t o = __shfl_xor_sync(H.mask, v[t], j, 16);
                    const bool asc = (((t * 16 + H.sl) & kk) == 0);
                    const bool lower = (H.sl & j) == 0;
                    const uint64_t mn = v[t] < o ? v[t] : o;
                    const uint64_t mx = v[t] < o ? o : v[t];
                    v[t] = (lower == asc) ? mn : mx;
                }
            }
        }
    }
}

template <int E>
__device__ __forceinline__ void half_sort_e(uint64_t* keys, int nc, const HalfWarp& H) {
    uint64_t v[E];
#pragma unroll
    for (int t = 0; t < E; t++) {
        const int e = t * 16 + H.sl;
        v[t] = (e < nc) ? keys[e] : kEmptyKey;
    }
    half_bitonic<E>(v, H);
    H.sync();
#pragma unroll
    for (int t = 0; t < E; t++) {
        const int e = t * 16 + H.sl;
        if (e < nc) keys[e] = v[t];
    }
    H.sync();
}

// sorts keys[0..nc) ascending, nc <= 16 * NT: rank counting up to 16 keys, bitonic above
template <int NT>
__device__ __forceinline__ void half_sort_keys(uint64_t* keys, int nc, const HalfWarp& H) {
    if (nc <= 1) return;
    if (nc <= 16) {
        const uint64_t mine = H.sl < nc ? keys[H.sl] : 0;
        int rank = 0;
        for (int j = 0; j < nc; j++) {
            const uint64_t o = keys[j];
            rank += (o < mine || (o == mine && j < H.sl)) ? 1 : 0;
        }
        H.sync();
        if (H.sl < nc) keys[rank] = mine;
        H.sync();
    } else if (nc <= 32) {
        half_sort_e<2>(keys, nc, H);
    } else if (NT >= 4 && nc <= 64) {
        half_sort_e<(NT >= 4 ? 4 : 2)>(keys, nc, H);
    } else if (NT >= 6 && nc <= 128) {
        half_sort_e<(NT >= 6 ? 8 : 2)>(keys, nc, H);
    } else {
        half_sort_e<(NT >= 10 ? 16 : 2)>(keys, nc, H);
    }
}

// continues a visited insert whose first 16 probe slots were all taken
static __device__ __noinline__ void half_visited_insert_from(uint32_t* tab, uint32_t mask, uint32_t id,
                                                             uint32_t h, int sl, uint32_t hmask) {
    for (uint32_t probe = 16; probe <= mask; probe += 16) {
        const uint32_t s = (h + probe + (uint32_t)sl) & mask;
        const uint32_t empty = __ballot_sync(hmask, tab[s] == kEmptyId) & hmask;
        if (empty) {
            if ((uint32_t)sl == (uint32_t)(__ffs(empty) - 1) % 16u) tab[s] = id;
            break;
        }
    }
}

// ---- the paired persistent search ---------------------------------------------------------
// Each half pulls queries from A.queue (over A.order) until the queue is drained. UNI: one
// (Ls, k) for the launch (A.Ls / A.k); otherwise per query (A.ls_arr / A.k_arr).
template <int CH, bool Signed, int FW, bool UNI>
__device__ void flat_pair_run(const FlatArgs& A, unsigned char* wmem, uint32_t* gfilter,
                              uint32_t* gvisited, int lane) {
    constexpr int NT = 2 * CH;  // 16-entry chunks of an adjacency row
    constexpr bool SFILT = FW > 0;
    constexpr FlatLayout K = make_flat_layout(0u, 32u * CH, (uint32_t)FW, 0u);
    const HalfWarp H(lane);
    const int sl = H.sl;
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
    const int4* q4 = reinterpret_cast<const int4*>(qwords);
    const int64_t limit = A.limit;
    const int deg_lim = (int)A.deg_lim;
    const bool nir = A.norm_in_row != 0;

    // this half's query (u < 0: none in progress)
    uint32_t q = 0, Ls = 0, k = 0, qid = 0, fmask = 0, vmask = 0, vshift = 0;
    int max_visits = 0;
    int32_t qq = 0;
    int fsize = 0, u = -1, u2 = -1, flags = 0, nvis = 0, comps = 0;
    uint32_t pred = kEmptyId;
    uint32_t apred[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) apred[t] = kEmptyId;

    for (;;) {
        // ---- a half without a query takes the next one --------------------------------
        if (u < 0) {
            uint32_t slot = 0;
            if (sl == 0) slot = atomicAdd(A.queue, 1u);
            slot = __shfl_sync(H.mask, slot, H.base);
            if (slot >= A.nq) break;
            q = A.order[slot];
            Ls = UNI ? A.Ls : A.ls_arr[q];
            k = UNI ? A.k : A.k_arr[q];
            qid = A.qbase + q;
            fmask = (1u << flat_filter_bits(Ls)) - 1u;
            const uint32_t vcap = flat_visited_cap(Ls);
            vmask = vcap - 1u;
            vshift = 32u - (uint32_t)ceil_log2_u64(vcap);
            max_visits = (int)(vcap / 2u);
            // query row (zero padded): lane sl fills words sl and sl + 16
            {
                const uint8_t* src = A.queries + (size_t)q * A.qstride;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint32_t wd = (uint32_t)sl + 16u * h;
                    uint32_t wv = 0;
#pragma unroll
                    for (int b = 0; b < 4; b++) {
                        const uint32_t i = 4u * wd + b;
                        const uint32_t v = (i < A.dim) ? (uint32_t)src[i] : 0u;
                        wv |= v << (8 * b);
                    }
                    qwords[wd] = wv;
                }
            }
            // clear this query's tables (sizes are multiples of 64 words, 16-byte aligned)
            {
                const uint4 e4 = make_uint4(kEmptyId, kEmptyId, kEmptyId, kEmptyId);
                uint4* f4 = reinterpret_cast<uint4*>(filter);
                for (uint32_t i = sl; i < (fmask + 1u) / 4u; i += 16) f4[i] = e4;
                uint4* v4 = reinterpret_cast<uint4*>(vtab);
                for (uint32_t i = sl; i < vcap / 4u; i += 16) v4[i] = e4;
                if (sl < (int)(kVisitedBits / 128u)) reinterpret_cast<uint4*>(vbits)[sl] = make_uint4(0, 0, 0, 0);
            }
            H.sync();
            {
                int32_t s = partial_sq<Signed>(q4[sl & 7]);
#pragma unroll
                for (int off = 4; off > 0; off >>= 1) s += __shfl_xor_sync(H.mask, s, off, 8);
                qq = s;
            }
            // start point: F = {(d(q, start), start)}, one distance
            if (sl == 0) pend[0] = A.start;
            H.sync();
            half_row_distances<Signed>(A.rows, pend, pdist, 1, q4, qq, A.dim, nir, H);
            if (sl == 0) {
                fkey[0] = pack_key(pdist[0], A.start);
                fvis[0] = 0;
            }
            H.sync();
            fsize = 1;
            u = 0;
            u2 = -1;
            flags = 0;
            nvis = 0;
            comps = 1;
            pred = kEmptyId;
        }

        // ---- one expansion (flat_query's loop body) ---------------------------------------
        const uint64_t cur_key = fkey[u];
        const uint32_t cur = key_id(cur_key);
        uint32_t a[NT];
        if (cur == pred) {
#pragma unroll
            for (int t = 0; t < NT; t++) a[t] = apred[t];
        } else {
            const uint32_t* row = A.adj + (size_t)cur * A.gs;
#pragma unroll
            for (int t = 0; t < NT; t++) {
                const int j = t * 16 + sl;
                a[t] = (j < deg_lim) ? __ldg(row + j) : kEmptyId;
            }
        }
        if (sl == 0) fvis[u] = 1;
        const uint32_t vhome = visited_home(cur, vshift);
        const uint32_t vslot = (vhome + (uint32_t)sl) & vmask;
        const uint32_t vprobe = vtab[vslot];
        if (sl == 0) {
            const uint32_t b = visited_bit(cur);
            vbits[b >> 5] |= 1u << (b & 31u);
        }
        nvis++;
        const bool over = nvis > max_visits;
        if (over) {
            flags |= PGB_FLAG_OVERFLOW;
        } else {
            const int32_t cutoff = (fsize < (int)Ls) ? INT_MAX : key_dist(fkey[fsize - 1]);
            const uint32_t lt = H.lt, gt = H.gt;

            // ---- lossy filter in row order -> pending ids --------------------------------
            int np = 0;
            if (SFILT) {
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    const uint32_t x = a[t];
                    const bool part = x != kEmptyId && !(A.excl && x == qid);
                    const uint32_t slot =
                        part ? (uint32_t)(hash64_2(x) & fmask) : (0x80000000u | (uint32_t)(t * 16 + sl));
                    const uint32_t peers = __match_any_sync(H.mask, slot);
                    const uint32_t before = peers & lt;
                    const int src = before ? 31 - __clz(before) : lane;
                    const uint32_t prev = __shfl_sync(H.mask, x, src);
                    bool seen;
                    if (before) seen = part && prev == x;
                    else seen = part && filter[slot] == x;
                    H.sync();
                    if (part && (peers & gt) == 0) filter[slot] = x;
                    const bool pass = part && !seen;
                    const uint32_t m = H.ballot(pass);
                    if (pass) pend[np + __popc(m & lt)] = x;
                    np += __popc(m);
                    H.sync();
                }
            } else {
                uint32_t slot[NT], mem[NT];
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    const uint32_t x = a[t];
                    const bool part = x != kEmptyId && !(A.excl && x == qid);
                    slot[t] = part ? (uint32_t)(hash64_2(x) & fmask)
                                   : (0x80000000u | (uint32_t)(t * 16 + sl));
                    mem[t] = part ? filter[slot[t]] : kEmptyId;
                }
                uint32_t* sslot = reinterpret_cast<uint32_t*>(ckey);  // scratch: slots of row
                uint32_t* sid = sslot + 16 * NT;                        // and ids
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    const uint32_t x = a[t];
                    const bool part = x != kEmptyId && !(A.excl && x == qid);
                    const uint32_t peers = __match_any_sync(H.mask, slot[t]);
                    const uint32_t before = peers & lt;
                    const int src = before ? 31 - __clz(before) : lane;
                    const uint32_t prev = __shfl_sync(H.mask, x, src);
                    bool seen;
                    if (before) {
                        seen = part && prev == x;
                    } else {
                        seen = part && mem[t] == x;
                        if (part)
                            for (int p = t * 16 - 1; p >= 0; p--)
                                if (sslot[p] == slot[t]) {
                                    seen = sid[p] == x;
                                    break;
                                }
                    }
                    H.sync();
                    sslot[t * 16 + sl] = slot[t];
                    sid[t * 16 + sl] = x;
                    if (part && (peers & gt) == 0) filter[slot[t]] = x;
                    const bool pass = part && !seen;
                    const uint32_t m = H.ballot(pass);
                    if (pass) pend[np + __popc(m & lt)] = x;
                    np += __popc(m);
                    H.sync();
                }
            }
            comps += np;

            // ---- distances --------------------------------------------------------------
            half_row_distances<Signed>(A.rows, pend, pdist, np, q4, qq, A.dim, nir, H);

            // ---- candidates under the cutoff, in arrival order ---------------------------
            int nc = 0;
            for (int base = 0; base < np; base += 16) {
                const int i = base + sl;
                const bool c = i < np && pdist[i] < cutoff;
                const uint32_t m = H.ballot(c);
                if (c) ckey[nc + __popc(m & lt)] = pack_key(pdist[i], pend[i]);
                nc += __popc(m);
            }
            H.sync();
            uint64_t best = (u2 >= 0 && u2 < fsize) ? fkey[u2] : kEmptyKey;

            int unew = u;
            int ne = 0;
            if (nc > 0) {
                half_sort_keys<NT>(ckey, nc, H);
                // ---- multiset set_union: copy `rep` of a key enters iff rep >= copies in F
                bool found = false;
                for (int base = 0; base < nc; base += 16) {
                    const int i = base + sl;
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
                    const uint32_t m = H.ballot(enter);
                    const int pos = hi + ne + __popc(m & lt);
                    const bool keep = enter && pos < (int)Ls;
                    const uint32_t mk = H.ballot(keep);
                    const uint32_t mnv = H.ballot(keep && !vis);
                    if (mnv && !found) {
                        const uint64_t k0 = __shfl_sync(H.mask, key, __ffs(mnv) - 1);
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
                H.sync();
            }
            pred = (best != kEmptyKey) ? key_id(best) : kEmptyId;
            if (pred != kEmptyId) {
                const uint32_t* prow = A.adj + (size_t)pred * A.gs;
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    const int j = t * 16 + sl;
                    apred[t] = (j < deg_lim) ? __ldg(prow + j) : kEmptyId;
                }
            }

            int from;
            if (ne > 0) {
                unew = u + lower_bound_key(ekey, ne, cur_key);
                const int first = epos[0];
                for (int top = fsize - 1; top >= first; top -= 16) {
                    const int i = top - sl;
                    const bool act = i >= first;
                    uint64_t key = 0;
                    uint8_t vis = 0;
                    int np2 = 0;
                    if (act) {
                        key = fkey[i];
                        vis = fvis[i];
                        np2 = i + lower_bound_key(ekey, ne, key);
                    }
                    H.sync();
                    if (act && np2 < (int)Ls) {
                        fkey[np2] = key;
                        fvis[np2] = vis;
                    }
                    H.sync();
                }
                int minpos = INT_MAX;
                for (int j = sl; j < ne; j += 16) {
                    fkey[epos[j]] = ekey[j];
                    fvis[epos[j]] = evis[j];
                    if (!evis[j]) minpos = min(minpos, epos[j]);
                }
                H.sync();
                fsize = min((int)Ls, fsize + ne);

                // ---- cut (only a changed frontier can need one) -------------------------
                if (fsize > (int)k) {
                    const float thr = (float)(A.cut * (double)key_dist(fkey[k]));
                    const uint64_t last = fkey[fsize - 1];
                    const float dl = (float)key_dist(last);
                    const bool any_cut = thr < dl || (thr == dl && 0u < key_id(last));
                    int newsize = fsize;
                    for (int base = 0; any_cut && base < fsize; base += 16) {
                        const int i = base + sl;
                        bool after = false;
                        if (i < fsize) {
                            const uint64_t e = fkey[i];
                            const float de = (float)key_dist(e);
                            after = thr < de || (thr == de && 0u < key_id(e));
                        }
                        const uint32_t m = H.ballot(after);
                        if (m) {
                            newsize = base + H.first(m);
                            break;
                        }
                    }
                    fsize = newsize;
                }
                minpos = (int)__reduce_min_sync(H.mask, (unsigned)minpos);
                from = min(unew, minpos);
            } else {
                from = (u2 >= 0) ? u2 : u + 1;
            }

            // ---- next unvisited ------------------------------------------------------------
            u = -1;
            u2 = -1;
            for (int base = from; base < fsize; base += 16) {
                const int i = base + sl;
                const bool un = i < fsize && !fvis[i];
                const uint32_t m = H.ballot(un) >> H.base;
                if (m) {
                    u = base + __ffs(m) - 1;
                    const uint32_t rest = m & (m - 1);
                    u2 = rest ? base + __ffs(rest) - 1 : -1;
                    break;
                }
            }
            // second half of the visited insert
            {
                const uint32_t empty = H.ballot(vprobe == kEmptyId);
                if (empty) {
                    if (lane == __ffs(empty) - 1) vtab[vslot] = cur;
                } else {
                    half_visited_insert_from(vtab, vmask, cur, vhome, sl, H.mask);
                }
            }
            if (u >= 0 && key_id(fkey[u]) == pred) {
#pragma unroll
                for (int t = 0; t < NT; t++)
                    if (apred[t] != kEmptyId) prefetch_row_l2(A.rows + (size_t)apred[t] * kRowBytes);
            }
            H.sync();
        }

        // ---- a finished query: first k of the frontier, counts, flags ---------------------
        if (over || u < 0 || (int64_t)nvis >= limit) {
            if (fsize < (int)k) flags |= PGB_FLAG_SHORT;
            uint32_t* oid = A.ids + (size_t)q * A.out_stride;
            int32_t* od = A.dists + (size_t)q * A.out_stride;
            for (uint32_t j = sl; j < k; j += 16) {
                const bool have = (int)j < fsize;
                const uint64_t e = have ? fkey[j] : 0;
                oid[j] = have ? key_id(e) : kEmptyId;
                od[j] = have ? key_dist(e) : INT_MAX;
            }
            if (sl == 0 && A.stats) {
                pgb_query_stats s;
                s.dist_comps = comps;
                s.expansions = nvis;
                s.flags = flags;
                s.reserved = 0;
                A.stats[q] = s;
            }
            H.sync();
            u = -1;
        }
    }
}

}  // namespace pgb
