// oracle.cpp -- CPU restatement of the graph beam search path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA path: only the
// tests, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg load it.
// The product (libpgb.so) never links, calls or falls back to it.
//
// It restates, sequentially and with plain STL containers, the semantics that the
// reference's CUDA kernels reproduce from ParlayANN (commit 45587ba, absent here):
//   * flat beam search      : cuda/busqueda.cu:151-499   (kernelBusqueda)
//   * filter / hashes / order: cuda/utiles_gpu.cuh:12-36 (hash64_2, hash64, menor)
//   * exact visited multiset: cuda/busqueda.cu:57-82, overflow rule :205-208
//   * HNSW layered search   : cuda/busqueda_hnsw.cu:215-456 (kernelHnsw)
//   * filter sizes          : cuda/busqueda.cu:536-540, cuda/busqueda_hnsw.cu:556-559
//   * distance              : cuda/lectores.cpp:172-179 (distanciaCPU)
//   * recall with ties      : cuda/evaluacion.cpp:56-80 (calcularRecall)
// The flat search is written the way ParlayANN writes beam_search (std::set_union /
// std::set_difference on (dist, id)-sorted vectors) so that the multiset semantics the
// reference emulates with copy counts come out of the STL algorithms themselves.
//
// Parity status: pinned against outputs of the reference's own kernels (rebuilt for
// sm_100a from the reference sources by oracle/Makefile into oracle/_ref/) on the
// committed fixtures in tests/golden/.

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <unordered_set>
#include <vector>

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kFlagOverflow = 1;  // cuda/busqueda.cuh:14
constexpr int kFlagShort = 2;     // cuda/busqueda.cuh:15

// parlaylib hash64_2 (cuda/utiles_gpu.cuh:12-17)
inline uint64_t hash64_2(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// parlaylib hash64 (cuda/utiles_gpu.cuh:21-31); HNSW uses it for entry points only
inline uint64_t hash64(uint64_t u) {
    uint64_t v = u * 3935559000370003845ull + 2691343689449507681ull;
    v ^= v >> 21;
    v ^= v << 37;
    v ^= v >> 4;
    v *= 4768777513237032717ull;
    v ^= v << 20;
    v ^= v >> 41;
    v ^= v << 5;
    return v;
}

inline int ceil_log2(uint64_t x) {
    int b = 0;
    while ((1ull << b) < x) b++;
    return b;
}

inline uint64_t next_pow2(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

struct Pair {
    uint32_t id;
    int32_t d;
};

// (dist, id) order (cuda/utiles_gpu.cuh:34-36)
inline bool less_pair(const Pair& a, const Pair& b) {
    return a.d < b.d || (a.d == b.d && a.id < b.id);
}

struct Vectors {
    const uint8_t* data;  // n rows of `stride` bytes, first `dim` bytes meaningful
    uint32_t dim;
    uint32_t stride;
    int is_signed;
    const uint8_t* row(uint32_t i) const { return data + (size_t)i * stride; }
};

// squared L2 in exact integer arithmetic (cuda/lectores.cpp:172-179)
inline int32_t sq_l2(const uint8_t* a, const uint8_t* b, uint32_t dim, int is_signed) {
    int32_t s = 0;
    if (is_signed) {
        const int8_t* x = reinterpret_cast<const int8_t*>(a);
        const int8_t* y = reinterpret_cast<const int8_t*>(b);
        for (uint32_t i = 0; i < dim; i++) {
            int32_t t = (int32_t)x[i] - (int32_t)y[i];
            s += t * t;
        }
    } else {
        for (uint32_t i = 0; i < dim; i++) {
            int32_t t = (int32_t)a[i] - (int32_t)b[i];
            s += t * t;
        }
    }
    return s;
}

template <typename F>
void parallel_for(uint32_t n, int nthreads, F&& f) {
    if (nthreads <= 1 || n < 2) {
        for (uint32_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++)
        pool.emplace_back([&]() {
            for (;;) {
                uint32_t i = next.fetch_add(16);
                if (i >= n) break;
                uint32_t e = std::min(n, i + 16);
                for (; i < e; i++) f(i);
            }
        });
    for (auto& th : pool) th.join();
}

struct FlatParams {
    uint32_t k, Ls;
    double cut;
    int64_t limit;  // <= 0: no limit (n)
    uint32_t degree_limit;
    int exclude_query_id;
    uint32_t query_id_base;
    uint32_t start;
};

// One query of ParlayANN beam_search as restated by cuda/busqueda.cu:151-499.
void flat_one(const Vectors& base, uint32_t n, const uint64_t* offsets, const uint32_t* degrees,
              const uint32_t* edges, const uint8_t* q, uint32_t qid, const FlatParams& P,
              uint32_t* ids_out, int32_t* dists_out, int32_t* comps_out, int32_t* exps_out,
              int32_t* flags_out) {
    const uint32_t Ls = P.Ls;
    // filter size (cuda/busqueda.cu:536-538): bits = max(10, ceil(log2(Ls*Ls)) - 2)
    const int bits = std::max(10, ceil_log2((uint64_t)Ls * Ls) - 2);
    const uint32_t mask = (1u << bits) - 1;
    std::vector<uint32_t> filter((size_t)mask + 1, kEmpty);
    // lossy "has been seen" filter; the start point is not inserted (busqueda.cu:166-173)
    auto has_been_seen = [&](uint32_t a) {
        uint32_t s = (uint32_t)(hash64_2(a) & mask);
        if (filter[s] == a) return true;
        filter[s] = a;
        return false;
    };
    // visited-table overflow rule (busqueda.cu:540, :205-208)
    const uint64_t max_visits = next_pow2(8ull * Ls + 128) / 2;
    const int64_t limit = (P.limit <= 0) ? (int64_t)n : P.limit;

    std::vector<Pair> frontier{{P.start, sq_l2(q, base.row(P.start), base.dim, base.is_signed)}};
    std::vector<Pair> visited;  // sorted multiset
    std::vector<Pair> unvisited{frontier[0]};
    std::vector<Pair> candidates, merged;
    std::vector<uint32_t> keep;
    int64_t comps = 1, num_visited = 0;
    int flags = 0;

    while (!unvisited.empty() && num_visited < limit) {
        const Pair current = unvisited[0];
        visited.insert(std::upper_bound(visited.begin(), visited.end(), current, less_pair),
                       current);
        num_visited++;
        if ((uint64_t)num_visited > max_visits) {
            flags |= kFlagOverflow;
            break;
        }
        keep.clear();
        const uint32_t deg = degrees[current.id];
        const uint32_t ne = std::min(deg, P.degree_limit);
        const uint32_t* row = edges + offsets[current.id];
        for (uint32_t i = 0; i < ne; i++) {
            uint32_t a = row[i];
            // the wrapper's `a == p.id()` test compares against the QUERY index
            if (P.exclude_query_id && a == qid) continue;
            if (has_been_seen(a)) continue;
            keep.push_back(a);
        }
        const int32_t cutoff = (frontier.size() < Ls) ? INT_MAX : frontier.back().d;
        candidates.clear();
        for (uint32_t a : keep) {
            int32_t d = sq_l2(q, base.row(a), base.dim, base.is_signed);
            comps++;
            if (d >= cutoff) continue;
            candidates.push_back({a, d});
        }
        std::sort(candidates.begin(), candidates.end(), less_pair);
        merged.clear();
        std::set_union(frontier.begin(), frontier.end(), candidates.begin(), candidates.end(),
                       std::back_inserter(merged), less_pair);
        if (merged.size() > Ls) merged.resize(Ls);
        // cut (busqueda.cu:445-464): threshold computed in double, held in float,
        // compared in (float dist, id) order against the pair {0, thr}
        if (P.k > 0 && merged.size() > P.k) {
            const float thr = (float)(P.cut * (double)merged[P.k].d);
            auto it = std::upper_bound(merged.begin(), merged.end(), thr,
                                       [](float t, const Pair& e) {
                                           float de = (float)e.d;
                                           return t < de || (t == de && 0u < e.id);
                                       });
            merged.resize((size_t)(it - merged.begin()));
        }
        frontier.swap(merged);
        unvisited.clear();
        std::set_difference(frontier.begin(), frontier.end(), visited.begin(), visited.end(),
                            std::back_inserter(unvisited), less_pair);
    }
    if (frontier.size() < P.k) flags |= kFlagShort;
    for (uint32_t j = 0; j < P.k; j++) {
        ids_out[j] = (j < frontier.size()) ? frontier[j].id : kEmpty;
        dists_out[j] = (j < frontier.size()) ? frontier[j].d : INT_MAX;
    }
    *comps_out = (int32_t)comps;
    *exps_out = (int32_t)num_visited;
    *flags_out = flags;
}

struct HnswParams {
    uint32_t k, Ls;
    int64_t limit;  // layer-0 limit_eval; <= 0 or >= n: n
};

struct HnswGraph {
    uint32_t n;
    const uint32_t* levels;      // top level of each node
    const uint32_t* node_point;  // base point stored by each node
    const uint64_t* first_list;  // index of node i's level-0 list in list_offsets
    const uint64_t* list_offsets;
    const uint32_t* list_sizes;
    const uint32_t* ids;
    const uint32_t* entries;
    uint32_t num_entries;
};

// One query of ParlayANN HNSW search as restated by cuda/busqueda_hnsw.cu:215-456.
void hnsw_one(const Vectors& base, const HnswGraph& g, const uint8_t* q, const HnswParams& P,
              uint32_t* ids_out, int32_t* dists_out, int32_t* comps_out, int32_t* exps_out,
              int32_t* flags_out) {
    auto dist_node = [&](uint32_t node) {
        return sq_l2(q, base.row(g.node_point[node]), base.dim, base.is_signed);
    };
    const uint32_t Ls = P.Ls;
    // layer-0 filter bits (busqueda_hnsw.cu:556-557)
    const int bits0 = (Ls > 2) ? ceil_log2(Ls) * 2 - 2 : 2;
    // is_inw overflow rule (busqueda_hnsw.cu:559, :428-431)
    const uint64_t cap_inw = next_pow2(32ull * Ls + 2048);
    const uint64_t limit0 = (P.limit > 0 && (uint64_t)P.limit < g.n) ? (uint64_t)P.limit : g.n;
    const int top = (int)g.levels[g.entries[0]];

    std::vector<uint32_t> eps(g.entries, g.entries + g.num_entries);
    std::vector<Pair> W;     // workset, (dist, id) order
    std::vector<Pair> cand;  // ordered by dist only, distinct dists
    int64_t comps = 0, exps = 0;
    int flags = 0;

    auto cand_insert = [&](int32_t d, uint32_t id) {
        auto it = std::lower_bound(cand.begin(), cand.end(), d,
                                   [](const Pair& e, int32_t x) { return e.d < x; });
        if (it != cand.end() && it->d == d) return;  // std::set by distance
        cand.insert(it, Pair{id, d});
    };
    auto w_insert = [&](int32_t d, uint32_t id) {
        Pair p{id, d};
        W.insert(std::upper_bound(W.begin(), W.end(), p, less_pair), p);
    };

    for (int layer = top; layer >= 0; layer--) {
        const uint32_t ef = (layer > 0) ? 1 : Ls;
        const int bits = (layer > 0) ? 2 : bits0;
        const uint32_t mask = (1u << bits) - 1;
        const uint64_t limit = (layer > 0) ? UINT64_MAX : limit0;
        std::vector<uint32_t> vis((size_t)mask + 1, kEmpty);
        std::unordered_set<uint32_t> inw;
        cand.clear();
        W.clear();
        uint64_t inserted = 0;
        for (uint32_t pe : eps) {
            vis[hash64(pe) & mask] = pe;
            int32_t d = dist_node(pe);
            inw.insert(pe);
            cand_insert(d, pe);
            w_insert(d, pe);  // not trimmed
            comps++;
            inserted++;
        }
        uint64_t cnt_eval = 0;
        while (!cand.empty()) {
            if (cand.front().d > W.back().d) break;
            if (++cnt_eval > limit) break;
            const uint32_t u = cand.front().id;
            cand.erase(cand.begin());
            exps++;
            const uint64_t li = g.first_list[u] + (uint64_t)layer;
            const uint32_t* nb = g.ids + g.list_offsets[li];
            const uint32_t deg = g.list_sizes[li];
            std::vector<uint32_t> pend;
            for (uint32_t i = 0; i < deg; i++) {
                uint32_t pv = nb[i];
                uint32_t h = (uint32_t)(hash64_2(pv) & mask);
                if (vis[h] == pv) continue;
                vis[h] = pv;
                pend.push_back(pv);
            }
            comps += (int64_t)pend.size();
            for (uint32_t pv : pend) {
                int32_t d = dist_node(pv);
                if (!(W.size() < ef || d < W.back().d)) continue;
                if (!inw.insert(pv).second) continue;
                cand_insert(d, pv);
                w_insert(d, pv);
                if (W.size() > ef) W.pop_back();
                if (cand.size() > ef) cand.pop_back();
                inserted++;
            }
            if (inserted > cap_inw / 2) {
                flags |= kFlagOverflow;
                break;
            }
        }
        if (layer > 0) eps.assign(1, W.back().id);
    }
    if (W.size() < P.k) flags |= kFlagShort;
    for (uint32_t j = 0; j < P.k; j++) {
        ids_out[j] = (j < W.size()) ? g.node_point[W[j].id] : kEmpty;
        dists_out[j] = (j < W.size()) ? W[j].d : INT_MAX;
    }
    *comps_out = (int32_t)comps;
    *exps_out = (int32_t)exps;
    *flags_out = flags;
}

}  // namespace

extern "C" {

// Flat-graph beam search over a CSR graph (ParlayANN Graph layout: degrees + edges).
// base/queries: rows of `*_stride` bytes whose first `dim` bytes are the vector.
int oracle_flat_search(const uint8_t* base, uint32_t n, uint32_t dim, uint32_t base_stride,
                       int is_signed, const uint32_t* degrees, const uint32_t* edges,
                       const uint8_t* queries, uint32_t nq, uint32_t query_stride, uint32_t k,
                       uint32_t Ls, double cut, int64_t limit, uint32_t degree_limit,
                       int exclude_query_id, uint32_t query_id_base, uint32_t start,
                       uint32_t* ids, int32_t* dists, int32_t* comps, int32_t* exps,
                       int32_t* flags, int nthreads) {
    if (!base || !degrees || !edges || !queries || n == 0 || Ls == 0 || start >= n) return 1;
    std::vector<uint64_t> offsets((size_t)n + 1, 0);
    for (uint32_t i = 0; i < n; i++) offsets[i + 1] = offsets[i] + degrees[i];
    Vectors V{base, dim, base_stride, is_signed};
    FlatParams P{k, Ls, cut, limit, degree_limit ? degree_limit : UINT32_MAX,
                 exclude_query_id, query_id_base, start};
    parallel_for(nq, nthreads, [&](uint32_t i) {
        flat_one(V, n, offsets.data(), degrees, edges, queries + (size_t)i * query_stride,
                 query_id_base + i, P, ids + (size_t)i * k, dists + (size_t)i * k, comps + i,
                 exps + i, flags + i);
    });
    return 0;
}

// HNSW search. Lists are laid out node by node, levels 0..levels[i] for node i
// (the order of the HNSW v3 file, cuda/hnsw.h:11-16); list_sizes has one entry per list.
int oracle_hnsw_search(const uint8_t* base, uint32_t dim, uint32_t base_stride, int is_signed,
                       uint32_t n, const uint32_t* levels, const uint32_t* node_point,
                       const uint32_t* list_sizes, const uint32_t* ids_flat,
                       const uint32_t* entries, uint32_t num_entries, const uint8_t* queries,
                       uint32_t nq, uint32_t query_stride, uint32_t k, uint32_t Ls,
                       int64_t limit, uint32_t* ids, int32_t* dists, int32_t* comps,
                       int32_t* exps, int32_t* flags, int nthreads) {
    if (!base || n == 0 || num_entries == 0 || Ls == 0) return 1;
    std::vector<uint64_t> first_list(n), list_offsets;
    uint64_t nl = 0, off = 0;
    for (uint32_t i = 0; i < n; i++) {
        first_list[i] = nl;
        for (uint32_t l = 0; l <= levels[i]; l++) {
            list_offsets.push_back(off);
            off += list_sizes[nl];
            nl++;
        }
    }
    HnswGraph g{n, levels, node_point, first_list.data(), list_offsets.data(), list_sizes,
                ids_flat, entries, num_entries};
    Vectors V{base, dim, base_stride, is_signed};
    HnswParams P{k, Ls, limit};
    parallel_for(nq, nthreads, [&](uint32_t i) {
        hnsw_one(V, g, queries + (size_t)i * query_stride, P, ids + (size_t)i * k,
                 dists + (size_t)i * k, comps + i, exps + i, flags + i);
    });
    return 0;
}

// recall@k with distance ties (cuda/evaluacion.cpp:56-80)
double oracle_recall(const uint32_t* gt_ids, const float* gt_dists, uint32_t nq, uint32_t gt_k,
                     const uint32_t* ids, uint32_t k) {
    long long total = 0;
    for (uint32_t q = 0; q < nq; q++) {
        const uint32_t* truth = gt_ids + (size_t)q * gt_k;
        const float* dtruth = gt_dists + (size_t)q * gt_k;
        uint32_t end = gt_k;
        if (gt_k != k) {
            float ref = dtruth[k - 1];
            for (uint32_t i = k; i < gt_k; i++)
                if (!(std::fabs(ref - dtruth[i]) < 1e-6f)) {
                    end = i;
                    break;
                }
        }
        std::vector<uint32_t> mine(ids + (size_t)q * k, ids + (size_t)(q + 1) * k);
        std::sort(mine.begin(), mine.end());
        mine.erase(std::unique(mine.begin(), mine.end()), mine.end());
        for (uint32_t x : mine)
            if (std::find(truth, truth + end, x) != truth + end) total++;
    }
    return (double)total / nq / k;
}

// int32 squared L2 of explicit (query, point) pairs: the distance known-answer
// procedure of cuda/paso1_carga.cu:54-123.
void oracle_pair_distances(const uint8_t* base, uint32_t base_stride, const uint8_t* queries,
                           uint32_t query_stride, uint32_t dim, int is_signed,
                           const uint32_t* pairs, uint64_t npairs, int32_t* out) {
    for (uint64_t i = 0; i < npairs; i++)
        out[i] = sq_l2(queries + (size_t)pairs[2 * i] * query_stride,
                       base + (size_t)pairs[2 * i + 1] * base_stride, dim, is_signed);
}

}  // extern "C"
