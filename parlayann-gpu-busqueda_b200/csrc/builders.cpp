// builders.cpp -- CPU graph builders for the four graph families the search serves.
//
// The reference only searches graphs that ParlayANN built on the CPU
// (ParlayANN-ppopp24 @45587ba, not vendored; reference cpu_baseline/setup.sh:45-52).
// These are this project's own builders, written from the published algorithm
// descriptions: Vamana (DiskANN, NeurIPS'19) with ParlayANN's batch insertion by
// prefix doubling (PPoPP'24), HCNNG (Munoz et al., Pattern Recognition'19),
// NN-descent initialised from cluster trees (Dong et al., WWW'11; PyNNDescent), and
// HNSW (Malkov & Yashunin, TPAMI'18). Search parity never depends on them: the oracle
// and the GPU read the same graph file.
//
// Every builder is deterministic for a given seed and independent of the thread
// count: each batch searches a read-only snapshot of the graph and edge merges are
// applied in a fixed (sorted) order.

#include <cmath>
#include <cstdio>
#include <memory>
#include <mutex>
#include <numeric>

#include "builders.h"

namespace pgb {
namespace {

// Adjacency with a fixed number of slots per node.
struct Adjacency {
    uint32_t n = 0, slots = 0;
    uint32_t* adj = nullptr;  // n * slots
    uint32_t* deg = nullptr;  // n
    const uint32_t* row(uint32_t i) const { return adj + (size_t)i * slots; }
    uint32_t* row(uint32_t i) { return adj + (size_t)i * slots; }
};

// Per-thread scratch: epoch-stamped membership over all n points.
struct Scratch {
    std::vector<uint32_t> mark;
    uint32_t epoch = 0;
    std::vector<DistId> frontier;
    std::vector<uint8_t> expanded;
    void begin(uint32_t n) {
        if (mark.size() != n) {
            mark.assign(n, 0);
            epoch = 0;
        }
        if (++epoch == 0) {
            std::fill(mark.begin(), mark.end(), 0);
            epoch = 1;
        }
    }
    bool test_and_set(uint32_t i) {
        if (mark[i] == epoch) return true;
        mark[i] = epoch;
        return false;
    }
};

// Greedy beam search used while building: returns every expanded node with its distance.
void build_search(const HostVectors& V, const Adjacency& G, const uint8_t* q,
                  const std::vector<uint32_t>& starts, uint32_t L, Scratch& s,
                  std::vector<DistId>& visited) {
    visited.clear();
    s.begin(V.n);
    auto& F = s.frontier;
    auto& E = s.expanded;
    F.clear();
    E.clear();
    for (uint32_t st : starts) {
        if (s.test_and_set(st)) continue;
        DistId e{V.dist_to(q, st), st};
        auto it = std::upper_bound(F.begin(), F.end(), e);
        E.insert(E.begin() + (it - F.begin()), 0);
        F.insert(it, e);
    }
    if (F.size() > L) {
        F.resize(L);
        E.resize(L);
    }
    size_t cur = 0;
    for (;;) {
        while (cur < F.size() && E[cur]) cur++;
        if (cur >= F.size()) break;
        E[cur] = 1;
        const DistId u = F[cur];
        visited.push_back(u);
        const uint32_t* r = G.row(u.id);
        const uint32_t dg = G.deg[u.id];
        for (uint32_t j = 0; j < dg; j++) {
            uint32_t nb = r[j];
            if (s.test_and_set(nb)) continue;
            int32_t d = V.dist_to(q, nb);
            if (F.size() == L && !(d < F.back().d)) continue;
            DistId e{d, nb};
            auto it = std::upper_bound(F.begin(), F.end(), e);
            size_t pos = (size_t)(it - F.begin());
            F.insert(it, e);
            E.insert(E.begin() + pos, 0);
            if (F.size() > L) {
                F.pop_back();
                E.pop_back();
            }
            if (pos < cur) cur = pos;
        }
    }
}

// RobustPrune (DiskANN): keep c unless an already kept o has alpha * d(o, c) <= d(p, c).
void robust_prune(const HostVectors& V, uint32_t p, std::vector<DistId>& cand, float alpha,
                  uint32_t R, std::vector<uint32_t>& out) {
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end(),
                           [](const DistId& a, const DistId& b) { return a.id == b.id; }),
               cand.end());
    out.clear();
    for (const DistId& c : cand) {
        if (out.size() >= R) break;
        if (c.id == p) continue;
        bool keep = true;
        for (uint32_t o : out)
            if (alpha * (float)V.dist(o, c.id) <= (float)c.d) {
                keep = false;
                break;
            }
        if (keep) out.push_back(c.id);
    }
}

std::vector<uint32_t> permutation(uint32_t n, uint64_t seed) {
    std::vector<uint32_t> p(n);
    std::iota(p.begin(), p.end(), 0u);
    SplitMix64 rng(seed);
    for (uint32_t i = n; i > 1; i--) std::swap(p[i - 1], p[rng.below(i)]);
    return p;
}

// Adds the reverse of every new edge p -> q of a batch; overfull rows are re-pruned.
void add_reverse_edges(const HostVectors& V, Adjacency& G, const std::vector<uint32_t>& batch,
                       float alpha, uint32_t R, int nthreads) {
    std::vector<std::pair<uint32_t, uint32_t>> pairs;  // (q, p)
    for (uint32_t p : batch) {
        const uint32_t* r = G.row(p);
        for (uint32_t j = 0; j < G.deg[p]; j++) pairs.emplace_back(r[j], p);
    }
    std::sort(pairs.begin(), pairs.end());
    std::vector<size_t> starts;
    for (size_t i = 0; i < pairs.size(); i++)
        if (i == 0 || pairs[i].first != pairs[i - 1].first) starts.push_back(i);
    starts.push_back(pairs.size());
    parallel_for(starts.size() - 1, nthreads, [&](size_t g) {
        thread_local std::vector<DistId> cand;
        thread_local std::vector<uint32_t> out;
        const uint32_t q = pairs[starts[g]].first;
        uint32_t* r = G.row(q);
        uint32_t dg = G.deg[q];
        cand.clear();
        for (uint32_t j = 0; j < dg; j++) cand.push_back({V.dist(q, r[j]), r[j]});
        size_t added = 0;
        for (size_t i = starts[g]; i < starts[g + 1]; i++) {
            uint32_t p = pairs[i].second;
            bool present = false;
            for (uint32_t j = 0; j < dg; j++)
                if (r[j] == p) {
                    present = true;
                    break;
                }
            if (!present && p != q) {
                cand.push_back({V.dist(q, p), p});
                added++;
            }
        }
        if (added == 0) return;
        if (cand.size() <= R) {
            for (size_t j = dg; j < cand.size(); j++) r[j] = cand[j].id;
            G.deg[q] = (uint32_t)cand.size();
        } else {
            robust_prune(V, q, cand, alpha, R, out);
            for (size_t j = 0; j < out.size(); j++) r[j] = out[j];
            for (size_t j = out.size(); j < G.slots; j++) r[j] = kNoNeighbor;
            G.deg[q] = (uint32_t)out.size();
        }
    }, 16);
}

// Random two-pivot partition tree: leaves of at most `leaf` points (HCNNG / NN-descent init).
void cluster_leaves(const HostVectors& V, std::vector<uint32_t>& ids, uint32_t leaf,
                    uint64_t seed, std::vector<std::pair<size_t, size_t>>& leaves) {
    leaves.clear();
    std::vector<std::pair<size_t, size_t>> stack{{0, ids.size()}};
    SplitMix64 rng(seed);
    while (!stack.empty()) {
        auto [b, e] = stack.back();
        stack.pop_back();
        size_t m = e - b;
        if (m <= leaf) {
            leaves.emplace_back(b, e);
            continue;
        }
        uint32_t a = ids[b + rng.below(m)];
        uint32_t c = ids[b + rng.below(m)];
        size_t mid = b;
        if (a != c) {
            // closer to a goes left; partition in place
            std::vector<uint32_t> left, right;
            left.reserve(m);
            right.reserve(m);
            for (size_t i = b; i < e; i++) {
                uint32_t x = ids[i];
                if (V.dist(x, a) <= V.dist(x, c)) left.push_back(x);
                else right.push_back(x);
            }
            std::copy(left.begin(), left.end(), ids.begin() + b);
            std::copy(right.begin(), right.end(), ids.begin() + b + left.size());
            mid = b + left.size();
        }
        if (mid == b || mid == e) mid = b + m / 2;  // degenerate split
        stack.emplace_back(b, mid);
        stack.emplace_back(mid, e);
    }
    std::sort(leaves.begin(), leaves.end());
}

// exact k nearest neighbours of every point of a leaf, within the leaf
void leaf_knn(const HostVectors& V, const uint32_t* pts, size_t m, uint32_t k,
              std::vector<std::vector<DistId>>& knn) {
    knn.assign(m, {});
    uint32_t kk = (uint32_t)std::min<size_t>(k, m - 1);
    std::vector<DistId> row;
    for (size_t i = 0; i < m; i++) {
        row.clear();
        for (size_t j = 0; j < m; j++)
            if (j != i) row.push_back({V.dist(pts[i], pts[j]), pts[j]});
        if (kk < row.size()) {
            std::nth_element(row.begin(), row.begin() + kk, row.end());
            row.resize(kk);
        }
        std::sort(row.begin(), row.end());
        knn[i] = row;
    }
}

struct DisjointSets {
    std::vector<uint32_t> p;
    explicit DisjointSets(size_t m) : p(m) { std::iota(p.begin(), p.end(), 0u); }
    uint32_t find(uint32_t x) {
        while (p[x] != x) x = p[x] = p[p[x]];
        return x;
    }
    bool unite(uint32_t a, uint32_t b) {
        a = find(a);
        b = find(b);
        if (a == b) return false;
        p[a] = b;
        return true;
    }
};

}  // namespace

std::vector<uint32_t> vamana_insertion_order(uint32_t n, uint64_t seed) {
    std::vector<uint32_t> order = permutation(n, seed);
    // point 0 first: it is the entry of every search
    auto it0 = std::find(order.begin(), order.end(), 0u);
    std::rotate(order.begin(), it0, it0 + 1);
    return order;
}

size_t vamana_max_batch(uint32_t n) { return std::max<size_t>(1, (size_t)(0.02 * n)); }

// ---------------------------------------------------------------------------
// Vamana (DiskANN) with prefix-doubling batch insertion. Start point 0, the point the
// search starts from (reference busqueda.cu:166-173).
int build_vamana(const HostVectors& V, uint32_t R, uint32_t L, float alpha, int passes,
                 uint64_t seed, int nthreads, uint32_t* out_deg, uint32_t* out_adj) {
    const uint32_t n = V.n;
    Adjacency G{n, R, out_adj, out_deg};
    std::fill(out_adj, out_adj + (size_t)n * R, kNoNeighbor);
    std::fill(out_deg, out_deg + n, 0u);
    if (n <= 1) return 0;
    const std::vector<uint32_t> order = vamana_insertion_order(n, seed);
    const std::vector<uint32_t> starts{0};
    const size_t max_batch = vamana_max_batch(n);
    for (int pass = 0; pass < passes; pass++) {
        const float a = (passes > 1 && pass == 0) ? 1.0f : alpha;
        size_t pos = (pass == 0) ? 1 : 0;
        size_t batch = 1;
        while (pos < n) {
            size_t end = std::min<size_t>(n, pos + batch);
            std::vector<uint32_t> ids(order.begin() + pos, order.begin() + end);
            std::vector<std::vector<uint32_t>> outs(ids.size());
            parallel_for(ids.size(), nthreads, [&](size_t i) {
                thread_local Scratch s;
                thread_local std::vector<DistId> visited;
                uint32_t p = ids[i];
                build_search(V, G, V.row(p), starts, L, s, visited);
                // in later passes the current out-neighbours stay candidates
                for (uint32_t j = 0; j < G.deg[p]; j++)
                    visited.push_back({V.dist(p, G.row(p)[j]), G.row(p)[j]});
                robust_prune(V, p, visited, a, R, outs[i]);
            }, 1);
            for (size_t i = 0; i < ids.size(); i++) {
                uint32_t p = ids[i];
                uint32_t* r = G.row(p);
                std::fill(r, r + R, kNoNeighbor);
                std::copy(outs[i].begin(), outs[i].end(), r);
                G.deg[p] = (uint32_t)outs[i].size();
            }
            add_reverse_edges(V, G, ids, a, R, nthreads);
            pos = end;
            batch = std::min(batch * 2, max_batch);
        }
    }
    return 0;
}

// ---------------------------------------------------------------------------
// HCNNG: `trees` random cluster trees with leaves of at most `leaf` points; in each
// leaf a degree-bounded minimum spanning tree (Kruskal over the leaf's 10-NN
// candidate edges, node degree <= mst_deg). Edges of all trees are concatenated per
// point, duplicates included, as HCNNG graphs keep them. Row capacity trees*mst_deg.
int build_hcnng(const HostVectors& V, uint32_t trees, uint32_t leaf, uint32_t mst_deg,
                uint64_t seed, int nthreads, uint32_t* out_deg, uint32_t* out_adj) {
    const uint32_t n = V.n;
    const uint32_t slots = trees * mst_deg;
    Adjacency G{n, slots, out_adj, out_deg};
    std::fill(out_adj, out_adj + (size_t)n * slots, kNoNeighbor);
    std::fill(out_deg, out_deg + n, 0u);
    if (n <= 1) return 0;
    std::vector<uint32_t> ids(n);
    std::vector<std::pair<size_t, size_t>> leaves;
    for (uint32_t t = 0; t < trees; t++) {
        std::iota(ids.begin(), ids.end(), 0u);
        cluster_leaves(V, ids, std::max<uint32_t>(leaf, 2), seed * 1000003ull + t, leaves);
        parallel_for(leaves.size(), nthreads, [&](size_t li) {
            auto [b, e] = leaves[li];
            size_t m = e - b;
            if (m < 2) return;
            const uint32_t* pts = ids.data() + b;
            std::vector<std::vector<DistId>> knn;
            leaf_knn(V, pts, m, 10, knn);
            std::vector<std::tuple<int32_t, uint32_t, uint32_t>> edges;
            // local index of each neighbour: map by sorting
            std::vector<std::pair<uint32_t, uint32_t>> idx(m);
            for (size_t i = 0; i < m; i++) idx[i] = {pts[i], (uint32_t)i};
            std::sort(idx.begin(), idx.end());
            auto local_of = [&](uint32_t id) {
                auto it = std::lower_bound(idx.begin(), idx.end(), std::make_pair(id, 0u));
                return it->second;
            };
            for (size_t i = 0; i < m; i++)
                for (const DistId& x : knn[i]) {
                    uint32_t j = local_of(x.id);
                    uint32_t a = (uint32_t)std::min<size_t>(i, j), c = (uint32_t)std::max<size_t>(i, j);
                    edges.emplace_back(x.d, a, c);
                }
            std::sort(edges.begin(), edges.end());
            edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
            DisjointSets ds(m);
            std::vector<uint32_t> degm(m, 0);
            for (auto& [d, a, c] : edges) {
                if (degm[a] >= mst_deg || degm[c] >= mst_deg) continue;
                if (!ds.unite(a, c)) continue;
                degm[a]++;
                degm[c]++;
                uint32_t pa = pts[a], pc = pts[c];
                G.row(pa)[G.deg[pa]++] = pc;
                G.row(pc)[G.deg[pc]++] = pa;
            }
        }, 1);
    }
    return 0;
}

// ---------------------------------------------------------------------------
// NN-descent (PyNNDescent flavour): k-NN lists initialised from `init_trees` cluster
// trees (exact k-NN inside leaves of `leaf` points), refined by local joins over
// neighbours-of-neighbours until fewer than delta*n*K updates, then undirected and
// RobustPrune(alpha)d down to K out-edges.
int build_nndescent(const HostVectors& V, uint32_t K, uint32_t init_trees, uint32_t leaf,
                    float alpha, float delta, uint32_t max_iters, uint64_t seed, int nthreads,
                    uint32_t* out_deg, uint32_t* out_adj) {
    const uint32_t n = V.n;
    std::fill(out_adj, out_adj + (size_t)n * K, kNoNeighbor);
    std::fill(out_deg, out_deg + n, 0u);
    if (n <= 1) return 0;
    std::vector<std::vector<DistId>> knn(n);
    std::vector<std::unique_ptr<std::mutex>> locks(1024);
    for (auto& l : locks) l = std::make_unique<std::mutex>();
    auto merge_into = [&](uint32_t p, const DistId& c) {
        auto& lst = knn[p];
        if (c.id == p) return false;
        for (const DistId& e : lst)
            if (e.id == c.id) return false;
        if (lst.size() >= K && !(c < lst.back())) return false;
        lst.insert(std::upper_bound(lst.begin(), lst.end(), c), c);
        if (lst.size() > K) lst.pop_back();
        return true;
    };
    std::vector<uint32_t> ids(n);
    std::vector<std::pair<size_t, size_t>> leaves;
    // the first tree's leaf neighbours are kept: points of small cluster pieces get
    // neighbours across cluster boundaries there, which the refined k-NN loses
    std::vector<std::vector<DistId>> seed_lists(n);
    for (uint32_t t = 0; t < init_trees; t++) {
        std::iota(ids.begin(), ids.end(), 0u);
        cluster_leaves(V, ids, std::max<uint32_t>(leaf, K + 1), seed * 7919ull + t, leaves);
        parallel_for(leaves.size(), nthreads, [&](size_t li) {
            auto [b, e] = leaves[li];
            size_t m = e - b;
            if (m < 2) return;
            std::vector<std::vector<DistId>> lk;
            leaf_knn(V, ids.data() + b, m, K, lk);
            for (size_t i = 0; i < m; i++) {
                uint32_t p = ids[b + i];
                for (const DistId& c : lk[i]) merge_into(p, c);  // leaves partition the points
                if (t == 0) seed_lists[p] = lk[i];
            }
        }, 1);
    }
    // local joins: candidates are neighbours of neighbours (forward and reverse)
    for (uint32_t it = 0; it < max_iters; it++) {
        std::vector<std::vector<uint32_t>> rev(n);
        for (uint32_t p = 0; p < n; p++)
            for (const DistId& e : knn[p]) rev[e.id].push_back(p);
        std::vector<std::vector<DistId>> next(knn);
        std::atomic<uint64_t> updates{0};
        parallel_for(n, nthreads, [&](size_t pi) {
            uint32_t p = (uint32_t)pi;
            thread_local std::vector<uint32_t> cand;
            cand.clear();
            for (const DistId& e : knn[p]) {
                for (const DistId& f : knn[e.id]) cand.push_back(f.id);
                for (uint32_t r : rev[e.id]) cand.push_back(r);
            }
            for (uint32_t r : rev[p]) cand.push_back(r);
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            auto& lst = next[p];
            uint64_t u = 0;
            for (uint32_t c : cand) {
                if (c == p) continue;
                bool have = false;
                for (const DistId& e : lst)
                    if (e.id == c) {
                        have = true;
                        break;
                    }
                if (have) continue;
                DistId x{V.dist(p, c), c};
                if (lst.size() >= K && !(x < lst.back())) continue;
                lst.insert(std::upper_bound(lst.begin(), lst.end(), x), x);
                if (lst.size() > K) lst.pop_back();
                u++;
            }
            updates += u;
        }, 32);
        knn.swap(next);
        if ((double)updates.load() < (double)delta * n * K) break;
    }
    // undirect and prune: k-NN + reverse k-NN + first-tree leaf neighbours, RobustPrune(alpha)
    std::vector<std::vector<DistId>> rev(n);
    for (uint32_t p = 0; p < n; p++)
        for (const DistId& e : knn[p]) rev[e.id].push_back({e.d, p});
    parallel_for(n, nthreads, [&](size_t pi) {
        uint32_t p = (uint32_t)pi;
        thread_local std::vector<DistId> cand;
        thread_local std::vector<uint32_t> out;
        cand.assign(knn[p].begin(), knn[p].end());
        cand.insert(cand.end(), rev[p].begin(), rev[p].end());
        cand.insert(cand.end(), seed_lists[p].begin(), seed_lists[p].end());
        robust_prune(V, p, cand, alpha, K, out);
        std::copy(out.begin(), out.end(), out_adj + (size_t)p * K);
        out_deg[p] = (uint32_t)out.size();
    }, 64);
    return 0;
}

// ---------------------------------------------------------------------------
// HNSW with batch insertion. Levels l = floor(-ln(U) * ml); level-0 rows hold 2M
// neighbours, upper rows M; neighbour selection by the HNSW heuristic with an alpha
// relaxation (keep c unless d(o, c) < alpha * d(p, c) for a kept o; alpha = 1 is the
// plain heuristic, alpha < 1 keeps more neighbours).

static void hnsw_select(const HostVectors& V, uint32_t p, std::vector<DistId>& cand,
                        float alpha, uint32_t cap, std::vector<uint32_t>& out) {
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end(),
                           [](const DistId& a, const DistId& b) { return a.id == b.id; }),
               cand.end());
    out.clear();
    for (const DistId& c : cand) {
        if (out.size() >= cap) break;
        if (c.id == p) continue;
        bool keep = true;
        for (uint32_t o : out)
            if ((float)V.dist(o, c.id) < alpha * (float)c.d) {
                keep = false;
                break;
            }
        if (keep) out.push_back(c.id);
    }
}

std::vector<uint32_t> hnsw_levels(uint32_t n, float ml, uint64_t seed) {
    std::vector<uint32_t> level(n, 0);
    SplitMix64 rng(seed);
    for (uint32_t i = 0; i < n; i++) {
        double u = rng.uniform();
        if (u <= 0) u = 1e-300;
        level[i] = (uint32_t)std::min(30.0, std::floor(-std::log(u) * ml));
    }
    return level;
}

std::vector<uint32_t> hnsw_insertion_order(uint32_t n, uint64_t seed) {
    return permutation(n, seed ^ 0x5bd1e995ull);
}

int build_hnsw(const HostVectors& V, uint32_t M, uint32_t efc, float ml, float alpha,
               uint64_t seed, int nthreads, HnswBuilt& H) {
    const uint32_t n = V.n;
    H.n = n;
    H.M = M;
    H.level = hnsw_levels(n, ml, seed);
    auto cap = [&](uint32_t l) { return l == 0 ? 2 * M : M; };
    H.first.resize(n);
    H.row_off.clear();
    uint64_t off = 0, nl = 0;
    for (uint32_t i = 0; i < n; i++) {
        H.first[i] = nl;
        for (uint32_t l = 0; l <= H.level[i]; l++) {
            H.row_off.push_back(off);
            off += cap(l);
            nl++;
        }
    }
    H.rows.assign(off, kNoNeighbor);
    H.sizes.assign(nl, 0);
    auto row = [&](uint32_t i, uint32_t l) { return H.rows.data() + H.row_off[H.first[i] + l]; };
    auto size = [&](uint32_t i, uint32_t l) -> uint32_t& { return H.sizes[H.first[i] + l]; };

    std::vector<uint32_t> order = hnsw_insertion_order(n, seed);
    uint32_t top = 0;
    H.entry = order[0];
    top = H.level[H.entry];
    const size_t max_batch = std::max<size_t>(1, (size_t)(0.02 * n));
    size_t pos = 1, batch = 1;
    while (pos < n) {
        size_t end = std::min<size_t>(n, pos + batch);
        std::vector<uint32_t> ids(order.begin() + pos, order.begin() + end);
        // out[i][l] = selected neighbours of ids[i] at level l
        std::vector<std::vector<std::vector<uint32_t>>> outs(ids.size());
        const uint32_t entry = H.entry, toplevel = top;
        parallel_for(ids.size(), nthreads, [&](size_t i) {
            thread_local Scratch s;
            thread_local std::vector<DistId> visited, F;
            const uint32_t p = ids[i];
            const uint8_t* q = V.row(p);
            uint32_t ep = entry;
            int32_t dep = V.dist_to(q, ep);
            // greedy descent through levels above the node's own
            for (int l = (int)toplevel; l > (int)H.level[p]; l--) {
                bool moved = true;
                while (moved) {
                    moved = false;
                    const uint32_t* r = H.rows.data() + H.row_off[H.first[ep] + l];
                    uint32_t sz = H.sizes[H.first[ep] + l];
                    for (uint32_t j = 0; j < sz; j++) {
                        int32_t d = V.dist_to(q, r[j]);
                        if (d < dep || (d == dep && r[j] < ep)) {
                            dep = d;
                            ep = r[j];
                            moved = true;
                        }
                    }
                }
            }
            outs[i].resize(H.level[p] + 1);
            std::vector<uint32_t> eps{ep};
            for (int l = (int)std::min(toplevel, H.level[p]); l >= 0; l--) {
                // beam search at level l with ef = efc over the snapshot
                s.begin(n);
                F.clear();
                std::vector<uint8_t> E;
                for (uint32_t e : eps)
                    if (!s.test_and_set(e)) {
                        DistId x{V.dist_to(q, e), e};
                        auto it = std::upper_bound(F.begin(), F.end(), x);
                        E.insert(E.begin() + (it - F.begin()), 0);
                        F.insert(it, x);
                    }
                size_t cur = 0;
                for (;;) {
                    while (cur < F.size() && E[cur]) cur++;
                    if (cur >= F.size()) break;
                    E[cur] = 1;
                    uint32_t u = F[cur].id;
                    const uint32_t* r = H.rows.data() + H.row_off[H.first[u] + l];
                    uint32_t sz = H.sizes[H.first[u] + l];
                    for (uint32_t j = 0; j < sz; j++) {
                        uint32_t nb = r[j];
                        if (s.test_and_set(nb)) continue;
                        int32_t d = V.dist_to(q, nb);
                        if (F.size() >= efc && !(d < F.back().d)) continue;
                        DistId x{d, nb};
                        auto it = std::upper_bound(F.begin(), F.end(), x);
                        size_t ps = (size_t)(it - F.begin());
                        F.insert(it, x);
                        E.insert(E.begin() + ps, 0);
                        if (F.size() > efc) {
                            F.pop_back();
                            E.pop_back();
                        }
                        if (ps < cur) cur = ps;
                    }
                }
                visited.assign(F.begin(), F.end());
                hnsw_select(V, p, visited, alpha, cap(l), outs[i][l]);
                eps.clear();
                for (const DistId& x : F) eps.push_back(x.id);
            }
        }, 1);
        // write forward edges
        for (size_t i = 0; i < ids.size(); i++) {
            uint32_t p = ids[i];
            for (uint32_t l = 0; l < outs[i].size(); l++) {
                uint32_t* r = row(p, l);
                std::copy(outs[i][l].begin(), outs[i][l].end(), r);
                size(p, l) = (uint32_t)outs[i][l].size();
            }
        }
        // reverse edges, grouped by (level, target) in sorted order
        std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> rev;  // (l, q, p)
        for (size_t i = 0; i < ids.size(); i++)
            for (uint32_t l = 0; l < outs[i].size(); l++)
                for (uint32_t qn : outs[i][l]) rev.emplace_back(l, qn, ids[i]);
        std::sort(rev.begin(), rev.end());
        std::vector<size_t> st;
        for (size_t i = 0; i < rev.size(); i++)
            if (i == 0 || std::get<0>(rev[i]) != std::get<0>(rev[i - 1]) ||
                std::get<1>(rev[i]) != std::get<1>(rev[i - 1]))
                st.push_back(i);
        st.push_back(rev.size());
        parallel_for(st.size() - 1, nthreads, [&](size_t g) {
            thread_local std::vector<DistId> cand;
            thread_local std::vector<uint32_t> out;
            uint32_t l = std::get<0>(rev[st[g]]), qn = std::get<1>(rev[st[g]]);
            if (H.level[qn] < l) return;
            uint32_t* r = row(qn, l);
            uint32_t& sz = size(qn, l);
            cand.clear();
            for (uint32_t j = 0; j < sz; j++) cand.push_back({V.dist(qn, r[j]), r[j]});
            size_t added = 0;
            for (size_t i = st[g]; i < st[g + 1]; i++) {
                uint32_t p = std::get<2>(rev[i]);
                bool present = p == qn;
                for (uint32_t j = 0; j < sz && !present; j++) present = r[j] == p;
                if (!present) {
                    cand.push_back({V.dist(qn, p), p});
                    added++;
                }
            }
            if (!added) return;
            if (cand.size() <= cap(l)) {
                for (size_t j = sz; j < cand.size(); j++) r[j] = cand[j].id;
                sz = (uint32_t)cand.size();
            } else {
                hnsw_select(V, qn, cand, alpha, cap(l), out);
                std::fill(r, r + cap(l), kNoNeighbor);
                std::copy(out.begin(), out.end(), r);
                sz = (uint32_t)out.size();
            }
        }, 16);
        for (uint32_t p : ids)
            if (H.level[p] > top) {
                top = H.level[p];
                H.entry = p;
            }
        pos = end;
        batch = std::min(batch * 2, max_batch);
    }
    return 0;
}

}  // namespace pgb
