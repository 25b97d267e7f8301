// host_common.h -- host-side helpers shared by the loaders, builders and C ABI.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace pgb {

constexpr uint32_t kNoNeighbor = 0xFFFFFFFFu;  // row padding (reference comun.h:22)

// exact int32 squared L2 between two rows of `dim` bytes
template <bool Signed>
inline int32_t sq_l2(const uint8_t* a, const uint8_t* b, uint32_t dim) {
    int32_t s = 0;
    if (Signed) {
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

struct HostVectors {
    const uint8_t* data = nullptr;  // n rows of `stride` bytes
    uint32_t n = 0, dim = 0, stride = 0;
    bool is_signed = true;
    const uint8_t* row(uint32_t i) const { return data + (size_t)i * stride; }
    int32_t dist(uint32_t i, uint32_t j) const {
        return is_signed ? sq_l2<true>(row(i), row(j), dim) : sq_l2<false>(row(i), row(j), dim);
    }
    int32_t dist_to(const uint8_t* q, uint32_t j) const {
        return is_signed ? sq_l2<true>(q, row(j), dim) : sq_l2<false>(q, row(j), dim);
    }
};

inline int default_threads() {
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

// dynamic-chunk parallel loop over [0, n)
template <typename F>
void parallel_for(size_t n, int nthreads, F&& f, size_t grain = 64) {
    if (nthreads <= 0) nthreads = default_threads();
    if (nthreads == 1 || n <= grain) {
        for (size_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    int nt = (int)std::min<size_t>((size_t)nthreads, (n + grain - 1) / grain);
    for (int t = 0; t < nt; t++)
        pool.emplace_back([&]() {
            for (;;) {
                size_t i = next.fetch_add(grain);
                if (i >= n) break;
                size_t e = std::min(n, i + grain);
                for (; i < e; i++) f(i);
            }
        });
    for (auto& th : pool) th.join();
}

// SplitMix64: the documented PRNG of the builders (seeded, thread-count independent)
struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t m) { return next() % m; }
};

struct DistId {
    int32_t d;
    uint32_t id;
    bool operator<(const DistId& o) const { return d < o.d || (d == o.d && id < o.id); }
    bool operator==(const DistId& o) const { return d == o.d && id == o.id; }
};

}  // namespace pgb
