// builders.h -- CPU graph builders (see builders.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "host_common.h"

namespace pgb {

// HNSW built in memory: one row of capacity (2M at level 0, M above) per (node, level).
struct HnswBuilt {
    uint32_t n = 0, M = 0;
    std::vector<uint32_t> level;
    std::vector<uint64_t> first;    // index of node i's level-0 row
    std::vector<uint32_t> rows;     // row storage
    std::vector<uint32_t> sizes;    // per (node, level)
    std::vector<uint64_t> row_off;  // per (node, level): offset in rows
    uint32_t entry = 0;
};

int build_vamana(const HostVectors& V, uint32_t R, uint32_t L, float alpha, int passes,
                 uint64_t seed, int nthreads, uint32_t* out_deg, uint32_t* out_adj);
// Vamana's insertion schedule, shared by the CPU and GPU builders: a seeded permutation
// with point 0 moved to the front, inserted in prefix-doubling batches 1, 2, 4, ... up
// to vamana_max_batch(n) points (2 % of n) per batch
std::vector<uint32_t> vamana_insertion_order(uint32_t n, uint64_t seed);
size_t vamana_max_batch(uint32_t n);
int build_hcnng(const HostVectors& V, uint32_t trees, uint32_t leaf, uint32_t mst_deg,
                uint64_t seed, int nthreads, uint32_t* out_deg, uint32_t* out_adj);
int build_nndescent(const HostVectors& V, uint32_t K, uint32_t init_trees, uint32_t leaf,
                    float alpha, float delta, uint32_t max_iters, uint64_t seed, int nthreads,
                    uint32_t* out_deg, uint32_t* out_adj);
int build_hnsw(const HostVectors& V, uint32_t M, uint32_t efc, float ml, float alpha,
               uint64_t seed, int nthreads, HnswBuilt& H);
// HNSW's node levels (floor(-ln(U) * ml), at most 30) and insertion order, shared by the
// CPU and GPU builders; insertion runs in the same prefix-doubling batches as Vamana's
std::vector<uint32_t> hnsw_levels(uint32_t n, float ml, uint64_t seed);
std::vector<uint32_t> hnsw_insertion_order(uint32_t n, uint64_t seed);

}  // namespace pgb
