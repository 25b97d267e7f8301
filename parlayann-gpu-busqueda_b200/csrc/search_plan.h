// search_plan.h -- launch planning for the flat and HNSW search kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pgb.h"
#include "search_flat.cuh"

namespace pgb {

struct FlatPlanRequest {
    uint32_t max_ls = 10;          // largest beam served by the launch
    uint32_t deg_lim = 32;         // adjacency entries read per row
    bool is_signed = true;
    bool batched = false;
    bool codes = false;            // plain schedule over 4-bit code rows (not batched)
    int warps_per_block = 0;       // 0: default (4)
    int max_blocks_per_sm = 0;     // 0: as many as fit
    // table placement: the lossy filter is read on every neighbour and stays in shared
    // memory up to 16 KB; the visited table is touched once per expansion and lives in
    // global memory (L2), which keeps more warps resident
    uint32_t filter_smem_limit = 16384;
    uint32_t visited_smem_limit = 0;
    bool force_filter_placement = false;
    bool filter_in_shared = true;
    bool force_visited_placement = false;
    bool visited_in_shared = true;
};

struct FlatPlan {
    int ch = 1;
    bool batched = false, is_signed = true, sfilt = true, svis = true;
    FlatLayout L{};
    uint32_t gfilter_words = 0, gvisited_words = 0;  // per warp, 0 when in shared memory
    int warps_per_block = 4, blocks_per_sm = 1, blocks = 1;
    uint64_t total_warps = 0;
    size_t smem_bytes = 0;
    void* kernel = nullptr;          // plain, or batched with per-query (Ls, k)
    void* kernel_uniform = nullptr;  // batched: one (Ls, k) for every query
};

int flat_chunks_for(uint32_t deg_lim);
pgb_status plan_flat(const FlatPlanRequest& rq, FlatPlan& P);
// A's table pointers must cover P.total_warps slices when the plan keeps them global.
// A batched launch with A.ls_arr == nullptr runs the uniform kernel on (A.Ls, A.k).
// ix (optional): the index whose L2 access-policy window, when set, the launch carries.
pgb_status launch_flat(const FlatPlan& P, FlatArgs A, cudaStream_t stream,
                       const pgb_index* ix = nullptr);

// process-wide count of search kernels launched (pgb_search_launches); a negative n takes
// back launches that were only captured into a graph
void count_launches(int64_t n);

}  // namespace pgb
