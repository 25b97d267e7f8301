// searcher.h -- the searcher object behind pgb_searcher_*.
#pragma once

#include <cuda_runtime.h>

#include "../../include/pgb.h"
#include "search_hnsw.h"
#include "search_plan.h"

struct pgb_searcher {
    pgb_index* index = nullptr;
    pgb_query_params params{};
    uint32_t max_queries = 0;
    pgb::FlatPlan flat{};
    uint32_t* gfilter = nullptr;   // flat: per-warp filters when not in shared memory
    uint32_t* gvisited = nullptr;  // flat: per-warp visited tables when not in shared
    pgb::HnswState hnsw{};
    // code rows (pgb_searcher_create_compressed): the search keeps `rerank` candidates per
    // query in cand / cand_d, re-ranked exactly into the caller's k
    bool codes = false;
    uint32_t rerank = 0;
    uint32_t* cand = nullptr;
    int32_t* cand_d = nullptr;
    // host-memory path staging
    uint8_t* q_dev = nullptr;
    uint32_t* ids_dev = nullptr;
    int32_t* dists_dev = nullptr;
    pgb_query_stats* stats_dev = nullptr;
    cudaStream_t stream = nullptr;
};

namespace pgb {
pgb_status cuda_status(cudaError_t e, const char* what);
pgb_status check_params(const pgb_index* ix, const pgb_query_params* p);
// the device address of page-locked host memory (a kernel reads and writes it over the
// bus, no staging copy), or null for pageable or device memory
void* pinned_device_ptr(const void* p);
}  // namespace pgb
