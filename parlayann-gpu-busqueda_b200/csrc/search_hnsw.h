// search_hnsw.h -- HNSW searcher state (scratch, epochs) and launch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pgb.h"

struct pgb_index;

namespace pgb {

struct HnswState {
    bool ready = false;
    int ch = 1;
    int fmode = 0;              // lossy filter: 0 shared, 1 global ids + shared bitmap, 2 global (epoch, id)
    uint32_t bits0 = 2;         // layer-0 filter bits
    uint32_t cap_inw = 0;       // the reference's is_inw capacity: overflow past half of it
    uint32_t filter_slots = 0;  // global filter slots per warp (0: shared)
    uint32_t wcap = 0;          // workset / candidate capacity
    uint32_t warp_bytes = 0;
    int warps_per_block = 4, blocks = 1;
    uint64_t total_warps = 0;
    size_t smem_bytes = 0;
    void* kernel = nullptr;
    unsigned long long* gfilter = nullptr; // global lossy filter per warp: 4-byte ids
                                           // (fmode 1) or (epoch, id) pairs (fmode 2)
    uint64_t epoch_base = 0;               // next unused epoch (tables start at epoch 0)
    uint64_t* d_epoch = nullptr;           // fmode 2: the same on the device, read by each
                                           // launch and advanced after it (captured
                                           // graphs replay with fresh epochs)
    uint32_t max_ls = 0;                   // the beam the state was prepared for
    uint32_t* queue = nullptr;             // next query of the running launch (zeroed per launch)
};

pgb_status hnsw_prepare(const pgb_index* ix, const pgb_query_params& p, HnswState& H);
pgb_status hnsw_launch(const pgb_index* ix, HnswState& H, const pgb_query_params& p,
                       const void* queries, uint32_t nq, uint32_t qstride, uint32_t* ids,
                       int32_t* dists, pgb_query_stats* stats, cudaStream_t stream);
// One launch at beam Ls <= H.max_ls and k, the outputs of query q at q * out_stride (the
// filter size and is_inw capacity follow Ls; the tables were sized for H.max_ls). With
// ls_arr / k_arr (device, every beam <= H.max_ls, every k <= out_stride) query q runs at
// its own beam and k, and the work queue hands the queries out in `order` (may be null).
// done (host-mapped, may be null): done[q] = done_seq once query q's outputs are visible.
pgb_status hnsw_launch_at(const pgb_index* ix, HnswState& H, uint32_t Ls, uint32_t k, int64_t limit,
                          const void* queries, uint32_t nq, uint32_t qstride, uint32_t* ids,
                          int32_t* dists, pgb_query_stats* stats, uint32_t out_stride,
                          cudaStream_t stream, const uint32_t* ls_arr = nullptr,
                          const uint32_t* k_arr = nullptr, const uint32_t* order = nullptr,
                          uint32_t* done = nullptr, uint32_t done_seq = 0);
// epochs one launch of nq queries uses, and their reservation on the host mirror of the
// device epoch word (a wrap enqueues a clear of the tables and of the word on `stream`)
uint64_t hnsw_epoch_need(const pgb_index* ix, uint32_t nq);
pgb_status hnsw_epoch_reserve(HnswState& H, uint64_t need, cudaStream_t stream);
// device bytes of the state's scratch tables
size_t hnsw_scratch_bytes(const HnswState& H);
void hnsw_release(HnswState& H);
// section totals of the HNSW kernel in the profiling build (added into acc; reset zeroes
// them); a no-op otherwise
cudaError_t hnsw_section_totals(unsigned long long* acc, bool reset);

}  // namespace pgb
