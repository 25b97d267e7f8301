// search_flat.cu -- launch planning for the flat-graph beam search kernels (plain and
// batched; the kernels themselves are in search_flat_kernels.cuh, compiled per adjacency
// chunk count by search_flat_ch*.cu).
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "errors.h"
#include "index.h"
#include "search_flat.cuh"
#include "search_hnsw.h"
#include "search_plan.h"

namespace pgb {

void* flat_kernel_ch1(FlatSchedule sched, bool is_signed, uint32_t filter_words);
void* flat_kernel_ch2(FlatSchedule sched, bool is_signed, uint32_t filter_words);
void* flat_kernel_ch3(FlatSchedule sched, bool is_signed, uint32_t filter_words);
void* flat_kernel_ch4(FlatSchedule sched, bool is_signed, uint32_t filter_words);
void* flat_kernel_ch8(FlatSchedule sched, bool is_signed, uint32_t filter_words);
cudaError_t flat_section_totals_ch1(unsigned long long* acc, bool reset);
cudaError_t flat_section_totals_ch2(unsigned long long* acc, bool reset);
cudaError_t flat_section_totals_ch3(unsigned long long* acc, bool reset);
cudaError_t flat_section_totals_ch4(unsigned long long* acc, bool reset);
cudaError_t flat_section_totals_ch8(unsigned long long* acc, bool reset);

namespace {

void* pick(int ch, FlatSchedule sched, bool is_signed, uint32_t filter_words) {
    switch (ch) {
        case 1: return flat_kernel_ch1(sched, is_signed, filter_words);
        case 2: return flat_kernel_ch2(sched, is_signed, filter_words);
        case 3: return flat_kernel_ch3(sched, is_signed, filter_words);
        case 4: return flat_kernel_ch4(sched, is_signed, filter_words);
        default: return flat_kernel_ch8(sched, is_signed, filter_words);
    }
}

}  // namespace

namespace {
std::atomic<int64_t> g_search_launches{0};
}  // namespace

void count_launches(int64_t n) { g_search_launches.fetch_add(n, std::memory_order_relaxed); }

int flat_chunks_for(uint32_t gs) {
    int ch = (int)((gs + 31) / 32);
    return ch <= 4 ? ch : 8;
}

pgb_status plan_flat(const FlatPlanRequest& rq, FlatPlan& P) {
    P = FlatPlan{};
    P.ch = flat_chunks_for(rq.deg_lim);
    P.batched = rq.batched;
    P.is_signed = rq.is_signed;
    const uint32_t ls = rq.max_ls;
    const uint32_t fwords = 1u << flat_filter_bits(ls);
    const uint32_t vwords = flat_visited_cap(ls);
    P.sfilt = rq.force_filter_placement ? rq.filter_in_shared
                                        : (4ull * fwords <= rq.filter_smem_limit);
    // the shared-filter kernels exist for 1,024 to 4,096 words (beams up to 128)
    if (P.sfilt && fwords > kSharedFilterMaxWords)
        return fail(PGB_ERR_BAD_ARG, "a shared-memory filter holds at most 4,096 slots (beams up to 128)");
    P.svis = rq.force_visited_placement ? rq.visited_in_shared
                                        : (4ull * vwords <= rq.visited_smem_limit);
    const uint32_t ls_cap = (ls + 7u) & ~7u;
    if (ls_cap > flat_fvis_cap(P.sfilt ? fwords : 0u))
        return fail(PGB_ERR_BAD_ARG, "beam above the kernels' frontier capacity");
    P.L = make_flat_layout(ls_cap, 32u * P.ch, P.sfilt ? fwords : 0u, P.svis ? vwords : 0u);
    P.gfilter_words = P.sfilt ? 0u : fwords;
    P.gvisited_words = P.svis ? 0u : vwords;
    const uint32_t kfw = P.sfilt ? fwords : 0u;
    if (rq.codes && rq.batched) return fail(PGB_ERR_BAD_ARG, "code rows are searched by the plain schedule only");
    const FlatSchedule sched = P.batched ? FlatSchedule::kBatched
                                         : (rq.codes ? FlatSchedule::kPlainCodes : FlatSchedule::kPlain);
    P.kernel = pick(P.ch, sched, P.is_signed, kfw);
    if (P.batched) P.kernel_uniform = pick(P.ch, FlatSchedule::kBatchedUniform, P.is_signed, kfw);
    if (!P.kernel || (P.batched && !P.kernel_uniform))
        return fail(PGB_ERR_BAD_ARG, "no kernel for this filter size");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(PGB_ERR_CUDA, "cudaGetDevice failed");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return fail(PGB_ERR_CUDA, "cudaGetDeviceProperties failed");
    const size_t smem_cap = prop.sharedMemPerBlockOptin;
    // at most 4 warps per block: the kernels are built for 128 threads, 9 blocks per SM
    const size_t warp_bytes = P.L.bytes;
    int wpb = rq.warps_per_block > 0 ? std::min(rq.warps_per_block, 4) : 4;
    while (wpb > 1 && (size_t)wpb * warp_bytes > smem_cap) wpb >>= 1;
    if ((size_t)wpb * warp_bytes > smem_cap)
        return fail(PGB_ERR_BAD_ARG, "beam too wide for shared memory with this placement");
    P.warps_per_block = wpb;
    P.smem_bytes = (size_t)wpb * warp_bytes;
    // the attribute belongs to the kernel, shared by every plan of it: set the device
    // maximum so that no later plan can shrink it under an earlier one
    cudaError_t e = cudaSuccess;
    for (void* kern : {P.kernel, P.kernel_uniform}) {
        if (!kern || e != cudaSuccess) continue;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
    }
    if (e != cudaSuccess)
        return fail(PGB_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    // blocks per SM: the smaller of the two batched kernels' figures (same launch bounds)
    int bps = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, P.kernel, wpb * 32, P.smem_bytes);
    if (e == cudaSuccess && P.kernel_uniform) {
        int bu = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bu, P.kernel_uniform, wpb * 32, P.smem_bytes);
        bps = std::min(bps, bu);
    }
    if (e != cudaSuccess || bps < 1)
        return fail(PGB_ERR_CUDA, "kernel does not fit on a multiprocessor");
    if (rq.max_blocks_per_sm > 0) bps = std::min(bps, rq.max_blocks_per_sm);
    P.blocks_per_sm = bps;
    P.blocks = bps * prop.multiProcessorCount;
    P.total_warps = (uint64_t)P.blocks * wpb;
    return PGB_OK;
}

pgb_status launch_flat(const FlatPlan& P, FlatArgs A, cudaStream_t stream, const pgb_index* ix) {
    A.L = P.L;
    A.gfilter_words = P.gfilter_words;
    A.gvisited_words = P.gvisited_words;
    void* args[] = {&A};
    // the work-queue form needs no more warps than queries (small serving batches)
    int blocks = P.blocks;
    if (P.batched)
        blocks = std::max(1, std::min(blocks, (int)((A.nq + P.warps_per_block - 1) / P.warps_per_block)));
    void* kern = (P.batched && !A.ls_arr) ? P.kernel_uniform : P.kernel;
    cudaError_t e;
    if (ix && ix->l2_bytes) {
        // the index's persisting window travels with the launch (and into a captured graph)
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(blocks);
        cfg.blockDim = dim3(P.warps_per_block * 32);
        cfg.dynamicSmemBytes = P.smem_bytes;
        cfg.stream = stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeAccessPolicyWindow;
        at[0].val.accessPolicyWindow.base_ptr = ix->l2_base;
        at[0].val.accessPolicyWindow.num_bytes = ix->l2_bytes;
        at[0].val.accessPolicyWindow.hitRatio = ix->l2_hit;
        at[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        at[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelExC(&cfg, kern, args);
    } else {
        e = cudaLaunchKernel(kern, dim3(blocks), dim3(P.warps_per_block * 32), args, P.smem_bytes, stream);
    }
    if (e != cudaSuccess)
        return fail(PGB_ERR_CUDA, std::string("search launch: ") + cudaGetErrorString(e));
    count_launches(1);
    return PGB_OK;
}

}  // namespace pgb

extern "C" uint64_t pgb_search_launches(void) {
    return (uint64_t)pgb::g_search_launches.load(std::memory_order_relaxed);
}

extern "C" pgb_status pgb_section_profile(uint64_t* out, uint32_t n, int reset) {
#ifdef PGB_SECTION_PROFILE
    if (!out || n < pgb::NUM_SECTIONS) return pgb::fail(PGB_ERR_BAD_ARG, "need NUM_SECTIONS slots");
    unsigned long long acc[pgb::NUM_SECTIONS] = {0};
    cudaError_t e = pgb::flat_section_totals_ch1(acc, reset != 0);
    if (e == cudaSuccess) e = pgb::flat_section_totals_ch2(acc, reset != 0);
    if (e == cudaSuccess) e = pgb::flat_section_totals_ch3(acc, reset != 0);
    if (e == cudaSuccess) e = pgb::flat_section_totals_ch4(acc, reset != 0);
    if (e == cudaSuccess) e = pgb::flat_section_totals_ch8(acc, reset != 0);
    if (e == cudaSuccess) e = pgb::hnsw_section_totals(acc, reset != 0);
    if (e != cudaSuccess) return pgb::fail(PGB_ERR_CUDA, cudaGetErrorString(e));
    for (int i = 0; i < pgb::NUM_SECTIONS; i++) out[i] = acc[i];
    return PGB_OK;
#else
    (void)out;
    (void)n;
    (void)reset;
    return pgb::fail(PGB_ERR_BAD_ARG, "library built without section profiling");
#endif
}
