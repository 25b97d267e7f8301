// search_flat.cu -- the two schedules of the flat-graph beam search.
//
// plain   : the drop-in. Persistent grid, warp w takes queries w, w+W, ... (the
//           reference's schedule, cuda/busqueda.cu:151-152), one Ls and k per launch.
// batched : persistent grid whose warps pull queries from a device counter over a
//           longest-beam-first order, each query with its own Ls and k; tables sized
//           for the batch's largest Ls. Same per-query code, identical neighbours.
#include <algorithm>
#include <cstdio>

#include "errors.h"
#include "search_flat.cuh"
#include "search_plan.h"

// resident 128-thread blocks per SM the flat kernels are compiled for (registers per
// thread = 65536 / (128 * this)): 9 -> 56 registers, 36 warps per SM
#ifndef PGB_MIN_BLOCKS
#define PGB_MIN_BLOCKS 9
#endif

namespace pgb {

#ifdef PGB_SECTION_PROFILE
__device__ unsigned long long g_section_cycles[NUM_SECTIONS];
// zero the warp's counters on entry, fold them into the device totals on exit
#define PGB_PROF_ENTER()                                                                \
    do {                                                                                \
        if (lane < NUM_SECTIONS)                                                        \
            reinterpret_cast<unsigned long long*>(wmem + A.L.off_prof)[lane] = 0ull;    \
        __syncwarp();                                                                   \
    } while (0)
#define PGB_PROF_EXIT()                                                                 \
    do {                                                                                \
        __syncwarp();                                                                   \
        if (lane < NUM_SECTIONS)                                                        \
            atomicAdd(&g_section_cycles[lane],                                          \
                      reinterpret_cast<unsigned long long*>(wmem + A.L.off_prof)[lane]); \
    } while (0)
#else
#define PGB_PROF_ENTER()
#define PGB_PROF_EXIT()
#endif

template <int CH, bool Signed, bool SFILT>
__global__ void __launch_bounds__(128, PGB_MIN_BLOCKS) flat_plain_kernel(FlatArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t gw = blockIdx.x * wpb + w;
    const uint32_t total = gridDim.x * wpb;
    unsigned char* wmem = smem + (size_t)w * A.L.bytes;
    uint32_t* gf = A.gfilter ? A.gfilter + (size_t)gw * A.gfilter_words : nullptr;
    uint32_t* gv = A.gvisited ? A.gvisited + (size_t)gw * A.gvisited_words : nullptr;
    PGB_PROF_ENTER();
    for (uint32_t q = gw; q < A.nq; q += total)
        flat_query<CH, Signed, SFILT>(A, wmem, gf, gv, q, A.Ls, A.k, lane);
    PGB_PROF_EXIT();
}

template <int CH, bool Signed, bool SFILT>
__global__ void __launch_bounds__(128, PGB_MIN_BLOCKS) flat_batched_kernel(FlatArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t gw = blockIdx.x * wpb + w;
    unsigned char* wmem = smem + (size_t)w * A.L.bytes;
    uint32_t* gf = A.gfilter ? A.gfilter + (size_t)gw * A.gfilter_words : nullptr;
    uint32_t* gv = A.gvisited ? A.gvisited + (size_t)gw * A.gvisited_words : nullptr;
    PGB_PROF_ENTER();
    for (;;) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(A.queue, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if (slot >= A.nq) break;
        const uint32_t q = A.order[slot];
        flat_query<CH, Signed, SFILT>(A, wmem, gf, gv, q, A.ls_arr[q], A.k_arr[q], lane);
    }
    PGB_PROF_EXIT();
}

namespace {

using KernelFn = void (*)(FlatArgs);

template <int CH, bool Signed, bool SFILT>
KernelFn pick_kernel(bool batched) {
    return batched ? flat_batched_kernel<CH, Signed, SFILT> : flat_plain_kernel<CH, Signed, SFILT>;
}

template <int CH>
KernelFn pick_ch(bool batched, bool is_signed, bool sfilt) {
    if (is_signed) return sfilt ? pick_kernel<CH, true, true>(batched) : pick_kernel<CH, true, false>(batched);
    return sfilt ? pick_kernel<CH, false, true>(batched) : pick_kernel<CH, false, false>(batched);
}

KernelFn pick(int ch, bool batched, bool is_signed, bool sfilt) {
    switch (ch) {
        case 1: return pick_ch<1>(batched, is_signed, sfilt);
        case 2: return pick_ch<2>(batched, is_signed, sfilt);
        case 3: return pick_ch<3>(batched, is_signed, sfilt);
        case 4: return pick_ch<4>(batched, is_signed, sfilt);
        default: return pick_ch<8>(batched, is_signed, sfilt);
    }
}

}  // namespace

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
    P.svis = rq.force_visited_placement ? rq.visited_in_shared
                                        : (4ull * vwords <= rq.visited_smem_limit);
    const uint32_t ls_cap = (ls + 7u) & ~7u;
    P.L = make_flat_layout(ls_cap, 32u * P.ch, P.sfilt ? fwords : 0u, P.svis ? vwords : 0u);
    P.gfilter_words = P.sfilt ? 0u : fwords;
    P.gvisited_words = P.svis ? 0u : vwords;
    P.kernel = (void*)pick(P.ch, P.batched, P.is_signed, P.sfilt);

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(PGB_ERR_CUDA, "cudaGetDevice failed");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return fail(PGB_ERR_CUDA, "cudaGetDeviceProperties failed");
    const size_t smem_cap = prop.sharedMemPerBlockOptin;
    // at most 4 warps per block: the kernels are built for 128 threads, 9 blocks per SM
    int wpb = rq.warps_per_block > 0 ? std::min(rq.warps_per_block, 4) : 4;
    while (wpb > 1 && (size_t)wpb * P.L.bytes > smem_cap) wpb >>= 1;
    if ((size_t)wpb * P.L.bytes > smem_cap)
        return fail(PGB_ERR_BAD_ARG, "beam too wide for shared memory with this placement");
    P.warps_per_block = wpb;
    P.smem_bytes = (size_t)wpb * P.L.bytes;
    // the attribute belongs to the kernel, shared by every plan of it: set the device
    // maximum so that no later plan can shrink it under an earlier one
    cudaError_t e = cudaFuncSetAttribute(P.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_cap);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(P.kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess)
        return fail(PGB_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    int bps = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, P.kernel, wpb * 32, P.smem_bytes);
    if (e != cudaSuccess || bps < 1)
        return fail(PGB_ERR_CUDA, "kernel does not fit on a multiprocessor");
    if (rq.max_blocks_per_sm > 0) bps = std::min(bps, rq.max_blocks_per_sm);
    P.blocks_per_sm = bps;
    P.blocks = bps * prop.multiProcessorCount;
    P.total_warps = (uint64_t)P.blocks * wpb;
    return PGB_OK;
}

pgb_status launch_flat(const FlatPlan& P, FlatArgs A, cudaStream_t stream) {
    A.L = P.L;
    A.gfilter_words = P.gfilter_words;
    A.gvisited_words = P.gvisited_words;
    void* args[] = {&A};
    // the work-queue form needs no more warps than queries (small serving batches)
    int blocks = P.blocks;
    if (P.batched)
        blocks = std::max(1, std::min(blocks, (int)((A.nq + P.warps_per_block - 1) / P.warps_per_block)));
    cudaError_t e = cudaLaunchKernel(P.kernel, dim3(blocks), dim3(P.warps_per_block * 32), args,
                                     P.smem_bytes, stream);
    if (e != cudaSuccess)
        return fail(PGB_ERR_CUDA, std::string("search launch: ") + cudaGetErrorString(e));
    return PGB_OK;
}

}  // namespace pgb

extern "C" pgb_status pgb_section_profile(uint64_t* out, uint32_t n, int reset) {
#ifdef PGB_SECTION_PROFILE
    if (!out || n < pgb::NUM_SECTIONS) return pgb::fail(PGB_ERR_BAD_ARG, "need NUM_SECTIONS slots");
    cudaError_t e = cudaMemcpyFromSymbol(out, pgb::g_section_cycles, 8 * pgb::NUM_SECTIONS);
    if (e == cudaSuccess && reset) {
        unsigned long long zero[pgb::NUM_SECTIONS] = {0};
        e = cudaMemcpyToSymbol(pgb::g_section_cycles, zero, sizeof(zero));
    }
    if (e != cudaSuccess) return pgb::fail(PGB_ERR_CUDA, cudaGetErrorString(e));
    return PGB_OK;
#else
    (void)out;
    (void)n;
    (void)reset;
    return pgb::fail(PGB_ERR_BAD_ARG, "library built without section profiling");
#endif
}
