// search_flat_kernels.cuh -- the two schedules of the flat-graph beam search, included
// by search_flat_ch{1,2,3,4,8}.cu: each of those compiles the kernels of one adjacency
// chunk count, so the variants build in parallel.
//
// plain   : the drop-in. Persistent grid, warp w takes queries w, w+W, ... (the
//           reference's schedule, cuda/busqueda.cu:151-152), one Ls and k per launch.
// batched : persistent grid whose warps pull queries from a device counter over a
//           longest-beam-first order, each query with its own Ls and k; tables sized
//           for the batch's largest Ls. Same per-query code, identical neighbours.
#pragma once

#include "search_flat.cuh"

// resident 128-thread blocks per SM the flat kernels are compiled for (registers per
// thread = 65536 / (128 * this)): 9 -> 56 registers, 36 warps per SM
#ifndef PGB_MIN_BLOCKS
#define PGB_MIN_BLOCKS 9
#endif

namespace pgb {

#ifdef PGB_SECTION_PROFILE
// device variables belong to one translation unit: each kernel file keeps its own totals
// and pgb_section_profile adds them up
static __device__ unsigned long long g_section_cycles[NUM_SECTIONS];
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

// C4: the rows are 4-bit code rows (schedule kPlainCodes)
template <int CH, bool Signed, int FW, bool C4 = false>
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
        flat_query<CH, Signed, FW, C4>(A, wmem, gf, gv, q, A.Ls, A.k, lane);
    PGB_PROF_EXIT();
}

// UNI: every query of the launch has the same (Ls, k), read from A.Ls / A.k like the
// plain kernel does (kernel parameters, which spare the registers that a per-query pair
// holds through the search); otherwise each query's pair comes from A.ls_arr / A.k_arr.
template <int CH, bool Signed, int FW, bool UNI>
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
        if (UNI)
            flat_query<CH, Signed, FW, false, true>(A, wmem, gf, gv, q, A.Ls, A.k, lane);
        else
            flat_query<CH, Signed, FW, false, true>(A, wmem, gf, gv, q, A.ls_arr[q], A.k_arr[q], lane);
        if (A.done) publish_query_done(A.done, q, A.done_seq, lane);
    }
    PGB_PROF_EXIT();
}

template <int CH, bool Signed, int FW>
void* flat_kernel_of(FlatSchedule sched) {
    switch (sched) {
        case FlatSchedule::kPlain: return (void*)flat_plain_kernel<CH, Signed, FW>;
        case FlatSchedule::kBatched: return (void*)flat_batched_kernel<CH, Signed, FW, false>;
        case FlatSchedule::kPlainCodes: return (void*)flat_plain_kernel<CH, Signed, FW, true>;
        default: return (void*)flat_batched_kernel<CH, Signed, FW, true>;
    }
}

// this chunk count's kernel for (schedule, element type, shared-filter words); null for
// a filter size without a kernel
template <int CH>
void* flat_kernel_ch(FlatSchedule sched, bool is_signed, uint32_t filter_words) {
    switch (filter_words) {
        case 0: return is_signed ? flat_kernel_of<CH, true, 0>(sched) : flat_kernel_of<CH, false, 0>(sched);
        case 1024: return is_signed ? flat_kernel_of<CH, true, 1024>(sched) : flat_kernel_of<CH, false, 1024>(sched);
        case 2048: return is_signed ? flat_kernel_of<CH, true, 2048>(sched) : flat_kernel_of<CH, false, 2048>(sched);
        case 4096: return is_signed ? flat_kernel_of<CH, true, 4096>(sched) : flat_kernel_of<CH, false, 4096>(sched);
        default: return nullptr;
    }
}

// this translation unit's profile totals, added into acc[NUM_SECTIONS]; reset zeroes them
inline cudaError_t flat_section_totals(unsigned long long* acc, bool reset) {
#ifdef PGB_SECTION_PROFILE
    unsigned long long v[NUM_SECTIONS];
    cudaError_t e = cudaMemcpyFromSymbol(v, g_section_cycles, sizeof(v));
    if (e != cudaSuccess) return e;
    for (int i = 0; i < NUM_SECTIONS; i++) acc[i] += v[i];
    if (reset) {
        unsigned long long zero[NUM_SECTIONS] = {0};
        e = cudaMemcpyToSymbol(g_section_cycles, zero, sizeof(zero));
    }
    return e;
#else
    (void)acc;
    (void)reset;
    return cudaSuccess;
#endif
}

}  // namespace pgb
