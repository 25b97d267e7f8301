// device_common.cuh -- device primitives shared by the flat and HNSW search kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pgb {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kEmptyId = 0xFFFFFFFFu;      // row padding / empty table slot
constexpr uint64_t kEmptyKey = ~0ull;           // sentinel (dist, id) key, sorts last
constexpr int kRowBytes = 128;                  // every vector row occupies 128 bytes

// parlaylib hash64_2: filter slots must land where ParlayANN's land
// (reference cuda/utiles_gpu.cuh:12-17)
__device__ __forceinline__ uint64_t hash64_2(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// parlaylib hash64; HNSW marks its entry points with it (cuda/utiles_gpu.cuh:21-31)
__device__ __forceinline__ uint64_t hash64(uint64_t u) {
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

// (dist, id) packed so that unsigned order == ParlayANN's pair order
// (distances are >= 0 and below 2^24 for 128 bytes of 8-bit values)
__device__ __forceinline__ uint64_t pack_key(int32_t d, uint32_t id) {
    return ((uint64_t)(uint32_t)d << 32) | id;
}
__device__ __forceinline__ int32_t key_dist(uint64_t k) { return (int32_t)(k >> 32); }
__device__ __forceinline__ uint32_t key_id(uint64_t k) { return (uint32_t)k; }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
__device__ __forceinline__ uint32_t lanemask_gt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_gt;" : "=r"(m));
    return m;
}

// 16 bytes of one 128-byte row: dot(p, p) - 2 dot(p, q) over those bytes.
// Summed over the 8 lanes of a row this plus ||q||^2 is ||q - p||^2 exactly
// (the reference computes the same integer with a stored norm, cuda/distancia.cuh:43-58;
// here ||p||^2 comes from the row itself, so no norm array is gathered).
template <bool Signed>
__device__ __forceinline__ int32_t partial_l2(const int4 p, const int4 q) {
    int32_t pp, pq;
    if (Signed) {
        pp = __dp4a(p.x, p.x, 0);
        pp = __dp4a(p.y, p.y, pp);
        pp = __dp4a(p.z, p.z, pp);
        pp = __dp4a(p.w, p.w, pp);
        pq = __dp4a(p.x, q.x, 0);
        pq = __dp4a(p.y, q.y, pq);
        pq = __dp4a(p.z, q.z, pq);
        pq = __dp4a(p.w, q.w, pq);
    } else {
        pp = (int32_t)__dp4a((uint32_t)p.x, (uint32_t)p.x, 0u);
        pp = (int32_t)__dp4a((uint32_t)p.y, (uint32_t)p.y, (uint32_t)pp);
        pp = (int32_t)__dp4a((uint32_t)p.z, (uint32_t)p.z, (uint32_t)pp);
        pp = (int32_t)__dp4a((uint32_t)p.w, (uint32_t)p.w, (uint32_t)pp);
        pq = (int32_t)__dp4a((uint32_t)p.x, (uint32_t)q.x, 0u);
        pq = (int32_t)__dp4a((uint32_t)p.y, (uint32_t)q.y, (uint32_t)pq);
        pq = (int32_t)__dp4a((uint32_t)p.z, (uint32_t)q.z, (uint32_t)pq);
        pq = (int32_t)__dp4a((uint32_t)p.w, (uint32_t)q.w, (uint32_t)pq);
    }
    return pp - 2 * pq;
}

// dot(p, q) over 16 bytes
template <bool Signed>
__device__ __forceinline__ int32_t partial_dot(const int4 p, const int4 q) {
    if (Signed) {
        int32_t s = __dp4a(p.x, q.x, 0);
        s = __dp4a(p.y, q.y, s);
        s = __dp4a(p.z, q.z, s);
        return __dp4a(p.w, q.w, s);
    } else {
        uint32_t s = __dp4a((uint32_t)p.x, (uint32_t)q.x, 0u);
        s = __dp4a((uint32_t)p.y, (uint32_t)q.y, s);
        s = __dp4a((uint32_t)p.z, (uint32_t)q.z, s);
        return (int32_t)__dp4a((uint32_t)p.w, (uint32_t)q.w, s);
    }
}

// Rows of at most 124 meaningful bytes carry their squared norm (int32) in bytes
// 124..127; the query row has zeros there, so it drops out of every dot product.
constexpr uint32_t kNormInRowMaxDim = 124;

// Compressed rows: 4-bit codes, 64 bytes per row. Byte b of 32-bit word j of 16-byte
// word c holds dimension 32c + 8j + b in its low nibble and 32c + 8j + 4 + b in its high
// nibble (so the low nibbles pair with query word 8c + 2j, the high ones with 8c + 2j + 1,
// and the query row keeps its natural byte order). Bytes 60..63 hold the squared norm of
// the reconstructed row, which leaves room for 120 dimensions.
constexpr int kCodeRowBytes = 64;
constexpr uint32_t kCodeMaxDim = 120;

// acc + dot of the four query bytes q (signed when Signed) with four unsigned bytes c
template <bool Signed>
__device__ __forceinline__ int32_t dp4a_qc(uint32_t q, uint32_t c, int32_t acc) {
    int32_t d;
    if (Signed)
        asm("dp4a.s32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(q), "r"(c), "r"(acc));
    else
        asm("dp4a.u32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(q), "r"(c), "r"(acc));
    return d;
}

// dot of 16 code bytes (32 codes) with the 32 query bytes qa (the word's first 16
// dimensions) and qb (the next 16). The high nibbles are used in place (16 x code); their
// sum is a multiple of 16 and is divided by 16 at the end, exactly.
template <bool Signed>
__device__ __forceinline__ int32_t code_dot(const int4 v, const int4 qa, const int4 qb) {
    constexpr uint32_t lo = 0x0F0F0F0Fu, hi = 0xF0F0F0F0u;
    int32_t a = dp4a_qc<Signed>((uint32_t)qa.x, (uint32_t)v.x & lo, 0);
    int32_t b = dp4a_qc<Signed>((uint32_t)qa.y, (uint32_t)v.x & hi, 0);
    a = dp4a_qc<Signed>((uint32_t)qa.z, (uint32_t)v.y & lo, a);
    b = dp4a_qc<Signed>((uint32_t)qa.w, (uint32_t)v.y & hi, b);
    a = dp4a_qc<Signed>((uint32_t)qb.x, (uint32_t)v.z & lo, a);
    b = dp4a_qc<Signed>((uint32_t)qb.y, (uint32_t)v.z & hi, b);
    a = dp4a_qc<Signed>((uint32_t)qb.z, (uint32_t)v.w & lo, a);
    b = dp4a_qc<Signed>((uint32_t)qb.w, (uint32_t)v.w & hi, b);
    return a + (b >> 4);
}

template <bool Signed>
__device__ __forceinline__ int32_t partial_sq(const int4 q) {
    if (Signed) {
        int32_t s = __dp4a(q.x, q.x, 0);
        s = __dp4a(q.y, q.y, s);
        s = __dp4a(q.z, q.z, s);
        return __dp4a(q.w, q.w, s);
    } else {
        uint32_t s = __dp4a((uint32_t)q.x, (uint32_t)q.x, 0u);
        s = __dp4a((uint32_t)q.y, (uint32_t)q.y, s);
        s = __dp4a((uint32_t)q.z, (uint32_t)q.z, s);
        return (int32_t)__dp4a((uint32_t)q.w, (uint32_t)q.w, s);
    }
}

// Marks one query of a launch as finished for a host observer: every lane's output writes
// are made visible at system scope before lane 0 stores the flag (host-mapped memory).
__device__ __forceinline__ void publish_query_done(uint32_t* done, uint32_t q, uint32_t seq, int lane) {
    __threadfence_system();
    __syncwarp();
    if (lane == 0) *reinterpret_cast<volatile uint32_t*>(done + q) = seq;
}

// read-only 16-byte load through the non-coherent path
__device__ __forceinline__ int4 ldg16(const void* p) {
    return __ldg(reinterpret_cast<const int4*>(p));
}

// Hint: bring the line of one 128-byte row into L2 (no register or completion cost).
__device__ __forceinline__ void prefetch_row_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Loads a query of `dim` bytes (any alignment) into a zero-padded 128-byte row in
// shared memory: lane l fills bytes 4l..4l+3.
__device__ __forceinline__ void load_query_row(const uint8_t* src, uint32_t dim, int lane,
                                               uint32_t* dst_words) {
    uint32_t w = 0;
#pragma unroll
    for (int b = 0; b < 4; b++) {
        uint32_t i = 4u * lane + b;
        uint32_t v = (i < dim) ? (uint32_t)src[i] : 0u;
        w |= v << (8 * b);
    }
    dst_words[lane] = w;
}

}  // namespace pgb
