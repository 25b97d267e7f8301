// index.h -- device-resident index: 128-byte vector rows + fixed-stride adjacency.
//
// HBM layout
//   rows       : n x 128 B, vector bytes then zeros (int8 d=100 or uint8 d=128); when
//                the vector has at most 124 bytes, its int32 squared norm fills bytes
//                124..127, so no separate norm array is gathered (d=128: recomputed)
//   adj        : n x gs u32, gs = degree rounded up to 32 (128-byte aligned rows),
//                padded with 0xFFFFFFFF (reference GrafoGPU, cuda/datos_gpu.h:19-28)
//   HNSW       : level-0 matrix n x g0s; upper levels one block of gas ids per
//                (node, level >= 1) at upper_start[node] + level - 1; vectors in node
//                order (reference HnswGPU, cuda/hnsw.h:37-59)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pgb.h"

struct pgb_index {
    int device = 0;
    uint32_t n = 0, dim = 0;
    pgb_elem elem = PGB_INT8;
    bool is_hnsw = false;
    bool norm_in_row = false;  // rows hold their squared norm in bytes 124..127
    uint8_t* rows = nullptr;  // point order
    // flat graph
    uint32_t* adj = nullptr;
    uint32_t G = 0, gs = 0;
    // HNSW
    uint32_t n_nodes = 0;
    uint32_t* adj0 = nullptr;
    uint32_t G0 = 0, g0s = 0;
    uint32_t* adju = nullptr;
    uint32_t GA = 0, gas = 0;
    uint32_t* upper_start = nullptr;
    uint32_t* node_point = nullptr;
    uint8_t* node_rows = nullptr;  // == rows when node i stores point i
    uint32_t entries[PGB_MAX_HNSW_ENTRIES] = {0};
    uint32_t n_entries = 0;
    uint32_t top_level = 0;
    uint64_t device_bytes = 0;
    // flat graphs, after pgb_index_compress: n x 64-byte 4-bit code rows; dimension d of a
    // row is code_step * code + code_off_host[d] (code_off: the offsets as one 128-byte
    // row of element values on the device)
    uint8_t* codes = nullptr;
    uint8_t* code_off = nullptr;
    int32_t code_step = 0;
    int32_t code_off_host[PGB_MAX_DIM] = {0};
    // L2 access-policy window given to every flat search launch over this index
    // (pgb_index_set_l2_window): [l2_base, l2_base + l2_bytes) persists with ratio l2_hit
    void* l2_base = nullptr;
    size_t l2_bytes = 0;
    float l2_hit = 0.f;
};

namespace pgb {
// RAII device selection for entry points
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};
}  // namespace pgb
