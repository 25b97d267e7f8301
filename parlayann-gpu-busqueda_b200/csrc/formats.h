// formats.h -- readers / writers of the on-disk formats the reference reads.
//   vectors : [n u32][dim u32][n*dim bytes]               (cuda/lectores.h:7-15)
//   graph   : [n u32][maxdeg u32][deg n*u32][edges u32..]  (cuda/lectores.h:17-27)
//   HNSW v3 : "HNSW" | version u32 | code_U u64 | size_node u64 | dim u32 | m_l f32 |
//             m u32 | efc u32 | alpha f32 | n u32 | n*(level u32, point u32) |
//             per node, level 0..level: count u64 + ids u32 | entries: count u64 + ids
//                                                          (cuda/hnsw.h:11-16)
//   GT      : [nq u32][k u32][ids nq*k u32][dists nq*k f32] (cuda/lectores.h:29-36)
// Every reader checks the exact file size / end of file and the id ranges, as the
// reference readers do (cuda/lectores.cpp:62-144, cuda/hnsw_lector.cpp:14-111), but
// reports a status instead of exiting.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pgb {

struct VectorFile {
    uint32_t n = 0, dim = 0;
    std::vector<uint8_t> data;  // n*dim
};

struct GraphFile {
    uint32_t n = 0, max_degree = 0;
    std::vector<uint32_t> degrees;
    std::vector<uint32_t> edges;
};

struct HnswFile {
    uint32_t n = 0, dim = 0, m = 0, efc = 0;
    float ml = 0, alpha = 0;
    std::vector<uint32_t> levels, node_point;
    std::vector<uint32_t> list_sizes;  // per (node, level), node-major
    std::vector<uint32_t> ids;
    std::vector<uint32_t> entries;
};

// return "" on success, else an error message; *io tells IO vs FORMAT failures
std::string read_vectors(const std::string& path, VectorFile& out, bool* io);
std::string read_graph(const std::string& path, GraphFile& out, bool* io);
std::string read_hnsw(const std::string& path, HnswFile& out, bool* io);
std::string write_graph(const std::string& path, uint32_t n, uint32_t slots,
                        const uint32_t* degrees, const uint32_t* adjacency);
std::string write_hnsw(const std::string& path, const HnswFile& h);

}  // namespace pgb
