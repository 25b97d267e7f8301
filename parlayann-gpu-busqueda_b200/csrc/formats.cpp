// formats.cpp -- file readers / writers (see formats.h for the layouts).
#include "formats.h"

#include <cstdio>
#include <cstring>
#include <memory>

namespace pgb {
namespace {

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};

bool file_size(FILE* f, uint64_t& sz) {
    if (fseeko(f, 0, SEEK_END) != 0) return false;
    off_t e = ftello(f);
    if (e < 0) return false;
    sz = (uint64_t)e;
    return fseeko(f, 0, SEEK_SET) == 0;
}

template <typename T>
bool read_exact(FILE* f, T* dst, size_t count) {
    return fread(dst, sizeof(T), count, f) == count;
}

std::string msg(const std::string& path, const char* what) { return path + ": " + what; }

}  // namespace

std::string read_vectors(const std::string& path, VectorFile& v, bool* io) {
    *io = true;
    File F;
    F.f = fopen(path.c_str(), "rb");
    if (!F.f) return msg(path, "cannot open");
    uint64_t sz = 0;
    if (!file_size(F.f, sz)) return msg(path, "cannot stat");
    uint32_t hdr[2];
    *io = false;
    if (sz < 8 || !read_exact(F.f, hdr, 2)) return msg(path, "truncated header");
    v.n = hdr[0];
    v.dim = hdr[1];
    if (sz != 8 + (uint64_t)v.n * v.dim) return msg(path, "size does not match header");
    v.data.resize((size_t)v.n * v.dim);
    *io = true;
    if (!read_exact(F.f, v.data.data(), v.data.size())) return msg(path, "short read");
    return "";
}

std::string read_graph(const std::string& path, GraphFile& g, bool* io) {
    *io = true;
    File F;
    F.f = fopen(path.c_str(), "rb");
    if (!F.f) return msg(path, "cannot open");
    uint64_t sz = 0;
    if (!file_size(F.f, sz)) return msg(path, "cannot stat");
    uint32_t hdr[2];
    *io = false;
    if (sz < 8 || !read_exact(F.f, hdr, 2)) return msg(path, "truncated header");
    g.n = hdr[0];
    g.max_degree = hdr[1];
    if (sz < 8 + 4ull * g.n) return msg(path, "truncated degrees");
    g.degrees.resize(g.n);
    if (!read_exact(F.f, g.degrees.data(), g.n)) return msg(path, "short read");
    uint64_t total = 0;
    for (uint32_t i = 0; i < g.n; i++) {
        if (g.degrees[i] > g.max_degree) return msg(path, "degree above max degree");
        total += g.degrees[i];
    }
    if (sz != 8 + 4ull * g.n + 4ull * total) return msg(path, "size does not match degrees");
    g.edges.resize(total);
    if (!read_exact(F.f, g.edges.data(), total)) return msg(path, "short read");
    for (uint64_t e = 0; e < total; e++)
        if (g.edges[e] >= g.n) return msg(path, "edge out of range");
    return "";
}

std::string read_hnsw(const std::string& path, HnswFile& h, bool* io) {
    *io = true;
    File F;
    F.f = fopen(path.c_str(), "rb");
    if (!F.f) return msg(path, "cannot open");
    std::vector<char> buf;
    {
        char tmp[1 << 16];
        size_t got;
        while ((got = fread(tmp, 1, sizeof(tmp), F.f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
    }
    *io = false;
    size_t pos = 0;
    bool ok = true;
    auto rd = [&](void* dst, size_t bytes) {
        if (!ok || pos + bytes > buf.size()) {
            ok = false;
            return;
        }
        memcpy(dst, buf.data() + pos, bytes);
        pos += bytes;
    };
    char magic[4];
    rd(magic, 4);
    if (!ok || memcmp(magic, "HNSW", 4) != 0) return msg(path, "not an HNSW model");
    uint32_t version = 0;
    rd(&version, 4);
    if (!ok || version != 3) return msg(path, "HNSW version is not 3");
    uint64_t skip;
    rd(&skip, 8);  // code_U
    rd(&skip, 8);  // size_node
    rd(&h.dim, 4);
    rd(&h.ml, 4);
    rd(&h.m, 4);
    rd(&h.efc, 4);
    rd(&h.alpha, 4);
    rd(&h.n, 4);
    if (!ok) return msg(path, "truncated header");
    if ((uint64_t)h.n * 8 > buf.size()) return msg(path, "node count exceeds file");
    h.levels.resize(h.n);
    h.node_point.resize(h.n);
    for (uint32_t i = 0; i < h.n && ok; i++) {
        rd(&h.levels[i], 4);
        rd(&h.node_point[i], 4);
        if (h.levels[i] > 64) return msg(path, "level out of range");
    }
    if (!ok) return msg(path, "truncated node table");
    h.list_sizes.clear();
    h.ids.clear();
    for (uint32_t i = 0; i < h.n && ok; i++)
        for (uint32_t l = 0; l <= h.levels[i] && ok; l++) {
            uint64_t cnt = 0;
            rd(&cnt, 8);
            if (!ok) break;
            if (cnt > (buf.size() - pos) / 4) return msg(path, "list exceeds file");
            h.list_sizes.push_back((uint32_t)cnt);
            for (uint64_t j = 0; j < cnt; j++) {
                uint32_t v = 0;
                rd(&v, 4);
                if (v >= h.n) return msg(path, "neighbour out of range");
                h.ids.push_back(v);
            }
        }
    if (!ok) return msg(path, "truncated lists");
    uint64_t ne = 0;
    rd(&ne, 8);
    if (!ok || ne > (buf.size() - pos) / 4) return msg(path, "truncated entries");
    h.entries.resize(ne);
    for (uint64_t i = 0; i < ne; i++) rd(&h.entries[i], 4);
    if (!ok) return msg(path, "truncated entries");
    if (pos != buf.size()) return msg(path, "trailing bytes after entries");
    for (uint32_t e : h.entries)
        if (e >= h.n) return msg(path, "entry point out of range");
    return "";
}

std::string write_graph(const std::string& path, uint32_t n, uint32_t slots,
                        const uint32_t* degrees, const uint32_t* adj) {
    File F;
    F.f = fopen(path.c_str(), "wb");
    if (!F.f) return msg(path, "cannot create");
    uint32_t maxdeg = 0;
    for (uint32_t i = 0; i < n; i++) maxdeg = std::max(maxdeg, degrees[i]);
    uint32_t hdr[2] = {n, maxdeg};
    bool ok = fwrite(hdr, 4, 2, F.f) == 2;
    ok = ok && fwrite(degrees, 4, n, F.f) == n;
    for (uint32_t i = 0; i < n && ok; i++)
        ok = fwrite(adj + (size_t)i * slots, 4, degrees[i], F.f) == degrees[i];
    if (!ok) return msg(path, "write failed");
    return "";
}

std::string write_hnsw(const std::string& path, const HnswFile& h) {
    File F;
    F.f = fopen(path.c_str(), "wb");
    if (!F.f) return msg(path, "cannot create");
    bool ok = true;
    auto wr = [&](const void* p, size_t bytes) { ok = ok && fwrite(p, 1, bytes, F.f) == bytes; };
    wr("HNSW", 4);
    uint32_t version = 3;
    wr(&version, 4);
    uint64_t code_u = 0, size_node = 0;
    wr(&code_u, 8);
    wr(&size_node, 8);
    wr(&h.dim, 4);
    wr(&h.ml, 4);
    wr(&h.m, 4);
    wr(&h.efc, 4);
    wr(&h.alpha, 4);
    wr(&h.n, 4);
    for (uint32_t i = 0; i < h.n; i++) {
        wr(&h.levels[i], 4);
        wr(&h.node_point[i], 4);
    }
    size_t li = 0, off = 0;
    for (uint32_t i = 0; i < h.n; i++)
        for (uint32_t l = 0; l <= h.levels[i]; l++) {
            uint64_t cnt = h.list_sizes[li++];
            wr(&cnt, 8);
            wr(h.ids.data() + off, 4 * cnt);
            off += cnt;
        }
    uint64_t ne = h.entries.size();
    wr(&ne, 8);
    wr(h.entries.data(), 4 * ne);
    if (!ok) return msg(path, "write failed");
    return "";
}

}  // namespace pgb
