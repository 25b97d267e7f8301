// Drives the C++ interface (pgb_buscador.hpp) the way the reference's search driver drives
// BuscadorGPU (cuda/paso2_busqueda.cu:106-149): load the base and the graph, upload the
// queries, preparar / lanzar / copy idsDev, distsDev, compDev, banderasDev back, liberar.
// usage: buscador_golden flat|hnsw <base> <queries> <graph> <Ls> <visit|-1> <k> <cut> <out>
// out: [nq u32][k u32][ids][dists][comp][flags], the reference harness's layout.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "pgb_buscador.hpp"

static std::vector<int8_t> read_i8bin(const char* path, uint32_t& n, uint32_t& dim) {
    FILE* f = fopen(path, "rb");
    if (!f) throw pgb::Error(PGB_ERR_IO, path);
    uint32_t hdr[2];
    if (fread(hdr, 4, 2, f) != 2) throw pgb::Error(PGB_ERR_FORMAT, path);
    n = hdr[0];
    dim = hdr[1];
    std::vector<int8_t> v((size_t)n * dim);
    if (fread(v.data(), 1, v.size(), f) != v.size()) throw pgb::Error(PGB_ERR_FORMAT, path);
    fclose(f);
    return v;
}

int main(int argc, char** argv) {
    if (argc != 10) {
        fprintf(stderr, "usage: %s flat|hnsw base queries graph Ls visit k cut out\n", argv[0]);
        return 2;
    }
    try {
        const std::string mode = argv[1];
        pgb::Indice indice = (mode == "flat") ? pgb::Indice::cargarPlano(argv[2], argv[4])
                                              : pgb::Indice::cargarHnsw(argv[2], argv[4]);
        uint32_t nq = 0, dim = 0;
        std::vector<int8_t> q = read_i8bin(argv[3], nq, dim);
        void* qdev = nullptr;
        pgb::check_cuda(cudaMalloc(&qdev, q.size()), "queries");
        pgb::check_cuda(cudaMemcpy(qdev, q.data(), q.size(), cudaMemcpyHostToDevice), "queries");

        pgb::ConfigBusqueda cfg;
        cfg.Ls = atoi(argv[5]);
        const long visit = atol(argv[6]);
        cfg.limite = visit < 0 ? 0 : visit;
        cfg.k = atoi(argv[7]);
        cfg.cut = atof(argv[8]);

        pgb::BuscadorGPU b;
        b.preparar(indice, nq, cfg);
        b.lanzar(qdev, 0);
        pgb::check_cuda(cudaDeviceSynchronize(), "search");
        std::vector<uint32_t> ids((size_t)nq * cfg.k);
        std::vector<int> dists(ids.size()), comp(nq), flags(nq);
        pgb::check_cuda(cudaMemcpy(ids.data(), b.idsDev, ids.size() * 4, cudaMemcpyDeviceToHost), "ids");
        pgb::check_cuda(cudaMemcpy(dists.data(), b.distsDev, dists.size() * 4, cudaMemcpyDeviceToHost), "dists");
        pgb::check_cuda(cudaMemcpy(comp.data(), b.compDev, nq * 4, cudaMemcpyDeviceToHost), "comp");
        pgb::check_cuda(cudaMemcpy(flags.data(), b.banderasDev, nq * 4, cudaMemcpyDeviceToHost), "flags");
        b.liberar();
        cudaFree(qdev);

        FILE* f = fopen(argv[9], "wb");
        if (!f) throw pgb::Error(PGB_ERR_IO, argv[9]);
        uint32_t hdr[2] = {nq, (uint32_t)cfg.k};
        fwrite(hdr, 4, 2, f);
        fwrite(ids.data(), 4, ids.size(), f);
        fwrite(dists.data(), 4, dists.size(), f);
        fwrite(comp.data(), 4, comp.size(), f);
        fwrite(flags.data(), 4, flags.size(), f);
        fclose(f);
    } catch (const pgb::Error& e) {
        fprintf(stderr, "error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
    return 0;
}
