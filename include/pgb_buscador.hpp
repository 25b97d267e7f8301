// pgb_buscador.hpp -- C++ host interface over the C ABI (pgb.h), shaped like the
// reference's search classes so a caller of the reference switches by renaming includes:
//
//   reference (cuda/busqueda.cuh:6-61, cuda/hnsw.h:65-86)   here
//   ConfigBusqueda{Ls, limite, k, cut}                      pgb::ConfigBusqueda (+ degree_limit,
//                                                           excluir_consulta, base_consulta)
//   subirVectores / subirGrafo / subirHnsw                  pgb::Indice::plano / ::hnsw / ::cargar*
//   BuscadorGPU::preparar(grafo, nq, cfg)                   pgb::BuscadorGPU::preparar(indice, nq, cfg)
//   BuscadorGPU::lanzar(base, consultas, grafo, stream)     pgb::BuscadorGPU::lanzar(consultas, stream)
//   BuscadorGPU::liberar()                                  pgb::BuscadorGPU::liberar()
//   idsDev / distsDev / compDev / banderasDev               same members (device, owned)
//   BANDERA_DESBORDE / BANDERA_FRONTERA_CORTA               PGB_FLAG_OVERFLOW / PGB_FLAG_SHORT
//
// Differences, by design: the index (vectors + graph) is uploaded once into an Indice and
// the searcher keeps a pointer to it; consultas are the caller's device rows of dim bytes
// (no norm array); failures throw pgb::Error (status + message) where the reference
// prints and exits (cuda/comun.h:57-65); the HNSW searcher uses the same class.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pgb.h"

namespace pgb {

struct Error : std::runtime_error {
    pgb_status status;
    Error(pgb_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(pgb_status s) {
    if (s != PGB_OK)
        throw Error(s, std::string(pgb_status_string(s)) + ": " + pgb_last_error());
}

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(PGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

struct ConfigBusqueda {
    int Ls = 10;                    // beam width (beamSize)
    long limite = 0;                // max expansions ("visit"); 0 -> n
    int k = 10;                     // neighbours returned
    double cut = 1.35;              // frontier cut
    uint32_t degree_limit = 0;      // 0 -> max degree
    bool excluir_consulta = true;   // skip neighbour == query index, as ParlayANN's wrapper
    uint32_t base_consulta = 0;     // index of the first query of a launch

    pgb_query_params params() const {
        pgb_query_params p{};
        p.k = (uint32_t)k;
        p.beam_size = (uint32_t)Ls;
        p.cut = cut;
        p.limit = limite;
        p.degree_limit = degree_limit;
        p.exclude_query_id = excluir_consulta ? 1u : 0u;
        p.query_id_base = base_consulta;
        return p;
    }
};

// Device-resident vectors + graph (flat or HNSW). Move-only.
class Indice {
  public:
    Indice() = default;
    Indice(const Indice&) = delete;
    Indice& operator=(const Indice&) = delete;
    Indice(Indice&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    Indice& operator=(Indice&& o) noexcept {
        std::swap(h_, o.h_);
        return *this;
    }
    ~Indice() { pgb_index_destroy(h_); }

    static Indice plano(const void* vectores, uint32_t n, uint32_t dim, pgb_elem tipo,
                        const uint32_t* grados, const uint32_t* aristas, int dispositivo = 0) {
        Indice ix;
        check(pgb_index_create_flat(dispositivo, vectores, n, dim, tipo, grados, aristas, &ix.h_));
        return ix;
    }
    static Indice cargarPlano(const std::string& vectores, const std::string& grafo,
                              pgb_elem tipo = PGB_INT8, int dispositivo = 0) {
        Indice ix;
        check(pgb_index_load_flat(dispositivo, vectores.c_str(), tipo, grafo.c_str(), &ix.h_));
        return ix;
    }
    static Indice cargarHnsw(const std::string& vectores, const std::string& modelo,
                             pgb_elem tipo = PGB_INT8, int dispositivo = 0) {
        Indice ix;
        check(pgb_index_load_hnsw(dispositivo, vectores.c_str(), tipo, modelo.c_str(), &ix.h_));
        return ix;
    }
    pgb_index_info info() const {
        pgb_index_info i{};
        check(pgb_index_get_info(h_, &i));
        return i;
    }
    pgb_index* get() const { return h_; }

  private:
    pgb_index* h_ = nullptr;
};

// BuscadorGPU / BuscadorHnsw: scratch and outputs for one (index, nq, config).
class BuscadorGPU {
  public:
    uint32_t* idsDev = nullptr;   // numConsultas * k
    int* distsDev = nullptr;      // numConsultas * k
    int* compDev = nullptr;       // distance computations per query
    int* banderasDev = nullptr;   // PGB_FLAG_* per query
    int* expansionesDev = nullptr;
    uint32_t numConsultas = 0;
    ConfigBusqueda cfg;

    BuscadorGPU() = default;
    BuscadorGPU(const BuscadorGPU&) = delete;
    BuscadorGPU& operator=(const BuscadorGPU&) = delete;
    ~BuscadorGPU() { liberar(); }

    void preparar(const Indice& indice, uint32_t nq, const ConfigBusqueda& c) {
        liberar();
        cfg = c;
        numConsultas = nq;
        indice_ = &indice;
        pgb_query_params p = c.params();
        check(pgb_searcher_create(indice.get(), nq, &p, &s_));
        check_cuda(cudaMalloc(&idsDev, sizeof(uint32_t) * nq * c.k), "idsDev");
        check_cuda(cudaMalloc(&distsDev, sizeof(int) * nq * c.k), "distsDev");
        check_cuda(cudaMalloc(&stats_, sizeof(pgb_query_stats) * nq), "stats");
        check_cuda(cudaMalloc(&compDev, sizeof(int) * nq), "compDev");
        check_cuda(cudaMalloc(&banderasDev, sizeof(int) * nq), "banderasDev");
        check_cuda(cudaMalloc(&expansionesDev, sizeof(int) * nq), "expansionesDev");
    }

    // consultas: device rows of the index dim bytes, `paso` bytes apart (0: dim)
    void lanzar(const void* consultas, cudaStream_t stream = 0, uint32_t paso = 0) {
        if (!s_) throw Error(PGB_ERR_BAD_ARG, "lanzar before preparar");
        const uint32_t dim = indice_->info().dim;
        check(pgb_searcher_search(s_, consultas, numConsultas, paso ? paso : dim, idsDev,
                                  distsDev, stats_, stream));
        // split the stats records into the reference's per-query arrays
        const size_t w = sizeof(pgb_query_stats);
        check_cuda(cudaMemcpy2DAsync(compDev, sizeof(int), (const char*)stats_, w, sizeof(int),
                                     numConsultas, cudaMemcpyDeviceToDevice, stream), "comp");
        check_cuda(cudaMemcpy2DAsync(expansionesDev, sizeof(int), (const char*)stats_ + 4, w,
                                     sizeof(int), numConsultas, cudaMemcpyDeviceToDevice, stream),
                   "expansiones");
        check_cuda(cudaMemcpy2DAsync(banderasDev, sizeof(int), (const char*)stats_ + 8, w,
                                     sizeof(int), numConsultas, cudaMemcpyDeviceToDevice, stream),
                   "banderas");
    }

    void liberar() {
        pgb_searcher_destroy(s_);
        s_ = nullptr;
        cudaFree(idsDev);
        cudaFree(distsDev);
        cudaFree(stats_);
        cudaFree(compDev);
        cudaFree(banderasDev);
        cudaFree(expansionesDev);
        idsDev = nullptr;
        distsDev = nullptr;
        stats_ = nullptr;
        compDev = banderasDev = expansionesDev = nullptr;
    }

  private:
    const Indice* indice_ = nullptr;
    pgb_searcher* s_ = nullptr;
    pgb_query_stats* stats_ = nullptr;
};

// The same searcher serves HNSW indexes; the name mirrors the reference.
using BuscadorHnsw = BuscadorGPU;

}  // namespace pgb
