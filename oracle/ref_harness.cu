// ref_harness.cu -- drives the reference's own search kernels on files we choose.
//
// TEST INFRASTRUCTURE ONLY (oracle pinning). oracle/Makefile compiles this file together
// with the reference's sources, read in place from the reference tree (busqueda.cu,
// busqueda_hnsw.cu, datos_gpu.cu, lectores.cpp, hnsw_lector.cpp), into oracle/_ref/.
// Nothing of the reference is copied into this repository. The binary runs on a B200 and
// writes the reference's outputs, which tests/golden/make_golden.py turns into fixtures.
//
// It calls the reference's public pieces exactly as its drivers do
// (cuda/comparacion1.cu:172-176,212-247): leerVectoresI8bin -> subirVectores,
// leerGrafoParlay -> subirGrafo / leerHnsw -> subirHnsw, BuscadorGPU / BuscadorHnsw
// preparar + lanzar, then copies idsDev / distsDev / compDev / banderasDev back.
//
// usage:
//   ref_search flat <base.i8bin> <queries.i8bin> <graph> <Ls> <visit|-1> <k> <cut> <out>
//   ref_search hnsw <base.i8bin> <queries.i8bin> <hnsw>  <Ls> <visit|-1> <k> <cut> <out>
// out: [nq u32][k u32][ids nq*k u32][dists nq*k i32][comp nq i32][flags nq i32]
//
// REF_TIME_REPS=N (optional): after the checked launch, time the reference's lanzar:
// 3 untimed launches, then N launches, each after a 512 MiB write that flushes the L2,
// bracketed by CUDA events on the launch stream; prints one JSON line on stdout.

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "busqueda.cuh"
#include "hnsw.h"
#include "lectores.h"

template <class Launch>
static void time_launches(int reps, uint32_t nq, Launch launch) {
    const size_t flush_bytes = 512ull << 20;
    void* flush = nullptr;
    CHECK_CUDA(cudaMalloc(&flush, flush_bytes));
    cudaEvent_t a, b;
    CHECK_CUDA(cudaEventCreate(&a));
    CHECK_CUDA(cudaEventCreate(&b));
    for (int i = 0; i < 3; i++) launch();
    CHECK_CUDA(cudaDeviceSynchronize());
    double total_ms = 0;
    for (int i = 0; i < reps; i++) {
        CHECK_CUDA(cudaMemsetAsync(flush, i & 0xff, flush_bytes, 0));
        CHECK_CUDA(cudaEventRecord(a, 0));
        launch();
        CHECK_CUDA(cudaEventRecord(b, 0));
        CHECK_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        CHECK_CUDA(cudaEventElapsedTime(&ms, a, b));
        total_ms += ms;
    }
    const double avg = total_ms / reps;
    printf("{\"reference_kernel_ms\": %.6f, \"qps\": %.1f, \"queries\": %u, \"reps\": %d}\n", avg,
           nq / (avg * 1e-3), nq, reps);
    CHECK_CUDA(cudaEventDestroy(a));
    CHECK_CUDA(cudaEventDestroy(b));
    CHECK_CUDA(cudaFree(flush));
}

int main(int argc, char** argv) {
    if (argc != 10) {
        fprintf(stderr, "usage: %s flat|hnsw base queries graph Ls visit k cut out\n", argv[0]);
        return 2;
    }
    const std::string mode = argv[1];
    VectoresHost base = leerVectoresI8bin(argv[2]);
    VectoresHost queries = leerVectoresI8bin(argv[3]);
    ConfigBusqueda cfg;
    cfg.Ls = atoi(argv[5]);
    long visit = atol(argv[6]);
    cfg.k = atoi(argv[7]);
    cfg.cut = atof(argv[8]);
    const uint32_t nq = queries.n;
    const int reps = getenv("REF_TIME_REPS") ? atoi(getenv("REF_TIME_REPS")) : 0;

    VectoresGPU baseGPU, queriesGPU;
    subirVectores(base, baseGPU);
    subirVectores(queries, queriesGPU);

    std::vector<uint32_t> ids((size_t)nq * cfg.k);
    std::vector<int> dists((size_t)nq * cfg.k), comp(nq), flags(nq);
    auto fetch = [&](uint32_t* idsDev, int* distsDev, int* compDev, int* flagsDev) {
        CHECK_CUDA(cudaDeviceSynchronize());
        CHECK_CUDA(cudaMemcpy(ids.data(), idsDev, ids.size() * 4, cudaMemcpyDeviceToHost));
        CHECK_CUDA(cudaMemcpy(dists.data(), distsDev, dists.size() * 4, cudaMemcpyDeviceToHost));
        CHECK_CUDA(cudaMemcpy(comp.data(), compDev, comp.size() * 4, cudaMemcpyDeviceToHost));
        CHECK_CUDA(cudaMemcpy(flags.data(), flagsDev, flags.size() * 4, cudaMemcpyDeviceToHost));
    };

    if (mode == "flat") {
        GrafoHost g = leerGrafoParlay(argv[4]);
        GrafoGPU gg;
        subirGrafo(g, gg);
        // the driver passes n when no visit limit is configured (comparacion1.cu:240)
        cfg.limite = (visit < 0) ? (long)gg.n : visit;
        BuscadorGPU b;
        b.preparar(gg, nq, cfg);
        b.lanzar(baseGPU, queriesGPU, gg, 0);
        fetch(b.idsDev, b.distsDev, b.compDev, b.banderasDev);
        if (reps > 0) time_launches(reps, nq, [&] { b.lanzar(baseGPU, queriesGPU, gg, 0); });
        b.liberar();
        liberarGrafo(gg);
    } else if (mode == "hnsw") {
        HnswHost h = leerHnsw(argv[4]);
        HnswGPU hg;
        subirHnsw(h, base, baseGPU, hg);
        cfg.limite = visit;  // BuscadorHnsw::lanzar maps <= 0 to n (busqueda_hnsw.cu:610)
        BuscadorHnsw b;
        b.preparar(hg, nq, cfg);
        b.lanzar(queriesGPU, hg, 0);
        fetch(b.idsDev, b.distsDev, b.compDev, b.banderasDev);
        if (reps > 0) time_launches(reps, nq, [&] { b.lanzar(queriesGPU, hg, 0); });
        b.liberar();
        liberarHnsw(hg);
    } else {
        fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 2;
    }

    FILE* f = fopen(argv[9], "wb");
    if (!f) {
        fprintf(stderr, "cannot write %s\n", argv[9]);
        return 1;
    }
    uint32_t hdr[2] = {nq, (uint32_t)cfg.k};
    fwrite(hdr, 4, 2, f);
    fwrite(ids.data(), 4, ids.size(), f);
    fwrite(dists.data(), 4, dists.size(), f);
    fwrite(comp.data(), 4, comp.size(), f);
    fwrite(flags.data(), 4, flags.size(), f);
    fclose(f);
    liberarVectores(baseGPU);
    liberarVectores(queriesGPU);
    return 0;
}
