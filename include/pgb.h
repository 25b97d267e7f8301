/* pgb.h -- C ABI of the B200 graph beam search (ParlayANN search API as a drop-in).
 *
 * Plain C: pointers, sizes, status codes. No exceptions cross this boundary and no
 * call exits the process (the reference's CHECK_CUDA exits, cuda/comun.h:57-65; here
 * every failure is a pgb_status plus a message from pgb_last_error()).
 *
 * What each group replaces in the reference (paths inside the reference project):
 *   pgb_index_*     <- subirVectores / subirGrafo / subirHnsw + the readers
 *                      (cuda/datos_gpu.cu:8-81, cuda/busqueda_hnsw.cu:462-530,
 *                      cuda/lectores.cpp:62-170, cuda/hnsw_lector.cpp:14-111)
 *   pgb_searcher_*  <- BuscadorGPU / BuscadorHnsw preparar, lanzar, liberar
 *                      (cuda/busqueda.cuh:36-61, cuda/busqueda.cu:525-594,
 *                      cuda/hnsw.h:65-86, cuda/busqueda_hnsw.cu:551-645)
 *   pgb_query_params <- ConfigBusqueda (cuda/busqueda.cuh:6-11) extended to ParlayANN's
 *                      QueryParams{k, beamSize, cut, limit, degree_limit}
 *   pgb_query_stats <- compDev / banderasDev (cuda/busqueda.cuh:43-46) + expansions
 *   pgb_recall      <- calcularRecall (cuda/evaluacion.cpp:56-80)
 *   pgb_batch_*, pgb_server_* have no counterpart in the reference: the batched
 *                      persistent form and the serving loop built on top of the plain
 *                      warp-per-query search, returning identical neighbours.
 *   pgb_build_*     <- ParlayANN's CPU graph builders (absent from the reference; it
 *                      clones them at run time, cpu_baseline/setup.sh:45-52).
 *
 * Memory: an index owns its device copy of vectors and graph and is read-only after
 * creation. A searcher / batch owns its scratch; outputs are caller-owned device
 * buffers (pgb_searcher_search) or host buffers (pgb_searcher_search_host).
 * Threading: one index may be searched from several host threads, each with its own
 * searcher and stream.
 */
#ifndef PGB_H_
#define PGB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pgb_status {
    PGB_OK = 0,
    PGB_ERR_BAD_ARG = 1,     /* invalid argument or size beyond a supported maximum */
    PGB_ERR_OOM = 2,         /* device or pinned allocation failed                  */
    PGB_ERR_CUDA = 3,        /* a CUDA runtime call failed                          */
    PGB_ERR_OVERFLOW = 4,    /* a capacity counter would wrap (reuse limit reached) */
    PGB_ERR_IO = 5,          /* file could not be opened / read / written           */
    PGB_ERR_FORMAT = 6,      /* file or arrays violate the format                   */
    PGB_ERR_BUSY = 7,        /* server: no free slot or memory for the request      */
    PGB_ERR_TIMEOUT = 8,     /* a bounded wait gave up                              */
    PGB_ERR_NOT_FOUND = 9    /* server: unknown ticket                              */
} pgb_status;

/* element type of the vectors */
typedef enum pgb_elem { PGB_INT8 = 0, PGB_UINT8 = 1 } pgb_elem;

#define PGB_NO_NEIGHBOR 0xFFFFFFFFu /* output padding id (reference SIN_VECINO)      */
#define PGB_FLAG_OVERFLOW 1         /* visited table past half capacity (BANDERA_DESBORDE) */
#define PGB_FLAG_SHORT 2            /* frontier ended with fewer than k entries       */
#define PGB_MAX_DEGREE 256          /* rows wider than this are rejected              */
#define PGB_MAX_BEAM 1024           /* largest beam size (Ls) accepted                */
#define PGB_MAX_K 1024              /* largest k accepted                             */
#define PGB_MAX_DIM 128             /* vectors are stored as 128-byte rows            */
#define PGB_MAX_HNSW_ENTRIES 8      /* reference MAX_ENTRADAS_HNSW (cuda/hnsw.h:9)    */

typedef struct pgb_query_params {
    uint32_t k;                /* neighbours returned                                  */
    uint32_t beam_size;        /* Ls: frontier width (HNSW: layer-0 ef)                */
    double cut;                /* frontier cut factor (flat graphs; reference 1.35)    */
    int64_t limit;             /* max expansions ("visit"); <= 0 means n               */
    uint32_t degree_limit;     /* first degree_limit row entries used; 0 = max degree  */
    uint32_t exclude_query_id; /* 1: skip neighbour id == query index, as ParlayANN's
                                  wrapper does with `a == p.id()` (flat graphs only)   */
    uint32_t query_id_base;    /* query index of the first query of the call           */
    uint32_t reserved;
} pgb_query_params;

typedef struct pgb_query_stats {
    int32_t dist_comps;  /* distance computations, counted as the reference does */
    int32_t expansions;  /* frontier nodes expanded                              */
    int32_t flags;       /* PGB_FLAG_* bits                                       */
    int32_t reserved;
} pgb_query_stats;

typedef struct pgb_index_info {
    uint32_t n_points;
    uint32_t dim;
    uint32_t elem;          /* pgb_elem                                   */
    uint32_t is_hnsw;
    uint32_t max_degree;    /* flat: G; HNSW: level-0 degree G0            */
    uint32_t upper_degree;  /* HNSW: upper-level degree GA; flat: 0        */
    uint32_t top_level;     /* HNSW only                                  */
    uint32_t n_entries;     /* HNSW only                                  */
    uint64_t device_bytes;  /* vectors + graph resident on the device     */
} pgb_index_info;

typedef struct pgb_index pgb_index;
typedef struct pgb_searcher pgb_searcher;
typedef struct pgb_batch pgb_batch;
typedef struct pgb_server pgb_server;

/* ---- errors ---------------------------------------------------------------- */
const char* pgb_status_string(pgb_status s);
/* message of the last failing call on this host thread ("" if none) */
const char* pgb_last_error(void);
/* 1 if a CUDA device of compute capability 10.x is visible, else 0 */
int pgb_device_available(void);

/* ---- index ------------------------------------------------------------------- */
/* Flat fixed-degree graph (Vamana/DiskANN, HCNNG, PyNNDescent) from host arrays.
 * vectors: n rows of dim bytes (int8 or uint8, packed). Graph in ParlayANN's layout:
 * degrees[n], edges = all rows concatenated (sum(degrees) ids < n). */
pgb_status pgb_index_create_flat(int device, const void* vectors, uint32_t n, uint32_t dim,
                                 pgb_elem elem, const uint32_t* degrees,
                                 const uint32_t* edges, pgb_index** out);
/* HNSW from host arrays in the order of the ParlayANN HNSW v3 file (cuda/hnsw.h:11-16):
 * per node i (0..n_nodes-1) its top level levels[i] and stored point node_point[i];
 * list_sizes / ids: the neighbour lists of node 0 levels 0..levels[0], node 1, ... */
pgb_status pgb_index_create_hnsw(int device, const void* vectors, uint32_t n_points,
                                 uint32_t dim, pgb_elem elem, uint32_t n_nodes,
                                 const uint32_t* levels, const uint32_t* node_point,
                                 const uint32_t* list_sizes, const uint32_t* ids,
                                 const uint32_t* entries, uint32_t n_entries,
                                 pgb_index** out);
/* From files: .i8bin / .u8bin vectors ([n u32][dim u32][n*dim bytes]), a ParlayANN
 * graph ([n u32][maxdeg u32][deg n*u32][edges]) or HNSW v3 model. */
pgb_status pgb_index_load_flat(int device, const char* vectors_path, pgb_elem elem,
                               const char* graph_path, pgb_index** out);
pgb_status pgb_index_load_hnsw(int device, const char* vectors_path, pgb_elem elem,
                               const char* hnsw_path, pgb_index** out);
pgb_status pgb_index_get_info(const pgb_index* index, pgb_index_info* out);
/* Reads and checks a file on the host only (no GPU): kind 0 = vectors, 1 = flat graph,
 * 2 = HNSW v3 model, with the reference readers' checks (exact size / end of file, ids in
 * range; cuda/lectores.cpp:62-170, cuda/hnsw_lector.cpp:14-111). info (may be NULL)
 * receives {n, dim | max degree | dim, total bytes | edges | lists, 0 | 0 | entries}. */
pgb_status pgb_file_check(const char* path, int kind, uint64_t info[4]);
pgb_status pgb_index_destroy(pgb_index* index);

/* Exact squared L2 distances of (query, point) pairs, computed by the search kernels' own
 * row code (dp4a over 128-byte rows): the library's form of the reference's load-and-verify
 * step (cuda/paso1_carga.cu:33-123), which checks GPU distances of random and ground-truth
 * pairs against the CPU distance (cuda/lectores.cpp:172-179). Device pointers: queries (nq
 * rows of index dim bytes, query_stride apart), pairs[2 * npairs] = (query row, point id)
 * and out[npairs] (int32). Synchronous on `stream`. A pair naming a query >= nq or a point
 * >= n gets INT32_MIN and the call returns PGB_ERR_BAD_ARG. */
pgb_status pgb_index_distances(const pgb_index* index, const void* queries, uint32_t nq,
                               uint32_t query_stride, const uint32_t* pairs, uint64_t npairs,
                               int32_t* out, void* stream);

/* Gather calibration: the int32 squared L2 distance of one query (device, index dim bytes)
 * to count rows named by ids (device) into out, computed with lanes_per_row threads per
 * 128-byte row (1, 4, 8 or 32). Asynchronous on `stream`. It measures the device's random
 * row-gather rate, as the reference's micro_distancias.cu:19-63 does for its kernels;
 * lanes_per_row 4 is the search kernels' own row code. Ids >= n get INT32_MIN. */
pgb_status pgb_gather_probe(const pgb_index* index, const void* query, const uint32_t* ids,
                            uint64_t count, int32_t* out, uint32_t lanes_per_row, void* stream);

/* L2 residency (no counterpart in the reference): an access-policy window over one region
 * of a flat index -- PGB_L2_ROWS (the 128-byte vector rows), PGB_L2_CODES (the 64-byte
 * code rows of pgb_index_compress) or PGB_L2_GRAPH (the adjacency rows) -- carried by every
 * later flat search launch over the index (plain, compressed, batched, served, and CUDA
 * graphs captured after the call). The window covers the region's first
 * min(size, max_bytes (0: no limit), device maximum) bytes; the persisting set-aside of
 * this process is set to min(window, device maximum), and window_bytes / hit_ratio (may
 * be NULL) receive what was set. Lines in the window stay in L2 across launches and
 * against other traffic. PGB_L2_NONE removes the window, demotes persisting lines and
 * returns the set-aside to none (so does pgb_index_destroy). The set-aside is one per
 * process: the last call made wins. */
#define PGB_L2_NONE 0u
#define PGB_L2_ROWS 1u
#define PGB_L2_CODES 2u
#define PGB_L2_GRAPH 3u
pgb_status pgb_index_set_l2_window(pgb_index* index, uint32_t region, uint64_t max_bytes,
                                   uint64_t* window_bytes, float* hit_ratio);

/* ---- plain warp-per-query search (the drop-in) ------------------------------------ */
/* preparar: scratch for up to max_queries queries with these params. */
pgb_status pgb_searcher_create(pgb_index* index, uint32_t max_queries,
                               const pgb_query_params* params, pgb_searcher** out);
/* lanzar: asynchronous on `stream` (a cudaStream_t; NULL = legacy default stream).
 * queries: device pointer, nq rows of index dim bytes, `query_stride` bytes apart.
 * Outputs (device): ids[nq*k], dists[nq*k], stats[nq] (stats may be NULL). Rows of
 * queries that end with fewer than k entries are padded with PGB_NO_NEIGHBOR/INT32_MAX. */
pgb_status pgb_searcher_search(pgb_searcher* s, const void* queries, uint32_t nq,
                               uint32_t query_stride, uint32_t* ids, int32_t* dists,
                               pgb_query_stats* stats, void* stream);
/* Same search from and to HOST memory, synchronous: copies the queries in, searches,
 * copies ids / dists / stats (stats may be NULL) out. When every buffer is page-locked,
 * the launch reads and writes them directly and no staging copy is made. */
pgb_status pgb_searcher_search_host(pgb_searcher* s, const void* queries, uint32_t nq,
                                    uint32_t query_stride, uint32_t* ids, int32_t* dists,
                                    pgb_query_stats* stats);
/* liberar */
pgb_status pgb_searcher_destroy(pgb_searcher* s);

/* ---- compressed rows (no counterpart in the reference) -----------------------------
 * 4-bit codes, 64 bytes per point next to the 128-byte vector rows: the compressed form
 * the reference's paper points to (BANG's PQ, paper/paper.tex:134-136), here as a scalar
 * code whose distances stay exact integers. Dimension d of a point is stored as a code c
 * in 0..15 standing for v = step * c + offsets[d] (c = round half up of (x - offsets[d]) /
 * step, clamped), so a search over the codes is exactly the search over the
 * reconstructed vectors v. Flat graphs with dim <= 120 only.
 * pgb_index_compress: step == 0 chooses step (1..17) and offsets from per-dimension
 * histograms, minimising the total squared reconstruction error (ties: smaller step, then
 * smaller offset); otherwise the given step and offsets[dim] are used (each v must stay
 * inside the element's range). Replaces earlier codes of the index. */
pgb_status pgb_index_compress(pgb_index* index, int32_t step, const int32_t* offsets);
/* The index's step, offsets[dim] (may be NULL) and code rows (n x 64 bytes into host
 * memory; may be NULL). */
pgb_status pgb_index_get_codes(const pgb_index* index, int32_t* step, int32_t* offsets,
                               uint8_t* codes);
/* A searcher over the code rows (plain schedule): ParlayANN's beam search with params on
 * the reconstructed vectors keeps the first `rerank` entries of each final frontier
 * (k <= rerank <= beam_size), which are then re-ranked by their exact distance to the
 * vector rows (ties by id); ids / dists receive the k best. pgb_searcher_search and
 * pgb_searcher_search_host run it; stats are those of the search over the codes, as if
 * it returned `rerank` neighbours (PGB_FLAG_SHORT: fewer than `rerank` entries). */
pgb_status pgb_searcher_create_compressed(pgb_index* index, uint32_t max_queries,
                                          const pgb_query_params* params, uint32_t rerank,
                                          pgb_searcher** out);

/* ---- plain search without device allocation (no counterpart in the reference) ------
 * For callers that may not allocate device memory at query time: cudaMalloc and cudaFree
 * can synchronise the whole device (stalling every other stream of a serving process),
 * and a host framework's caching allocator may already hold the device's free memory.
 * The same plain kernel and results as pgb_searcher_search with these params, but with
 * its per-warp visited tables in one fixed array inside the library
 * (PGB_NOALLOC_SCRATCH_BYTES on every device that loads the library, held until exit)
 * instead of a searcher's scratch; the lossy filter stays in shared memory, which caps
 * the beam at PGB_NOALLOC_MAX_BEAM (larger beams fail with PGB_ERR_BAD_ARG). Flat-graph
 * indexes only. Wide beams run on fewer warps, as many as the array holds tables for.
 * The first call on each device (made with that device current) looks up the array's
 * device address; make that first call before any stream capture. Every call on a device
 * shares the one array: calls whose kernels overlap on the GPU (other streams, other host
 * threads) race on it and return wrong neighbours, so order them on one stream or
 * synchronise between them. Nothing in the array has to start at zero: each query clears
 * its own table before use. Arguments and outputs as pgb_searcher_search; any nq. */
#define PGB_NOALLOC_SCRATCH_BYTES (16u << 20)
#define PGB_NOALLOC_MAX_BEAM 128u
pgb_status pgb_search_flat_noalloc(const pgb_index* index, const pgb_query_params* params,
                                   const void* queries, uint32_t nq, uint32_t query_stride,
                                   uint32_t* ids, int32_t* dists, pgb_query_stats* stats,
                                   void* stream);

/* ---- batched persistent form (no counterpart in the reference) -----------------------
 * One persistent launch serves queries of different beam sizes and k: warps pull the next
 * query from a device counter over a longest-beam-first order, so a long beam never holds
 * a block. Neighbours are identical to pgb_searcher_search with the same per-query params.
 * Outputs use a row stride of max_k; row q holds k_q entries then padding. On an HNSW
 * index the launch runs the HNSW kernel (cut, degree_limit, exclude_query_id and the
 * placement options do not apply). */
typedef struct pgb_batch_options {
    uint32_t max_queries;
    uint32_t max_beam;          /* largest Ls planned                                   */
    uint32_t max_k;             /* largest k planned; output row stride                 */
    double cut;
    int64_t limit;              /* <= 0: n                                              */
    uint32_t degree_limit;      /* 0: graph max degree                                  */
    uint32_t exclude_query_id;
    uint32_t query_id_base;
    uint32_t warps_per_block;   /* 1, 2 or 4; 0: default (4) / tuned                    */
    uint32_t filter_placement;  /* 0 auto, 1 shared memory (max_beam <= 128), 2 global  */
    uint32_t visited_placement; /* 0 auto, 1 shared memory, 2 global memory             */
    uint32_t blocks_per_sm;     /* cap on resident blocks per SM; 0: all that fit / tuned */
} pgb_batch_options;

typedef struct pgb_batch_config {
    uint32_t warps_per_block, blocks, filter_in_shared, visited_in_shared;
    uint32_t shared_bytes_per_warp;
    float tuned_ms;             /* time of the chosen config in the last tune (0: untuned) */
} pgb_batch_config;

pgb_status pgb_batch_create(pgb_index* index, const pgb_batch_options* opt, pgb_batch** out);
/* Host step: per-query beam sizes and k (host arrays of nq); uploads the work order. */
pgb_status pgb_batch_plan(pgb_batch* b, const uint32_t* beam_sizes, const uint32_t* ks,
                          uint32_t nq);
/* Device step: one launch over the planned queries (device pointers); capturable. */
pgb_status pgb_batch_search(pgb_batch* b, const void* queries, uint32_t query_stride,
                            uint32_t* ids, int32_t* dists, pgb_query_stats* stats,
                            void* stream);
/* Same launch from and to HOST memory, synchronous: upload of the planned queries,
 * one launch, download of ids / dists / stats (stats may be NULL); row stride max_k.
 * When every buffer is page-locked (cudaHostAlloc / cudaHostRegister / torch
 * pin_memory), the launch reads and writes them directly and no staging copy is made. */
pgb_status pgb_batch_search_host(pgb_batch* b, const void* queries, uint32_t query_stride,
                                 uint32_t* ids, int32_t* dists, pgb_query_stats* stats);
/* Autotuner: times the candidate launch shapes (warps per block; all resident blocks per
 * SM, three quarters or five eighths of them) and table placements on the planned
 * queries (outputs are overwritten) and keeps the fastest. Synchronous. */
pgb_status pgb_batch_tune(pgb_batch* b, const void* queries, uint32_t query_stride,
                          uint32_t* ids, int32_t* dists, pgb_query_stats* stats);
pgb_status pgb_batch_get_config(const pgb_batch* b, pgb_batch_config* out);
/* CUDA graph of (counter reset + launch) for these buffers; replay on any stream. */
pgb_status pgb_batch_capture(pgb_batch* b, const void* queries, uint32_t query_stride,
                             uint32_t* ids, int32_t* dists, pgb_query_stats* stats);
pgb_status pgb_batch_replay(pgb_batch* b, void* stream);
pgb_status pgb_batch_destroy(pgb_batch* b);

/* ---- serving (no counterpart in the reference) ----------------------------------------
 * A request loop over one flat-graph or HNSW index. submit() copies the query and admits
 * the request into a bounded pool (PGB_ERR_BUSY when full; the pool is sized by the device
 * memory budget). A dispatcher thread continuously packs whatever has arrived into
 * batches (longest beam first) and launches them on up to max_inflight streams, so
 * requests that arrive while others are on the GPU start as soon as a stream and slots
 * free up, overlapping with them (on an HNSW index too, each request at its own beam
 * and k). Each request gets exactly the neighbours that pgb_searcher_search returns
 * for it alone with the same params (exclusion quirk off; cut and degree_limit apply to
 * flat graphs). */
typedef struct pgb_server_options {
    uint32_t max_beam;       /* largest beam a request may ask for                       */
    uint32_t max_k;          /* largest k a request may ask for                          */
    uint32_t max_batch;      /* requests per launch (0: 1024)                            */
    uint32_t max_inflight;   /* launches on the GPU at once (0: 4)                       */
    uint64_t memory_budget;  /* device bytes for the pool (0: half of the free memory)   */
    double cut;              /* as pgb_query_params                                      */
    int64_t limit;
    uint32_t degree_limit;
    uint32_t max_wait_us;    /* hold a partial batch at most this long while launches are
                                in flight, to grow it (0: launch at once)                */
} pgb_server_options;

typedef struct pgb_server_stats {
    uint64_t submitted, completed, rejected, launches;
    uint32_t pending, in_flight, pool_slots, streams;
    double p50_us, p99_us;   /* submit-to-completion latency over the last 65,536 requests */
    double mean_batch;       /* requests per launch                                         */
} pgb_server_stats;

pgb_status pgb_server_create(pgb_index* index, const pgb_server_options* opt,
                             pgb_server** out);
/* query: host memory, index dim bytes; the ticket names the request in poll() */
pgb_status pgb_server_submit(pgb_server* s, const void* query, uint32_t beam_size, uint32_t k,
                             uint64_t* ticket);
/* Waits up to timeout_us for the request; PGB_ERR_TIMEOUT if it is not done yet. On
 * success copies k ids / dists (and stats, may be NULL) and releases the ticket. */
pgb_status pgb_server_poll(pgb_server* s, uint64_t ticket, uint32_t timeout_us, uint32_t* ids,
                           int32_t* dists, pgb_query_stats* stats);
/* A burst: n queries query_stride bytes apart with their own beam sizes and k. Admits the
 * longest prefix that fits; *admitted tells how many (tickets[0..admitted)); PGB_OK even
 * when only part of the burst fit, PGB_ERR_BUSY when none did. */
pgb_status pgb_server_submit_many(pgb_server* s, const void* queries, uint32_t n,
                                  uint32_t query_stride, const uint32_t* beam_sizes,
                                  const uint32_t* ks, uint64_t* tickets, uint32_t* admitted);
/* Non-blocking sweep over n tickets: done[i] = 1 and row i of ids / dists (stride max_k)
 * and stats[i] (may be NULL) filled for every finished request, whose ticket is released;
 * done[i] = 0 otherwise. *n_done counts the finished ones. Unknown tickets are skipped. */
pgb_status pgb_server_poll_many(pgb_server* s, const uint64_t* tickets, uint32_t n,
                                uint32_t* ids, int32_t* dists, pgb_query_stats* stats,
                                uint8_t* done, uint32_t* n_done);
pgb_status pgb_server_get_stats(pgb_server* s, pgb_server_stats* out);
/* completes the requests in flight, then frees everything */
pgb_status pgb_server_destroy(pgb_server* s);

/* ---- evaluation ---------------------------------------------------------------- */
/* recall@k with distance ties (big-ann-benchmarks compute_recall_with_distance_ties). */
double pgb_recall(const uint32_t* gt_ids, const float* gt_dists, uint32_t nq, uint32_t gt_k,
                  const uint32_t* ids, uint32_t k);

/* Search kernels (flat, HNSW, re-rank, pair distances) this process has launched through
 * the library so far, each replay of a captured batch graph counting its kernels: a host
 * counter for checking how many launches a timed region made. */
uint64_t pgb_search_launches(void);

/* ---- section profiler ----------------------------------------------------------------
 * In a library built with the section profiler (libpgb_prof.so), each flat-search warp adds
 * the clock cycles of every search phase to device totals (the reference's -DPERFIL
 * sections, cuda/busqueda.cuh:17-29). out receives n >= 10 counters: setup, visit,
 * filter, distances, sort, union, shift, cut+next cycles, then expansions and queries.
 * reset != 0 zeroes them after the read. Other builds return PGB_ERR_BAD_ARG. */
pgb_status pgb_section_profile(uint64_t* out, uint32_t n, int reset);

/* ---- graph builders (CPU, deterministic for a seed) ---------------------------------
 * vectors: n packed rows of dim bytes. nthreads <= 0: all host threads.
 * Outputs: degrees[n] and a padded n x slots adjacency (PGB_NO_NEIGHBOR padding),
 * slots = R (Vamana), trees*mst_deg (HCNNG), K (NN-descent). */
pgb_status pgb_build_vamana(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                            uint32_t R, uint32_t L, float alpha, int passes, uint64_t seed,
                            int nthreads, uint32_t* degrees, uint32_t* adjacency);
/* The same Vamana construction on GPU `device`. No counterpart in the reference, which
 * searches CPU-built graphs; it is the GPU construction the reference plans
 * (README.md:336-350: prefix-doubling batches, a search per new point, one warp per
 * point for the prune, reverse edges through a radix sort, no atomics in the order).
 * Identical insertion order, batches, search, prune and reverse-edge rules, so
 * degrees/adjacency equal pgb_build_vamana's for the same arguments. Host inputs and
 * outputs; dim <= 128. */
pgb_status pgb_build_vamana_gpu(int device, const void* vectors, uint32_t n, uint32_t dim,
                                pgb_elem elem, uint32_t R, uint32_t L, float alpha, int passes,
                                uint64_t seed, uint32_t* degrees, uint32_t* adjacency);
pgb_status pgb_build_hcnng(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                           uint32_t trees, uint32_t leaf, uint32_t mst_deg, uint64_t seed,
                           int nthreads, uint32_t* degrees, uint32_t* adjacency);
/* The same HCNNG construction on GPU `device` (no counterpart in the reference; the HCNNG
 * step of its planned GPU construction, README.md:351-353: exact 10-NN inside each
 * cluster-tree leaf, a degree-bounded MST per leaf, one warp per leaf). Identical trees,
 * leaf neighbours, MST order and row order, so degrees/adjacency equal pgb_build_hcnng's
 * for the same arguments. dim <= 128, leaf <= 1024, n < 2^31. */
pgb_status pgb_build_hcnng_gpu(int device, const void* vectors, uint32_t n, uint32_t dim,
                               pgb_elem elem, uint32_t trees, uint32_t leaf, uint32_t mst_deg,
                               uint64_t seed, uint32_t* degrees, uint32_t* adjacency);
pgb_status pgb_build_nndescent(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                               uint32_t K, uint32_t init_trees, uint32_t leaf, float alpha,
                               float delta, uint32_t max_iters, uint64_t seed, int nthreads,
                               uint32_t* degrees, uint32_t* adjacency);
/* HNSW written straight to an HNSW v3 model file. */
pgb_status pgb_build_hnsw(const void* vectors, uint32_t n, uint32_t dim, pgb_elem elem,
                          uint32_t M, uint32_t ef_construction, float ml, float alpha,
                          uint64_t seed, int nthreads, const char* path);
/* The same HNSW construction on GPU `device` (no counterpart in the reference; the HNSW
 * step of its planned GPU construction, README.md:350): identical levels, insertion
 * batches, descent, per-level search, selection and reverse-edge rules, so the file is
 * byte-identical to pgb_build_hnsw's for the same arguments. dim <= 128. */
pgb_status pgb_build_hnsw_gpu(int device, const void* vectors, uint32_t n, uint32_t dim,
                              pgb_elem elem, uint32_t M, uint32_t ef_construction, float ml,
                              float alpha, uint64_t seed, const char* path);
/* ParlayANN graph file from a padded adjacency (row i: degrees[i] ids, stride slots). */
pgb_status pgb_write_graph(const char* path, uint32_t n, uint32_t slots,
                           const uint32_t* degrees, const uint32_t* adjacency);

#ifdef __cplusplus
}
#endif
#endif /* PGB_H_ */
