"""Python host side over the C ABI: index, searcher (BuscadorGPU / BuscadorHnsw), builders.

Mirrors the reference's search interface (reference cuda/busqueda.cuh:36-61,
cuda/hnsw.h:65-86): a searcher is prepared for (graph, number of queries, config)
(``preparar``), launched asynchronously on a stream (``lanzar``) and released
(``liberar``). ConfigBusqueda{Ls, limite, k, cut} becomes QueryParams with ParlayANN's
names {k, beam_size, cut, limit, degree_limit}. Errors raise PgbError (the reference
exits the process instead).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .formats import Graph, Hnsw


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())


def _elem(dtype) -> int:
    return N.PGB_INT8 if np.dtype(dtype) == np.int8 else N.PGB_UINT8


@dataclass
class QueryParams:
    """ParlayANN QueryParams; defaults are the reference's ConfigBusqueda
    (Ls=10, no visit limit, k=10, cut=1.35)."""
    k: int = 10
    beam_size: int = 10
    cut: float = 1.35
    limit: int = 0                 # <= 0: n
    degree_limit: int = 0          # 0: graph max degree
    exclude_query_id: bool = True  # ParlayANN wrapper's `a == p.id()` quirk (flat graphs)
    query_id_base: int = 0

    def to_c(self) -> N.QueryParams:
        return N.QueryParams(self.k, self.beam_size, float(self.cut), int(self.limit),
                             self.degree_limit, 1 if self.exclude_query_id else 0,
                             self.query_id_base, 0)


class Index:
    """Device-resident index (vectors + graph). Read-only after creation."""

    def __init__(self, handle: int, dtype, device: int = 0):
        self._h = C.c_void_p(handle)
        self.dtype = np.dtype(dtype)
        self.device = device
        info = N.IndexInfo()
        N.check(N.lib.pgb_index_get_info(self._h, C.byref(info)))
        self.info = info

    @classmethod
    def flat(cls, vectors: np.ndarray, graph: Graph, device: int = 0) -> "Index":
        v = np.ascontiguousarray(vectors)
        deg = np.ascontiguousarray(graph.degrees, dtype=np.uint32)
        edges = np.ascontiguousarray(graph.edges, dtype=np.uint32)
        h = C.c_void_p()
        N.check(N.lib.pgb_index_create_flat(device, _ptr(v), v.shape[0], v.shape[1],
                                            _elem(v.dtype), _ptr(deg),
                                            _ptr(edges) if edges.size else 0, C.byref(h)))
        return cls(h.value, v.dtype, device)

    @classmethod
    def hnsw(cls, vectors: np.ndarray, h: Hnsw, device: int = 0) -> "Index":
        v = np.ascontiguousarray(vectors)
        arrs = [np.ascontiguousarray(a, dtype=np.uint32)
                for a in (h.levels, h.node_point, h.list_sizes, h.ids, h.entries)]
        out = C.c_void_p()
        N.check(N.lib.pgb_index_create_hnsw(device, _ptr(v), v.shape[0], v.shape[1],
                                            _elem(v.dtype), h.n, *[_ptr(a) for a in arrs[:4]],
                                            _ptr(arrs[4]), len(arrs[4]), C.byref(out)))
        return cls(out.value, v.dtype, device)

    @classmethod
    def load_flat(cls, vectors_path: str, graph_path: str, dtype=np.int8, device: int = 0):
        h = C.c_void_p()
        N.check(N.lib.pgb_index_load_flat(device, vectors_path.encode(), _elem(dtype),
                                          graph_path.encode(), C.byref(h)))
        return cls(h.value, dtype, device)

    @classmethod
    def load_hnsw(cls, vectors_path: str, hnsw_path: str, dtype=np.int8, device: int = 0):
        h = C.c_void_p()
        N.check(N.lib.pgb_index_load_hnsw(device, vectors_path.encode(), _elem(dtype),
                                          hnsw_path.encode(), C.byref(h)))
        return cls(h.value, dtype, device)

    @property
    def handle(self):
        return self._h

    def compress(self, step: int = 0, offsets=None) -> None:
        """4-bit code rows next to the vectors (flat graphs, dim <= 120): dimension d is
        stored as c in 0..15 standing for step * c + offsets[d]. step 0 chooses step and
        offsets from the data (least squared reconstruction error)."""
        off = None if offsets is None else np.ascontiguousarray(offsets, dtype=np.int32)
        N.check(N.lib.pgb_index_compress(self._h, int(step), _ptr(off)))
        self.info = N.IndexInfo()
        N.check(N.lib.pgb_index_get_info(self._h, C.byref(self.info)))

    def set_l2_window(self, region: str, max_bytes: int = 0):
        """Persisting L2 window over "rows", "codes" or "graph" (None / "none" removes it),
        carried by every later flat search launch; returns (window bytes, hit ratio)."""
        r = {None: N.L2_NONE, "none": N.L2_NONE, "rows": N.L2_ROWS, "codes": N.L2_CODES,
             "graph": N.L2_GRAPH}[region]
        wb, hr = C.c_uint64(), C.c_float()
        N.check(N.lib.pgb_index_set_l2_window(self._h, r, int(max_bytes), C.byref(wb),
                                              C.byref(hr)))
        return wb.value, hr.value

    def distances(self, queries, pairs, stream: int = 0) -> np.ndarray:
        """Exact int32 squared L2 of (query row, point id) pairs by the search kernels' row
        code. queries: [nq, dim] (numpy or CUDA tensor); pairs: [npairs, 2] uint32."""
        import torch
        dev = torch.device("cuda", self.device)
        q = queries if hasattr(queries, "data_ptr") else torch.from_numpy(
            np.ascontiguousarray(queries).view(np.uint8)).to(dev)
        pr = pairs if hasattr(pairs, "data_ptr") else torch.from_numpy(
            np.ascontiguousarray(pairs, dtype=np.uint32).view(np.int32)).to(dev)
        npairs = pr.shape[0]
        out = torch.empty(max(1, npairs), dtype=torch.int32, device=dev)
        N.check(N.lib.pgb_index_distances(self._h, _ptr(q), q.shape[0], q.stride(0), _ptr(pr),
                                          npairs, _ptr(out), C.c_void_p(stream)))
        return out[:npairs].cpu().numpy()

    def gather_probe(self, query, ids, lanes_per_row: int, out=None, stream: int = 0):
        """Distances of one device query row to the rows `ids` (CUDA uint32 tensor) with
        lanes_per_row threads per row; returns the output tensor (asynchronous)."""
        import torch
        if out is None:
            out = torch.empty(ids.shape[0], dtype=torch.int32, device=ids.device)
        N.check(N.lib.pgb_gather_probe(self._h, _ptr(query), _ptr(ids), ids.shape[0], _ptr(out),
                                       lanes_per_row, C.c_void_p(stream)))
        return out

    def codes(self, rows: bool = True):
        """(step, offsets int32 [dim], code rows uint8 [n, 64] or None)."""
        step = C.c_int32()
        off = np.zeros(self.info.dim, dtype=np.int32)
        codes = np.empty((self.info.n_points, 64), dtype=np.uint8) if rows else None
        N.check(N.lib.pgb_index_get_codes(self._h, C.byref(step), _ptr(off), _ptr(codes)))
        return step.value, off, codes

    def close(self):
        if self._h:
            N.lib.pgb_index_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Searcher:
    """BuscadorGPU / BuscadorHnsw: prepare once for (index, max queries, params)."""

    def __init__(self, index: Index, max_queries: int, params: QueryParams, rerank: int = 0):
        """rerank > 0: search the index's code rows (Index.compress) keeping `rerank`
        candidates per query (k <= rerank <= beam_size), re-ranked exactly into k."""
        self.index, self.params, self.max_queries = index, params, max_queries
        self.rerank = rerank
        self._cp = params.to_c()
        h = C.c_void_p()
        if rerank:
            N.check(N.lib.pgb_searcher_create_compressed(index.handle, max_queries,
                                                         C.byref(self._cp), rerank, C.byref(h)))
        else:
            N.check(N.lib.pgb_searcher_create(index.handle, max_queries, C.byref(self._cp),
                                              C.byref(h)))
        self._h = h

    def lanzar(self, queries, ids, dists, stats=None, stream: int = 0, query_stride=None):
        """Asynchronous search of device queries into device outputs (torch tensors or
        raw pointers); ``stream`` is a cudaStream_t value (0 = default stream)."""
        nq = queries.shape[0]
        stride = query_stride or (queries.stride(0) if hasattr(queries, "stride") else queries.shape[1])
        N.check(N.lib.pgb_searcher_search(self._h, _ptr(queries), nq, stride, _ptr(ids),
                                          _ptr(dists), _ptr(stats), C.c_void_p(stream)))

    def search_device(self, queries, stream: int = 0):
        """torch CUDA uint8/int8 queries [nq, dim] -> (ids, dists, stats) torch tensors."""
        import torch
        nq, k = queries.shape[0], self.params.k
        ids = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
        dists = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
        stats = torch.empty((nq, 4), dtype=torch.int32, device=queries.device)
        self.lanzar(queries, ids, dists, stats, stream)
        return ids, dists, stats

    def search(self, queries: np.ndarray):
        """Host queries -> host (ids uint32 [nq,k], dists int32 [nq,k], stats int32 [nq,4]),
        synchronous (query upload, search, result download)."""
        q = np.ascontiguousarray(queries)
        nq, k = q.shape[0], self.params.k
        ids = np.empty((nq, k), dtype=np.uint32)
        dists = np.empty((nq, k), dtype=np.int32)
        stats = np.empty((nq, 4), dtype=np.int32)
        N.check(N.lib.pgb_searcher_search_host(self._h, _ptr(q), nq, q.shape[1], _ptr(ids),
                                               _ptr(dists), _ptr(stats)))
        return ids, dists, stats

    def liberar(self):
        if self._h:
            N.lib.pgb_searcher_destroy(self._h)
            self._h = C.c_void_p()

    close = liberar

    def __del__(self):
        try:
            self.liberar()
        except Exception:
            pass


def recall(gt_ids: np.ndarray, gt_dists: np.ndarray, ids: np.ndarray, k: int) -> float:
    """recall@k with distance ties (big-ann-benchmarks compute_recall_with_distance_ties;
    reference cuda/evaluacion.cpp:56-80)."""
    gi = np.ascontiguousarray(gt_ids, dtype=np.uint32)
    gd = np.ascontiguousarray(gt_dists, dtype=np.float32)
    ii = np.ascontiguousarray(ids[:, :k], dtype=np.uint32)
    r = N.lib.pgb_recall(_ptr(gi), _ptr(gd), gi.shape[0], gi.shape[1], _ptr(ii), k)
    if r < 0:
        raise ValueError("recall: bad arguments")
    return r


# ---- builders (CPU, deterministic) ----------------------------------------------------
def build_vamana(x: np.ndarray, R: int = 32, L: int = 64, alpha: float = 1.2, passes: int = 1,
                 seed: int = 0, threads: int = 0) -> Graph:
    x = np.ascontiguousarray(x)
    deg = np.empty(x.shape[0], dtype=np.uint32)
    adj = np.empty((x.shape[0], R), dtype=np.uint32)
    N.check(N.lib.pgb_build_vamana(_ptr(x), x.shape[0], x.shape[1], _elem(x.dtype), R, L,
                                   alpha, passes, seed, threads, _ptr(deg), _ptr(adj)))
    return Graph.from_padded(deg, adj)


def build_vamana_gpu(x: np.ndarray, R: int = 32, L: int = 64, alpha: float = 1.2,
                     passes: int = 1, seed: int = 0, device: int = 0) -> Graph:
    """build_vamana on the GPU: the same graph for the same arguments."""
    x = np.ascontiguousarray(x)
    deg = np.empty(x.shape[0], dtype=np.uint32)
    adj = np.empty((x.shape[0], R), dtype=np.uint32)
    N.check(N.lib.pgb_build_vamana_gpu(device, _ptr(x), x.shape[0], x.shape[1], _elem(x.dtype),
                                       R, L, alpha, passes, seed, _ptr(deg), _ptr(adj)))
    return Graph.from_padded(deg, adj)


def build_hcnng(x: np.ndarray, trees: int = 30, leaf: int = 1000, mst_deg: int = 3,
                seed: int = 0, threads: int = 0) -> Graph:
    x = np.ascontiguousarray(x)
    slots = trees * mst_deg
    deg = np.empty(x.shape[0], dtype=np.uint32)
    adj = np.empty((x.shape[0], slots), dtype=np.uint32)
    N.check(N.lib.pgb_build_hcnng(_ptr(x), x.shape[0], x.shape[1], _elem(x.dtype), trees, leaf,
                                  mst_deg, seed, threads, _ptr(deg), _ptr(adj)))
    return Graph.from_padded(deg, adj)


def build_hcnng_gpu(x: np.ndarray, trees: int = 30, leaf: int = 1000, mst_deg: int = 3,
                    seed: int = 0, device: int = 0) -> Graph:
    """build_hcnng on the GPU: the same graph for the same arguments (leaf <= 1024)."""
    x = np.ascontiguousarray(x)
    slots = trees * mst_deg
    deg = np.empty(x.shape[0], dtype=np.uint32)
    adj = np.empty((x.shape[0], slots), dtype=np.uint32)
    N.check(N.lib.pgb_build_hcnng_gpu(device, _ptr(x), x.shape[0], x.shape[1], _elem(x.dtype),
                                      trees, leaf, mst_deg, seed, _ptr(deg), _ptr(adj)))
    return Graph.from_padded(deg, adj)


def build_nndescent(x: np.ndarray, K: int = 40, init_trees: int = 10, leaf: int = 1000,
                    alpha: float = 1.2, delta: float = 0.05, max_iters: int = 8, seed: int = 0,
                    threads: int = 0) -> Graph:
    x = np.ascontiguousarray(x)
    deg = np.empty(x.shape[0], dtype=np.uint32)
    adj = np.empty((x.shape[0], K), dtype=np.uint32)
    N.check(N.lib.pgb_build_nndescent(_ptr(x), x.shape[0], x.shape[1], _elem(x.dtype), K,
                                      init_trees, leaf, alpha, delta, max_iters, seed, threads,
                                      _ptr(deg), _ptr(adj)))
    return Graph.from_padded(deg, adj)


def build_hnsw(x: np.ndarray, path: str, M: int = 32, ef_construction: int = 128,
               ml: float = 0.36, alpha: float = 0.83, seed: int = 0, threads: int = 0) -> None:
    x = np.ascontiguousarray(x)
    N.check(N.lib.pgb_build_hnsw(_ptr(x), x.shape[0], x.shape[1], _elem(x.dtype), M,
                                 ef_construction, ml, alpha, seed, threads, path.encode()))


def build_hnsw_gpu(x: np.ndarray, path: str, M: int = 32, ef_construction: int = 128,
                   ml: float = 0.36, alpha: float = 0.83, seed: int = 0, device: int = 0) -> None:
    """build_hnsw on the GPU: the same file for the same arguments."""
    x = np.ascontiguousarray(x)
    N.check(N.lib.pgb_build_hnsw_gpu(device, _ptr(x), x.shape[0], x.shape[1], _elem(x.dtype), M,
                                     ef_construction, ml, alpha, seed, path.encode()))


def file_check(path: str, kind: str):
    """C-reader validation of a file on the host: kind 'vectors', 'graph' or 'hnsw'.
    Returns the 4 info counters; raises PgbError (IO or FORMAT) on a bad file."""
    info = (C.c_uint64 * 4)()
    k = {"vectors": 0, "graph": 1, "hnsw": 2}[kind]
    N.check(N.lib.pgb_file_check(path.encode(), k, info))
    return list(info)


def device_available() -> bool:
    return bool(N.lib.pgb_device_available())


def search_launches() -> int:
    """Search kernels this process has launched through the library (graph replays count
    their kernels)."""
    return int(N.lib.pgb_search_launches())


class Batch:
    """Batched persistent form: one launch over queries with per-query (Ls, k).

    plan() is the host step (longest beam first work order); search()/replay() are
    device-only and return the same neighbours as Searcher with the same params.
    Output rows have stride max_k. warps_per_block, filter_placement,
    visited_placement and blocks_per_sm (a cap on resident blocks per SM) fix parts of
    the launch shape (0: automatic); tune() times the rest on the planned queries."""

    def __init__(self, index: Index, max_queries: int, max_beam: int, max_k: int,
                 cut: float = 1.35, limit: int = 0, degree_limit: int = 0,
                 exclude_query_id: bool = True, query_id_base: int = 0,
                 warps_per_block: int = 0, filter_placement: int = 0, visited_placement: int = 0,
                 blocks_per_sm: int = 0):
        self.index, self.max_k = index, max_k
        self._opt = N.BatchOptions(max_queries, max_beam, max_k, float(cut), int(limit),
                                   degree_limit, 1 if exclude_query_id else 0, query_id_base,
                                   warps_per_block, filter_placement, visited_placement,
                                   blocks_per_sm)
        h = C.c_void_p()
        N.check(N.lib.pgb_batch_create(index.handle, C.byref(self._opt), C.byref(h)))
        self._h = h
        self.nq = 0

    def plan(self, beam_sizes, ks):
        ls = np.ascontiguousarray(beam_sizes, dtype=np.uint32)
        kk = np.ascontiguousarray(ks, dtype=np.uint32)
        assert ls.shape == kk.shape
        N.check(N.lib.pgb_batch_plan(self._h, _ptr(ls), _ptr(kk), ls.shape[0]))
        self.nq = ls.shape[0]

    def _args(self, queries, ids, dists, stats):
        stride = queries.stride(0) if hasattr(queries, "stride") else queries.shape[1]
        return _ptr(queries), stride, _ptr(ids), _ptr(dists), _ptr(stats)

    def search(self, queries, ids, dists, stats=None, stream: int = 0):
        q, st, i, d, s = self._args(queries, ids, dists, stats)
        N.check(N.lib.pgb_batch_search(self._h, q, st, i, d, s, C.c_void_p(stream)))

    def search_host(self, queries: np.ndarray, ids=None, dists=None, stats=None):
        """Host queries (planned count) -> host ids/dists/stats, synchronous. Pass pinned
        numpy/torch buffers to avoid staging copies in the driver."""
        q = queries if not isinstance(queries, np.ndarray) else np.ascontiguousarray(queries)
        if ids is None:
            ids = np.empty((self.nq, self.max_k), dtype=np.uint32)
            dists = np.empty((self.nq, self.max_k), dtype=np.int32)
            stats = np.empty((self.nq, 4), dtype=np.int32)
        stride = q.stride(0) if hasattr(q, "stride") else q.shape[1]
        N.check(N.lib.pgb_batch_search_host(self._h, _ptr(q), stride, _ptr(ids), _ptr(dists),
                                            _ptr(stats)))
        return ids, dists, stats

    def tune(self, queries, ids, dists, stats=None):
        q, st, i, d, s = self._args(queries, ids, dists, stats)
        N.check(N.lib.pgb_batch_tune(self._h, q, st, i, d, s))
        return self.config()

    def config(self) -> dict:
        c = N.BatchConfig()
        N.check(N.lib.pgb_batch_get_config(self._h, C.byref(c)))
        return {f: getattr(c, f) for f, _ in N.BatchConfig._fields_}

    def capture(self, queries, ids, dists, stats=None):
        q, st, i, d, s = self._args(queries, ids, dists, stats)
        N.check(N.lib.pgb_batch_capture(self._h, q, st, i, d, s))

    def replay(self, stream: int = 0):
        N.check(N.lib.pgb_batch_replay(self._h, C.c_void_p(stream)))

    def outputs(self, device):
        """Device output buffers (torch) of the right shape for this batch."""
        import torch
        ids = torch.empty((self.nq, self.max_k), dtype=torch.int32, device=device)
        dists = torch.empty((self.nq, self.max_k), dtype=torch.int32, device=device)
        stats = torch.empty((self.nq, 4), dtype=torch.int32, device=device)
        return ids, dists, stats

    def close(self):
        if self._h:
            N.lib.pgb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (pgb_server_*): submit() -> ticket, poll(ticket)."""

    BUSY, TIMEOUT = 7, 8

    def __init__(self, index: Index, max_beam: int, max_k: int, max_batch: int = 0,
                 max_inflight: int = 0, memory_budget: int = 0, cut: float = 1.35,
                 limit: int = 0, degree_limit: int = 0, max_wait_us: int = 0):
        self.index, self.max_k = index, max_k
        self._opt = N.ServerOptions(max_beam, max_k, max_batch, max_inflight, memory_budget,
                                    float(cut), int(limit), degree_limit, max_wait_us)
        h = C.c_void_p()
        N.check(N.lib.pgb_server_create(index.handle, C.byref(self._opt), C.byref(h)))
        self._h = h

    def submit(self, query: np.ndarray, beam_size: int, k: int):
        """Returns the ticket, or None when the pool is full (PGB_ERR_BUSY)."""
        q = np.ascontiguousarray(query)
        t = C.c_uint64()
        st = N.lib.pgb_server_submit(self._h, _ptr(q), beam_size, k, C.byref(t))
        if st == self.BUSY:
            return None
        N.check(st)
        return t.value

    def poll(self, ticket: int, k: int, timeout_us: int = 0):
        """(ids, dists, stats) when done, None on timeout."""
        ids = np.empty(k, np.uint32)
        dists = np.empty(k, np.int32)
        stats = np.empty(4, np.int32)
        st = N.lib.pgb_server_poll(self._h, ticket, timeout_us, _ptr(ids), _ptr(dists),
                                   _ptr(stats))
        if st == self.TIMEOUT:
            return None
        N.check(st)
        return ids, dists, stats

    def submit_many(self, queries: np.ndarray, beam_sizes, ks):
        """Burst submission; returns the tickets of the admitted prefix (may be empty)."""
        q = np.ascontiguousarray(queries)
        ls = np.ascontiguousarray(beam_sizes, dtype=np.uint32)
        kk = np.ascontiguousarray(ks, dtype=np.uint32)
        t = np.empty(len(q), np.uint64)
        got = C.c_uint32()
        st = N.lib.pgb_server_submit_many(self._h, _ptr(q), len(q), q.shape[1], _ptr(ls),
                                          _ptr(kk), _ptr(t), C.byref(got))
        if st == self.BUSY:
            return t[:0]
        N.check(st)
        return t[:got.value]

    def poll_many(self, tickets: np.ndarray):
        """Non-blocking: (done mask, ids [n, max_k], dists [n, max_k], stats [n, 4])."""
        t = np.ascontiguousarray(tickets, dtype=np.uint64)
        n = len(t)
        ids = np.empty((n, self.max_k), np.uint32)
        dists = np.empty((n, self.max_k), np.int32)
        stats = np.empty((n, 4), np.int32)
        done = np.zeros(n, np.uint8)
        cnt = C.c_uint32()
        N.check(N.lib.pgb_server_poll_many(self._h, _ptr(t), n, _ptr(ids), _ptr(dists),
                                           _ptr(stats), _ptr(done), C.byref(cnt)))
        return done.astype(bool), ids, dists, stats

    def stats(self) -> dict:
        s = N.ServerStats()
        N.check(N.lib.pgb_server_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in N.ServerStats._fields_}

    def close(self):
        if self._h:
            N.lib.pgb_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
