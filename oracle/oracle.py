"""ctypes front end of liboracle.so, the CPU restatement of the search path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs, always as the checker, never as the thing measured
against itself or shipped. See oracle.cpp for the reference lines it restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    vp, u32, i32, i64 = C.c_void_p, C.c_uint32, C.c_int, C.c_int64
    lib.oracle_flat_search.restype = C.c_int
    lib.oracle_flat_search.argtypes = [vp, u32, u32, u32, i32, vp, vp, vp, u32, u32, u32, u32,
                                       C.c_double, i64, u32, i32, u32, u32, vp, vp, vp, vp, vp,
                                       i32]
    lib.oracle_hnsw_search.restype = C.c_int
    lib.oracle_hnsw_search.argtypes = [vp, u32, u32, i32, u32, vp, vp, vp, vp, vp, u32, vp, u32,
                                       u32, u32, u32, i64, vp, vp, vp, vp, vp, i32]
    lib.oracle_recall.restype = C.c_double
    lib.oracle_recall.argtypes = [vp, vp, u32, u32, vp, u32]
    lib.oracle_pair_distances.restype = None
    lib.oracle_pair_distances.argtypes = [vp, u32, vp, u32, u32, i32, vp, C.c_uint64, vp]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _p(a):
    return a.ctypes.data


def flat_search(base, degrees, edges, queries, k, Ls, cut=1.35, limit=0, degree_limit=0,
                exclude_query_id=True, query_id_base=0, start=0, threads=0):
    """ParlayANN beam_search over a CSR graph; returns ids, dists, comps, expansions, flags."""
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries)
    degrees = np.ascontiguousarray(degrees, dtype=np.uint32)
    edges = np.ascontiguousarray(edges, dtype=np.uint32)
    if edges.size == 0:
        edges = np.zeros(1, np.uint32)
    nq = queries.shape[0]
    ids = np.empty((nq, k), np.uint32)
    dists = np.empty((nq, k), np.int32)
    comps = np.empty(nq, np.int32)
    exps = np.empty(nq, np.int32)
    flags = np.empty(nq, np.int32)
    threads = threads or os.cpu_count() or 1
    rc = lib().oracle_flat_search(_p(base), base.shape[0], base.shape[1], base.shape[1],
                                  int(base.dtype == np.int8), _p(degrees), _p(edges),
                                  _p(queries), nq, queries.shape[1], k, Ls, cut, limit,
                                  degree_limit, int(exclude_query_id), query_id_base, start,
                                  _p(ids), _p(dists), _p(comps), _p(exps), _p(flags), threads)
    if rc != 0:
        raise ValueError("oracle_flat_search: bad arguments")
    return ids, dists, comps, exps, flags


def hnsw_search(base, h, queries, k, Ls, limit=0, threads=0):
    """ParlayANN HNSW search over a formats.Hnsw model."""
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries)
    arrs = [np.ascontiguousarray(a, dtype=np.uint32)
            for a in (h.levels, h.node_point, h.list_sizes, h.ids, h.entries)]
    if arrs[3].size == 0:
        arrs[3] = np.zeros(1, np.uint32)
    nq = queries.shape[0]
    ids = np.empty((nq, k), np.uint32)
    dists = np.empty((nq, k), np.int32)
    comps = np.empty(nq, np.int32)
    exps = np.empty(nq, np.int32)
    flags = np.empty(nq, np.int32)
    threads = threads or os.cpu_count() or 1
    rc = lib().oracle_hnsw_search(_p(base), base.shape[1], base.shape[1],
                                  int(base.dtype == np.int8), h.n, *[_p(a) for a in arrs],
                                  len(arrs[4]), _p(queries), nq, queries.shape[1], k, Ls, limit,
                                  _p(ids), _p(dists), _p(comps), _p(exps), _p(flags), threads)
    if rc != 0:
        raise ValueError("oracle_hnsw_search: bad arguments")
    return ids, dists, comps, exps, flags


def recall(gt_ids, gt_dists, ids, k):
    gi = np.ascontiguousarray(gt_ids, dtype=np.uint32)
    gd = np.ascontiguousarray(gt_dists, dtype=np.float32)
    ii = np.ascontiguousarray(ids[:, :k], dtype=np.uint32)
    return lib().oracle_recall(_p(gi), _p(gd), gi.shape[0], gi.shape[1], _p(ii), k)


def pair_distances(base, queries, pairs):
    base = np.ascontiguousarray(base)
    queries = np.ascontiguousarray(queries)
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    out = np.empty(pairs.shape[0], np.int32)
    lib().oracle_pair_distances(_p(base), base.shape[1], _p(queries), queries.shape[1],
                                base.shape[1], int(base.dtype == np.int8), _p(pairs),
                                pairs.shape[0], _p(out))
    return out


def brute_force_knn(base, queries, k):
    """Exact k-NN by int64 numpy arithmetic (small cases): ids sorted by (dist, id)."""
    b = base.astype(np.int64)
    q = queries.astype(np.int64)
    d = (q * q).sum(1)[:, None] + (b * b).sum(1)[None, :] - 2 * q @ b.T
    order = np.lexsort((np.broadcast_to(np.arange(b.shape[0]), d.shape), d), axis=1)[:, :k]
    return order.astype(np.uint32), np.take_along_axis(d, order, 1).astype(np.int64)
