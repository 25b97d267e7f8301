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


# ---- compressed rows (4-bit codes) --------------------------------------------------
# The library's code rows (pgb_index_compress, parlayann-gpu-busqueda_b200/csrc/codes.cu)
# store dimension d of a point as c in 0..15 standing for v = step * c + offsets[d]; the
# search over them is ParlayANN's beam search on the reconstructed vectors v, followed by
# an exact re-rank of the first `rerank` frontier entries. The reference has no such
# format; these functions restate the library's rules so the parity check is exact.

def code_histograms(base):
    """Per-dimension 256-bin histograms of value - lo (lo = -128 for int8, 0 for uint8)."""
    b = np.asarray(base)
    v = b.astype(np.int64) + (128 if b.dtype == np.int8 else 0)
    h = np.zeros((b.shape[1], 256), np.int64)
    for d in range(b.shape[1]):
        h[d] = np.bincount(v[:, d], minlength=256)
    return h


def _codes_of(x, step, off):
    num = 2 * (x - off) + step  # round half up of (x - off) / step, clamped to 0..15
    return np.where(num < 0, 0, np.minimum(15, num // (2 * step)))


def choose_codes(hist, signed):
    """The step in 1..17 and per-dimension offsets minimising the total squared
    reconstruction error (ties: smaller step, then smaller offset), every reconstructed
    value inside the element's range."""
    lo, hi = (-128, 127) if signed else (0, 255)
    dim = hist.shape[0]
    x = np.arange(256, dtype=np.int64) + lo
    best = None
    for s in range(1, (hi - lo) // 15 + 1):
        offs = np.arange(lo, hi - 15 * s + 1, dtype=np.int64)
        # err[o, d] = sum_x hist[d, x] (x - v(x))^2
        c = _codes_of(x[None, :], s, offs[:, None])            # [o, x]
        e2 = (x[None, :] - (s * c + offs[:, None])) ** 2         # [o, x]
        err = e2 @ hist.T                                        # [o, d]
        j = np.argmin(err, axis=0)                               # first (smallest) offset
        total = int(err[j, np.arange(dim)].sum())
        if best is None or total < best[0]:
            best = (total, s, offs[j].astype(np.int32))
    return best[1], best[2]


def encode_codes(base, step, offsets):
    """(code rows uint8 [n, 64] in the library's nibble layout, reconstructed vectors of
    the base's dtype)."""
    b = np.asarray(base)
    n, dim = b.shape
    off = np.asarray(offsets, np.int64)[:dim]
    c = _codes_of(b.astype(np.int64), step, off[None, :])
    v = step * c + off[None, :]
    rows = np.zeros((n, 64), np.uint8)
    d = np.arange(dim)
    byte = (d >> 5) * 16 + ((d >> 3) & 3) * 4 + (d & 3)
    shift = 4 * ((d >> 2) & 1)
    for j in range(dim):
        rows[:, byte[j]] |= (c[:, j] << shift[j]).astype(np.uint8)
    norm = (v * v).sum(1).astype(np.uint32)
    rows[:, 60:64] = norm.view(np.uint8).reshape(n, 4)
    return rows, v.astype(b.dtype)


def exact_rerank(base, queries, cand, k):
    """The first k of each row of candidate ids (padding 0xFFFFFFFF dropped) by exact
    squared distance, ties by id; padded with 0xFFFFFFFF / INT32_MAX."""
    b = np.asarray(base).astype(np.int64)
    q = np.asarray(queries).astype(np.int64)
    nq = cand.shape[0]
    ids = np.full((nq, k), 0xFFFFFFFF, np.uint32)
    dists = np.full((nq, k), np.iinfo(np.int32).max, np.int32)
    for i in range(nq):
        c = cand[i][cand[i] != 0xFFFFFFFF].astype(np.int64)
        if c.size == 0:
            continue
        d = ((b[c] - q[i][None, :]) ** 2).sum(1)
        order = np.lexsort((c, d))[:k]
        ids[i, :order.size] = c[order]
        dists[i, :order.size] = d[order]
    return ids, dists


def compressed_search(base, degrees, edges, queries, k, Ls, rerank, step, offsets, **kw):
    """Beam search over the reconstructed vectors keeping `rerank` entries, then the exact
    re-rank to k; returns ids, dists and the search's comps, expansions, flags."""
    _, v = encode_codes(base, step, offsets)
    cid, _, comps, exps, flags = flat_search(v, degrees, edges, queries, rerank, Ls, **kw)
    ids, dists = exact_rerank(base, queries, cid, k)
    return ids, dists, comps, exps, flags
