"""pgb_search_flat_noalloc, the plain flat-graph search for callers that may not allocate
device memory while they serve queries (cudaMalloc / cudaFree can synchronise the whole
device and stall a serving process's other streams, and a host framework's caching
allocator may already hold the free memory). It keeps its visited tables in a fixed array
inside the library; here it must return exactly what the searcher entry point
(pgb_searcher_search) returns for the same params -- integer ids, distances and counters,
so the tolerance is zero -- on two calls in a row (the second one finds the first call's
tables left in the shared array).

This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu

PGB_ERR_BAD_ARG = 1


def _noalloc(N, index, params, q, ids, dists, stats):
    cp = params.to_c()
    return N.lib.pgb_search_flat_noalloc(index.handle, C.byref(cp), C.c_void_p(q.data_ptr()),
                                         q.shape[0], q.stride(0), C.c_void_p(ids.data_ptr()),
                                         C.c_void_p(dists.data_ptr()),
                                         C.c_void_p(stats.data_ptr()), None)


@pytest.mark.parametrize("Ls,k,degree_limit", [(40, 10, 0), (128, 50, 0), (20, 10, 16)])
def test_noalloc_matches_searcher_on_two_calls(pgb, golden, gpu, Ls, k, degree_limit):
    import torch
    N = pgb.search.N
    base, queries = golden.vectors_for("vamana")
    # several queries per warp, so that warps reuse their tables within a call too
    qh = np.ascontiguousarray(np.tile(queries, (max(1, 6000 // len(queries)), 1)))
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    params = pgb.QueryParams(k=k, beam_size=Ls, degree_limit=degree_limit)
    q = torch.from_numpy(qh).cuda()
    nq = q.shape[0]
    want = pgb.Searcher(index, nq, params)
    wid, wd, ws = want.search_device(q)
    torch.cuda.synchronize()
    want.liberar()
    # outputs allocated by the caller, once; the entry point itself allocates nothing
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dists = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    stats = torch.empty((nq, 4), dtype=torch.int32, device="cuda")
    for call in range(2):
        for t in (ids, dists, stats):
            t.fill_(-7)
        st = _noalloc(N, index, params, q, ids, dists, stats)
        assert st == 0, N.lib.pgb_last_error().decode()
        torch.cuda.synchronize()
        assert_same(f"ids call {call}", ids.cpu().numpy(), wid.cpu().numpy())
        assert_same(f"dists call {call}", dists.cpu().numpy(), wd.cpu().numpy())
        assert_same(f"stats call {call}", stats[:, :3].cpu().numpy(), ws[:, :3].cpu().numpy())
    index.close()


def test_noalloc_rejects_beam_above_maximum_and_hnsw(pgb, golden, gpu):
    import torch
    N = pgb.search.N
    base, queries = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    q = torch.from_numpy(np.ascontiguousarray(queries)).cuda()
    ids = torch.empty((len(queries), 10), dtype=torch.int32, device="cuda")
    dists = torch.empty_like(ids)
    stats = torch.empty((len(queries), 4), dtype=torch.int32, device="cuda")
    st = _noalloc(N, index, pgb.QueryParams(k=10, beam_size=129), q, ids, dists, stats)
    assert st == PGB_ERR_BAD_ARG
    assert b"maximum of 128" in N.lib.pgb_last_error()
    index.close()
    hindex = pgb.Index.hnsw(base, golden.hnsw["hnsw"])
    st = _noalloc(N, hindex, pgb.QueryParams(k=10, beam_size=10), q, ids, dists, stats)
    assert st == PGB_ERR_BAD_ARG
    assert b"flat-graph indexes only" in N.lib.pgb_last_error()
    hindex.close()
