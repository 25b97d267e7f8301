"""Compressed rows (4-bit codes) through the C ABI: the chosen step and offsets, the code
rows, and the search over them followed by the exact re-rank, all bit-exact with the
oracle's restatement (beam search over the reconstructed vectors, then an exact re-rank of
the first `rerank` frontier entries)."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu

CFGS = [  # (Ls, rerank, k): shared filters, the global filter (Ls 300), k above 32
    (10, 10, 10), (40, 10, 10), (40, 40, 10), (80, 40, 10), (150, 100, 10), (300, 300, 10),
    (64, 64, 50),
]


def blobs(dtype, dim, n=1500, nq=64, seed=0):
    rng = np.random.default_rng(seed + dim)
    lo, hi = (-128, 128) if dtype == np.int8 else (0, 256)
    centers = rng.integers(lo // 2, hi // 2 if lo else hi, size=(16, dim))
    lab = rng.integers(0, 16, size=n + nq)
    x = np.clip(centers[lab] + rng.normal(0, 20, size=(n + nq, dim)), lo, hi - 1).astype(dtype)
    return x[:n], x[n:]


def check_codes(pgb, oracle, index, base):
    step, off, rows = index.codes()
    ostep, ooff = oracle.choose_codes(oracle.code_histograms(base), base.dtype == np.int8)
    assert step == ostep
    assert_same("offsets", off, ooff)
    orows, _ = oracle.encode_codes(base, step, off)
    assert_same("code rows", rows, orows)
    return step, off


def run_compressed(pgb, oracle, base, queries, g, Ls, R, k, host=True):
    index = pgb.Index.flat(base, g)
    index.compress()
    step, off = check_codes(pgb, oracle, index, base)
    s = pgb.Searcher(index, len(queries), pgb.QueryParams(k=k, beam_size=Ls), rerank=R)
    ids, dists, stats = s.search(queries)
    s.close()
    index.close()
    o = oracle.compressed_search(base, g.degrees, g.edges, queries, k, Ls, R, step, off)
    return (ids, dists, stats), o


@pytest.mark.parametrize("graph_name", ["vamana", "hcnng", "nnd", "ties_vamana"])
@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: "L%d_R%d_k%d" % c)
def test_compressed_matches_oracle(pgb, oracle, golden, gpu, graph_name, cfg):
    Ls, R, k = cfg
    base, queries = golden.vectors_for(graph_name)
    (ids, dists, stats), (oid, od, oc, oe, of) = run_compressed(
        pgb, oracle, base, queries, golden.graphs[graph_name], Ls, R, k)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    assert_same("expansions", stats[:, 1], oe)
    assert_same("flags", stats[:, 2], of)


@pytest.mark.parametrize("dtype", [np.int8, np.uint8])
@pytest.mark.parametrize("dim", [5, 37, 64, 100, 120])
def test_compressed_dims_and_types(pgb, oracle, gpu, dtype, dim):
    base, queries = blobs(dtype, dim)
    g = pgb.build_vamana(base, R=24, L=48, alpha=1.2, seed=dim)
    (ids, dists, stats), (oid, od, oc, oe, of) = run_compressed(
        pgb, oracle, base, queries, g, 32, 20, 10)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)


def test_explicit_step_and_offsets(pgb, oracle, golden, gpu):
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    rng = np.random.default_rng(3)
    step = 9
    off = rng.integers(-128, 128 - 15 * step + 1, size=base.shape[1]).astype(np.int32)
    index = pgb.Index.flat(base, g)
    index.compress(step, off)
    s2, o2, rows = index.codes()
    assert s2 == step
    assert_same("offsets", o2, off)
    assert_same("code rows", rows, oracle.encode_codes(base, step, off)[0])
    s = pgb.Searcher(index, len(queries), pgb.QueryParams(k=10, beam_size=40), rerank=30)
    ids, dists, stats = s.search(queries)
    oid, od, oc, _, _ = oracle.compressed_search(base, g.degrees, g.edges, queries, 10, 40, 30,
                                                 step, off)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    # a second compress replaces the codes
    index.compress()
    assert index.codes(rows=False)[0] == oracle.choose_codes(oracle.code_histograms(base), True)[0]


def test_compressed_pinned_and_device_paths(pgb, oracle, golden, gpu):
    """The same results through page-locked host buffers (read and written by the launch)
    and through device tensors on a stream."""
    import torch
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    index = pgb.Index.flat(base, g)
    index.compress()
    step, off, _ = index.codes(rows=False)
    nq, k = len(queries), 10
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=k, beam_size=64), rerank=48)
    oid, od, oc, _, _ = oracle.compressed_search(base, g.degrees, g.edges, queries, k, 64, 48,
                                                 step, off)
    qp = torch.from_numpy(queries).pin_memory()
    ip = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    dp = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    from parlayann_gpu_busqueda_b200 import _native as N
    import ctypes as C
    N.check(N.lib.pgb_searcher_search_host(s._h, qp.data_ptr(), nq, queries.shape[1],
                                           ip.data_ptr(), dp.data_ptr(), None))
    assert_same("pinned ids", ip.numpy().view(np.uint32), oid)
    assert_same("pinned dists", dp.numpy(), od)
    qd = torch.from_numpy(queries).cuda()
    ids, dists, stats = s.search_device(qd)
    torch.cuda.synchronize()
    assert_same("device ids", ids.cpu().numpy().view(np.uint32), oid)
    assert_same("device dists", dists.cpu().numpy(), od)
    assert_same("device comps", stats[:, 0].cpu().numpy(), oc)
    s.close()
    index.close()


def test_compressed_arguments(pgb, golden, gpu):
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    index = pgb.Index.flat(base, g)
    p = pgb.QueryParams(k=10, beam_size=40)
    with pytest.raises(pgb.PgbError):  # no codes yet
        pgb.Searcher(index, 8, p, rerank=20)
    with pytest.raises(pgb.PgbError):
        index.codes()
    index.compress()
    for bad in (5, 41):  # below k, above beam_size
        with pytest.raises(pgb.PgbError):
            pgb.Searcher(index, 8, p, rerank=bad)
    with pytest.raises(pgb.PgbError):  # step out of range
        index.compress(18, np.full(base.shape[1], -128, np.int32))
    with pytest.raises(pgb.PgbError):  # offset + 15 * step above 127
        index.compress(9, np.full(base.shape[1], 0, np.int32))
    index.close()
    wide = np.zeros((64, 121), np.int8)
    gw = pgb.build_vamana(wide, R=8, L=16, alpha=1.2, seed=0)
    iw = pgb.Index.flat(wide, gw)
    with pytest.raises(pgb.PgbError):  # more than 120 dimensions
        iw.compress()
    iw.close()
    h = pgb.Index.hnsw(base, golden.hnsw["hnsw"])
    with pytest.raises(pgb.PgbError):
        h.compress()
    h.close()
