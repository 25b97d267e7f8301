"""Parity of the CUDA flat-graph search with the oracle (bit-exact ids, int32 distances,
distance counts, expansions and flags), through the C ABI."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu

FLAT_CFGS = [  # (Ls, visit, k, cut) -- the reference's (Ls, visit) configs at small scale
    (10, 3, 10, 1.35), (10, 8, 10, 1.35), (10, 0, 10, 1.35), (20, 0, 10, 1.35),
    (40, 0, 10, 1.35), (80, 0, 10, 1.35), (40, 0, 10, 0.9), (64, 0, 50, 1.35),
    (150, 0, 10, 1.35), (300, 0, 10, 1.35),
]


def run_both(pgb, oracle, base, queries, graph, Ls, visit, k, cut, **kw):
    index = pgb.Index.flat(base, graph)
    p = pgb.QueryParams(k=k, beam_size=Ls, cut=cut, limit=visit, **kw)
    s = pgb.Searcher(index, len(queries), p)
    ids, dists, stats = s.search(queries)
    s.liberar()
    index.close()
    o = oracle.flat_search(base, graph.degrees, graph.edges, queries, k, Ls, cut=cut, limit=visit,
                           degree_limit=kw.get("degree_limit", 0),
                           exclude_query_id=kw.get("exclude_query_id", True),
                           query_id_base=kw.get("query_id_base", 0))
    return (ids, dists, stats), o


@pytest.mark.parametrize("graph_name", ["vamana", "hcnng", "nnd", "ties_vamana"])
@pytest.mark.parametrize("cfg", FLAT_CFGS, ids=lambda c: "L%d_v%d_k%d_c%g" % c)
def test_flat_matches_oracle(pgb, oracle, golden, gpu, graph_name, cfg):
    Ls, visit, k, cut = cfg
    base, queries = golden.vectors_for(graph_name)
    (ids, dists, stats), (oid, od, oc, oe, of) = run_both(
        pgb, oracle, base, queries, golden.graphs[graph_name], Ls, visit, k, cut)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    assert_same("expansions", stats[:, 1], oe)
    assert_same("flags", stats[:, 2], of)


def test_searchers_with_different_beams_coexist(pgb, oracle, golden, gpu):
    """Several live searchers of one kernel variant keep working after each other's
    creation (their launch shapes differ; none may shrink another's limits)."""
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    index = pgb.Index.flat(base, g)
    wide = pgb.Searcher(index, len(queries), pgb.QueryParams(k=10, beam_size=120))
    narrow = pgb.Searcher(index, len(queries), pgb.QueryParams(k=10, beam_size=12))
    for s, Ls in ((wide, 120), (narrow, 12), (wide, 120)):
        ids, dists, _ = s.search(queries)
        oid, od, *_ = oracle.flat_search(base, g.degrees, g.edges, queries, 10, Ls)
        assert_same(f"ids Ls={Ls}", ids, oid)
        assert_same(f"dists Ls={Ls}", dists, od)


def test_query_id_base_and_exclusion_off(pgb, oracle, golden, gpu):
    """The exclusion quirk follows query_id_base; with exclusion off every id is eligible."""
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    for excl, qb in ((True, 37), (False, 0)):
        (ids, dists, st), (oid, od, oc, oe, of) = run_both(
            pgb, oracle, base, queries, g, 30, 0, 10, 1.35, exclude_query_id=excl,
            query_id_base=qb)
        assert_same(f"ids excl={excl}", ids, oid)
        assert_same(f"comps excl={excl}", st[:, 0], oc)


@pytest.mark.parametrize("deg_lim", [1, 7, 20, 31])
def test_degree_limit(pgb, oracle, golden, gpu, deg_lim):
    base, queries = golden.vectors_for("hcnng")
    g = golden.graphs["hcnng"]
    (ids, dists, st), (oid, od, oc, oe, of) = run_both(
        pgb, oracle, base, queries, g, 40, 0, 10, 1.35, degree_limit=deg_lim)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", st[:, 0], oc)


def test_concurrent_searchers_share_an_index(pgb, golden, gpu):
    """The threading contract: an index is read-only once created, so several host threads
    may search it at once, each through its own searcher (own stream, own scratch). Four
    threads on a flat and an HNSW index, at different beams, five rounds each: every round
    returns the single-thread answer."""
    import threading
    base, queries = golden.vectors_for("vamana")
    flat = pgb.Index.flat(base, golden.graphs["vamana"])
    hnsw = pgb.Index.hnsw(base, golden.hnsw["hnsw"])
    cfgs = [(flat, 20, 10), (flat, 64, 50), (hnsw, 50, 10), (hnsw, 300, 20)]
    expect = []
    for ix, Ls, k in cfgs:
        s = pgb.Searcher(ix, len(queries), pgb.QueryParams(k=k, beam_size=Ls))
        expect.append(s.search(queries))
        s.liberar()
    bad = []

    def worker(i):
        ix, Ls, k = cfgs[i]
        s = pgb.Searcher(ix, len(queries), pgb.QueryParams(k=k, beam_size=Ls))
        try:
            for r in range(5):
                ids, dists, st = s.search(queries)
                if not (np.array_equal(ids, expect[i][0]) and np.array_equal(dists, expect[i][1])
                        and np.array_equal(st, expect[i][2])):
                    bad.append((i, r))
        finally:
            s.liberar()

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(len(cfgs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not bad, bad
    flat.close()
    hnsw.close()


@pytest.mark.parametrize("kind", ["flat", "hnsw"])
def test_searcher_host_path_pinned_buffers(pgb, golden, gpu, kind):
    """pgb_searcher_search_host with page-locked buffers: the launch reads the queries (at
    their stride) and writes the results through them; the answers are those of the
    staged path."""
    import torch
    base, queries = golden.vectors_for("vamana")
    index = (pgb.Index.flat(base, golden.graphs["vamana"]) if kind == "flat"
             else pgb.Index.hnsw(base, golden.hnsw["hnsw"]))
    nq, k = len(queries), 10
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=k, beam_size=50))
    want_i, want_d, want_s = s.search(queries)  # pageable numpy: staging copies
    wide = torch.zeros((nq, 112), dtype=torch.uint8).pin_memory()  # rows 112 bytes apart
    wide[:, :queries.shape[1]] = torch.from_numpy(queries.view(np.uint8))
    ids = torch.full((nq, k), -1, dtype=torch.int32).pin_memory()
    dists = torch.full((nq, k), -1, dtype=torch.int32).pin_memory()
    st = torch.zeros((nq, 4), dtype=torch.int32).pin_memory()
    lib = pgb._native.lib
    pgb._native.check(lib.pgb_searcher_search_host(s._h, wide.data_ptr(), nq, 112, ids.data_ptr(),
                                                   dists.data_ptr(), st.data_ptr()))
    assert_same("ids", ids.numpy().view(np.uint32), want_i)
    assert_same("dists", dists.numpy(), want_d)
    assert_same("stats", st.numpy()[:, :3], want_s[:, :3])
    s.liberar()
    index.close()
