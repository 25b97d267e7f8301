"""The batched persistent form returns, query by query, the oracle's answer for that
query's own (Ls, k) -- whatever launch shape or table placement the tuner picks."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


def oracle_rows(oracle, base, graph, queries, ls, ks, max_k, **kw):
    ids = np.full((len(queries), max_k), 0xFFFFFFFF, np.uint32)
    dists = np.full((len(queries), max_k), 0, np.int32)
    comps = np.zeros(len(queries), np.int32)
    exps = np.zeros(len(queries), np.int32)
    for L in np.unique(ls):
        for k in np.unique(ks):
            sel = np.nonzero((ls == L) & (ks == k))[0]
            if not len(sel):
                continue
            for q in sel:  # query index matters (exclusion quirk): one call per query
                o = oracle.flat_search(base, graph.degrees, graph.edges, queries[q:q + 1], int(k),
                                       int(L), query_id_base=int(q), **kw)
                ids[q, :k], dists[q, :k], comps[q], exps[q] = o[0][0], o[1][0], o[2][0], o[3][0]
    return ids, dists, comps, exps


@pytest.mark.parametrize("graph_name", ["vamana", "hcnng"])
def test_batch_mixed_beams_match_oracle(pgb, oracle, golden, gpu, graph_name):
    import torch
    base, queries = golden.vectors_for(graph_name)
    graph = golden.graphs[graph_name]
    rng = np.random.default_rng(11)
    nq = len(queries)
    ls = rng.choice([10, 16, 25, 40, 63, 100, 160], size=nq).astype(np.uint32)
    ks = rng.choice([10, 50], size=nq).astype(np.uint32)
    max_k = 50
    index = pgb.Index.flat(base, graph)
    b = pgb.Batch(index, nq, max_beam=int(ls.max()), max_k=max_k)
    b.plan(ls, ks)
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    ids, dists, stats = b.outputs(q.device)
    b.search(q, ids, dists, stats)
    torch.cuda.synchronize()
    oid, od, oc, oe = oracle_rows(oracle, base, graph, queries, ls, ks, max_k)
    got_i = ids.cpu().numpy().view(np.uint32)
    got_d = dists.cpu().numpy()
    st = stats.cpu().numpy()
    for qi in range(nq):
        k = ks[qi]
        assert_same(f"q{qi} ids", got_i[qi, :k], oid[qi, :k])
        assert_same(f"q{qi} dists", got_d[qi, :k], od[qi, :k])
    assert_same("comps", st[:, 0], oc)
    assert_same("expansions", st[:, 1], oe)
    # every tuned configuration and the captured graph give the same answer
    cfg = b.tune(q, ids, dists, stats)
    assert cfg["tuned_ms"] > 0
    b.capture(q, ids, dists, stats)
    ids.fill_(0)
    b.replay()
    torch.cuda.synchronize()
    for qi in range(nq):
        k = ks[qi]
        assert_same(f"replay q{qi}", ids.cpu().numpy().view(np.uint32)[qi, :k], oid[qi, :k])
    b.close()
    index.close()


@pytest.mark.parametrize("placement", [(1, 1), (1, 2), (2, 1), (2, 2)])
def test_batch_placements_identical(pgb, golden, gpu, placement):
    import torch
    base, queries = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    nq = len(queries)
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=80))
    want_i, want_d, _ = s.search(queries)
    b = pgb.Batch(index, nq, max_beam=80, max_k=10, filter_placement=placement[0],
                  visited_placement=placement[1], warps_per_block=2)
    b.plan(np.full(nq, 80), np.full(nq, 10))
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    ids, dists, stats = b.outputs(q.device)
    b.search(q, ids, dists, stats)
    torch.cuda.synchronize()
    cfg = b.config()
    assert cfg["filter_in_shared"] == (placement[0] == 1)
    assert cfg["visited_in_shared"] == (placement[1] == 1)
    assert_same("ids", ids.cpu().numpy().view(np.uint32), want_i)
    assert_same("dists", dists.cpu().numpy(), want_d)


@pytest.mark.parametrize("kind", ["vamana", "hnsw"])
@pytest.mark.parametrize("blocks_per_sm", [1, 3, 0])
def test_batch_resident_block_cap_identical(pgb, golden, gpu, kind, blocks_per_sm):
    """A cap on resident blocks per SM (a tuner candidate, or the caller's option) only
    changes how many warps share the queue: the neighbours are the plain search's, and
    tune() with a fixed cap keeps it."""
    import torch
    base, queries = golden.vectors_for(kind)
    index = (pgb.Index.hnsw(base, golden.hnsw[kind]) if kind == "hnsw"
             else pgb.Index.flat(base, golden.graphs[kind]))
    nq = len(queries)
    want_i, want_d, want_s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=40)).search(queries)
    b = pgb.Batch(index, nq, max_beam=40, max_k=10, blocks_per_sm=blocks_per_sm)
    b.plan(np.full(nq, 40), np.full(nq, 10))
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    ids, dists, stats = b.outputs(q.device)
    b.tune(q, ids, dists, stats)
    cfg = b.config()
    if blocks_per_sm:
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        assert cfg["blocks"] == blocks_per_sm * sms, cfg
    ids.fill_(0)
    b.search(q, ids, dists, stats)
    torch.cuda.synchronize()
    assert_same("ids", ids.cpu().numpy().view(np.uint32), want_i)
    assert_same("dists", dists.cpu().numpy(), want_d)
    assert_same("stats", stats.cpu().numpy()[:, :3], want_s[:, :3])
    b.close()
    index.close()


def test_batch_uniform_and_per_query_kernels_agree(pgb, golden, gpu):
    """A plan whose queries share one (Ls, k) runs the uniform-batch kernel; changing one
    query's beam switches to the per-query kernel. Both give the plain search's output."""
    import torch
    base, queries = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    nq = len(queries)
    want = {ls: pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=ls)).search(queries)
            for ls in (49, 50)}
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    b = pgb.Batch(index, nq, max_beam=50, max_k=10)
    for beams in (np.full(nq, 50), np.where(np.arange(nq) == 3, 49, 50)):
        b.plan(beams, np.full(nq, 10))
        ids, dists, stats = b.outputs(q.device)
        b.search(q, ids, dists, stats)
        torch.cuda.synchronize()
        got_i, got_d = ids.cpu().numpy().view(np.uint32), dists.cpu().numpy()
        for qi in range(nq):
            wi, wd, _ = want[int(beams[qi])]
            assert_same(f"ids q{qi} Ls={beams[qi]}", got_i[qi], wi[qi])
            assert_same(f"dists q{qi} Ls={beams[qi]}", got_d[qi], wd[qi])
    b.close()
    index.close()


def test_batch_rejects_forced_shared_filter_above_4096_slots(pgb, golden, gpu):
    base, _ = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    with pytest.raises(pgb.PgbError) as e:
        pgb.Batch(index, 16, max_beam=129, max_k=10, filter_placement=1)
    assert "4,096 slots" in str(e.value)
    index.close()


def test_batch_host_path_matches_device(pgb, oracle, golden, gpu):
    base, queries = golden.vectors_for("nnd")
    graph = golden.graphs["nnd"]
    index = pgb.Index.flat(base, graph)
    nq = len(queries)
    b = pgb.Batch(index, nq, max_beam=40, max_k=10)
    b.plan(np.full(nq, 40), np.full(nq, 10))
    ids, dists, stats = b.search_host(queries)
    oid, od, oc, oe, of = oracle.flat_search(base, graph.degrees, graph.edges, queries, 10, 40)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)


@pytest.mark.parametrize("max_beam", [160, 300])
def test_batch_hnsw_mixed_beams_match_oracle(pgb, oracle, golden, gpu, max_beam):
    """HNSW in the batched form: each query at its own (Ls, k) in one launch of the HNSW
    kernel, tables sized for max_beam (300: the (epoch, id) global filter); the answer of
    every query, its distance count and its flags are the oracle's for its (Ls, k). A
    captured graph replays to the same answer, each replay with fresh filter epochs, also
    between direct launches of the same batch."""
    import torch
    base, queries = golden.vectors_for("hnsw")
    h = golden.hnsw["hnsw"]
    rng = np.random.default_rng(3)
    nq = len(queries)
    ls = rng.choice([10, 25, 50, 100, max_beam], size=nq).astype(np.uint32)
    ks = rng.choice([10, 20], size=nq).astype(np.uint32)
    index = pgb.Index.hnsw(base, h)
    b = pgb.Batch(index, nq, max_beam=max_beam, max_k=20)
    b.plan(ls, ks)
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    ids, dists, stats = b.outputs(q.device)
    b.search(q, ids, dists, stats)
    torch.cuda.synchronize()
    got_i = ids.cpu().numpy().view(np.uint32)
    got_d = dists.cpu().numpy()
    st = stats.cpu().numpy()
    for qi in range(nq):
        k = int(ks[qi])
        oi, od, oc, oe, of = oracle.hnsw_search(base, h, queries[qi:qi + 1], k, int(ls[qi]))
        assert_same(f"q{qi} ids", got_i[qi, :k], oi[0])
        assert_same(f"q{qi} dists", got_d[qi, :k], od[0])
        assert_same(f"q{qi} comps/exps/flags", st[qi, :3], [oc[0], oe[0], of[0]])
    cfg = b.tune(q, ids, dists, stats)
    assert cfg["tuned_ms"] > 0
    b.capture(q, ids, dists, stats)
    for r in range(4):
        ids.fill_(0)
        dists.fill_(0)
        if r == 2:
            b.search(q, ids, dists, stats)  # a direct launch between replays
        else:
            b.replay()
        torch.cuda.synchronize()
        rep_i = ids.cpu().numpy().view(np.uint32)
        rep_d = dists.cpu().numpy()
        for qi in range(nq):
            assert_same(f"replay {r} q{qi} ids", rep_i[qi, :ks[qi]], got_i[qi, :ks[qi]])
            assert_same(f"replay {r} q{qi} dists", rep_d[qi, :ks[qi]], got_d[qi, :ks[qi]])
    b.close()
    index.close()


@pytest.mark.parametrize("kind", ["flat", "hnsw"])
def test_batch_host_path_pinned_buffers(pgb, golden, gpu, kind):
    """Page-locked host buffers are read and written by the launch itself; pageable ones
    go through staging copies. Both give the device path's answers."""
    import torch
    base, queries = golden.vectors_for("vamana")
    index = (pgb.Index.flat(base, golden.graphs["vamana"]) if kind == "flat"
             else pgb.Index.hnsw(base, golden.hnsw["hnsw"]))
    nq = len(queries)
    rng = np.random.default_rng(7)
    ls = rng.choice([20, 40, 64], size=nq).astype(np.uint32)
    ks = rng.choice([5, 10], size=nq).astype(np.uint32)
    b = pgb.Batch(index, nq, max_beam=64, max_k=10)
    b.plan(ls, ks)
    i0, d0, s0 = b.search_host(queries)  # pageable numpy buffers
    q = torch.from_numpy(queries.view(np.uint8)).pin_memory()
    ids = torch.full((nq, 10), -1, dtype=torch.int32).pin_memory()
    dists = torch.full((nq, 10), -1, dtype=torch.int32).pin_memory()
    st = torch.zeros((nq, 4), dtype=torch.int32).pin_memory()
    for _ in range(2):
        b.search_host(q, ids, dists, st)
        gi = ids.numpy().view(np.uint32)
        for qi in range(nq):
            k = int(ks[qi])
            assert_same(f"ids q{qi}", gi[qi, :k], i0[qi, :k])
            assert_same(f"dists q{qi}", dists.numpy()[qi, :k], d0[qi, :k])
        assert_same("stats", st.numpy()[:, :3], s0[:, :3])
    b.close()
    index.close()


def test_search_launch_counter(pgb, golden, gpu):
    """pgb_search_launches counts one launch per search call and per graph replay; the
    launch recorded while capturing a graph is not a launch."""
    import torch
    base, queries = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    nq = len(queries)
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=20))
    c0 = pgb.search_launches()
    for _ in range(3):
        s.search_device(q)
    assert pgb.search_launches() - c0 == 3
    b = pgb.Batch(index, nq, max_beam=20, max_k=10)
    b.plan(np.full(nq, 20), np.full(nq, 10))
    ids, dists, stats = b.outputs(q.device)
    c1 = pgb.search_launches()
    b.search(q, ids, dists, stats)
    b.capture(q, ids, dists, stats)
    assert pgb.search_launches() - c1 == 1
    for _ in range(4):
        b.replay()
    torch.cuda.synchronize()
    assert pgb.search_launches() - c1 == 5
    b.close()
    s.liberar()
    index.close()
