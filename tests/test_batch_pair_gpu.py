"""The batched form's paired schedule (two queries per warp, one per 16-lane half) returns,
query by query, the oracle's answer for that query's own (Ls, k): ids, int32 distances,
distance counts, expansions and flags, for every graph family, table placement and
launch shape, with odd query counts (a half that finds the queue empty exits while the
other half finishes) and with the visit limit, the cut and the exclusion quirk varied."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


def oracle_answer(oracle, base, graph, queries, ls, ks, max_k, **kw):
    nq = len(queries)
    ids = np.full((nq, max_k), 0xFFFFFFFF, np.uint32)
    dists = np.zeros((nq, max_k), np.int32)
    st = np.zeros((nq, 3), np.int32)
    for q in range(nq):  # the query index matters (exclusion quirk): one call per query
        k = int(ks[q])
        o = oracle.flat_search(base, graph.degrees, graph.edges, queries[q:q + 1], k, int(ls[q]),
                               query_id_base=q, **kw)
        ids[q, :k], dists[q, :k] = o[0][0], o[1][0]
        st[q] = (o[2][0], o[3][0], o[4][0])
    return ids, dists, st


def run_pair(pgb, index, queries, ls, ks, max_k, **opt):
    import torch
    nq = len(queries)
    b = pgb.Batch(index, nq, max_beam=int(ls.max()), max_k=max_k, queries_per_warp=2, **opt)
    b.plan(ls, ks)
    q = torch.from_numpy(np.ascontiguousarray(queries).view(np.uint8)).cuda()
    ids, dists, stats = b.outputs(q.device)
    b.search(q, ids, dists, stats)
    torch.cuda.synchronize()
    cfg = b.config()
    assert cfg["queries_per_warp"] == 2
    out = ids.cpu().numpy().view(np.uint32), dists.cpu().numpy(), stats.cpu().numpy()
    return b, q, out


def check_rows(got, want, ks, tag):
    gi, gd, gs = got
    wi, wd, ws = want
    for qi in range(len(ks)):
        k = int(ks[qi])
        assert_same(f"{tag} q{qi} ids", gi[qi, :k], wi[qi, :k])
        assert_same(f"{tag} q{qi} dists", gd[qi, :k], wd[qi, :k])
    assert_same(f"{tag} comps/expansions/flags", gs[:, :3], ws)


@pytest.mark.parametrize("graph_name", ["vamana", "hcnng", "nnd", "ties_vamana"])
@pytest.mark.parametrize("placement", [(1, 2), (2, 2), (1, 1), (2, 1)])
def test_pair_mixed_beams_match_oracle(pgb, oracle, golden, gpu, graph_name, placement):
    base, queries = golden.vectors_for(graph_name)
    graph = golden.graphs[graph_name]
    rng = np.random.default_rng(5)
    nq = len(queries)
    beams = [10, 16, 25, 40, 63, 100] if placement[0] == 1 else [10, 40, 100, 160, 300]
    ls = rng.choice(beams, size=nq).astype(np.uint32)
    ks = rng.choice([1, 10, 50], size=nq).astype(np.uint32)
    index = pgb.Index.flat(base, graph)
    b, _, got = run_pair(pgb, index, queries, ls, ks, 50, filter_placement=placement[0],
                         visited_placement=placement[1], warps_per_block=2)
    want = oracle_answer(oracle, base, graph, queries, ls, ks, 50)
    check_rows(got, want, ks, f"{graph_name} {placement}")
    b.close()
    index.close()


@pytest.mark.parametrize("nq", [1, 2, 3, 31, 97])
def test_pair_odd_query_counts(pgb, oracle, golden, gpu, nq):
    base, queries = golden.vectors_for("vamana")
    graph = golden.graphs["vamana"]
    queries = np.ascontiguousarray(queries[:nq])
    ls = np.full(nq, 40, np.uint32)
    ks = np.full(nq, 10, np.uint32)
    index = pgb.Index.flat(base, graph)
    for wpb in (1, 4):
        b, _, got = run_pair(pgb, index, queries, ls, ks, 10, warps_per_block=wpb)
        check_rows(got, oracle_answer(oracle, base, graph, queries, ls, ks, 10), ks, f"wpb{wpb}")
        b.close()
    index.close()


@pytest.mark.parametrize("kw", [dict(limit=7), dict(cut=1.0), dict(cut=2.5),
                                dict(exclude_query_id=False), dict(degree_limit=20)])
def test_pair_params(pgb, oracle, golden, gpu, kw):
    base, queries = golden.vectors_for("hcnng")
    graph = golden.graphs["hcnng"]
    nq = len(queries)
    rng = np.random.default_rng(9)
    ls = rng.choice([12, 30, 64], size=nq).astype(np.uint32)
    ks = np.full(nq, 10, np.uint32)
    index = pgb.Index.flat(base, graph)
    b, _, got = run_pair(pgb, index, queries, ls, ks, 10, **kw)
    want = oracle_answer(oracle, base, graph, queries, ls, ks, 10, **kw)
    check_rows(got, want, ks, str(kw))
    b.close()
    index.close()


def test_pair_tuned_and_captured_identical(pgb, oracle, golden, gpu):
    """The tuner may pick either schedule; whatever it picks, and a captured graph of it,
    give the one-query-per-warp kernel's answer."""
    import torch
    base, queries = golden.vectors_for("vamana")
    graph = golden.graphs["vamana"]
    nq = len(queries)
    ls = np.full(nq, 40, np.uint32)
    ks = np.full(nq, 10, np.uint32)
    index = pgb.Index.flat(base, graph)
    b, q, got = run_pair(pgb, index, queries, ls, ks, 10)
    one = pgb.Batch(index, nq, max_beam=40, max_k=10, queries_per_warp=1)
    one.plan(ls, ks)
    i1, d1, s1 = one.outputs(q.device)
    one.search(q, i1, d1, s1)
    torch.cuda.synchronize()
    assert_same("pair vs single ids", got[0], i1.cpu().numpy().view(np.uint32))
    assert_same("pair vs single dists", got[1], d1.cpu().numpy())
    assert_same("pair vs single stats", got[2], s1.cpu().numpy())
    ids, dists, stats = b.outputs(q.device)
    b.tune(q, ids, dists, stats)
    b.capture(q, ids, dists, stats)
    for _ in range(2):
        ids.fill_(0)
        b.replay()
        torch.cuda.synchronize()
        assert_same("replay ids", ids.cpu().numpy().view(np.uint32), got[0])
    b.close()
    one.close()
    index.close()


def test_pair_rejects_rows_above_128(pgb, golden, gpu):
    """Rows wider than 128 neighbours are served by one query per warp only."""
    rng = np.random.default_rng(0)
    n = 300
    base = rng.integers(-50, 50, size=(n, 16), dtype=np.int8)
    deg = np.full(n, 140, np.uint32)
    edges = np.concatenate([rng.choice(n, 140, replace=False) for _ in range(n)]).astype(np.uint32)
    from parlayann_gpu_busqueda_b200.formats import Graph
    index = pgb.Index.flat(base, Graph(n, 140, deg, edges))
    with pytest.raises(pgb.PgbError, match="128 neighbours"):
        pgb.Batch(index, 4, max_beam=20, max_k=10, queries_per_warp=2)
    index.close()
