"""Parity of the CUDA HNSW search with the oracle, through the C ABI."""
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu

HNSW_CFGS = [(10, 0, 10), (50, 0, 10), (100, 0, 10), (50, 5, 10), (20, 0, 20), (150, 0, 10),
             (300, 0, 10)]


@pytest.mark.parametrize("name", ["hnsw", "ties_hnsw"])
@pytest.mark.parametrize("cfg", HNSW_CFGS, ids=lambda c: "L%d_v%d_k%d" % c)
def test_hnsw_matches_oracle(pgb, oracle, golden, gpu, name, cfg):
    Ls, visit, k = cfg
    base, queries = golden.vectors_for(name)
    h = golden.hnsw[name]
    index = pgb.Index.hnsw(base, h)
    s = pgb.Searcher(index, len(queries), pgb.QueryParams(k=k, beam_size=Ls, limit=visit))
    ids, dists, stats = s.search(queries)
    s.liberar()
    index.close()
    oid, od, oc, oe, of = oracle.hnsw_search(base, h, queries, k, Ls, limit=visit)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    assert_same("expansions", stats[:, 1], oe)
    assert_same("flags", stats[:, 2], of)


@pytest.fixture(scope="module")
def hnsw_m24(pgb, golden, tmp_path_factory):
    """An M=24 model of the golden base: level-0 rows of up to 48 neighbours, so an
    expansion can pass more than 32 of them (two chunks of pending neighbours)."""
    p = str(tmp_path_factory.mktemp("hnsw") / "m24.hnsw")
    pgb.build_hnsw(golden.base, p, M=24, ef_construction=64, ml=0.4, alpha=1.0, seed=2)
    return pgb.read_hnsw(p)


@pytest.mark.parametrize("cfg", [(10, 0, 10), (50, 0, 10), (100, 0, 10), (300, 0, 10), (64, 7, 20)],
                         ids=lambda c: "L%d_v%d_k%d" % c)
def test_hnsw_two_chunk_rows_match_oracle(pgb, oracle, golden, gpu, hnsw_m24, cfg):
    Ls, visit, k = cfg
    index = pgb.Index.hnsw(golden.base, hnsw_m24)
    assert index.info.max_degree > 32
    s = pgb.Searcher(index, len(golden.queries), pgb.QueryParams(k=k, beam_size=Ls, limit=visit))
    ids, dists, stats = s.search(golden.queries)
    s.liberar()
    index.close()
    oid, od, oc, oe, of = oracle.hnsw_search(golden.base, hnsw_m24, golden.queries, k, Ls, limit=visit)
    assert (stats[:, 0] > 32).any()
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    assert_same("expansions", stats[:, 1], oe)
    assert_same("flags", stats[:, 2], of)


def with_duplicate_neighbours(h, seed):
    """The model with repeated ids inside its lists: in about half of the lists of three
    or more, the last entry becomes a copy of the first, and in a quarter of the lists of
    five or more, entry 3 a copy of entry 1 (another id between the copies, so on the
    4-slot upper-layer filters the second copy often passes the filter again)."""
    import dataclasses
    import numpy as np
    rng = np.random.default_rng(seed)
    ids = h.ids.copy()
    off, sz = h.list_offsets[:-1], h.list_sizes.astype(np.int64)
    a = np.flatnonzero((sz >= 3) & (rng.random(len(sz)) < 0.5))
    ids[off[a] + sz[a] - 1] = ids[off[a]]
    b = np.flatnonzero((sz >= 5) & (rng.random(len(sz)) < 0.25))
    ids[off[b] + 3] = ids[off[b] + 1]
    return dataclasses.replace(h, ids=ids)


@pytest.mark.parametrize("Ls", [10, 50, 150, 300])
def test_hnsw_duplicate_neighbours_match_oracle(pgb, oracle, golden, gpu, Ls):
    """Repeated ids in a row: only the first copy that passes the filter can be accepted
    (is_inw), and every copy that passes costs a distance."""
    import numpy as np
    import torch
    base, queries = golden.vectors_for("hnsw")
    h = with_duplicate_neighbours(golden.hnsw["hnsw"], 5)
    index = pgb.Index.hnsw(base, h)
    nq = len(queries)
    oid, od, oc, oe, of = oracle.hnsw_search(base, h, queries, 10, Ls)
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=Ls))
    ids, dists, stats = s.search(queries)
    s.liberar()
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("stats", stats[:, :3], np.stack([oc, oe, of], 1))
    b = pgb.Batch(index, nq, max_beam=Ls, max_k=10)
    b.plan(np.full(nq, Ls), np.full(nq, 10))
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    bi, bd, bs = b.outputs(q.device)
    b.search(q, bi, bd, bs)
    torch.cuda.synchronize()
    assert_same("batched ids", bi.cpu().numpy().view(np.uint32), oid)
    assert_same("batched stats", bs.cpu().numpy()[:, :3], np.stack([oc, oe, of], 1))
    b.close()
    index.close()
