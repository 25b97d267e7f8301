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
