"""Edge cases of the search, through the C ABI, against the oracle: the smallest and the
largest beam (1 and PGB_MAX_BEAM = 1024), k above the beam (short frontiers padded with
0xFFFFFFFF / INT_MAX and flagged), an empty batch, and a two-point index."""
import numpy as np
import pytest

from conftest import assert_same
from test_search_gpu import run_both

pytestmark = pytest.mark.gpu

EDGES = [(1, 1), (1, 10), (5, 20), (1024, 10), (1024, 100)]


@pytest.mark.parametrize("Ls,k", EDGES, ids=lambda v: str(v))
def test_flat_extreme_beams_and_k(pgb, oracle, golden, gpu, Ls, k):
    base, queries = golden.vectors_for("vamana")
    q = queries[:32]
    (ids, dists, stats), (oid, od, oc, oe, of) = run_both(
        pgb, oracle, base, q, golden.graphs["vamana"], Ls, 0, k, 1.35)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    assert_same("expansions", stats[:, 1], oe)
    assert_same("flags", stats[:, 2], of)
    if k > Ls:
        # fewer than k entries can survive: padded rows and the short flag
        assert (stats[:, 2] & pgb.FLAG_SHORT).any()
        assert (ids == pgb.NO_NEIGHBOR).any()


@pytest.mark.parametrize("Ls,k", EDGES, ids=lambda v: str(v))
def test_hnsw_extreme_beams_and_k(pgb, oracle, golden, gpu, Ls, k):
    base, queries = golden.vectors_for("hnsw")
    h = golden.hnsw["hnsw"]
    q = queries[:32]
    index = pgb.Index.hnsw(base, h)
    s = pgb.Searcher(index, len(q), pgb.QueryParams(k=k, beam_size=Ls))
    ids, dists, stats = s.search(q)
    s.liberar()
    index.close()
    oid, od, oc, oe, of = oracle.hnsw_search(base, h, q, k, Ls)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    assert_same("expansions", stats[:, 1], oe)
    assert_same("flags", stats[:, 2], of)


def test_empty_batch_is_a_no_op(pgb, golden, gpu):
    base, queries = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    s = pgb.Searcher(index, 8, pgb.QueryParams(k=10, beam_size=20))
    ids, dists, stats = s.search(queries[:0])
    assert ids.shape == (0, 10) and dists.shape == (0, 10) and stats.shape == (0, 4)
    ids, dists, stats = s.search(queries[:4])  # still usable
    assert ids.shape == (4, 10)
    s.liberar()
    index.close()


def test_two_point_index(pgb, oracle, gpu):
    base = np.array([[1, 2, 3, 4], [-5, 6, -7, 8]], np.int8)
    queries = np.array([[0, 0, 0, 0], [-5, 6, -7, 9], [127, -128, 0, 1]], np.int8)
    g = pgb.Graph.from_padded(np.array([1, 1], np.uint32), np.array([[1], [0]], np.uint32))
    for Ls, k in ((1, 1), (2, 2), (4, 3)):
        (ids, dists, stats), (oid, od, oc, oe, of) = run_both(pgb, oracle, base, queries, g, Ls, 0,
                                                              k, 1.35, exclude_query_id=False)
        assert_same(f"ids {Ls},{k}", ids, oid)
        assert_same(f"dists {Ls},{k}", dists, od)
        assert_same(f"flags {Ls},{k}", stats[:, 2], of)
