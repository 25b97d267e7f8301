"""The L2 access-policy window (pgb_index_set_l2_window) changes where lines live, never
the results: plain, compressed and batched searches with a window over each region stay
bit-exact with the oracle."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("region", ["rows", "codes", "graph"])
def test_window_keeps_results(pgb, oracle, golden, gpu, region):
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    nq, k, Ls = len(queries), 10, 40
    index = pgb.Index.flat(base, g)
    index.compress()
    wb, hr = index.set_l2_window(region)
    region_bytes = {"rows": 128, "codes": 64, "graph": 4 * ((g.degrees.max() + 31) // 32 * 32)}[region]
    assert 0 < wb <= region_bytes * len(base)
    assert 0.0 < hr <= 1.0
    oid, od, oc, oe, of = oracle.flat_search(base, g.degrees, g.edges, queries, k, Ls)
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=k, beam_size=Ls))
    ids, dists, stats = s.search(queries)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)
    s.close()
    step, off, _ = index.codes(rows=False)
    cid, cd, cc, _, _ = oracle.compressed_search(base, g.degrees, g.edges, queries, k, Ls, 30,
                                                 step, off)
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=k, beam_size=Ls), rerank=30)
    ids, dists, stats = s.search(queries)
    assert_same("compressed ids", ids, cid)
    assert_same("compressed dists", dists, cd)
    s.close()
    b = pgb.Batch(index, nq, max_beam=Ls, max_k=k)
    b.plan(np.full(nq, Ls), np.full(nq, k))
    bi, bd, bs = b.search_host(queries)
    assert_same("batched ids", bi, oid)
    assert_same("batched dists", bd, od)
    b.close()
    assert index.set_l2_window(None) == (0, 0.0)
    index.close()


def test_window_arguments(pgb, golden, gpu):
    base, _ = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    with pytest.raises(pgb.PgbError):  # no code rows yet
        index.set_l2_window("codes")
    from parlayann_gpu_busqueda_b200 import _native as N
    import ctypes as C
    assert N.lib.pgb_index_set_l2_window(index.handle, 9, 0, None, None) != 0  # unknown region
    wb, _ = index.set_l2_window("rows", max_bytes=1 << 16)
    assert wb == 1 << 16
    index.close()  # destroys with the window set
    h = pgb.Index.hnsw(base, golden.hnsw["hnsw"])
    with pytest.raises(pgb.PgbError):
        h.set_l2_window("rows")
    h.close()
