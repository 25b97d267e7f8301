"""Parity across vector shapes: int8 / uint8, dims where the row carries its norm
(d <= 124) and where it is recomputed (d > 124), odd dims and strided query rows."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.int8, np.uint8])
@pytest.mark.parametrize("dim", [4, 37, 100, 124, 125, 128])
def test_dims_and_types(pgb, oracle, gpu, dtype, dim):
    rng = np.random.default_rng(dim)
    n, nq = 1500, 64
    lo, hi = (-128, 128) if dtype == np.int8 else (0, 256)
    centers = rng.integers(lo, hi, size=(16, dim))
    lab = rng.integers(0, 16, size=n + nq)
    x = np.clip(centers[lab] + rng.normal(0, 20, size=(n + nq, dim)), lo, hi - 1).astype(dtype)
    base, queries = x[:n], x[n:]
    g = pgb.build_vamana(base, R=24, L=48, alpha=1.2, seed=dim)
    index = pgb.Index.flat(base, g)
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=32))
    ids, dists, stats = s.search(queries)
    oid, od, oc, oe, of = oracle.flat_search(base, g.degrees, g.edges, queries, 10, 32)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)
    assert_same("comps", stats[:, 0], oc)


def test_strided_device_queries(pgb, oracle, golden, gpu):
    """Queries read from rows 160 bytes apart on the device (query_stride > dim)."""
    import torch
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    nq = len(queries)
    wide = np.zeros((nq, 160), np.uint8)
    wide[:, :100] = queries.view(np.uint8)
    q = torch.from_numpy(wide).cuda()
    index = pgb.Index.flat(base, g)
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=40))
    ids, dists, stats = s.search_device(q[:, :100])
    torch.cuda.synchronize()
    oid, od, *_ = oracle.flat_search(base, g.degrees, g.edges, queries, 10, 40)
    assert_same("ids", ids.cpu().numpy().view(np.uint32), oid)
    assert_same("dists", dists.cpu().numpy(), od)
