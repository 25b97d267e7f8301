"""The overflow rule on long walks: a query that expands more nodes than half the exact
visited table (flat graphs: nextpow2(8 Ls + 128) / 2) or inserts more ids than half of
is_inw (HNSW: nextpow2(32 Ls + 2048) / 2) stops there with PGB_FLAG_OVERFLOW, and its
answer, distance count and expansions are the oracle's (reference cuda/busqueda.cu:205-208,
cuda/busqueda_hnsw.cu:559).

The data make such walks: point i is a "thermometer" code of i (dimension j holds
clip(i - 254 j, 0, 254) - 127), so the distance between two points grows with the gap
between their indexes, and the graph links each point to the next two. Searching from
point 0 for the last point walks the whole chain; a query near the start stops early."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu

N = 5_000


def chain_data():
    i = np.arange(N)[:, None]
    j = np.arange(100)[None, :]
    base = (np.clip(i - 254 * j, 0, 254) - 127).astype(np.int8)
    deg = np.minimum(2, N - 1 - np.arange(N)).astype(np.uint32)
    edges = np.concatenate([np.arange(p + 1, p + 1 + d) for p, d in enumerate(deg)]).astype(np.uint32)
    targets = [N - 1, N - 7, N // 2, 3_000, 700, 129, 60, 5, 0]
    rng = np.random.default_rng(4)
    targets += list(rng.integers(0, N, 23))
    queries = base[np.array(targets)]
    return base, deg, edges, np.ascontiguousarray(queries)


@pytest.mark.parametrize("Ls", [10, 40, 100, 300])
def test_flat_overflow_matches_oracle(pgb, oracle, gpu, Ls):
    import torch
    from parlayann_gpu_busqueda_b200.formats import Graph
    base, deg, edges, queries = chain_data()
    index = pgb.Index.flat(base, Graph(N, 2, deg, edges))
    nq = len(queries)
    oi, od, oc, oe, of = oracle.flat_search(base, deg, edges, queries, 10, Ls)
    assert (of & pgb.FLAG_OVERFLOW).any() and not (of & pgb.FLAG_OVERFLOW).all()
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=Ls))
    ids, dists, st = s.search(queries)
    assert_same(f"plain Ls={Ls} ids", ids, oi)
    assert_same(f"plain Ls={Ls} dists", dists, od)
    assert_same(f"plain Ls={Ls} stats", st[:, :3], np.stack([oc, oe, of], 1))
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    placements = [(1, 1), (1, 2), (2, 1), (2, 2)] if Ls <= 128 else [(2, 1), (2, 2)]
    for fp, vp in placements:
        b = pgb.Batch(index, nq, max_beam=Ls, max_k=10, filter_placement=fp, visited_placement=vp)
        b.plan(np.full(nq, Ls), np.full(nq, 10))
        bi, bd, bs = b.outputs(q.device)
        b.search(q, bi, bd, bs)
        torch.cuda.synchronize()
        assert_same(f"batched {fp}{vp} ids", bi.cpu().numpy().view(np.uint32), oi)
        assert_same(f"batched {fp}{vp} stats", bs.cpu().numpy()[:, :3], np.stack([oc, oe, of], 1))
        b.close()
    s.liberar()
    index.close()


@pytest.mark.parametrize("Ls", [10, 40, 100])
def test_hnsw_overflow_matches_oracle(pgb, oracle, gpu, Ls):
    """A one-layer HNSW model over the same chain: is_inw fills up on the long walks."""
    import torch
    from parlayann_gpu_busqueda_b200.formats import Hnsw
    base, deg, edges, queries = chain_data()
    h = Hnsw(n=N, dim=100, m=2, efc=2, ml=0.0, alpha=1.0,
             levels=np.zeros(N, np.uint32), node_point=np.arange(N, dtype=np.uint32),
             list_sizes=deg.astype(np.uint32), ids=edges, entries=np.zeros(1, np.uint32))
    index = pgb.Index.hnsw(base, h)
    nq = len(queries)
    oi, od, oc, oe, of = oracle.hnsw_search(base, h, queries, 10, Ls)
    assert (of & pgb.FLAG_OVERFLOW).any() and not (of & pgb.FLAG_OVERFLOW).all()
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=Ls))
    ids, dists, st = s.search(queries)
    assert_same(f"hnsw Ls={Ls} ids", ids, oi)
    assert_same(f"hnsw Ls={Ls} dists", dists, od)
    assert_same(f"hnsw Ls={Ls} stats", st[:, :3], np.stack([oc, oe, of], 1))
    b = pgb.Batch(index, nq, max_beam=Ls, max_k=10)
    b.plan(np.full(nq, Ls), np.full(nq, 10))
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    bi, bd, bs = b.outputs(q.device)
    b.search(q, bi, bd, bs)
    torch.cuda.synchronize()
    assert_same(f"hnsw batched Ls={Ls} ids", bi.cpu().numpy().view(np.uint32), oi)
    assert_same(f"hnsw batched Ls={Ls} stats", bs.cpu().numpy()[:, :3], np.stack([oc, oe, of], 1))
    b.close()
    s.liberar()
    index.close()
