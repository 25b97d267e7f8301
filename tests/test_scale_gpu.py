"""Larger-scale structure: 200,000 int8 d=100 points of the 1M workload's law with a
Vamana R=64 L=128 graph and an HNSW M=16 model (both from the GPU builders), 2,048
queries. At these sizes every search path meets real contention: thousands of warps
pulling from the work queue, global lossy filters of up to 2^17 slots per warp (Ls 700),
global visited tables, rows of 64 neighbours, HNSW (epoch, id) filters above beam 256.
Plain and batched answers equal the oracle's on every query (ids, int32 distances,
distance counts, expansions, flags)."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu

N, NQ = 200_000, 2_048


@pytest.fixture(scope="module")
def scale(pgb, synth):
    base = synth.LAW_C2.sample(N, 7, 0)
    queries = synth.LAW_C2.sample(NQ, 7, 1)
    graph = pgb.build_vamana_gpu(base, R=64, L=128, alpha=1.2, seed=0)
    return base, queries, graph


def stats3(oc, oe, of):
    return np.stack([oc, oe, of], axis=1)


@pytest.mark.parametrize("Ls", [40, 316, 700])
def test_flat_scale_matches_oracle(pgb, oracle, gpu, scale, Ls):
    import torch
    base, queries, graph = scale
    index = pgb.Index.flat(base, graph)
    oi, od, oc, oe, of = oracle.flat_search(base, graph.degrees, graph.edges, queries, 10, Ls)
    s = pgb.Searcher(index, NQ, pgb.QueryParams(k=10, beam_size=Ls))
    ids, dists, st = s.search(queries)
    assert_same(f"plain Ls={Ls} ids", ids, oi)
    assert_same(f"plain Ls={Ls} dists", dists, od)
    assert_same(f"plain Ls={Ls} stats", st[:, :3], stats3(oc, oe, of))
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    b = pgb.Batch(index, NQ, max_beam=Ls, max_k=10)
    b.plan(np.full(NQ, Ls), np.full(NQ, 10))
    bi, bd, bs = b.outputs(q.device)
    b.tune(q, bi, bd, bs)
    b.capture(q, bi, bd, bs)
    bi.fill_(0)
    b.replay()
    torch.cuda.synchronize()
    assert_same(f"batched Ls={Ls} ids", bi.cpu().numpy().view(np.uint32), oi)
    assert_same(f"batched Ls={Ls} dists", bd.cpu().numpy(), od)
    assert_same(f"batched Ls={Ls} stats", bs.cpu().numpy()[:, :3], stats3(oc, oe, of))
    b.close()
    s.liberar()
    index.close()


@pytest.mark.parametrize("Ls", [79, 400])
def test_hnsw_scale_matches_oracle(pgb, oracle, gpu, scale, Ls, tmp_path):
    import torch
    base, queries, _ = scale
    path = str(tmp_path / "m16.hnsw")
    pgb.build_hnsw_gpu(base, path, M=16, ef_construction=64, ml=0.36, alpha=0.83, seed=0)
    h = pgb.read_hnsw(path)
    index = pgb.Index.hnsw(base, h)
    oi, od, oc, oe, of = oracle.hnsw_search(base, h, queries, 10, Ls)
    s = pgb.Searcher(index, NQ, pgb.QueryParams(k=10, beam_size=Ls))
    ids, dists, st = s.search(queries)
    assert_same(f"hnsw Ls={Ls} ids", ids, oi)
    assert_same(f"hnsw Ls={Ls} dists", dists, od)
    assert_same(f"hnsw Ls={Ls} stats", st[:, :3], stats3(oc, oe, of))
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    b = pgb.Batch(index, NQ, max_beam=Ls, max_k=10)
    b.plan(np.full(NQ, Ls), np.full(NQ, 10))
    bi, bd, bs = b.outputs(q.device)
    b.capture(q, bi, bd, bs)
    for _ in range(2):
        bi.fill_(0)
        b.replay()
        torch.cuda.synchronize()
        assert_same(f"hnsw batched Ls={Ls} ids", bi.cpu().numpy().view(np.uint32), oi)
        assert_same(f"hnsw batched Ls={Ls} stats", bs.cpu().numpy()[:, :3], stats3(oc, oe, of))
    b.close()
    s.liberar()
    index.close()
