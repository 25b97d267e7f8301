"""Known-answer test of the distance, the reference's load-and-verify step
(cuda/paso1_carga.cu:33-123) restated: the search kernels' own row code
(pgb_index_distances: dp4a over 128-byte rows, the norm folded into the row padding for
d <= 124) gives exactly the CPU restatement's int32 squared L2 (cuda/lectores.cpp:172-179)
for 200,000 random (query, point) pairs and for every (query, ground-truth neighbour)
pair of 1,000 queries, on int8 d=100 and uint8 d=128 data, and at the extremes of both
element types."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


def chain_graph(n):
    """The smallest valid flat graph: point i -> point i + 1 (the distance needs none)."""
    from parlayann_gpu_busqueda_b200.formats import Graph
    return Graph(n, 1, np.ones(n, np.uint32), ((np.arange(n) + 1) % n).astype(np.uint32))


@pytest.mark.parametrize("law_name,n", [("LAW_C2", 200_000), ("LAW_C4", 100_000)])
def test_pair_distances_known_answer(pgb, oracle, synth, gpu, law_name, n):
    from parlayann_gpu_busqueda_b200 import groundtruth
    law = getattr(synth, law_name)
    base, queries = synth.dataset(law, n, 1_000, seed=0)
    index = pgb.Index.flat(base, chain_graph(n))
    rng = np.random.default_rng(1)
    pairs = np.stack([rng.integers(0, len(queries), 200_000),
                      rng.integers(0, n, 200_000)], axis=1).astype(np.uint32)
    got = index.distances(queries, pairs)
    assert_same("random pairs", got, oracle.pair_distances(base, queries, pairs))
    # an independent int64 restatement on a sample of them
    s = pairs[:5_000]
    d64 = ((queries[s[:, 0]].astype(np.int64) - base[s[:, 1]].astype(np.int64)) ** 2).sum(1)
    assert_same("random pairs, int64", got[:5_000].astype(np.int64), d64)
    # ground-truth pairs: each query with its 10 exact neighbours (GPU brute force), whose
    # float distances are the same integers
    gt_i, gt_d = groundtruth.knn_gpu(base, queries, 10)
    gp = np.stack([np.repeat(np.arange(len(queries)), 10), gt_i.ravel()], axis=1).astype(np.uint32)
    got_gt = index.distances(queries, gp)
    assert_same("ground-truth pairs", got_gt, oracle.pair_distances(base, queries, gp))
    assert_same("ground-truth pairs vs gt distances", got_gt.astype(np.float32), gt_d.ravel())
    index.close()


@pytest.mark.parametrize("dtype,dim", [(np.int8, 100), (np.uint8, 128), (np.int8, 7),
                                       (np.uint8, 124)])
def test_pair_distances_extremes(pgb, oracle, gpu, dtype, dim):
    info = np.iinfo(dtype)
    rows = [np.full(dim, info.min), np.full(dim, info.max), np.zeros(dim),
            np.resize([info.min, info.max], dim), np.resize([info.max, 0, info.min], dim)]
    base = np.stack(rows).astype(dtype)
    index = pgb.Index.flat(base, chain_graph(len(base)))
    pairs = np.array([(i, j) for i in range(len(base)) for j in range(len(base))], np.uint32)
    got = index.distances(base, pairs)
    want = ((base[pairs[:, 0]].astype(np.int64) - base[pairs[:, 1]].astype(np.int64)) ** 2).sum(1)
    assert_same("extremes", got.astype(np.int64), want)
    assert_same("extremes vs oracle", got, oracle.pair_distances(base, base, pairs))
    # the largest distance of the element type is reached and exact
    assert got.max() == dim * (int(info.max) - int(info.min)) ** 2
    index.close()


def test_pair_distances_reject_out_of_range(pgb, gpu):
    base = np.zeros((10, 16), np.int8)
    index = pgb.Index.flat(base, chain_graph(10))
    with pytest.raises(pgb.PgbError, match="out of range"):
        index.distances(base[:2], np.array([[0, 3], [0, 10]], np.uint32))
    with pytest.raises(pgb.PgbError, match="out of range"):
        index.distances(base[:2], np.array([[2, 3]], np.uint32))
    index.close()


@pytest.mark.parametrize("dtype,dim", [(np.int8, 100), (np.uint8, 128), (np.int8, 33)])
def test_gather_probe_layouts_agree(pgb, oracle, gpu, dtype, dim):
    """The gather calibration's four layouts (1, 4, 8 and 32 threads per row) compute the
    exact distances of the pair-distance entry point; ids past the table give INT32_MIN."""
    import torch
    rng = np.random.default_rng(2)
    info = np.iinfo(dtype)
    n = 5_000
    base = rng.integers(info.min, int(info.max) + 1, size=(n, dim)).astype(dtype)
    query = rng.integers(info.min, int(info.max) + 1, size=(1, dim)).astype(dtype)
    index = pgb.Index.flat(base, chain_graph(n))
    ids = rng.integers(0, n, 20_011).astype(np.uint32)
    ids[::997] = n + 7  # out of range
    want = oracle.pair_distances(base, query, np.stack([np.zeros_like(ids), np.minimum(ids, n - 1)], 1))
    want = np.where(ids >= n, np.iinfo(np.int32).min, want)
    q = torch.from_numpy(query.view(np.uint8)[0].copy()).cuda()
    tid = torch.from_numpy(ids.view(np.int32)).cuda()
    for lanes in (1, 4, 8, 32):
        got = index.gather_probe(q, tid, lanes)
        torch.cuda.synchronize()
        assert_same(f"{lanes} lanes/row", got.cpu().numpy(), want)
    with pytest.raises(pgb.PgbError, match="lanes_per_row"):
        index.gather_probe(q, tid, 2)
    index.close()
