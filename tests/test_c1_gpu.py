"""The small plain-method workload at its full shape: 10,000 int8 d=100 vectors from the
64-centre mixture (centres uniform in [-40, 40], sigma 12, seed 0), 1,000 queries of the
same law, a Vamana graph R=32 L=64 alpha=1.2, k=10 and Ls in {10, 20, 40, 80}.

For every beam, the plain searcher, the batched form and the CPU restatement agree on
every query's ids, int32 distances, distance count, expansions and flags; recall@10
(with distance ties, against exact ground truth) is highest at the widest beam and
above 0.9 there."""
import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu

BEAMS = (10, 20, 40, 80)


@pytest.fixture(scope="module")
def c1(pgb, synth):
    base, queries = synth.c1(seed=0)
    assert base.shape == (10_000, 100) and queries.shape == (1_000, 100)
    graph = pgb.build_vamana(base, R=32, L=64, alpha=1.2, seed=0)
    return base, queries, graph


def test_c1_plain_and_batched_match_oracle(pgb, oracle, gpu, c1):
    import torch
    from parlayann_gpu_busqueda_b200 import groundtruth
    base, queries, graph = c1
    nq = len(queries)
    index = pgb.Index.flat(base, graph)
    q = torch.from_numpy(queries.view(np.uint8)).cuda()
    gt_i, gt_d = groundtruth.knn_gpu(base, queries, 100)
    recalls = []
    for Ls in BEAMS:
        oi, od, oc, oe, of = oracle.flat_search(base, graph.degrees, graph.edges, queries, 10, Ls)
        s = pgb.Searcher(index, nq, pgb.QueryParams(k=10, beam_size=Ls))
        ids, dists, st = s.search(queries)
        assert_same(f"plain Ls={Ls} ids", ids, oi)
        assert_same(f"plain Ls={Ls} dists", dists, od)
        assert_same(f"plain Ls={Ls} comps", st[:, 0], oc)
        assert_same(f"plain Ls={Ls} expansions", st[:, 1], oe)
        assert_same(f"plain Ls={Ls} flags", st[:, 2], of)
        s.liberar()
        b = pgb.Batch(index, nq, max_beam=Ls, max_k=10)
        b.plan(np.full(nq, Ls, np.uint32), np.full(nq, 10, np.uint32))
        bi, bd, bs = b.outputs(q.device)
        b.search(q, bi, bd, bs)
        torch.cuda.synchronize()
        assert_same(f"batched Ls={Ls} ids", bi.cpu().numpy().view(np.uint32), oi)
        assert_same(f"batched Ls={Ls} dists", bd.cpu().numpy(), od)
        bst = bs.cpu().numpy()
        assert_same(f"batched Ls={Ls} stats", bst[:, :3], np.stack([oc, oe, of], axis=1))
        b.close()
        recalls.append(pgb.recall(gt_i, gt_d, oi, 10))
    index.close()
    assert recalls[-1] >= max(recalls[:-1]), recalls
    assert recalls[-1] > 0.9, recalls
