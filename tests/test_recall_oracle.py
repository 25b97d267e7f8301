"""Recall with distance ties, and properties of the oracle itself."""
import numpy as np


def recall_py(gt_ids, gt_d, ids, k):
    """Plain restatement of compute_recall_with_distance_ties (cuda/evaluacion.cpp:56-80)."""
    total = 0
    for q in range(len(gt_ids)):
        end = gt_ids.shape[1]
        if gt_ids.shape[1] != k:
            ref = gt_d[q, k - 1]
            for i in range(k, gt_ids.shape[1]):
                if not abs(ref - gt_d[q, i]) < 1e-6:
                    end = i
                    break
        total += len(set(ids[q, :k].tolist()) & set(gt_ids[q, :end].tolist()))
    return total / len(gt_ids) / k


def test_recall_with_ties_matches_restatement(pgb, oracle):
    rng = np.random.default_rng(3)
    nq, kg = 200, 100
    gt_d = np.sort(rng.integers(0, 40, size=(nq, kg)), axis=1).astype(np.float32)  # many ties
    gt_ids = np.stack([rng.permutation(1000)[:kg] for _ in range(nq)]).astype(np.uint32)
    ids = gt_ids[:, :10].copy()
    flip = rng.random(ids.shape) < 0.3
    ids[flip] = rng.integers(0, 1000, size=flip.sum())
    ids[:, 3] = ids[:, 2]  # duplicate ids count once
    ids[:5, -1] = 0xFFFFFFFF
    want = recall_py(gt_ids, gt_d, ids, 10)
    assert abs(pgb.recall(gt_ids, gt_d, ids, 10) - want) < 1e-12
    assert abs(oracle.recall(gt_ids, gt_d, ids, 10) - want) < 1e-12
    # ties extend the ground-truth prefix: a 12th-ranked id at the 10th distance counts
    gt_d2 = np.zeros((1, 20), np.float32)
    gt_ids2 = np.arange(20, dtype=np.uint32)[None]
    got = np.array([[0, 1, 2, 3, 4, 5, 6, 7, 8, 15]], np.uint32)
    assert pgb.recall(gt_ids2, gt_d2, got, 10) == 1.0


def test_groundtruth_cpu_restatement(pgb, synth, oracle):
    from parlayann_gpu_busqueda_b200 import groundtruth
    base, q = synth.dataset(synth.LAW_C1, 3000, 40, seed=9)
    ids, d = groundtruth.knn_cpu(base, q, 25)
    oi, od = oracle.brute_force_knn(base, q, 25)
    assert np.array_equal(ids, oi) and np.array_equal(d, od.astype(np.float32))


def test_oracle_wide_beam_is_exact_over_reachable_points(pgb, oracle, golden):
    """With Ls >= n every reachable point enters the frontier, so the answer is the exact
    k-NN (the graph is connected from point 0)."""
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    ids, dists, *_ = oracle.flat_search(base, g.degrees, g.edges, queries, 10, base.shape[0],
                                        cut=10.0, exclude_query_id=False)
    gi, gd = oracle.brute_force_knn(base, queries, 10)
    assert np.array_equal(dists, gd)
    assert np.array_equal(ids, gi)


def test_oracle_limit_and_short_flag(pgb, oracle, golden):
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    _, _, comps, exps, flags = oracle.flat_search(base, g.degrees, g.edges, queries, 10, 40,
                                                  limit=3)
    assert (exps <= 3).all()
    _, _, _, _, flags = oracle.flat_search(base, g.degrees, g.edges, queries, 10, 40, cut=0.5)
    assert ((flags & 2) != 0).any()  # a cut below 1 shortens frontiers under k
