"""Ground truth: the GPU brute force (int8 GEMM, exact int32 distances, (dist, id) order)
against the int64 CPU restatement, on 1,000 queries -- the spot check behind every
recall figure. uint8 data goes through the -128 shift, which leaves distances unchanged."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("law_name,n,seed", [("LAW_C2", 20000, 3), ("LAW_C4", 12000, 5)])
def test_knn_gpu_equals_cpu(pgb, gpu, law_name, n, seed):
    from parlayann_gpu_busqueda_b200 import groundtruth, synthetic
    law = getattr(synthetic, law_name)
    base = law.sample(n, seed, 0)
    queries = law.sample(1000, seed, 1)
    gi, gd = groundtruth.knn_gpu(base, queries, 100, base_chunk=1 << 13, query_chunk=512)
    ci, cd = groundtruth.knn_cpu(base, queries, 100)
    assert np.array_equal(gd, cd), "distances"
    assert np.array_equal(gi, ci), "ids (ties broken by id)"
