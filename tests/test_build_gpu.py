"""GPU graph construction against the CPU builders: Vamana (pgb_build_vamana_gpu: the same
insertion order, batches, search, prune and reverse-edge rules), HNSW (pgb_build_hnsw_gpu:
byte-identical model files) and HCNNG (pgb_build_hcnng_gpu: the same trees, leaf
neighbours and MST order). The graphs must be identical -- degrees and every row, in
order."""
import os

import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


def both(pgb, x, **kw):
    cpu = pgb.build_vamana(x, **kw)
    gpu = pgb.build_vamana_gpu(x, **kw)
    return cpu, gpu


def assert_same_graph(tag, a, b):
    assert_same(f"{tag} degrees", b.degrees, a.degrees)
    assert_same(f"{tag} edges", b.edges, a.edges)


@pytest.mark.parametrize("R,L,alpha", [(32, 64, 1.2), (16, 40, 1.0), (64, 100, 1.2)])
def test_gpu_vamana_equals_cpu_int8(pgb, golden, gpu, R, L, alpha):
    cpu, g = both(pgb, golden.base, R=R, L=L, alpha=alpha, seed=0)
    assert_same_graph(f"R{R} L{L} a{alpha}", cpu, g)


def test_gpu_vamana_equals_cpu_uint8_d128(pgb, gpu):
    from parlayann_gpu_busqueda_b200.synthetic import LAW_C4
    x = LAW_C4.sample(3000, 3, 0)
    cpu, g = both(pgb, x, R=24, L=48, alpha=1.2, seed=5)
    assert_same_graph("uint8", cpu, g)


def test_gpu_vamana_two_passes_and_ties(pgb, golden, gpu):
    cpu, g = both(pgb, golden.base, R=24, L=48, alpha=1.2, passes=2, seed=1)
    assert_same_graph("2 passes", cpu, g)
    # duplicate vectors and equal distances everywhere
    cpu, g = both(pgb, golden.ties_base, R=16, L=32, alpha=1.2, seed=0)
    assert_same_graph("ties", cpu, g)


def test_gpu_vamana_retries_and_hubs_give_the_same_graph(pgb, golden, gpu):
    """Tiny first tables: most searches outgrow them and run again with larger ones, and
    most reverse-edge merges take the second (hub) launch; the graph must not change."""
    os.environ["PGB_BUILD_SMALL_TABLES"] = "1"
    try:
        g = pgb.build_vamana_gpu(golden.base, R=32, L=64, alpha=1.2, seed=0)
    finally:
        del os.environ["PGB_BUILD_SMALL_TABLES"]
    cpu = pgb.build_vamana(golden.base, R=32, L=64, alpha=1.2, seed=0)
    assert_same_graph("small tables", cpu, g)


def test_gpu_vamana_graph_searches_like_cpu_graph(pgb, oracle, golden, gpu):
    """The built graph is a working index: GPU search on it equals the oracle's."""
    g = pgb.build_vamana_gpu(golden.base, R=32, L=64, alpha=1.2, seed=0)
    index = pgb.Index.flat(golden.base, g)
    s = pgb.Searcher(index, len(golden.queries), pgb.QueryParams(k=10, beam_size=40))
    ids, dists, _ = s.search(golden.queries)
    s.liberar()
    index.close()
    oid, od, *_ = oracle.flat_search(golden.base, g.degrees, g.edges, golden.queries, 10, 40)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)


def hnsw_files(pgb, tmp_path, x, **kw):
    cpu_p, gpu_p = str(tmp_path / "cpu.hnsw"), str(tmp_path / "gpu.hnsw")
    pgb.build_hnsw(x, cpu_p, **kw)
    pgb.build_hnsw_gpu(x, gpu_p, **kw)
    return open(cpu_p, "rb").read(), open(gpu_p, "rb").read(), gpu_p


@pytest.mark.parametrize("M,efc,ml", [(16, 64, 0.36), (8, 32, 0.6)])
def test_gpu_hnsw_file_equals_cpu_int8(pgb, golden, gpu, tmp_path, M, efc, ml):
    cpu, g, _ = hnsw_files(pgb, tmp_path, golden.base, M=M, ef_construction=efc, ml=ml, alpha=0.83)
    assert g == cpu, "GPU HNSW file differs from the CPU builder's"


def test_gpu_hnsw_file_equals_cpu_uint8_and_ties(pgb, golden, gpu, tmp_path):
    from parlayann_gpu_busqueda_b200.synthetic import LAW_C4
    x = LAW_C4.sample(2500, 4, 0)
    cpu, g, _ = hnsw_files(pgb, tmp_path, x, M=12, ef_construction=40, ml=0.5, alpha=1.0, seed=3)
    assert g == cpu, "uint8"
    cpu, g, _ = hnsw_files(pgb, tmp_path, golden.ties_base, M=8, ef_construction=32, ml=0.5)
    assert g == cpu, "ties"


def test_gpu_hnsw_small_tables_and_search(pgb, oracle, golden, gpu, tmp_path):
    """Tiny first tables (retried searches, hub merges) give the same file, and the model
    searches like the oracle says."""
    os.environ["PGB_BUILD_SMALL_TABLES"] = "1"
    try:
        cpu, g, gpu_p = hnsw_files(pgb, tmp_path, golden.base, M=16, ef_construction=64, ml=0.36)
    finally:
        del os.environ["PGB_BUILD_SMALL_TABLES"]
    assert g == cpu
    h = pgb.read_hnsw(gpu_p)
    index = pgb.Index.hnsw(golden.base, h)
    s = pgb.Searcher(index, len(golden.queries), pgb.QueryParams(k=10, beam_size=50))
    ids, dists, _ = s.search(golden.queries)
    s.liberar()
    index.close()
    oid, od, *_ = oracle.hnsw_search(golden.base, h, golden.queries, 10, 50)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)


def test_gpu_hcnng_reproduces_the_golden_graph(pgb, golden, gpu):
    """c1s_hcnng.graph was written by the CPU builder with these arguments."""
    g = pgb.build_hcnng_gpu(golden.base, trees=10, leaf=400, mst_deg=3, seed=0)
    assert_same_graph("golden", golden.graphs["hcnng"], g)


@pytest.mark.parametrize("trees,leaf,mst_deg,seed", [(6, 300, 3, 3), (4, 1024, 2, 1), (3, 11, 4, 2),
                                                     (2, 2, 3, 5), (5, 64, 1, 0)])
def test_gpu_hcnng_equals_cpu_int8(pgb, golden, gpu, trees, leaf, mst_deg, seed):
    """Leaves of up to 1,024 points; of at most 11 (fewer than 10 neighbours each); of at
    most 2 (halved ranges everywhere); single-edge MST degree."""
    kw = dict(trees=trees, leaf=leaf, mst_deg=mst_deg, seed=seed)
    cpu = pgb.build_hcnng(golden.base, **kw)
    g = pgb.build_hcnng_gpu(golden.base, **kw)
    assert_same_graph(f"T{trees} leaf{leaf} mst{mst_deg}", cpu, g)


def test_gpu_hcnng_equals_cpu_uint8_d128_and_ties(pgb, golden, gpu):
    from parlayann_gpu_busqueda_b200.synthetic import LAW_C4
    x = LAW_C4.sample(3000, 3, 0)
    kw = dict(trees=5, leaf=700, mst_deg=3, seed=4)
    assert_same_graph("uint8", pgb.build_hcnng(x, **kw), pgb.build_hcnng_gpu(x, **kw))
    # every vector three times: equal distances everywhere
    kw = dict(trees=4, leaf=100, mst_deg=3, seed=0)
    assert_same_graph("ties", pgb.build_hcnng(golden.ties_base, **kw),
                      pgb.build_hcnng_gpu(golden.ties_base, **kw))


def test_gpu_hcnng_rejects_bad_arguments(pgb, golden, gpu):
    with pytest.raises(pgb.PgbError, match="1,024"):
        pgb.build_hcnng_gpu(golden.base, trees=2, leaf=1025)
    with pytest.raises(pgb.PgbError):
        pgb.build_hcnng_gpu(golden.base, trees=100, mst_deg=3)  # 300 slots > 256
    with pytest.raises(pgb.PgbError):
        pgb.build_hcnng_gpu(golden.base, trees=2, leaf=1)


def test_gpu_vamana_rejects_bad_arguments(pgb, golden, gpu):
    with pytest.raises(pgb.PgbError):
        pgb.build_vamana_gpu(golden.base, R=0, L=64)
    with pytest.raises(pgb.PgbError):
        pgb.build_vamana_gpu(np.zeros((10, 129), np.int8), R=8, L=16)
