"""_pgbpy, the pybind11 module for big-ann-benchmarks-style harnesses: an index loaded from
the reference's files, batch_search on numpy arrays, GPU Vamana / HCNNG / HNSW construction,
recall."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, assert_same

PKG = os.path.join(ROOT, "parlayann-gpu-busqueda_b200")


@pytest.fixture(scope="module")
def pgbpy(pgb):
    sys.path.insert(0, PKG)
    import _pgbpy
    return _pgbpy


def test_module_surface(pgbpy):
    for name in ("FlatIndex", "HNSWIndex", "Index", "build_vamana", "build_hcnng", "build_hnsw",
                 "compute_recall"):
        assert hasattr(pgbpy, name), name


def test_compute_recall_matches_package(pgb, pgbpy):
    rng = np.random.default_rng(3)
    gt = np.argsort(rng.random((50, 100)), axis=1).astype(np.uint32)
    gd = np.sort(rng.integers(0, 1000, (50, 100)), axis=1).astype(np.float32)
    got = gt[:, :10].copy()
    got[::3, 2] = 999999
    assert pgbpy.compute_recall(gt, gd, got, 10) == pgb.recall(gt, gd, got, 10)


@pytest.mark.gpu
def test_flat_batch_search_matches_oracle(pgb, pgbpy, oracle, golden, gpu):
    idx = pgbpy.FlatIndex(os.path.join(GOLDEN, "c1s_base.i8bin"),
                          os.path.join(GOLDEN, "c1s_vamana.graph"), "int8")
    assert idx.n == len(golden.base) and idx.dim == golden.base.shape[1]
    g = golden.graphs["vamana"]
    for Ls, k in ((20, 10), (64, 50)):
        ids, dists, st = idx.batch_search(golden.queries, knn=k, beam_size=Ls, stats=True)
        oid, od, oc, oe, of = oracle.flat_search(golden.base, g.degrees, g.edges, golden.queries, k,
                                                 Ls, exclude_query_id=False)
        assert_same(f"ids Ls={Ls}", ids, oid)
        assert_same(f"dists Ls={Ls}", dists, od)
        assert_same(f"comps Ls={Ls}", st[:, 0], oc)


@pytest.mark.gpu
def test_hnsw_batch_search_matches_oracle(pgb, pgbpy, oracle, golden, gpu):
    idx = pgbpy.HNSWIndex(os.path.join(GOLDEN, "c1s_base.i8bin"), os.path.join(GOLDEN, "c1s.hnsw"),
                          "int8")
    ids, dists = idx.batch_search(golden.queries, knn=10, beam_size=50)
    oid, od, *_ = oracle.hnsw_search(golden.base, golden.hnsw["hnsw"], golden.queries, 10, 50)
    assert_same("ids", ids, oid)
    assert_same("dists", dists, od)


@pytest.mark.gpu
def test_build_vamana_equals_cpu_builder(pgb, pgbpy, golden, gpu):
    deg, adj = pgbpy.build_vamana(golden.base, R=32, L=64, alpha=1.2, seed=0)
    c = pgb.build_vamana(golden.base, R=32, L=64, alpha=1.2, seed=0)
    g = pgb.Graph.from_padded(deg, adj)
    assert_same("degrees", g.degrees, c.degrees)
    assert_same("edges", g.edges, c.edges)


@pytest.mark.gpu
def test_build_hcnng_and_hnsw_equal_cpu_builders(pgb, pgbpy, golden, gpu, tmp_path):
    deg, adj = pgbpy.build_hcnng(golden.base, trees=4, leaf=300, mst_deg=3, seed=1)
    c = pgb.build_hcnng(golden.base, trees=4, leaf=300, mst_deg=3, seed=1)
    g = pgb.Graph.from_padded(deg, adj)
    assert_same("hcnng degrees", g.degrees, c.degrees)
    assert_same("hcnng edges", g.edges, c.edges)
    pg, pc = str(tmp_path / "g.hnsw"), str(tmp_path / "c.hnsw")
    pgbpy.build_hnsw(golden.base, pg, M=8, ef_construction=32, ml=0.5, alpha=1.0, seed=0)
    pgb.build_hnsw(golden.base, pc, M=8, ef_construction=32, ml=0.5, alpha=1.0, seed=0)
    assert open(pg, "rb").read() == open(pc, "rb").read()
