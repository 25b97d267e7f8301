"""CPU graph builders: valid graphs, deterministic for a seed whatever the thread count,
navigable from the start point 0, and searchable to high recall (checked by the oracle)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def small(synth):
    return synth.dataset(synth.LAW_C1, 1500, 50, seed=5)


def reach(g):
    off = g.offsets
    seen = np.zeros(g.n, bool)
    seen[0] = True
    frontier = [0]
    while frontier:
        nxt = []
        for u in frontier:
            for v in g.edges[off[u]:off[u + 1]]:
                if not seen[v]:
                    seen[v] = True
                    nxt.append(v)
        frontier = nxt
    return seen.mean()


BUILDERS = {
    "vamana": lambda pgb, x, t: pgb.build_vamana(x, R=24, L=48, alpha=1.2, seed=3, threads=t),
    "vamana2": lambda pgb, x, t: pgb.build_vamana(x, R=16, L=32, alpha=1.2, passes=2, seed=3,
                                                  threads=t),
    "hcnng": lambda pgb, x, t: pgb.build_hcnng(x, trees=6, leaf=300, mst_deg=3, seed=3, threads=t),
    "nnd": lambda pgb, x, t: pgb.build_nndescent(x, K=16, init_trees=3, leaf=300, seed=3,
                                                 threads=t),
}


@pytest.mark.parametrize("name", list(BUILDERS))
def test_builder_valid_deterministic_navigable(pgb, oracle, small, name):
    base, queries = small
    g1 = BUILDERS[name](pgb, base, 1)
    g8 = BUILDERS[name](pgb, base, 8)
    assert np.array_equal(g1.degrees, g8.degrees) and np.array_equal(g1.edges, g8.edges)
    assert (g1.edges < g1.n).all()
    off = g1.offsets
    self_loops = sum(int((g1.edges[off[i]:off[i + 1]] == i).any()) for i in range(g1.n))
    assert self_loops == 0
    assert reach(g1) > 0.99
    gi, gd = oracle.brute_force_knn(base, queries, 10)
    ids = oracle.flat_search(base, g1.degrees, g1.edges, queries, 10, 64,
                             exclude_query_id=False)[0]
    hits = np.mean([len(set(a) & set(b)) / 10 for a, b in zip(ids, gi)])
    assert hits > 0.9


def test_hcnng_keeps_duplicate_edges(pgb, small):
    base, _ = small
    g = pgb.build_hcnng(base, trees=10, leaf=300, mst_deg=3, seed=1)
    dup = sum(len(np.unique(g.row(i))) < len(g.row(i)) for i in range(g.n))
    assert dup > 0 and g.max_degree <= 30


def test_hnsw_builder_file(pgb, oracle, small, tmp_path):
    base, queries = small
    p = str(tmp_path / "m.hnsw")
    pgb.build_hnsw(base, p, M=8, ef_construction=40, ml=0.5, alpha=1.0, seed=2, threads=4)
    p2 = str(tmp_path / "m2.hnsw")
    pgb.build_hnsw(base, p2, M=8, ef_construction=40, ml=0.5, alpha=1.0, seed=2, threads=1)
    assert open(p, "rb").read() == open(p2, "rb").read()
    h = pgb.read_hnsw(p)
    top = h.levels[h.entries[0]]
    assert top == h.levels.max() and len(h.entries) == 1
    # every level-l neighbour exists at level l
    for i in range(0, h.n, 37):
        for level in range(int(h.levels[i]) + 1):
            nb = h.neighbours(i, level)
            assert (h.levels[nb] >= level).all()
    gi, _ = oracle.brute_force_knn(base, queries, 10)
    ids = oracle.hnsw_search(base, h, queries, 10, 64)[0]
    assert np.mean([len(set(a) & set(b)) / 10 for a, b in zip(ids, gi)]) > 0.9


def test_builder_argument_errors(pgb, small):
    base, _ = small
    with pytest.raises(pgb.PgbError):
        pgb.build_vamana(base, R=0)
    with pytest.raises(pgb.PgbError):
        pgb.build_hcnng(base, trees=100, mst_deg=3)  # 300 slots > 256
