"""Pins the oracle: on every committed case its outputs must equal, bit for bit, those of
the reference's own kernels (cuda/busqueda.cu kernelBusqueda, cuda/busqueda_hnsw.cu
kernelHnsw), which tests/golden/make_golden.py ran on a B200 and packed into
reference_outputs.npz."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_same

REF = np.load(os.path.join(GOLDEN, "reference_outputs.npz"))


def _cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.cases()


CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_equals_reference_kernels(oracle, golden, case):
    name, g, mode, Ls, visit, k, cut = case
    base, queries = golden.vectors_for(g)
    if mode == "flat":
        graph = golden.graphs[g]
        ids, dists, comps, exps, flags = oracle.flat_search(
            base, graph.degrees, graph.edges, queries, k, Ls, cut=cut,
            limit=visit if visit > 0 else 0, exclude_query_id=True)
    else:
        ids, dists, comps, exps, flags = oracle.hnsw_search(
            base, golden.hnsw[g], queries, k, Ls, limit=visit if visit > 0 else 0)
    assert_same(f"{name} ids", ids, REF[name + "__ids"])
    assert_same(f"{name} dists", dists, REF[name + "__dists"])
    assert_same(f"{name} comps", comps, REF[name + "__comp"])
    assert_same(f"{name} flags", flags, REF[name + "__flags"])


def test_golden_cases_exercise_the_quirks(pgb, golden):
    """The committed cases cover duplicate edges (multiset union), the query-index
    exclusion, short frontiers and visit limits."""
    h = golden.graphs["hcnng"]
    dup_rows = sum(len(np.unique(h.row(i))) < len(h.row(i)) for i in range(h.n))
    assert dup_rows > h.n // 4
    # queries 0..99 coincide with base ids 0..99: the exclusion is active
    assert golden.queries.shape[0] <= golden.base.shape[0]
    short = sum(int(((REF[c[0] + "__flags"] & 2) != 0).sum()) for c in CASES)
    assert short > 0
    assert any(c[5] > 0 for c in CASES)
