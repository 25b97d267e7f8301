import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)

import __graft_entry__ as ge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (compute capability 10.x)")


@pytest.fixture(scope="session")
def pgb():
    return ge.load_package()


@pytest.fixture(scope="session")
def oracle():
    return ge.load_oracle()


@pytest.fixture(scope="session")
def synth(pgb):
    from parlayann_gpu_busqueda_b200 import synthetic
    return synthetic


@pytest.fixture(scope="session")
def gpu(pgb):
    """Fails (never skips) when the CUDA path cannot run: GPU tests must not pass silently."""
    if not pgb.device_available():
        pytest.fail("no compute capability 10.x device: the CUDA path cannot run")
    return True


class Golden:
    """The committed inputs of tests/golden (see make_golden.py)."""

    def __init__(self, pgb):
        g = lambda f: os.path.join(GOLDEN, f)  # noqa: E731
        self.base = pgb.read_vectors(g("c1s_base.i8bin"))
        self.queries = pgb.read_vectors(g("c1s_queries.i8bin"))
        self.ties_base = pgb.read_vectors(g("ties_base.i8bin"))
        self.ties_queries = pgb.read_vectors(g("ties_queries.i8bin"))
        files = {"vamana": "c1s_vamana.graph", "hcnng": "c1s_hcnng.graph",
                 "nnd": "c1s_nnd.graph", "ties_vamana": "ties_vamana.graph"}
        self.graphs = {name: pgb.read_graph(g(f)) for name, f in files.items()}
        self.hnsw = {"hnsw": pgb.read_hnsw(g("c1s.hnsw")), "ties_hnsw": pgb.read_hnsw(g("ties.hnsw"))}

    def vectors_for(self, graph_name):
        if graph_name.startswith("ties"):
            return self.ties_base, self.ties_queries
        return self.base, self.queries


@pytest.fixture(scope="session")
def golden(pgb):
    return Golden(pgb)


def assert_same(tag, got, want):
    """Bit-exact comparison with a readable first difference."""
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, f"{tag}: shape {got.shape} != {want.shape}"
    bad = np.argwhere(got != want)
    if bad.size:
        i = tuple(bad[0])
        row = i[0]
        raise AssertionError(f"{tag}: {len(bad)} differences, first at {i}: got {got[i]} want "
                             f"{want[i]}; row got {got[row][:12]} want {want[row][:12]}")
