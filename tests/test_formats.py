"""File formats: Python writers/readers round-trip, and the C readers (the ones the index
loaders use) accept good files and reject truncated or corrupt ones with a status, as the
reference readers reject them with an exit (cuda/lectores.cpp:62-170,
cuda/hnsw_lector.cpp:14-111)."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN


def test_vectors_round_trip(pgb, tmp_path):
    x = np.random.default_rng(0).integers(-128, 128, size=(57, 100)).astype(np.int8)
    p = str(tmp_path / "v.i8bin")
    pgb.write_vectors(p, x)
    assert np.array_equal(pgb.read_vectors(p), x)
    assert pgb.file_check(p, "vectors")[:3] == [57, 100, 5700]
    u = x.view(np.uint8)
    pgb.write_vectors(p, u)
    assert np.array_equal(pgb.read_vectors(p, np.uint8), u)


def test_graph_round_trip_and_padding(pgb, tmp_path):
    g = pgb.read_graph(os.path.join(GOLDEN, "c1s_hcnng.graph"))
    p = str(tmp_path / "g.graph")
    pgb.write_graph(p, g)
    g2 = pgb.read_graph(p)
    assert np.array_equal(g.degrees, g2.degrees) and np.array_equal(g.edges, g2.edges)
    pad = g.padded()
    assert pad.shape == (g.n, g.max_degree)
    assert (pad[np.arange(g.max_degree)[None, :] >= g.degrees[:, None]] == 0xFFFFFFFF).all()
    assert np.array_equal(pgb.Graph.from_padded(g.degrees, pad).edges, g.edges)
    info = pgb.file_check(p, "graph")
    assert info[:3] == [g.n, g.max_degree, len(g.edges)]


def test_hnsw_round_trip(pgb, tmp_path):
    h = pgb.read_hnsw(os.path.join(GOLDEN, "c1s.hnsw"))
    p = str(tmp_path / "m.hnsw")
    pgb.write_hnsw(p, h)
    assert open(p, "rb").read() == open(os.path.join(GOLDEN, "c1s.hnsw"), "rb").read()
    assert pgb.file_check(p, "hnsw") == [h.n, h.dim, len(h.list_sizes), len(h.entries)]
    assert (h.neighbours(int(h.entries[0]), 1) < h.n).all()


def test_gt_round_trip(pgb, tmp_path):
    ids = np.arange(30, dtype=np.uint32).reshape(3, 10)
    d = np.arange(30, dtype=np.float32).reshape(3, 10)
    p = str(tmp_path / "gt")
    pgb.write_gt(p, ids, d)
    i2, d2 = pgb.read_gt(p)
    assert np.array_equal(ids, i2) and np.array_equal(d, d2)


def _corrupt(tmp_path, name, data):
    p = str(tmp_path / name)
    open(p, "wb").write(data)
    return p


@pytest.mark.parametrize("case", ["truncated", "trailing", "edge_out_of_range", "degree_over_max"])
def test_c_graph_reader_rejects(pgb, tmp_path, case):
    raw = bytearray(open(os.path.join(GOLDEN, "c1s_vamana.graph"), "rb").read())
    n, maxdeg = struct.unpack_from("<II", raw, 0)
    if case == "truncated":
        raw = raw[:-4]
    elif case == "trailing":
        raw += b"\0\0\0\0"
    elif case == "edge_out_of_range":
        struct.pack_into("<I", raw, len(raw) - 4, n + 5)
    else:
        struct.pack_into("<I", raw, 8, maxdeg + 1)
    p = _corrupt(tmp_path, "bad.graph", bytes(raw))
    with pytest.raises(pgb.PgbError) as e:
        pgb.file_check(p, "graph")
    assert e.value.status == 6  # PGB_ERR_FORMAT


@pytest.mark.parametrize("case", ["magic", "version", "truncated", "trailing", "neighbour"])
def test_c_hnsw_reader_rejects(pgb, tmp_path, case):
    raw = bytearray(open(os.path.join(GOLDEN, "c1s.hnsw"), "rb").read())
    if case == "magic":
        raw[:4] = b"HNSX"
    elif case == "version":
        struct.pack_into("<I", raw, 4, 2)
    elif case == "truncated":
        raw = raw[:-3]
    elif case == "trailing":
        raw += b"\1"
    else:
        # first neighbour id of node 0 level 0 (after the 48-byte header and node table)
        n = struct.unpack_from("<I", raw, 44)[0]
        off = 48 + 8 * n + 8
        struct.pack_into("<I", raw, off, n + 1)
    p = _corrupt(tmp_path, "bad.hnsw", bytes(raw))
    with pytest.raises(pgb.PgbError) as e:
        pgb.file_check(p, "hnsw")
    assert e.value.status == 6


def test_c_vector_reader_rejects_size_mismatch_and_missing(pgb, tmp_path):
    p = _corrupt(tmp_path, "bad.i8bin", struct.pack("<II", 10, 100) + b"\0" * 999)
    with pytest.raises(pgb.PgbError) as e:
        pgb.file_check(p, "vectors")
    assert e.value.status == 6
    with pytest.raises(pgb.PgbError) as e:
        pgb.file_check(str(tmp_path / "missing.i8bin"), "vectors")
    assert e.value.status == 5  # PGB_ERR_IO
