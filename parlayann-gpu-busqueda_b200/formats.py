"""numpy readers / writers of the reference's file formats.

vectors  : [n u32][dim u32][n*dim int8|uint8]                (reference cuda/lectores.h:7-15)
graph    : [n u32][maxdeg u32][deg n*u32][edges]             (cuda/lectores.h:17-27)
HNSW v3  : see read_hnsw                                      (cuda/hnsw.h:11-16)
GT       : [nq u32][k u32][ids nq*k u32][dists nq*k f32]      (cuda/lectores.h:29-36)
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np


def write_vectors(path: str, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x)
    assert x.ndim == 2 and x.dtype in (np.int8, np.uint8)
    with open(path, "wb") as f:
        f.write(np.array(x.shape, dtype=np.uint32).tobytes())
        f.write(x.tobytes())


def read_vectors(path: str, dtype=np.int8) -> np.ndarray:
    raw = np.fromfile(path, dtype=np.uint8)
    n, d = np.frombuffer(raw[:8].tobytes(), dtype=np.uint32)
    if raw.size != 8 + int(n) * int(d):
        raise ValueError(f"{path}: size does not match header")
    return raw[8:].view(dtype).reshape(int(n), int(d))


@dataclass
class Graph:
    """ParlayANN flat graph: degrees[n] + rows concatenated (CSR without offsets)."""
    n: int
    max_degree: int
    degrees: np.ndarray
    edges: np.ndarray

    @property
    def offsets(self) -> np.ndarray:
        off = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(self.degrees, out=off[1:])
        return off

    def row(self, i: int) -> np.ndarray:
        off = self.offsets
        return self.edges[off[i]:off[i + 1]]

    @staticmethod
    def from_padded(degrees: np.ndarray, adj: np.ndarray) -> "Graph":
        degrees = np.ascontiguousarray(degrees, dtype=np.uint32)
        mask = np.arange(adj.shape[1])[None, :] < degrees[:, None]
        edges = np.ascontiguousarray(adj[mask], dtype=np.uint32)
        return Graph(int(adj.shape[0]), int(degrees.max(initial=0)), degrees, edges)

    def padded(self, slots: int | None = None) -> np.ndarray:
        slots = slots or max(self.max_degree, 1)
        out = np.full((self.n, slots), 0xFFFFFFFF, dtype=np.uint32)
        mask = np.arange(slots)[None, :] < self.degrees[:, None]
        out[mask] = self.edges
        return out


def write_graph(path: str, g: Graph) -> None:
    with open(path, "wb") as f:
        f.write(np.array([g.n, g.max_degree], dtype=np.uint32).tobytes())
        f.write(np.ascontiguousarray(g.degrees, dtype=np.uint32).tobytes())
        f.write(np.ascontiguousarray(g.edges, dtype=np.uint32).tobytes())


def read_graph(path: str) -> Graph:
    raw = np.fromfile(path, dtype=np.uint32)
    n, maxdeg = int(raw[0]), int(raw[1])
    deg = raw[2:2 + n].copy()
    edges = raw[2 + n:].copy()
    if edges.size != int(deg.sum(dtype=np.int64)):
        raise ValueError(f"{path}: size does not match degrees")
    if (deg > maxdeg).any() or (edges >= n).any():
        raise ValueError(f"{path}: degree or edge out of range")
    return Graph(n, maxdeg, deg, edges)


@dataclass
class Hnsw:
    """ParlayANN HNSW v3 model: per node its top level and stored point; the lists of
    node 0 levels 0..levels[0], node 1, ...; entry points."""
    n: int
    dim: int
    m: int
    efc: int
    ml: float
    alpha: float
    levels: np.ndarray
    node_point: np.ndarray
    list_sizes: np.ndarray
    ids: np.ndarray
    entries: np.ndarray
    first_list: np.ndarray = field(default=None, repr=False)
    list_offsets: np.ndarray = field(default=None, repr=False)

    def __post_init__(self):
        self.first_list = np.zeros(self.n, dtype=np.int64)
        np.cumsum(self.levels[:-1].astype(np.int64) + 1, out=self.first_list[1:])
        self.list_offsets = np.zeros(len(self.list_sizes) + 1, dtype=np.int64)
        np.cumsum(self.list_sizes, out=self.list_offsets[1:])

    def neighbours(self, node: int, level: int) -> np.ndarray:
        li = int(self.first_list[node]) + level
        return self.ids[self.list_offsets[li]:self.list_offsets[li + 1]]


def read_hnsw(path: str) -> Hnsw:
    buf = open(path, "rb").read()
    if buf[:4] != b"HNSW":
        raise ValueError(f"{path}: not an HNSW model")
    version, = struct.unpack_from("<I", buf, 4)
    if version != 3:
        raise ValueError(f"{path}: version {version}")
    dim, ml, m, efc, alpha, n = struct.unpack_from("<IfIIfI", buf, 24)
    pos = 48
    tab = np.frombuffer(buf, dtype=np.uint32, count=2 * n, offset=pos).reshape(n, 2)
    levels, node_point = tab[:, 0].copy(), tab[:, 1].copy()
    pos += 8 * n
    sizes, chunks = [], []
    for i in range(n):
        for _ in range(int(levels[i]) + 1):
            cnt, = struct.unpack_from("<Q", buf, pos)
            pos += 8
            chunks.append(np.frombuffer(buf, dtype=np.uint32, count=cnt, offset=pos))
            sizes.append(cnt)
            pos += 4 * cnt
    ne, = struct.unpack_from("<Q", buf, pos)
    pos += 8
    entries = np.frombuffer(buf, dtype=np.uint32, count=ne, offset=pos).copy()
    pos += 4 * ne
    if pos != len(buf):
        raise ValueError(f"{path}: trailing bytes")
    ids = np.concatenate(chunks).astype(np.uint32) if chunks else np.zeros(0, np.uint32)
    return Hnsw(n, dim, m, efc, ml, alpha, levels, node_point,
                np.array(sizes, dtype=np.uint32), ids, entries)


def write_hnsw(path: str, h: Hnsw) -> None:
    with open(path, "wb") as f:
        f.write(b"HNSW")
        f.write(struct.pack("<IQQ", 3, 0, 0))
        f.write(struct.pack("<IfIIfI", h.dim, h.ml, h.m, h.efc, h.alpha, h.n))
        f.write(np.stack([h.levels, h.node_point], axis=1).astype(np.uint32).tobytes())
        for li, sz in enumerate(h.list_sizes):
            f.write(struct.pack("<Q", int(sz)))
            f.write(h.ids[h.list_offsets[li]:h.list_offsets[li + 1]].astype(np.uint32).tobytes())
        f.write(struct.pack("<Q", len(h.entries)))
        f.write(np.asarray(h.entries, dtype=np.uint32).tobytes())


def write_gt(path: str, ids: np.ndarray, dists: np.ndarray) -> None:
    nq, k = ids.shape
    with open(path, "wb") as f:
        f.write(np.array([nq, k], dtype=np.uint32).tobytes())
        f.write(np.ascontiguousarray(ids, dtype=np.uint32).tobytes())
        f.write(np.ascontiguousarray(dists, dtype=np.float32).tobytes())


def read_gt(path: str):
    raw = np.fromfile(path, dtype=np.uint32)
    nq, k = int(raw[0]), int(raw[1])
    ids = raw[2:2 + nq * k].reshape(nq, k).copy()
    dists = raw[2 + nq * k:2 + 2 * nq * k].view(np.float32).reshape(nq, k).copy()
    return ids, dists
