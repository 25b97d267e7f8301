"""Exact k-nearest-neighbour ground truth by brute force on the GPU.

Distances are exact int32: ||q||^2 + ||p||^2 - 2 q.p with q.p from an int8 x int8 -> int32
GEMM (uint8 data is shifted by -128, which leaves every difference unchanged). Written in
the reference's GT layout with float distances ([nq][k] ids, [nq][k] f32;
cuda/lectores.h:29-36). Used to evaluate recall, not on the search path.
"""
from __future__ import annotations

import numpy as np


def _as_int8(x: np.ndarray) -> np.ndarray:
    if x.dtype == np.int8:
        return x
    return (x.astype(np.int16) - 128).astype(np.int8)


def knn_gpu(base: np.ndarray, queries: np.ndarray, k: int = 100, device: int = 0,
            base_chunk: int = 1 << 18, query_chunk: int = 4096):
    """(ids uint32 [nq,k], dists float32 [nq,k]) sorted by (distance, id)."""
    import torch

    dev = torch.device("cuda", device)
    b8 = _as_int8(base)
    q8 = _as_int8(queries)
    dim = b8.shape[1]
    dpad = (dim + 15) // 16 * 16
    B = torch.zeros((b8.shape[0], dpad), dtype=torch.int8, device=dev)
    B[:, :dim] = torch.from_numpy(b8).to(dev)
    bn = (B.to(torch.int32) ** 2).sum(1)
    nq = q8.shape[0]
    out_i = np.empty((nq, k), dtype=np.uint32)
    out_d = np.empty((nq, k), dtype=np.float32)
    for qs in range(0, nq, query_chunk):
        qe = min(nq, qs + query_chunk)
        Q = torch.zeros((max(qe - qs, 17), dpad), dtype=torch.int8, device=dev)
        Q[: qe - qs, :dim] = torch.from_numpy(q8[qs:qe]).to(dev)
        qn = (Q.to(torch.int32) ** 2).sum(1)
        best_d = None
        best_i = None
        for bs in range(0, B.shape[0], base_chunk):
            be = min(B.shape[0], bs + base_chunk)
            Bc = B[bs:be]
            if Bc.shape[0] % 8:
                pad = 8 - Bc.shape[0] % 8
                Bc = torch.cat([Bc, torch.zeros((pad, dpad), dtype=torch.int8, device=dev)])
            dot = torch._int_mm(Q, Bc.t().contiguous())[:, : be - bs]
            d = qn[:, None] + bn[None, bs:be] - 2 * dot
            # (dist, id) order: key = dist * 2^32 + id in int64
            key = d.to(torch.int64) * (1 << 32) + torch.arange(bs, be, device=dev)[None, :]
            kk = min(k, be - bs)
            top = torch.topk(key, kk, dim=1, largest=False, sorted=True).values
            if best_d is None:
                best_d = top
            else:
                best_d = torch.topk(torch.cat([best_d, top], 1), k, dim=1, largest=False,
                                    sorted=True).values
        keys = best_d[: qe - qs]
        out_i[qs:qe] = (keys & 0xFFFFFFFF).cpu().numpy().astype(np.uint32)
        out_d[qs:qe] = (keys >> 32).cpu().numpy().astype(np.float32)
    del best_i
    return out_i, out_d


def knn_cpu(base: np.ndarray, queries: np.ndarray, k: int = 100):
    """Same answer in int64 numpy (spot checks of knn_gpu on small sets)."""
    b = base.astype(np.int64)
    q = queries.astype(np.int64)
    d = (q * q).sum(1)[:, None] + (b * b).sum(1)[None, :] - 2 * q @ b.T
    key = d * (1 << 32) + np.arange(b.shape[0])[None, :]
    part = np.argpartition(key, min(k, b.shape[0] - 1), axis=1)[:, :k]
    top = np.take_along_axis(key, part, 1)
    order = np.argsort(top, axis=1)
    top = np.take_along_axis(top, order, 1)
    return (top & 0xFFFFFFFF).astype(np.uint32), (top >> 32).astype(np.float32)
