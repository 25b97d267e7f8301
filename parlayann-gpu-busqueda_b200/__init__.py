"""B200 graph beam search: ParlayANN's search API over hand-written sm_100a kernels.

Importing the package loads lib/libpgb.so (the C ABI of include/pgb.h); there is no
CPU fallback for the search.
"""
from . import _native
from ._native import PgbError, NO_NEIGHBOR, FLAG_OVERFLOW, FLAG_SHORT
from .formats import (Graph, Hnsw, read_graph, read_gt, read_hnsw, read_vectors, write_graph,
                      write_gt, write_hnsw, write_vectors)
from .search import (Batch, Index, QueryParams, Searcher, Server, build_hcnng, build_hcnng_gpu, build_hnsw,
                     build_nndescent, build_hnsw_gpu, build_vamana, build_vamana_gpu, device_available,
                     file_check, recall, search_launches)

__all__ = [
    "PgbError", "NO_NEIGHBOR", "FLAG_OVERFLOW", "FLAG_SHORT", "Graph", "Hnsw", "read_graph",
    "read_gt", "read_hnsw", "read_vectors", "write_graph", "write_gt", "write_hnsw",
    "write_vectors", "Batch", "Index", "Server", "QueryParams", "Searcher", "build_hcnng",
    "build_hcnng_gpu", "build_hnsw", "build_nndescent", "build_hnsw_gpu", "build_vamana",
    "build_vamana_gpu", "device_available", "file_check", "recall", "search_launches",
]
