"""ctypes binding of libpgb.so (the C ABI declared in include/pgb.h).

The library is built in-tree (``lib/libpgb.so``). There is no fallback: if it is
missing, importing the package raises ImportError naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# PGB_LIB selects another in-tree build of the same C ABI (e.g. lib/libpgb_prof.so)
LIB_PATH = os.environ.get("PGB_LIB") or os.path.join(_HERE, "lib", "libpgb.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C {os.path.join(_HERE, 'csrc')}` "
        "(or __graft_entry__.build())")

lib = C.CDLL(LIB_PATH)

# ---- types -----------------------------------------------------------------------------
PGB_OK = 0
STATUS_NAMES = {0: "PGB_OK", 1: "PGB_ERR_BAD_ARG", 2: "PGB_ERR_OOM", 3: "PGB_ERR_CUDA",
                4: "PGB_ERR_OVERFLOW", 5: "PGB_ERR_IO", 6: "PGB_ERR_FORMAT", 7: "PGB_ERR_BUSY",
                8: "PGB_ERR_TIMEOUT", 9: "PGB_ERR_NOT_FOUND"}
PGB_INT8, PGB_UINT8 = 0, 1
NO_NEIGHBOR = 0xFFFFFFFF
FLAG_OVERFLOW, FLAG_SHORT = 1, 2


class QueryParams(C.Structure):
    _fields_ = [("k", C.c_uint32), ("beam_size", C.c_uint32), ("cut", C.c_double),
                ("limit", C.c_int64), ("degree_limit", C.c_uint32),
                ("exclude_query_id", C.c_uint32), ("query_id_base", C.c_uint32),
                ("reserved", C.c_uint32)]


class QueryStats(C.Structure):
    _fields_ = [("dist_comps", C.c_int32), ("expansions", C.c_int32), ("flags", C.c_int32),
                ("reserved", C.c_int32)]


class IndexInfo(C.Structure):
    _fields_ = [("n_points", C.c_uint32), ("dim", C.c_uint32), ("elem", C.c_uint32),
                ("is_hnsw", C.c_uint32), ("max_degree", C.c_uint32),
                ("upper_degree", C.c_uint32), ("top_level", C.c_uint32),
                ("n_entries", C.c_uint32), ("device_bytes", C.c_uint64)]


class PgbError(RuntimeError):
    """A pgb_status other than PGB_OK, with the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


vp, u32, i32, i64, u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_int64, C.c_uint64
P_u32 = C.POINTER(C.c_uint32)


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("pgb_status_string", C.c_char_p, C.c_int)
_sig("pgb_last_error", C.c_char_p)
_sig("pgb_device_available", C.c_int)
_sig("pgb_index_create_flat", C.c_int, C.c_int, vp, u32, u32, C.c_int, vp, vp, C.POINTER(vp))
_sig("pgb_index_create_hnsw", C.c_int, C.c_int, vp, u32, u32, C.c_int, u32, vp, vp, vp, vp,
     vp, u32, C.POINTER(vp))
_sig("pgb_index_load_flat", C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_char_p, C.POINTER(vp))
_sig("pgb_index_load_hnsw", C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_char_p, C.POINTER(vp))
_sig("pgb_index_get_info", C.c_int, vp, C.POINTER(IndexInfo))
_sig("pgb_index_destroy", C.c_int, vp)
_sig("pgb_searcher_create", C.c_int, vp, u32, C.POINTER(QueryParams), C.POINTER(vp))
_sig("pgb_searcher_search", C.c_int, vp, vp, u32, u32, vp, vp, vp, vp)
_sig("pgb_searcher_search_host", C.c_int, vp, vp, u32, u32, vp, vp, vp)
_sig("pgb_searcher_destroy", C.c_int, vp)
_sig("pgb_index_compress", C.c_int, vp, i32, vp)
_sig("pgb_search_launches", u64)
_sig("pgb_gather_probe", C.c_int, vp, vp, vp, u64, vp, u32, vp)
_sig("pgb_index_distances", C.c_int, vp, vp, u32, u32, vp, u64, vp, vp)
_sig("pgb_index_set_l2_window", C.c_int, vp, u32, u64, C.POINTER(u64), C.POINTER(C.c_float))
L2_NONE, L2_ROWS, L2_CODES, L2_GRAPH = 0, 1, 2, 3
_sig("pgb_index_get_codes", C.c_int, vp, C.POINTER(i32), vp, vp)
_sig("pgb_searcher_create_compressed", C.c_int, vp, u32, C.POINTER(QueryParams), u32,
     C.POINTER(vp))
_sig("pgb_search_flat_noalloc", C.c_int, vp, C.POINTER(QueryParams), vp, u32, u32, vp, vp, vp,
     vp)
_sig("pgb_recall", C.c_double, vp, vp, u32, u32, vp, u32)
_sig("pgb_build_vamana", C.c_int, vp, u32, u32, C.c_int, u32, u32, C.c_float, C.c_int, u64,
     C.c_int, vp, vp)
_sig("pgb_build_vamana_gpu", C.c_int, C.c_int, vp, u32, u32, C.c_int, u32, u32, C.c_float,
     C.c_int, u64, vp, vp)
_sig("pgb_build_hnsw_gpu", C.c_int, C.c_int, vp, u32, u32, C.c_int, u32, u32, C.c_float,
     C.c_float, u64, C.c_char_p)
_sig("pgb_build_hcnng", C.c_int, vp, u32, u32, C.c_int, u32, u32, u32, u64, C.c_int, vp, vp)
_sig("pgb_build_hcnng_gpu", C.c_int, C.c_int, vp, u32, u32, C.c_int, u32, u32, u32, u64, vp,
     vp)
_sig("pgb_build_nndescent", C.c_int, vp, u32, u32, C.c_int, u32, u32, u32, C.c_float,
     C.c_float, u32, u64, C.c_int, vp, vp)
_sig("pgb_build_hnsw", C.c_int, vp, u32, u32, C.c_int, u32, u32, C.c_float, C.c_float, u64,
     C.c_int, C.c_char_p)
_sig("pgb_write_graph", C.c_int, C.c_char_p, u32, u32, vp, vp)
_sig("pgb_section_profile", C.c_int, vp, u32, C.c_int)
_sig("pgb_file_check", C.c_int, C.c_char_p, C.c_int, vp)
SECTION_NAMES = ["setup", "visit", "filter", "distances", "sort", "union", "shift", "cut_next",
                 "expansions", "queries", "n_pending", "n_cand", "n_enter", "no_cand",
                 "pred_hit"]
N_TIMED_SECTIONS = 8  # the rest are event counts


def check(status: int) -> None:
    if status != PGB_OK:
        msg = lib.pgb_last_error()
        raise PgbError(status, msg.decode() if msg else "")


class BatchOptions(C.Structure):
    _fields_ = [("max_queries", C.c_uint32), ("max_beam", C.c_uint32), ("max_k", C.c_uint32),
                ("cut", C.c_double), ("limit", C.c_int64), ("degree_limit", C.c_uint32),
                ("exclude_query_id", C.c_uint32), ("query_id_base", C.c_uint32),
                ("warps_per_block", C.c_uint32), ("filter_placement", C.c_uint32),
                ("visited_placement", C.c_uint32), ("blocks_per_sm", C.c_uint32)]


class BatchConfig(C.Structure):
    _fields_ = [("warps_per_block", C.c_uint32), ("blocks", C.c_uint32),
                ("filter_in_shared", C.c_uint32), ("visited_in_shared", C.c_uint32),
                ("shared_bytes_per_warp", C.c_uint32), ("tuned_ms", C.c_float)]


_sig("pgb_batch_create", C.c_int, vp, C.POINTER(BatchOptions), C.POINTER(vp))
_sig("pgb_batch_plan", C.c_int, vp, vp, vp, u32)
_sig("pgb_batch_search", C.c_int, vp, vp, u32, vp, vp, vp, vp)
_sig("pgb_batch_tune", C.c_int, vp, vp, u32, vp, vp, vp)
_sig("pgb_batch_search_host", C.c_int, vp, vp, u32, vp, vp, vp)
_sig("pgb_batch_get_config", C.c_int, vp, C.POINTER(BatchConfig))
_sig("pgb_batch_capture", C.c_int, vp, vp, u32, vp, vp, vp)
_sig("pgb_batch_replay", C.c_int, vp, vp)
_sig("pgb_batch_destroy", C.c_int, vp)


class ServerOptions(C.Structure):
    _fields_ = [("max_beam", C.c_uint32), ("max_k", C.c_uint32), ("max_batch", C.c_uint32),
                ("max_inflight", C.c_uint32), ("memory_budget", C.c_uint64), ("cut", C.c_double),
                ("limit", C.c_int64), ("degree_limit", C.c_uint32), ("max_wait_us", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("rejected", C.c_uint64),
                ("launches", C.c_uint64), ("pending", C.c_uint32), ("in_flight", C.c_uint32),
                ("pool_slots", C.c_uint32), ("streams", C.c_uint32), ("p50_us", C.c_double),
                ("p99_us", C.c_double), ("mean_batch", C.c_double)]


_sig("pgb_server_create", C.c_int, vp, C.POINTER(ServerOptions), C.POINTER(vp))
_sig("pgb_server_submit", C.c_int, vp, vp, u32, u32, C.POINTER(C.c_uint64))
_sig("pgb_server_poll", C.c_int, vp, C.c_uint64, u32, vp, vp, vp)
_sig("pgb_server_get_stats", C.c_int, vp, C.POINTER(ServerStats))
_sig("pgb_server_submit_many", C.c_int, vp, vp, u32, u32, vp, vp, vp, C.POINTER(C.c_uint32))
_sig("pgb_server_poll_many", C.c_int, vp, vp, u32, vp, vp, vp, vp, C.POINTER(C.c_uint32))
_sig("pgb_server_destroy", C.c_int, vp)
