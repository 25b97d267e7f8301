"""The C-ABI library loads on a machine without a GPU, exports every entry point that
include/pgb.h declares, and reports errors as status codes (never exits)."""
import ctypes as C
import os
import re

import numpy as np

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pgb.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pgb_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_function_is_exported(pgb):
    names = declared_functions()
    assert len(names) >= 30
    lib = C.CDLL(pgb._native.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in pgb.h but not exported: {missing}"


def test_status_strings_and_last_error(pgb):
    lib = pgb._native.lib
    for s in range(10):
        assert lib.pgb_status_string(s)
    # a bad call sets the thread's last error and returns a status
    st = lib.pgb_write_graph(b"/nonexistent/x.graph", 0, 0, None, None)
    assert st == 1
    assert b"write_graph" in lib.pgb_last_error()


def test_index_creation_without_gpu_is_an_error_not_an_exit(pgb):
    if pgb.device_available():
        return  # on a GPU machine creation succeeds; covered by the gpu tests
    x = np.zeros((4, 8), np.int8)
    deg = np.array([1, 1, 1, 1], np.uint32)
    edges = np.array([1, 2, 3, 0], np.uint32)
    h = C.c_void_p()
    st = pgb._native.lib.pgb_index_create_flat(0, x.ctypes.data, 4, 8, 0, deg.ctypes.data,
                                               edges.ctypes.data, C.byref(h))
    assert st == 3 and not h.value  # PGB_ERR_CUDA
    assert b"device" in pgb._native.lib.pgb_last_error()


def test_argument_checks(pgb):
    lib = pgb._native.lib
    h = C.c_void_p()
    x = np.zeros((4, 8), np.int8)
    deg = np.array([1, 1, 1, 300], np.uint32)
    edges = np.zeros(303, np.uint32)
    assert lib.pgb_index_create_flat(0, x.ctypes.data, 4, 8, 0, deg.ctypes.data,
                                     edges.ctypes.data, C.byref(h)) == 1  # degree > 256
    assert lib.pgb_index_create_flat(0, x.ctypes.data, 4, 200, 0, deg.ctypes.data,
                                     edges.ctypes.data, C.byref(h)) == 1  # dim > 128
    deg = np.array([1, 1, 1, 1], np.uint32)
    edges = np.array([1, 2, 3, 9], np.uint32)
    assert lib.pgb_index_create_flat(0, x.ctypes.data, 4, 8, 0, deg.ctypes.data,
                                     edges.ctypes.data, C.byref(h)) == 6  # edge out of range
    assert lib.pgb_searcher_create(None, 1, None, C.byref(h)) == 1
    assert lib.pgb_recall(None, None, 0, 0, None, 0) < 0


def test_section_profile_absent_from_the_product_build(pgb):
    buf = (C.c_uint64 * 10)()
    if pgb._native.LIB_PATH.endswith("libpgb.so"):
        assert pgb._native.lib.pgb_section_profile(buf, 10, 0) == 1
