"""The C++ interface (include/pgb_buscador.hpp) builds against the C ABI on any machine,
and on a B200 reproduces the reference kernels' golden outputs through the same
preparar / lanzar / liberar sequence the reference's drivers use."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "buscador_golden.cpp")
LIBDIR = os.path.join(ROOT, "parlayann-gpu-busqueda_b200", "lib")


def build(tmp_path):
    exe = str(tmp_path / "buscador_golden")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           "-I", "/usr/local/cuda/include", SRC, "-o", exe, "-L", LIBDIR, "-lpgb",
           f"-Wl,-rpath,{LIBDIR}", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_cpp_interface_compiles_and_links(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", [("vamana", "c1s_vamana.graph", "flat", 40, -1, 10, 1.35),
                                  ("hcnng", "c1s_hcnng.graph", "flat", 10, 8, 10, 1.35),
                                  ("hnsw", "c1s.hnsw", "hnsw", 50, -1, 10, 1.35)])
def test_cpp_interface_reproduces_reference_outputs(tmp_path, gpu, case):
    name, gfile, mode, Ls, visit, k, cut = case
    exe = build(tmp_path)
    out = str(tmp_path / "out.bin")
    subprocess.run([exe, mode, os.path.join(GOLDEN, "c1s_base.i8bin"),
                    os.path.join(GOLDEN, "c1s_queries.i8bin"), os.path.join(GOLDEN, gfile),
                    str(Ls), str(visit), str(k), str(cut), out], check=True)
    raw = np.fromfile(out, dtype=np.uint32)
    nq, kk = int(raw[0]), int(raw[1])
    ids = raw[2:2 + nq * kk].reshape(nq, kk)
    dists = raw[2 + nq * kk:2 + 2 * nq * kk].view(np.int32).reshape(nq, kk)
    comp = raw[2 + 2 * nq * kk:2 + 2 * nq * kk + nq].view(np.int32)
    flags = raw[2 + 2 * nq * kk + nq:].view(np.int32)
    ref = np.load(os.path.join(GOLDEN, "reference_outputs.npz"))
    key = (f"{name}_L{Ls}_v{visit}_k{k}_c{cut}" if mode == "flat"
           else f"{name}_L{Ls}_v{visit}_k{k}")
    assert np.array_equal(ids, ref[key + "__ids"])
    assert np.array_equal(dists, ref[key + "__dists"])
    assert np.array_equal(comp, ref[key + "__comp"])
    assert np.array_equal(flags, ref[key + "__flags"])
