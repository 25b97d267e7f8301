"""Golden fixtures that pin the oracle against the reference's own search kernels.

Three steps (the first and last run here, the middle one on a B200):
  python tests/golden/make_golden.py inputs
      writes the committed inputs: seeded int8 d=100 vector sets and graphs of the four
      families (our builders; the search semantics do not depend on them)
  python tests/golden/make_golden.py run-reference OUTDIR
      runs oracle/_ref/ref_search -- the reference's kernels compiled for sm_100a from
      the reference sources by oracle/Makefile -- on every case, one output file each
  python tests/golden/make_golden.py collect OUTDIR
      packs the reference outputs into tests/golden/reference_outputs.npz

The reference reads only int8 vectors with d = 100 (cuda/comun.h:17, lectores.cpp:129),
so every case uses that shape.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# (case name, vector set, graph file, mode, Ls, visit, k, cut)
SETS = {"c1s": ("c1s_base.i8bin", "c1s_queries.i8bin"),
        "ties": ("ties_base.i8bin", "ties_queries.i8bin")}
GRAPHS = {"vamana": ("c1s", "c1s_vamana.graph"), "hcnng": ("c1s", "c1s_hcnng.graph"),
          "nnd": ("c1s", "c1s_nnd.graph"), "hnsw": ("c1s", "c1s.hnsw"),
          "ties_vamana": ("ties", "ties_vamana.graph"), "ties_hnsw": ("ties", "ties.hnsw")}


def cases():
    out = []
    flat_cfgs = [(10, 3, 10, 1.35), (10, 8, 10, 1.35), (10, -1, 10, 1.35), (20, -1, 10, 1.35),
                 (40, -1, 10, 1.35), (80, -1, 10, 1.35), (40, -1, 10, 0.9), (64, -1, 50, 1.35),
                 (150, -1, 10, 1.35)]
    for g in ("vamana", "hcnng", "nnd", "ties_vamana"):
        for Ls, visit, k, cut in flat_cfgs:
            out.append((f"{g}_L{Ls}_v{visit}_k{k}_c{cut}", g, "flat", Ls, visit, k, cut))
    for g in ("hnsw", "ties_hnsw"):
        for Ls, visit, k in [(10, -1, 10), (50, -1, 10), (100, -1, 10), (50, 5, 10), (20, -1, 20),
                             (150, -1, 10)]:
            out.append((f"{g}_L{Ls}_v{visit}_k{k}", g, "hnsw", Ls, visit, k, 1.35))
    return out


def _pkg():
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    return ge.load_package()


def make_inputs():
    pgb = _pkg()
    from parlayann_gpu_busqueda_b200 import synthetic as syn
    base, queries = syn.dataset(syn.LAW_C1, 2000, 100, seed=0)
    pgb.write_vectors(os.path.join(HERE, "c1s_base.i8bin"), base)
    pgb.write_vectors(os.path.join(HERE, "c1s_queries.i8bin"), queries)
    # exact ties: every vector appears three times; queries include copies of base rows
    rng = np.random.default_rng(7)
    uniq, _ = syn.dataset(syn.LAW_C1, 300, 1, seed=3)
    tb = np.repeat(uniq, 3, axis=0)[rng.permutation(900)]
    tq = np.concatenate([tb[rng.choice(900, 30, replace=False)],
                         syn.dataset(syn.LAW_C1, 10, 30, seed=4)[1]])
    pgb.write_vectors(os.path.join(HERE, "ties_base.i8bin"), tb)
    pgb.write_vectors(os.path.join(HERE, "ties_queries.i8bin"), tq)
    pgb.write_graph(os.path.join(HERE, "c1s_vamana.graph"),
                    pgb.build_vamana(base, R=32, L=64, alpha=1.2, seed=0))
    pgb.write_graph(os.path.join(HERE, "c1s_hcnng.graph"),
                    pgb.build_hcnng(base, trees=10, leaf=400, mst_deg=3, seed=0))
    pgb.write_graph(os.path.join(HERE, "c1s_nnd.graph"),
                    pgb.build_nndescent(base, K=24, init_trees=4, leaf=400, seed=0))
    pgb.build_hnsw(base, os.path.join(HERE, "c1s.hnsw"), M=8, ef_construction=48, ml=0.5,
                   alpha=1.0, seed=0)
    pgb.write_graph(os.path.join(HERE, "ties_vamana.graph"),
                    pgb.build_vamana(tb, R=16, L=32, alpha=1.2, seed=1))
    pgb.build_hnsw(tb, os.path.join(HERE, "ties.hnsw"), M=6, ef_construction=32, ml=0.6,
                   alpha=1.0, seed=1)


def run_reference(outdir):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_search")
    os.makedirs(outdir, exist_ok=True)
    for name, g, mode, Ls, visit, k, cut in cases():
        vset, gfile = GRAPHS[g]
        b, q = SETS[vset]
        cmd = [exe, mode, os.path.join(HERE, b), os.path.join(HERE, q), os.path.join(HERE, gfile),
               str(Ls), str(visit), str(k), str(cut), os.path.join(outdir, name + ".bin")]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    print(f"{len(cases())} reference runs written to {outdir}")


def read_ref_output(path):
    raw = np.fromfile(path, dtype=np.uint32)
    nq, k = int(raw[0]), int(raw[1])
    o = 2
    ids = raw[o:o + nq * k].reshape(nq, k)
    o += nq * k
    dists = raw[o:o + nq * k].view(np.int32).reshape(nq, k)
    o += nq * k
    comp = raw[o:o + nq].view(np.int32)
    flags = raw[o + nq:o + 2 * nq].view(np.int32)
    return ids, dists, comp, flags


def collect(outdir):
    arrays = {}
    for name, *_ in cases():
        ids, dists, comp, flags = read_ref_output(os.path.join(outdir, name + ".bin"))
        arrays[name + "__ids"] = ids
        arrays[name + "__dists"] = dists
        arrays[name + "__comp"] = comp
        arrays[name + "__flags"] = flags
    np.savez_compressed(os.path.join(HERE, "reference_outputs.npz"), **arrays)
    print(f"packed {len(cases())} cases")


if __name__ == "__main__":
    cmd = sys.argv[1]
    if cmd == "inputs":
        make_inputs()
    elif cmd == "run-reference":
        run_reference(sys.argv[2])
    elif cmd == "collect":
        collect(sys.argv[2])
    else:
        raise SystemExit(__doc__)
