"""Full-size parity check against the reference's own kernels (test infrastructure).

Runs the reference's BuscadorGPU / BuscadorHnsw (oracle/_ref/ref_search, built from the
reference sources by oracle/Makefile) and this library's searcher on the bench's 1M
workload (rank 0's 29,316 queries, k=10, cut 1.35, no visit limit) over one graph family,
and compares ids, distances, distance counts and flags query by query.

    python oracle/compare_ref.py vamana|hcnng|nnd|hnsw [Ls ...]      (needs a GPU)

Default beams: each family's recall@10 >= 0.90 operating point (40 / 16 / 79 / 79).
Prints one JSON line per beam; exits 1 if anything differs.
"""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
import __graft_entry__ as ge  # noqa: E402

DEFAULT_LS = {"vamana": 40, "hcnng": 16, "nnd": 79, "hnsw": 79}


def read_ref(path):
    """ref_search output: [nq u32][k u32] ids[nq][k] dists[nq][k] comps[nq] flags[nq]."""
    raw = np.fromfile(path, dtype=np.uint32)
    nq, k = int(raw[0]), int(raw[1])
    o = 2
    ids = raw[o:o + nq * k].reshape(nq, k)
    o += nq * k
    dists = raw[o:o + nq * k].view(np.int32).reshape(nq, k)
    o += nq * k
    comps = raw[o:o + nq].view(np.int32)
    o += nq
    flags = raw[o:o + nq].view(np.int32)
    return ids, dists, comps, flags


def main():
    kind = sys.argv[1] if len(sys.argv) > 1 else "hnsw"
    beams = [int(a) for a in sys.argv[2:]] or [DEFAULT_LS[kind]]
    pgb = ge.load_package()
    d = bench.data_dir()
    if kind == "hnsw":
        base, h = bench.load_hnsw(pgb)
        queries = bench.rank_queries(0)
        index = pgb.Index.hnsw(base, h)
        mode, model = "hnsw", os.path.join(d, bench.HNSW_FILE)
    else:
        base, queries, graph = bench.load_workload(pgb, 0, lambda: None, kind)
        index = pgb.Index.flat(base, graph)
        mode, model = "flat", os.path.join(d, bench.GRAPHS[kind][0])
    qp = os.path.join(d, "c2_q0.i8bin")
    pgb.write_vectors(qp, queries)
    ok = True
    for Ls in beams:
        out = os.path.join(d, "ref_%s_L%d.bin" % (kind, Ls))
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_search"), mode,
                        os.path.join(d, "c2_base.i8bin"), qp, model, str(Ls), "-1", "10", "1.35",
                        out], check=True)
        rid, rd, rc, rf = read_ref(out)
        # flat graphs: the reference skips a neighbour equal to the query's index (its
        # wrapper's p.id()); the searcher's default exclusion reproduces that
        s = pgb.Searcher(index, len(queries), pgb.QueryParams(k=rid.shape[1], beam_size=Ls, cut=1.35))
        ids, dists, stats = s.search(queries)
        s.liberar()
        res = {"graph": kind, "Ls": Ls, "nq": int(rid.shape[0]),
               "ids_equal": bool(np.array_equal(ids.view(np.uint32), rid)),
               "dists_equal": bool(np.array_equal(dists, rd)),
               "comps_equal": bool(np.array_equal(stats[:, 0], rc)),
               "flags_equal": bool(np.array_equal(stats[:, 2], rf)),
               "comps_per_query": float(rc.mean())}
        ok &= all(v for kk, v in res.items() if kk.endswith("_equal"))
        print(json.dumps(res), flush=True)
    index.close()
    sys.exit(0 if ok else 1)


if __name__ == "__main__":
    main()
