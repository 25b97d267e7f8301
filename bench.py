"""Benchmark: QPS at recall@10 = 0.90, batched vs plain warp-per-query kernel, on B200.

Workload (one GPU): 1,000,000 int8 d=100 vectors (seeded Gaussian mixture standing in
for MSSPACEV-1M), Vamana R=64 L=128 alpha=1.2, 29,316 queries, k=10. A step is one search
of all queries. The operating point is the smallest beam of the 18-value sweep whose
recall@10 (with distance ties, against exact GPU brute force) is >= 0.90.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank searches its own 29,316 queries against its own replica of
the index (weak scaling, no collective on the data path); the step time is the max over
ranks. ``--impl reference`` times the CPU restatement of the reference's search
(oracle/, all host threads) on the same workload; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import __graft_entry__ as ge  # noqa: E402

N_BASE = 1_000_000
N_QUERIES = 29_316
K = 10
R, L_BUILD, ALPHA = 64, 128, 1.2
TARGET_RECALL = 0.90
POLL_HEAD = 4096  # serving client: outstanding tickets polled per pass, oldest first
PARITY_SAMPLE = 1024  # queries of each full-size parity check against the oracle
METRIC = "QPS @ recall@10=0.90, batched vs plain kernel, 1 B200; serving p50/p99 latency"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def data_dir():
    d = os.environ.get("PGB_DATA", os.path.join(ROOT, "_data"))
    os.makedirs(d, exist_ok=True)
    return d


def standalone(name):
    """A numpy-only module of the package (formats, synthetic) loaded by itself, without
    importing the package (which maps lib/libpgb.so): the reference arm reads the data
    files with these and runs only the CPU restatement."""
    import importlib.util
    key = "pgb_standalone_" + name
    if key in sys.modules:
        return sys.modules[key]
    spec = importlib.util.spec_from_file_location(
        key, os.path.join(ROOT, "parlayann-gpu-busqueda_b200", name + ".py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[key] = mod
    spec.loader.exec_module(mod)
    return mod


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# the four graph families of the 1M workload, as the reference's runs name them; Vamana
# and HCNNG graphs come from the GPU builders, whose graphs are the CPU builders'
# (tests/test_build_gpu.py)
GRAPHS = {
    "vamana": ("c2_vamana_R64_L128_a1.2.graph", "Vamana R64 L128 alpha1.2",
               lambda pgb, x: pgb.build_vamana_gpu(x, R=R, L=L_BUILD, alpha=ALPHA, seed=0)),
    "hcnng": ("c2_hcnng_T30_L1000_m3.graph", "HCNNG 30 trees leaf1000 MST3",
              lambda pgb, x: pgb.build_hcnng_gpu(x, trees=30, leaf=1000, mst_deg=3, seed=0)),
    "nnd": ("c2_nnd_K40.graph", "PyNNDescent K40 alpha1.2",
            lambda pgb, x: pgb.build_nndescent(x, K=40, init_trees=10, leaf=1000, alpha=1.2,
                                               seed=0)),
}
HNSW_FILE = "c2_hnsw_M32_efc128.hnsw"


def load_base(pgb):
    from parlayann_gpu_busqueda_b200 import synthetic as syn
    base_p = os.path.join(data_dir(), "c2_base.i8bin")
    if not os.path.exists(base_p):
        base = syn.LAW_C2.sample(N_BASE, 0, 0)
        pgb.write_vectors(base_p + ".tmp", base)
        os.replace(base_p + ".tmp", base_p)
    return pgb.read_vectors(base_p)


def load_workload(pgb, rank, barrier, kind="vamana", nq=N_QUERIES):
    """Base vectors, this rank's queries and a flat graph (built once, cached on disk)."""
    fname, _, build = GRAPHS[kind]
    graph_p = os.path.join(data_dir(), fname)
    if rank == 0:
        base = load_base(pgb)
        if not os.path.exists(graph_p):
            t = time.time()
            g = build(pgb, base)
            log(f"built {kind} 1M in {time.time() - t:.1f} s")
            pgb.write_graph(graph_p + ".tmp", g)
            os.replace(graph_p + ".tmp", graph_p)
    barrier()
    base = load_base(pgb)
    graph = pgb.read_graph(graph_p)
    return base, rank_queries(rank, nq), graph


def rank_queries(rank, nq=N_QUERIES):
    """This rank's shard of the query stream: its own seeded draw from the base's law
    (stream 1 + rank), so that no two ranks search the same queries."""
    from parlayann_gpu_busqueda_b200 import synthetic as syn
    return syn.LAW_C2.sample(nq, 0, 1 + rank)


def max_over_ranks(x, device, world):
    """The largest of every rank's x (a step time): all ranks take part in the same
    all-reduce, so the slowest rank sets the whole job's time."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, steps, seconds):
    """Units all ranks processed in `steps` steps over the slowest rank's time."""
    return units_per_rank * world * steps / seconds


def load_hnsw(pgb):
    p = os.path.join(data_dir(), HNSW_FILE)
    base = load_base(pgb)
    if not os.path.exists(p):
        # the GPU builder writes the CPU builder's file (tests/test_build_gpu.py)
        t = time.time()
        pgb.build_hnsw_gpu(base, p + ".tmp", M=32, ef_construction=128, ml=0.36, alpha=0.83, seed=0)
        os.replace(p + ".tmp", p)
        log(f"built HNSW 1M on the GPU in {time.time() - t:.1f} s")
    return base, pgb.read_hnsw(p)


def ground_truth(base, queries, rank, device):
    from parlayann_gpu_busqueda_b200 import groundtruth, formats
    p = os.path.join(data_dir(), f"c2_gt100_q{rank}.bin")
    if os.path.exists(p):
        return formats.read_gt(p)
    ids, dists = groundtruth.knn_gpu(base, queries, 100, device)
    formats.write_gt(p + f".tmp{rank}", ids, dists)
    os.replace(p + f".tmp{rank}", p)
    return ids, dists


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while active."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu, self.proc, self.file = gpu_index, None, None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.file:
            return None
        self.file.flush()
        rows = [r.split(", ") for r in open(self.file.name).read().strip().splitlines() if r]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        m = json.load(open(p))
        return float(m["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def prepare_data(args):
    """--prepare: the 1M base, rank 0's queries' ground truth and the Vamana graph, built
    and cached on disk (the reference arm runs this in a separate, untimed process)."""
    import torch
    torch.cuda.set_device(0)
    pgb = ge.load_package()
    base, queries, _ = load_workload(pgb, 0, lambda: None)
    ground_truth(base, queries, 0, 0)


def run_reference(args, rank):
    """CPU restatement of the reference search (oracle) on the host cores. This process
    reads the data with the package's numpy-only readers and never maps the library; a
    cold data cache is filled first by `bench.py --prepare` in a child process."""
    if rank != 0:
        return
    fmt, syn = standalone("formats"), standalone("synthetic")
    base_p = os.path.join(data_dir(), "c2_base.i8bin")
    graph_p = os.path.join(data_dir(), GRAPHS["vamana"][0])
    gt_p = os.path.join(data_dir(), "c2_gt100_q0.bin")
    if not (os.path.exists(base_p) and os.path.exists(graph_p) and os.path.exists(gt_p)):
        t = time.time()
        subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--prepare"], check=True)
        log(f"data prepared in {time.time() - t:.1f} s (separate process, untimed)")
    oracle = ge.load_oracle()
    base = fmt.read_vectors(base_p)
    graph = fmt.read_graph(graph_p)
    queries = syn.LAW_C2.sample(N_QUERIES, 0, 1)
    Ls = int(os.environ.get("PGB_REF_LS", "0"))
    formats = fmt
    if not Ls:
        # same rule as our arm: smallest sweep beam reaching the target recall
        LS_SWEEP = syn.LS_SWEEP
        gi, gd = formats.read_gt(gt_p) if os.path.exists(gt_p) else (None, None)
        Ls = 40
        if gi is not None:
            sample = slice(0, 2000)
            for ls in LS_SWEEP:
                ids = oracle.flat_search(base, graph.degrees, graph.edges, queries[sample], K, ls)[0]
                if oracle.recall(gi[sample], gd[sample], ids, K) >= TARGET_RECALL:
                    Ls = ls
                    break
    threads = os.cpu_count() or 1
    # bounded sample: every step searches the first `sample` queries on all threads
    sample = min(N_QUERIES, int(os.environ.get("PGB_REF_SAMPLE", "8192")))
    q = np.ascontiguousarray(queries[:sample])
    for _ in range(args.warmup):
        oracle.flat_search(base, graph.degrees, graph.edges, q, K, Ls, threads=threads)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        oracle.flat_search(base, graph.degrees, graph.edges, q, K, Ls, threads=threads)
        times.append(time.perf_counter() - t)
    # the reference's protocol (comparacion1.cu:76-101): warm-up, then the best step
    qps = sample / min(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * min(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8", "data": "synthetic",
        "config": {"workload": "1M int8 d=100 Vamana R64 L128 a1.2, k=10", "Ls": Ls,
                   "queries_per_step": sample, "mean_step_qps": sample * len(times) / sum(times)},
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"first {sample} of {N_QUERIES} queries at Ls={Ls}",
                         "protocol": f"{args.warmup} warm-up steps, then the best of {args.steps}"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def section_shares(pgb, run, steps):
    """Section cycle shares and event counts per expansion of `steps` calls of run() under
    the profiling library (None under the plain library)."""
    if not os.environ.get("PGB_LIB", "").endswith("libpgb_prof.so"):
        return None
    import ctypes
    names = pgb._native.SECTION_NAMES
    nt = pgb._native.N_TIMED_SECTIONS
    buf = (ctypes.c_uint64 * len(names))()
    pgb._native.check(pgb._native.lib.pgb_section_profile(buf, len(names), 1))
    for _ in range(steps):
        run()
    pgb._native.check(pgb._native.lib.pgb_section_profile(buf, len(names), 1))
    cyc = list(buf)[:nt]
    tot = sum(cyc)
    sections = {n: round(c / tot, 4) for n, c in zip(names, cyc)}
    n_exp = max(1, buf[nt])
    sections["cycles_per_expansion"] = tot / n_exp
    for n, c in zip(names[nt + 2:], list(buf)[nt + 2:]):
        sections[n + "_per_expansion"] = round(c / n_exp, 3)
    return sections


def run_profile_hnsw(args, local):
    """Launches only the HNSW search kernel (M=32 model of the 1M base) on a small query set;
    under the profiling library, its section shares (filter / distances / acceptance = sort /
    cand update = union / W update = shift)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    from parlayann_gpu_busqueda_b200.synthetic import LAW_C2
    base, h = load_hnsw(pgb)
    nq, Ls = args.profile_nq, args.profile_ls
    queries = LAW_C2.sample(nq, 0, 1)
    index = pgb.Index.hnsw(base, h, device=local)
    q = torch.from_numpy(np.ascontiguousarray(queries).view(np.uint8)).to(dev)
    sp = torch.cuda.current_stream(dev).cuda_stream
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=K, beam_size=Ls))
    ids = torch.empty((nq, K), dtype=torch.int32, device=dev)
    d = torch.empty_like(ids)
    st = torch.empty((nq, 4), dtype=torch.int32, device=dev)
    for _ in range(args.warmup + args.steps):
        s.lanzar(q, ids, d, st, sp)
    torch.cuda.synchronize(dev)

    def run():
        s.lanzar(q, ids, d, st, sp)
        torch.cuda.synchronize(dev)
    sections = section_shares(pgb, run, args.steps)
    stn = st.cpu().numpy()
    print(json.dumps({"profile": "hnsw", "nq": nq, "Ls": Ls, "sections": sections,
                      "comps": int(stn[:, 0].astype(np.int64).sum()),
                      "expansions": int(stn[:, 1].astype(np.int64).sum())}))


def run_profile(args, local):
    """Launches only the search kernels (plain, then batched) on a small query set; with
    --workload codes the plain launches search the 4-bit code rows (+ the re-rank)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    base, queries, graph = load_workload(pgb, 0, lambda: None)
    nq, Ls = args.profile_nq, args.profile_ls
    index = pgb.Index.flat(base, graph, device=local)
    codes = args.workload == "codes"
    if codes:
        index.compress()
    q = torch.from_numpy(np.ascontiguousarray(queries[:nq]).view(np.uint8)).to(dev)
    sp = torch.cuda.current_stream(dev).cuda_stream
    s = pgb.Searcher(index, nq, pgb.QueryParams(k=K, beam_size=Ls), rerank=Ls if codes else 0)
    ids = torch.empty((nq, K), dtype=torch.int32, device=dev)
    d = torch.empty_like(ids)
    st = torch.empty((nq, 4), dtype=torch.int32, device=dev)
    b = pgb.Batch(index, nq, max_beam=Ls, max_k=K, warps_per_block=args.profile_wpb,
                  filter_placement=1, visited_placement=2)
    b.plan(np.full(nq, Ls, np.uint32), np.full(nq, K, np.uint32))
    for _ in range(args.warmup + args.steps):
        s.lanzar(q, ids, d, st, sp)
    for _ in range(args.warmup + args.steps):
        b.search(q, ids, d, st, sp)
    torch.cuda.synchronize(dev)
    stn = st.cpu().numpy()

    # section cycles of the batched launches only
    def run():
        b.search(q, ids, d, st, sp)
        torch.cuda.synchronize(dev)
    sections = section_shares(pgb, run, args.steps)
    print(json.dumps({"profile": True, "nq": nq, "Ls": Ls, "sections": sections,
                      "comps": int(stn[:, 0].astype(np.int64).sum()),
                      "expansions": int(stn[:, 1].astype(np.int64).sum()),
                      "row_stride": (int(index.info.max_degree) + 31) // 32 * 32}))


def oracle_agrees(oracle, base, kind, graph, queries, Ls, got):
    """True when the oracle's ids, int32 distances, distance counts, expansions and flags
    equal `got` = (ids, dists, stats) of the first PARITY_SAMPLE queries at beam Ls."""
    qs = np.ascontiguousarray(queries[:PARITY_SAMPLE])
    o = (oracle.hnsw_search(base, graph, qs, K, Ls) if kind == "hnsw"
         else oracle.flat_search(base, graph.degrees, graph.edges, qs, K, Ls))
    ids, dists, st = got
    return bool(np.array_equal(ids, o[0]) and np.array_equal(dists, o[1]) and
                np.array_equal(st[:, 0], o[2]) and np.array_equal(st[:, 1], o[3]) and
                np.array_equal(st[:, 2], o[4]))


def run_extras(args, pgb, torch, dev, local, base, queries, graph, gt_ids, gt_d, oracle, flush,
               Ls, swept):
    """After the headline, on one GPU: (1) full-size parity against the oracle on the first
    PARITY_SAMPLE queries -- Vamana at the smallest, the operating, the widest swept beam and
    at 316 (global filter and visited tables), and HCNNG, PyNNDescent and HNSW at their own
    recall@10 >= 0.90 beams; (2) those families' plain and batched QPS with the L2 flushed
    and their gather roofline; (3) 100k queries of uneven beams and k in one batched launch
    against the plain kernel once per (Ls, k), on the Vamana graph and the HNSW model; (4)
    the serving loop on both at two offered rates. Returns the blocks of the bench line."""
    from parlayann_gpu_busqueda_b200.synthetic import LS_SWEEP
    t_start = time.time()
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    q_dev = torch.from_numpy(queries.view(np.uint8)).to(dev)
    peak, _ = measured_peaks()
    ident = {}
    for ls in sorted({LS_SWEEP[0], Ls, max(swept)}):
        ident[f"vamana Ls={ls}"] = oracle_agrees(oracle, base, "vamana", graph, queries, ls, swept[ls])
    index = pgb.Index.flat(base, graph, device=local)
    wide = 316
    s = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=wide))
    wi, wd, ws = s.search_device(q_dev, sp)
    b = pgb.Batch(index, N_QUERIES, max_beam=wide, max_k=K)
    b.plan(np.full(N_QUERIES, wide, np.uint32), np.full(N_QUERIES, K, np.uint32))
    bi, bd, bs = b.outputs(dev)
    b.search(q_dev, bi, bd, bs, sp)
    torch.cuda.synchronize(dev)
    ident[f"vamana Ls={wide}"] = (
        oracle_agrees(oracle, base, "vamana", graph, queries, wide,
                      (wi.cpu().numpy().view(np.uint32)[:PARITY_SAMPLE],
                       wd.cpu().numpy()[:PARITY_SAMPLE], ws.cpu().numpy()[:PARITY_SAMPLE]))
        and bool(torch.equal(wi, bi) and torch.equal(wd, bd)))
    s.liberar()
    b.close()
    index.close()

    families = {}
    for kind in ("hcnng", "nnd", "hnsw"):
        t0 = time.time()
        if kind == "hnsw":
            _, fg = load_hnsw(pgb)
            index = pgb.Index.hnsw(base, fg, device=local)
        else:
            _, _, fg = load_workload(pgb, 0, lambda: None, kind)
            index = pgb.Index.flat(base, fg, device=local)
        setup_s = time.time() - t0
        fam_ls, sweep, kept = None, [], None
        for ls in LS_SWEEP:
            s = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=ls))
            ids, dists, st = s.search_device(q_dev, sp)
            torch.cuda.synchronize(dev)
            ids_h = ids.cpu().numpy().view(np.uint32)
            rec = pgb.recall(gt_ids, gt_d, ids_h, K)
            sweep.append([ls, round(rec, 5)])
            s.liberar()
            if rec >= TARGET_RECALL or ls == LS_SWEEP[-1]:
                fam_ls = ls
                kept = (ids_h[:PARITY_SAMPLE], dists.cpu().numpy()[:PARITY_SAMPLE],
                        st.cpu().numpy()[:PARITY_SAMPLE])
                break
        ident[f"{kind} Ls={fam_ls}"] = oracle_agrees(oracle, base, kind, fg, queries, fam_ls, kept)
        plain = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=fam_ls))
        p_ids = torch.empty((N_QUERIES, K), dtype=torch.int32, device=dev)
        p_d = torch.empty_like(p_ids)
        p_st = torch.empty((N_QUERIES, 4), dtype=torch.int32, device=dev)
        tp = _timed_events(torch, stream, lambda: plain.lanzar(q_dev, p_ids, p_d, p_st, sp),
                           args.steps, args.warmup, flush)
        b = pgb.Batch(index, N_QUERIES, max_beam=fam_ls, max_k=K)
        b.plan(np.full(N_QUERIES, fam_ls, np.uint32), np.full(N_QUERIES, K, np.uint32))
        bi, bd, bs = b.outputs(dev)
        cfg = b.tune(q_dev, bi, bd, bs)
        b.capture(q_dev, bi, bd, bs)
        tb = _timed_events(torch, stream, lambda: b.replay(sp), args.steps, args.warmup, flush)
        stn = p_st.cpu().numpy()
        gsz = (int(index.info.max_degree) + 31) // 32 * 32
        bytes_launch = float(128 * stn[:, 0].astype(np.int64).sum() +
                             4 * gsz * stn[:, 1].astype(np.int64).sum())
        mp, mb = sum(tp) / len(tp) / 1e3, sum(tb) / len(tb) / 1e3
        families[kind] = {
            "graph": GRAPHS[kind][1] if kind != "hnsw" else "HNSW M32 efc128",
            "Ls": fam_ls, "recall_at_10": dict((a, c) for a, c in sweep)[fam_ls],
            "plain_qps": N_QUERIES / mp, "batched_qps": N_QUERIES / mb,
            "batched_over_plain": mp / mb,
            "identical_neighbours": bool(torch.equal(p_ids, bi) and torch.equal(p_d, bd)),
            "frac": bytes_launch / mb / 1e9 / peak, "plain_frac": bytes_launch / mp / 1e9 / peak,
            "kernel": "hnsw_kernel" if kind == "hnsw" else "flat_batched_kernel",
            "comps_per_query": float(stn[:, 0].mean()),
            "expansions_per_query": float(stn[:, 1].mean()),
            "batched_config": cfg, "setup_s": round(setup_s, 1)}
        log(kind, families[kind])
        plain.liberar()
        b.close()
        index.close()

    # the batched form's own case: 100k queries of uneven beams and k in one launch
    mixed = {}
    mq = rank_queries(0, MIXED_NQ)
    for kind in ("vamana", "hnsw"):
        if kind == "hnsw":
            _, h = load_hnsw(pgb)
            index = pgb.Index.hnsw(base, h, device=local)
        else:
            index = pgb.Index.flat(base, graph, device=local)
        mixed[kind] = mixed_leg(pgb, torch, dev, index, mq, 3)
        log("mixed", kind, {k: v for k, v in mixed[kind].items() if k != "batched_config"})
        index.close()

    serving = {}
    rng = np.random.default_rng(1)
    seconds = float(os.environ.get("PGB_SERVE_SECONDS", "2"))
    for kind in ("vamana", "hnsw"):
        if kind == "hnsw":
            _, h = load_hnsw(pgb)
            index = pgb.Index.hnsw(base, h, device=local)
        else:
            index = pgb.Index.flat(base, graph, device=local)
        serving[kind] = [serve_rate(pgb, index, queries, gt_ids, gt_d, rate, seconds, rng)
                         for rate in (100_000, 1_000_000)]
        log("serving", kind, serving[kind])
        index.close()
    log(f"extras in {time.time() - t_start:.1f} s")
    return {"identical_to_oracle": ident, "families": families, "mixed": mixed,
            "serving": serving}


def gather_rate(pgb, torch, dev, index, query_dev, lanes, count, steps, warmup, flush,
                seed=0, sequential=False):
    """Row-gather rate of pgb_gather_probe: `count` rows (uniformly random ids, or 0..count-1
    in order) per step, L2 flushed before each step; returns (GB/s of 128-byte rows, the
    output of the last step)."""
    n = int(index.info.n_points)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    ids = (torch.arange(count, device=dev, dtype=torch.int64) % n if sequential else
           torch.randint(0, n, (count,), device=dev, generator=g)).to(torch.int32)
    out = torch.empty(count, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    t = _timed_events(torch, stream,
                      lambda: index.gather_probe(query_dev, ids, lanes, out, stream.cuda_stream),
                      steps, warmup, flush)
    return count * 128 / (sum(t) / len(t) / 1e3) / 1e9, out


def run_gather(args, local):
    """Gather calibration: the rate at which this B200 gathers random 128-byte rows with
    1, 4 (the search kernels' layout), 8 and 32 threads per row, from the 1M int8 d=100
    base (128 MB, about the size of L2) and from a 10M-row table (1.28 GB, HBM), L2
    flushed before every step; rows read in order give the streaming rate beside it. All
    layouts compute the same distances (checked)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    from parlayann_gpu_busqueda_b200.formats import Graph
    base = load_base(pgb)
    big = np.random.default_rng(5).integers(-128, 128, size=(10_000_000, 100), dtype=np.int8)
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)
    count = int(os.environ.get("PGB_GATHER_ROWS", str(20_000_000)))
    query = torch.from_numpy(rank_queries(0, 1).view(np.uint8)[0].copy()).to(dev)
    tables = {}
    peak, kind = measured_peaks()
    for name, x in (("1M rows (128 MB)", base), ("10M rows (1.28 GB)", big)):
        n = x.shape[0]
        chain = Graph(n, 1, np.ones(n, np.uint32), ((np.arange(n) + 1) % n).astype(np.uint32))
        index = pgb.Index.flat(x, chain, device=local)
        rows, ref = {}, None
        for lanes in (4, 1, 8, 32):
            gbs, out = gather_rate(pgb, torch, dev, index, query, lanes, count, args.steps,
                                   args.warmup, flush)
            if ref is None:
                ref = out.clone()
            rows[f"{lanes} lanes/row"] = {"gbs": gbs, "frac_of_hbm_peak": gbs / peak,
                                          "same_distances": bool(torch.equal(out, ref))}
            log(name, lanes, rows[f"{lanes} lanes/row"])
        seq, _ = gather_rate(pgb, torch, dev, index, query, 4, min(count, n), args.steps,
                             args.warmup, flush, sequential=True)
        rows["rows in order, 4 lanes/row"] = {"gbs": seq, "frac_of_hbm_peak": seq / peak}
        tables[name] = rows
        index.close()
    best = max(r["gbs"] for r in tables["10M rows (1.28 GB)"].values())
    print(json.dumps({
        "metric": "random 128-byte row gather rate, 1 B200", "value": best, "unit": "GB/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "dtype": "int8", "data": "synthetic",
        "config": {"workload": f"{count} rows per step, ids uniform at random; L2 flushed",
                   "tables": tables, "hbm_peak_gbs": peak, "peak_source": kind},
        "gpu_launches": _TIMED_LAUNCHES[0]}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: skip the other graph families' parity / QPS and the "
                         "serving leg (always skipped with more than one GPU)")
    ap.add_argument("--prepare", action="store_true",
                    help="build and cache the headline data (base, graph, ground truth), then exit")
    ap.add_argument("--profile", action="store_true",
                    help="small case for ncu: the 1M index, --profile-nq queries at --profile-ls, "
                         "warm-up then --steps launches of each kernel, nothing else")
    ap.add_argument("--profile-nq", type=int, default=8192)
    ap.add_argument("--profile-ls", type=int, default=40)
    ap.add_argument("--profile-wpb", type=int, default=4,
                    help="warps per block of the profiled batched launch")
    ap.add_argument("--workload", default="vamana",
                    choices=["vamana", "hcnng", "nnd", "hnsw", "mixed", "mixed_hnsw", "serving",
                             "serving_hnsw", "c4", "build", "codes", "gather", "sweep"],
                    help="vamana (default, the headline): plain vs batched at recall 0.90; "
                         "hcnng / nnd: the same on the other flat graphs; hnsw: HNSW search; "
                         "mixed / mixed_hnsw: 100k queries of uneven Ls and k in one launch "
                         "on the Vamana graph / the HNSW model; serving / "
                         "serving_hnsw: Poisson bursts through the request loop on the Vamana "
                         "graph / the HNSW model; c4: 10M uint8 d=128 Vamana, 100k queries, "
                         "Ls 20/50/100/200; build: GPU vs CPU Vamana, HNSW and HCNNG "
                         "construction on the 1M base; codes: 4-bit code rows + exact re-rank "
                         "vs vector rows, plain kernel, 1M Vamana; sweep: every family at "
                         "every sweep beam, plain and batched, against the oracle")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.prepare:
        prepare_data(args)
        return
    if args.profile:
        if args.workload == "hnsw":
            run_profile_hnsw(args, local)
        else:
            run_profile(args, local)
        return
    if args.workload in ("hnsw", "mixed", "mixed_hnsw", "serving", "serving_hnsw", "c4",
                         "build", "codes", "gather", "sweep") and args.impl == "ours":
        {"hnsw": run_hnsw, "mixed": run_mixed, "mixed_hnsw": lambda a, lo: run_mixed(a, lo, "hnsw"),
         "serving": run_serving,
         "serving_hnsw": lambda a, lo: run_serving(a, lo, "hnsw"), "c4": run_c4,
         "build": run_build, "codes": run_codes, "gather": run_gather,
         "sweep": run_sweep}[args.workload](args, local)
        return
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=1800),
                                device_id=dev)
        barrier = lambda: dist.barrier()  # noqa: E731
    else:
        barrier = lambda: None  # noqa: E731

    pgb = ge.load_package()
    from parlayann_gpu_busqueda_b200.synthetic import LS_SWEEP
    t0 = time.time()
    base, queries, graph = load_workload(pgb, rank, barrier, args.workload)
    gt_ids, gt_d = ground_truth(base, queries, rank, local)
    index = pgb.Index.flat(base, graph, device=local)
    log(f"rank {rank}: setup {time.time() - t0:.1f} s, index {index.info.device_bytes / 2**20:.0f} MiB")
    q_dev = torch.from_numpy(queries.view(np.uint8)).to(dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    # ---- operating point: smallest sweep beam with recall@10 >= 0.90 ---------------
    # (the first PARITY_SAMPLE rows of every swept beam are kept for the oracle check)
    sweep, Ls, swept = [], None, {}
    for ls in LS_SWEEP:
        s = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=ls))
        ids, dists, st = s.search_device(q_dev, sp)
        torch.cuda.synchronize(dev)
        ids_h = ids.cpu().numpy().view(np.uint32)
        rec = pgb.recall(gt_ids, gt_d, ids_h, K)
        sweep.append([ls, round(rec, 5)])
        swept[ls] = (ids_h[:PARITY_SAMPLE], dists.cpu().numpy()[:PARITY_SAMPLE],
                     st.cpu().numpy()[:PARITY_SAMPLE])
        s.liberar()
        if rec >= TARGET_RECALL and Ls is None:
            Ls = ls
        if Ls is not None and ls >= 2 * Ls:
            break
    if Ls is None:
        Ls = LS_SWEEP[-1]
    recall_at = dict((a, b) for a, b in sweep)[Ls]

    # L2 flush between timed steps (a write larger than the 126 MB L2)
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)

    launches = [0]  # search kernels launched inside the timed steps (the library's counter)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev = []
        c0 = pgb.search_launches()
        for _ in range(steps):
            flush.fill_(1)
            barrier()
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize(dev)
            barrier()
            ev.append(a.elapsed_time(b))
        launches[0] += pgb.search_launches() - c0
        return ev

    # ---- plain warp-per-query kernel (the drop-in) ----------------------------------
    plain = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=Ls))
    p_ids = torch.empty((N_QUERIES, K), dtype=torch.int32, device=dev)
    p_d = torch.empty_like(p_ids)
    p_st = torch.empty((N_QUERIES, 4), dtype=torch.int32, device=dev)
    run_plain = lambda: plain.lanzar(q_dev, p_ids, p_d, p_st, sp)  # noqa: E731

    # ---- batched persistent kernel: tuned, CUDA-graph captured -----------------------
    batch = pgb.Batch(index, N_QUERIES, max_beam=Ls, max_k=K)
    batch.plan(np.full(N_QUERIES, Ls, np.uint32), np.full(N_QUERIES, K, np.uint32))
    b_ids, b_d, b_st = batch.outputs(dev)
    tuned = batch.tune(q_dev, b_ids, b_d, b_st)
    batch.capture(q_dev, b_ids, b_d, b_st)
    run_batched = lambda: batch.replay(sp)  # noqa: E731

    clk = ClockSampler(local).__enter__()
    time.sleep(0.6)  # let the sampler come up before the timed region
    t_plain = timed(run_plain, args.steps, args.warmup)
    t_batch = timed(run_batched, args.steps, args.warmup)
    identical = bool(torch.equal(p_ids, b_ids) and torch.equal(p_d, b_d))

    # ---- end to end through the public host API (pinned host buffers) ---------------
    # the batched form's host entry point: query upload, one launch, result download
    q_host = torch.from_numpy(queries.view(np.uint8)).pin_memory()
    e_ids = torch.empty((N_QUERIES, K), dtype=torch.int32).pin_memory()
    e_d = torch.empty((N_QUERIES, K), dtype=torch.int32).pin_memory()
    lib = pgb._native.lib

    def run_e2e():
        pgb._native.check(lib.pgb_batch_search_host(batch._h, q_host.data_ptr(), queries.shape[1],
                                                    e_ids.data_ptr(), e_d.data_ptr(), None))

    for _ in range(args.warmup):
        run_e2e()
    e2e_t = []
    c0 = pgb.search_launches()
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize(dev)
        barrier()
        t = time.perf_counter()
        run_e2e()
        e2e_t.append(time.perf_counter() - t)
        barrier()
    launches[0] += pgb.search_launches() - c0
    clk.__exit__(None, None, None)
    clocks = clk.summary()
    e2e_ok = bool(np.array_equal(e_ids.numpy(), p_ids.cpu().numpy()))

    # ---- max over ranks ---------------------------------------------------------------
    tp_ms, tb_ms, te_s = (max_over_ranks(sum(xs), dev, world) for xs in (t_plain, t_batch, e2e_t))
    qps_plain = whole_job_rate(N_QUERIES, world, args.steps, tp_ms / 1e3)
    qps_batch = whole_job_rate(N_QUERIES, world, args.steps, tb_ms / 1e3)
    qps_e2e = whole_job_rate(N_QUERIES, world, args.steps, te_s)

    # ---- roofline of the plain kernel: algorithmic gather bytes per launch ----------
    st = p_st.cpu().numpy()
    G = int(index.info.max_degree)
    gs = (G + 31) // 32 * 32
    bytes_launch = float(128 * st[:, 0].astype(np.int64).sum() + 4 * gs * st[:, 1].astype(np.int64).sum())
    # the headline value is the batched kernel's: its launches carry the same per-query
    # work (identical neighbours, so identical comps / expansions)
    avg_batch_s = (sum(t_batch) / len(t_batch)) / 1e3
    avg_plain_s = (sum(t_plain) / len(t_plain)) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = bytes_launch / avg_batch_s / 1e9
    # empirical ceiling: random rows of this base gathered by the search's row code alone
    ceiling, _ = gather_rate(pgb, torch, dev, index, q_dev[0], 4, 20_000_000, 5, 2, flush)
    traffic = None
    tp = os.path.join(ROOT, "profiles", "flat_batched_c2_traffic.json")
    if os.path.exists(tp):
        tr = json.load(open(tp))
        if tr.get("Ls") == Ls and tr.get("nq") == N_QUERIES:
            traffic = tr.get("dram_bytes_per_launch")

    cpu_baseline = None
    if rank == 0 and not args.no_cpu_baseline:
        oracle = ge.load_oracle()
        sample = 8192
        qs = np.ascontiguousarray(queries[:sample])
        threads = os.cpu_count() or 1
        # the reference's protocol: one warm-up, then the best of 5 (comparacion1.cu:76-101)
        oracle.flat_search(base, graph.degrees, graph.edges, qs, K, Ls, threads=threads)
        ts = []
        for _ in range(5):
            t = time.perf_counter()
            o = oracle.flat_search(base, graph.degrees, graph.edges, qs, K, Ls, threads=threads)
            ts.append(time.perf_counter() - t)
        ps = p_st[:sample].cpu().numpy()
        assert (np.array_equal(o[0], p_ids[:sample].cpu().numpy().view(np.uint32)) and
                np.array_equal(o[1], p_d[:sample].cpu().numpy()) and
                np.array_equal(o[2], ps[:, 0]) and np.array_equal(o[3], ps[:, 1]) and
                np.array_equal(o[4], ps[:, 2])), \
            "CUDA result (ids, distances, counts or flags) differs from the CPU restatement"
        # the same restatement on one thread, on the first 1,024 of the sample
        q1 = np.ascontiguousarray(queries[:1024])
        t = time.perf_counter()
        oracle.flat_search(base, graph.degrees, graph.edges, q1, K, Ls, threads=1)
        one = len(q1) / (time.perf_counter() - t)
        cpu_baseline = {"value": sample / min(ts), "unit": "queries/s", "cores": threads,
                        "kind": "port",
                        "sample": f"first {sample} of {N_QUERIES} queries at Ls={Ls}, best of 5",
                        "one_thread_qps": one, "cpu_model": cpu_model()}

    # ---- beyond the headline (one GPU): oracle parity of every graph family at full size,
    # their QPS and gather roofline, and the serving loop's latency ------------------------
    extras = None
    if rank == 0 and world == 1 and not args.no_extras:
        oracle = ge.load_oracle()
        extras = run_extras(args, pgb, torch, dev, local, base, queries, graph, gt_ids, gt_d,
                            oracle, flush, Ls, swept)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": qps_batch,
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": tb_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int8",
            "data": "synthetic",
            "config": {
                "workload": "1M int8 d=100 Gaussian mixture (1024 centres, sigma 10, 30% zeros), "
                            f"{GRAPHS[args.workload][1]}, 29316 queries per GPU, k=10",
                "Ls": Ls, "recall_at_10": recall_at, "sweep_recall": sweep,
                "parallelism": f"queries sharded, index replicated x{world}",
                "l2": "flushed (512 MiB write) before every timed step; index 384 MB > L2",
                "plain_qps": qps_plain, "batched_qps": qps_batch,
                "batched_over_plain": qps_batch / qps_plain,
                "batched_config": tuned, "identical_neighbours": identical,
            },
            "e2e": {"value": qps_e2e, "unit": "queries/s", "api": "pgb_batch_search_host",
                    "h2d_bytes_per_step": int(queries.nbytes),
                    "d2h_bytes_per_step": int(2 * 4 * N_QUERIES * K),
                    "transfer": "pinned host buffers: the launch reads the queries from and "
                                "writes ids / dists to host memory over the bus",
                    "identical_neighbours": e2e_ok},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "kernel": "flat_batched_kernel", "bytes_per_launch": bytes_launch,
                         "avg_launch_ms": avg_batch_s * 1e3,
                         "plain_frac": bytes_launch / avg_plain_s / 1e9 / peak,
                         "gather_ceiling_gbs": ceiling,
                         "frac_of_gather_ceiling": achieved / ceiling,
                         "comps_per_query": float(st[:, 0].mean()),
                         "expansions_per_query": float(st[:, 1].mean())},
            "cpu_baseline": cpu_baseline,
            "clocks": clocks,
            # counted by the library: search kernels launched in the timed steps of the
            # plain, batched (graph replays) and end-to-end arms
            "gpu_launches": int(launches[0]),
        }
        if extras:
            line["config"]["identical_to_oracle"] = extras["identical_to_oracle"]
            line["families"] = extras["families"]
            line["mixed"] = extras["mixed"]
            line["serving"] = extras["serving"]
        print(json.dumps(line), flush=True)
    plain.liberar()
    batch.close()
    index.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# search kernels the library launched inside _timed_events' timed steps, for gpu_launches
_TIMED_LAUNCHES = [0]


def _timed_events(torch, stream, fn, steps, warmup, flush=None):
    pgb = ge.load_package()
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    out = []
    c0 = pgb.search_launches()
    for _ in range(steps):
        if flush is not None:
            flush.fill_(1)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    _TIMED_LAUNCHES[0] += pgb.search_launches() - c0
    return out


def run_hnsw(args, local):
    """HNSW (M=32, efConstruction=128) on the 1M workload: QPS at recall@10 >= 0.90."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    from parlayann_gpu_busqueda_b200.synthetic import LAW_C2, LS_SWEEP
    base, h = load_hnsw(pgb)
    queries = LAW_C2.sample(N_QUERIES, 0, 1)
    gt_ids, gt_d = ground_truth(base, queries, 0, local)
    index = pgb.Index.hnsw(base, h, device=local)
    q = torch.from_numpy(queries.view(np.uint8)).to(dev)
    stream = torch.cuda.current_stream(dev)
    sweep, Ls = [], None
    for ls in LS_SWEEP:
        s = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=ls))
        ids, _, _ = s.search_device(q, stream.cuda_stream)
        torch.cuda.synchronize()
        rec = pgb.recall(gt_ids, gt_d, ids.cpu().numpy().view(np.uint32), K)
        sweep.append([ls, round(rec, 5)])
        s.liberar()
        if rec >= TARGET_RECALL and Ls is None:
            Ls = ls
        if Ls is not None and ls >= 2 * Ls:
            break
    Ls = Ls or LS_SWEEP[-1]
    s = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=Ls))
    ids = torch.empty((N_QUERIES, K), dtype=torch.int32, device=dev)
    d = torch.empty_like(ids)
    st = torch.empty((N_QUERIES, 4), dtype=torch.int32, device=dev)
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)
    t = _timed_events(torch, stream, lambda: s.lanzar(q, ids, d, st, stream.cuda_stream),
                      args.steps, args.warmup, flush)
    stn = st.cpu().numpy()
    qps = N_QUERIES * len(t) / (sum(t) / 1e3)
    G0 = (int(index.info.max_degree) + 31) // 32 * 32
    bytes_launch = float(128 * stn[:, 0].astype(np.int64).sum() + 4 * G0 * stn[:, 1].astype(np.int64).sum())
    peak, kind = measured_peaks()
    achieved = bytes_launch / (sum(t) / len(t) / 1e3) / 1e9
    print(json.dumps({
        "metric": "QPS @ recall@10=0.90, HNSW search, 1 B200", "value": qps, "unit": "queries/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sum(t) / len(t), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8", "data": "synthetic",
        "config": {"workload": "1M int8 d=100 Gaussian mixture, HNSW M32 efc128, 29316 queries, k=10",
                   "Ls": Ls, "recall_at_10": dict((a, b) for a, b in sweep)[Ls], "sweep_recall": sweep,
                   "l2": "flushed before every timed step",
                   "comps_per_query": float(stn[:, 0].mean()),
                   "expansions_per_query": float(stn[:, 1].mean())},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": kind,
                     "kernel": "hnsw_kernel"},
        "gpu_launches": _TIMED_LAUNCHES[0]}), flush=True)


SWEEP_SAMPLE = 256  # queries of each sweep configuration checked against the oracle


def run_sweep(args, local):
    """The reference's full comparison grid (cuda/comparacion1.cu:33-36: every graph family
    at every beam of the sweep) on the 1M workload: Vamana, HCNNG, PyNNDescent and HNSW at
    the 18 beams 10..500, k=10, 29,316 queries. Per configuration: recall@10, plain and
    batched (tuned, captured) QPS with the L2 flushed before every timed step, the batched
    launch's gather roofline, plain and batched identical on every query, and the first
    SWEEP_SAMPLE queries identical to the oracle (ids, distances, counts, flags)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    oracle = ge.load_oracle()
    from parlayann_gpu_busqueda_b200.synthetic import LS_SWEEP
    base = load_base(pgb)
    queries = rank_queries(0)
    gt_ids, gt_d = ground_truth(base, queries, 0, local)
    q_dev = torch.from_numpy(queries.view(np.uint8)).to(dev)
    qs = np.ascontiguousarray(queries[:SWEEP_SAMPLE])
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)
    peak, kind_peak = measured_peaks()
    steps, warmup = max(1, min(args.steps, 5)), max(3, min(args.warmup, 3))
    t_start = time.time()
    table = {}
    for kind in ("vamana", "hcnng", "nnd", "hnsw"):
        if kind == "hnsw":
            _, fg = load_hnsw(pgb)
            index = pgb.Index.hnsw(base, fg, device=local)
        else:
            _, _, fg = load_workload(pgb, 0, lambda: None, kind)
            index = pgb.Index.flat(base, fg, device=local)
        gsz = (int(index.info.max_degree) + 31) // 32 * 32
        rows = []
        for ls in LS_SWEEP:
            plain = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=ls))
            p_ids = torch.empty((N_QUERIES, K), dtype=torch.int32, device=dev)
            p_d = torch.empty_like(p_ids)
            p_st = torch.empty((N_QUERIES, 4), dtype=torch.int32, device=dev)
            tp = _timed_events(torch, stream, lambda: plain.lanzar(q_dev, p_ids, p_d, p_st, sp),
                               steps, warmup, flush)
            b = pgb.Batch(index, N_QUERIES, max_beam=ls, max_k=K)
            b.plan(np.full(N_QUERIES, ls, np.uint32), np.full(N_QUERIES, K, np.uint32))
            bi, bd, bs = b.outputs(dev)
            b.tune(q_dev, bi, bd, bs)
            b.capture(q_dev, bi, bd, bs)
            tb = _timed_events(torch, stream, lambda: b.replay(sp), steps, warmup, flush)
            torch.cuda.synchronize(dev)
            ids_h = p_ids.cpu().numpy().view(np.uint32)
            stn = p_st.cpu().numpy()
            o = (oracle.hnsw_search(base, fg, qs, K, ls) if kind == "hnsw"
                 else oracle.flat_search(base, fg.degrees, fg.edges, qs, K, ls))
            same_oracle = bool(np.array_equal(ids_h[:SWEEP_SAMPLE], o[0]) and
                               np.array_equal(p_d.cpu().numpy()[:SWEEP_SAMPLE], o[1]) and
                               all(np.array_equal(stn[:SWEEP_SAMPLE, c], o[2 + c]) for c in range(3)))
            same_forms = bool(torch.equal(p_ids, bi) and torch.equal(p_d, bd) and
                              torch.equal(p_st[:, :3], bs[:, :3]))
            mp, mb = sum(tp) / len(tp) / 1e3, sum(tb) / len(tb) / 1e3
            bytes_launch = float(128 * stn[:, 0].astype(np.int64).sum() +
                                 4 * gsz * stn[:, 1].astype(np.int64).sum())
            rows.append({"Ls": ls, "recall_at_10": round(pgb.recall(gt_ids, gt_d, ids_h, K), 5),
                         "plain_qps": N_QUERIES / mp, "batched_qps": N_QUERIES / mb,
                         "batched_over_plain": mp / mb, "frac": bytes_launch / mb / 1e9 / peak,
                         "comps_per_query": float(stn[:, 0].mean()),
                         "expansions_per_query": float(stn[:, 1].mean()),
                         "identical_plain_batched": same_forms,
                         "identical_to_oracle": same_oracle})
            log(kind, rows[-1])
            plain.liberar()
            b.close()
        table[kind] = rows
        index.close()
    print(json.dumps({
        "metric": "QPS and recall@10 over the beam sweep, plain and batched, 1 B200",
        "unit": "queries/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "data": "synthetic", "dtype": "int8",
        "config": {"workload": "1M int8 d=100 Gaussian mixture, 29316 queries, k=10; Vamana R64 "
                               "L128, HCNNG 30x1000 MST3, PyNNDescent K40, HNSW M32 efc128",
                   "beams": LS_SWEEP, "l2": "flushed before every timed step",
                   "oracle_sample": SWEEP_SAMPLE, "peak_gbs": peak, "peak_source": kind_peak},
        "configurations": sum(len(v) for v in table.values()),
        "all_identical_to_oracle": all(r["identical_to_oracle"] for v in table.values() for r in v),
        "all_identical_plain_batched": all(r["identical_plain_batched"] for v in table.values()
                                           for r in v),
        "seconds": round(time.time() - t_start, 1), "table": table,
        "gpu_launches": _TIMED_LAUNCHES[0]}), flush=True)


def run_codes(args, local):
    """Compressed rows on the 1M Vamana workload: the plain kernel over 4-bit code rows
    (64 bytes per point; the 64 MB of codes fit in L2) with an exact re-rank of the whole
    final frontier (rerank = Ls), against the plain kernel over the 128-byte vector rows,
    each at its smallest sweep beam reaching recall@10 >= 0.90."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    from parlayann_gpu_busqueda_b200.synthetic import LS_SWEEP
    base, queries, graph = load_workload(pgb, 0, lambda: None)
    gt_ids, gt_d = ground_truth(base, queries, 0, local)
    index = pgb.Index.flat(base, graph, device=local)
    torch.cuda.synchronize()
    t0 = time.time()
    index.compress()
    compress_s = time.time() - t0
    step, off, _ = index.codes(rows=False)
    q = torch.from_numpy(queries.view(np.uint8)).to(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)
    gs = (int(index.info.max_degree) + 31) // 32 * 32
    peak, kind = measured_peaks()
    out = {}
    for name, rr in (("vector_rows", False), ("code_rows", True)):
        sweep, Ls = [], None
        for ls in LS_SWEEP:
            s = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=ls), rerank=ls if rr else 0)
            ids, _, _ = s.search_device(q, stream.cuda_stream)
            torch.cuda.synchronize()
            rec = pgb.recall(gt_ids, gt_d, ids.cpu().numpy().view(np.uint32), K)
            sweep.append([ls, round(rec, 5)])
            s.liberar()
            if rec >= TARGET_RECALL and Ls is None:
                Ls = ls
            if Ls is not None and ls >= 2 * Ls:
                break
        Ls = Ls or LS_SWEEP[-1]
        s = pgb.Searcher(index, N_QUERIES, pgb.QueryParams(k=K, beam_size=Ls), rerank=Ls if rr else 0)
        ids = torch.empty((N_QUERIES, K), dtype=torch.int32, device=dev)
        d = torch.empty_like(ids)
        st = torch.empty((N_QUERIES, 4), dtype=torch.int32, device=dev)
        # without an L2 window, then with one over this format's rows and over the graph
        # (the window's persisting lines survive the flush: that is what it is for)
        for window in (None, "codes" if rr else "rows", "graph"):
            wb, hr = index.set_l2_window(window)
            t = _timed_events(torch, stream, lambda: s.lanzar(q, ids, d, st, stream.cuda_stream),
                              args.steps, args.warmup, flush)
            stn = st.cpu().numpy().astype(np.int64)
            ms = sum(t) / len(t)
            row_b = 64 if rr else 128
            # gathered rows + adjacency rows (+ the re-rank's vector rows)
            bytes_launch = float(row_b * stn[:, 0].sum() + 4 * gs * stn[:, 1].sum()
                                 + (128 * Ls * N_QUERIES if rr else 0))
            achieved = bytes_launch / (ms / 1e3) / 1e9
            key = name if window is None else f"{name}_l2_window_{window}"
            out[key] = {"Ls": Ls, "rerank": Ls if rr else None, "qps": N_QUERIES / (ms / 1e3),
                        "ms_per_step": ms, "recall_at_10": dict((a, b) for a, b in sweep)[Ls],
                        "comps_per_query": float(stn[:, 0].mean()),
                        "expansions_per_query": float(stn[:, 1].mean()),
                        "algorithmic_gb_per_s": achieved, "frac_of_hbm_peak": achieved / peak}
            if window is None:
                out[key]["sweep_recall"] = sweep
            else:
                out[key]["l2_window"] = {"region": window, "bytes": wb, "hit_ratio": hr}
        index.set_l2_window(None)
        s.liberar()
    c, v = out["code_rows"], out["vector_rows"]
    print(json.dumps({
        "metric": "QPS @ recall@10=0.90, plain kernel over 4-bit code rows + exact re-rank, 1 B200",
        "value": c["qps"], "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": c["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8 (4-bit codes)", "data": "synthetic",
        "config": {"workload": "1M int8 d=100 Gaussian mixture, Vamana R64 L128 alpha1.2, "
                               "29316 queries, k=10",
                   "code_step": step, "compress_s": compress_s,
                   "l2": "flushed (512 MiB write) before every timed step",
                   "code_rows": c, "vector_rows": v,
                   "with_l2_window": {key: val for key, val in out.items() if "l2_window" in key},
                   "codes_over_vectors": c["qps"] / v["qps"]},
        "roofline": {"bound": "hbm", "achieved": c["algorithmic_gb_per_s"], "peak": peak,
                     "unit": "GB/s", "frac": c["frac_of_hbm_peak"], "traffic": None,
                     "peak_source": kind, "kernel": "flat_plain_kernel (code rows) + rerank_kernel"},
        "gpu_launches": _TIMED_LAUNCHES[0]}), flush=True)


def run_build(args, local):
    """Vamana construction on the 1M int8 d=100 base (R=64, L=128, alpha=1.2, seed 0): the
    GPU builder's wall time against the CPU builder on all host cores, and the two graphs
    compared entry by entry."""
    import torch
    torch.cuda.set_device(local)
    pgb = ge.load_package()
    base = load_base(pgb)
    times = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        g = pgb.build_vamana_gpu(base, R=R, L=L_BUILD, alpha=ALPHA, seed=0, device=local)
        times.append(time.perf_counter() - t)
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    c = pgb.build_vamana(base, R=R, L=L_BUILD, alpha=ALPHA, seed=0)
    t_cpu = time.perf_counter() - t
    identical = bool(np.array_equal(g.degrees, c.degrees) and np.array_equal(g.edges, c.edges))
    t_gpu = min(times)
    # HNSW M=32 efC=128 on the same base: GPU and CPU model files compared byte for byte
    hp_gpu = os.path.join(data_dir(), "build_gpu.hnsw")
    hp_cpu = os.path.join(data_dir(), "build_cpu.hnsw")
    torch.cuda.synchronize()
    t = time.perf_counter()
    pgb.build_hnsw_gpu(base, hp_gpu, M=32, ef_construction=128, ml=0.36, alpha=0.83, seed=0, device=local)
    h_gpu = time.perf_counter() - t
    t = time.perf_counter()
    pgb.build_hnsw(base, hp_cpu, M=32, ef_construction=128, ml=0.36, alpha=0.83, seed=0)
    h_cpu = time.perf_counter() - t
    with open(hp_gpu, "rb") as fa, open(hp_cpu, "rb") as fb:
        h_same = fa.read() == fb.read()
    for p in (hp_gpu, hp_cpu):
        os.unlink(p)
    # HCNNG 30 trees, leaves of 1,000, MST degree 3
    torch.cuda.synchronize()
    t = time.perf_counter()
    hg = pgb.build_hcnng_gpu(base, trees=30, leaf=1000, mst_deg=3, seed=0, device=local)
    c_gpu = time.perf_counter() - t
    t = time.perf_counter()
    hc = pgb.build_hcnng(base, trees=30, leaf=1000, mst_deg=3, seed=0)
    c_cpu = time.perf_counter() - t
    c_same = bool(np.array_equal(hg.degrees, hc.degrees) and np.array_equal(hg.edges, hc.edges))
    print(json.dumps({
        "metric": "Vamana build time, 1M int8 d=100, R=64 L=128 alpha=1.2, GPU vs CPU builder",
        "value": t_gpu, "unit": "s", "n_gpus": 1, "steps": len(times), "warmup": 0,
        "ms_per_step": t_gpu * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8", "data": "synthetic",
        "config": {"workload": "1M int8 d=100 Gaussian mixture, Vamana R64 L128 alpha1.2 seed 0, "
                               "prefix-doubling batches to 2% of n", "all_runs_s": times,
                   "identical_to_cpu_builder": identical,
                   "mean_degree": float(g.degrees.mean()),
                   "hnsw_M32_efc128": {"gpu_s": h_gpu, "cpu_s": h_cpu, "cpu_cores": os.cpu_count(),
                                       "file_identical_to_cpu_builder": bool(h_same)},
                   "hcnng_T30_leaf1000_mst3": {"gpu_s": c_gpu, "cpu_s": c_cpu, "cpu_cores": os.cpu_count(),
                                               "identical_to_cpu_builder": c_same,
                                               "mean_degree": float(hg.degrees.mean())},
                   "timing": "wall clock around the host call (upload, build, download)"},
        "cpu_baseline": {"value": t_cpu, "unit": "s", "cores": threads, "kind": "port",
                         "sample": "the same full 1M build by the CPU builder"},
        "gpu_launches": None}), flush=True)


C4_N, C4_NQ, C4_LS = 10_000_000, 100_000, (20, 50, 100, 200)


def load_c4(pgb):
    """10M uint8 d=128 base (4,096-centre law, 40 % zeros) and its Vamana R=64 L=128
    alpha=1.2 graph, generated and built once, cached on disk."""
    from parlayann_gpu_busqueda_b200.synthetic import LAW_C4
    base_p = os.path.join(data_dir(), "c4_base.u8bin")
    graph_p = os.path.join(data_dir(), "c4_vamana_R64_L128_a1.2.graph")
    if not os.path.exists(base_p):
        t = time.time()
        base = LAW_C4.sample(C4_N, 0, 0)
        pgb.write_vectors(base_p + ".tmp", base)
        os.replace(base_p + ".tmp", base_p)
        log(f"generated C4 base in {time.time() - t:.1f} s")
    base = pgb.read_vectors(base_p, np.uint8)
    if not os.path.exists(graph_p):
        t = time.time()
        g = pgb.build_vamana_gpu(base, R=R, L=L_BUILD, alpha=ALPHA, seed=0)
        pgb.write_graph(graph_p + ".tmp", g)
        os.replace(graph_p + ".tmp", graph_p)
        log(f"built C4 Vamana 10M on the GPU in {time.time() - t:.1f} s")
    return base, pgb.read_graph(graph_p), LAW_C4.sample(C4_NQ, 0, 1)


def run_c4(args, local):
    """Scale: 10M uint8 d=128 rows (1.28 GB) + Vamana R=64 (2.56 GB) resident in HBM,
    100,000 queries, k=10; plain and batched QPS, recall@10 and gather roofline at
    Ls 20 / 50 / 100 / 200."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    base, graph, queries = load_c4(pgb)
    gt_p = os.path.join(data_dir(), "c4_gt100.bin")
    from parlayann_gpu_busqueda_b200 import formats, groundtruth
    if os.path.exists(gt_p):
        gt_ids, gt_d = formats.read_gt(gt_p)
    else:
        t = time.time()
        gt_ids, gt_d = groundtruth.knn_gpu(base, queries, 100, local)
        formats.write_gt(gt_p + ".tmp", gt_ids, gt_d)
        os.replace(gt_p + ".tmp", gt_p)
        log(f"C4 ground truth in {time.time() - t:.1f} s")
    index = pgb.Index.flat(base, graph, device=local)
    q = torch.from_numpy(queries).to(dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)
    peak, kind = measured_peaks()
    gs = (int(index.info.max_degree) + 31) // 32 * 32
    oracle = ge.load_oracle()
    c4_sample = 512  # queries of the oracle check at every beam
    rows = []
    for ls in C4_LS:
        s = pgb.Searcher(index, C4_NQ, pgb.QueryParams(k=K, beam_size=ls))
        ids = torch.empty((C4_NQ, K), dtype=torch.int32, device=dev)
        d = torch.empty_like(ids)
        st = torch.empty((C4_NQ, 4), dtype=torch.int32, device=dev)
        tp = _timed_events(torch, stream, lambda: s.lanzar(q, ids, d, st, sp), args.steps,
                           args.warmup, flush)
        b = pgb.Batch(index, C4_NQ, max_beam=ls, max_k=K)
        b.plan(np.full(C4_NQ, ls, np.uint32), np.full(C4_NQ, K, np.uint32))
        bi, bd, bs = b.outputs(dev)
        b.tune(q, bi, bd, bs)
        b.capture(q, bi, bd, bs)
        tb = _timed_events(torch, stream, lambda: b.replay(sp), args.steps, args.warmup, flush)
        identical = bool(torch.equal(ids, bi) and torch.equal(d, bd))
        stn = st.cpu().numpy()
        ids_h = ids.cpu().numpy().view(np.uint32)
        rec = pgb.recall(gt_ids, gt_d, ids_h, K)
        o = oracle.flat_search(base, graph.degrees, graph.edges,
                               np.ascontiguousarray(queries[:c4_sample]), K, ls)
        same_oracle = bool(np.array_equal(ids_h[:c4_sample], o[0]) and
                           np.array_equal(d.cpu().numpy()[:c4_sample], o[1]) and
                           np.array_equal(stn[:c4_sample, 0], o[2]) and
                           np.array_equal(stn[:c4_sample, 1], o[3]) and
                           np.array_equal(stn[:c4_sample, 2], o[4]))
        bytes_launch = float(128 * stn[:, 0].astype(np.int64).sum() + 4 * gs * stn[:, 1].astype(np.int64).sum())
        mb = sum(tb) / len(tb) / 1e3
        rows.append({"Ls": ls, "recall_at_10": round(rec, 5),
                     "plain_qps": C4_NQ * len(tp) / (sum(tp) / 1e3),
                     "batched_qps": C4_NQ / mb, "identical_neighbours": identical,
                     "identical_to_oracle": same_oracle, "oracle_sample": c4_sample,
                     "comps_per_query": float(stn[:, 0].mean()),
                     "expansions_per_query": float(stn[:, 1].mean()),
                     "achieved_gbs": bytes_launch / mb / 1e9,
                     "frac": bytes_launch / mb / 1e9 / peak, "batched_config": b.config()})
        log(rows[-1])
        s.liberar()
        b.close()
    # headline row: the smallest beam at recall@10 >= 0.90
    head = next((r for r in rows if r["recall_at_10"] >= TARGET_RECALL), rows[-1])
    print(json.dumps({
        "metric": "QPS at Ls 20/50/100/200, 10M uint8 d=128 Vamana, batched vs plain, 1 B200",
        "value": head["batched_qps"], "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": C4_NQ / head["batched_qps"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "uint8",
        "data": "synthetic",
        "config": {"workload": "10M uint8 d=128 (4,096 centres, 40% zeros), Vamana R64 L128 "
                               "alpha1.2, 100,000 queries, k=10", "headline_Ls": head["Ls"],
                   "index_bytes": int(index.info.device_bytes),
                   "l2": "flushed (512 MiB write) before every timed step; index 3.8 GB > L2",
                   "rows": rows},
        "roofline": {"bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": head["frac"], "traffic": None, "peak_source": kind,
                     "kernel": "flat_batched_kernel"},
        "gpu_launches": _TIMED_LAUNCHES[0]}), flush=True)


MIXED_NQ = 100_000


def mixed_leg(pgb, torch, dev, index, queries, steps):
    """100,000 queries with Ls log-uniform in [10, 500] and k in {10, 50, 100} (seed 0): one
    batched launch (tuned, a CUDA graph) against the plain kernel launched once per distinct
    (Ls, k), the query-index exclusion off in both arms (the plain arm regroups queries).
    Returns the row of the bench line."""
    nq = len(queries)
    rng = np.random.default_rng(0)
    ls = np.rint(np.exp(rng.uniform(np.log(10), np.log(500), nq))).astype(np.uint32)
    ks = rng.choice(np.array([10, 50, 100], np.uint32), nq)
    q = torch.from_numpy(queries.view(np.uint8)).to(dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    b = pgb.Batch(index, nq, max_beam=int(ls.max()), max_k=100, exclude_query_id=False)
    b.plan(ls, ks)
    ids, d, st = b.outputs(dev)
    tuned = b.tune(q, ids, d, st)
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)
    b.capture(q, ids, d, st)
    tb = _timed_events(torch, stream, lambda: b.replay(sp), steps, 2, flush)
    # plain: the drop-in prepares one searcher per distinct (Ls, k) and launches it on
    # that group's queries; preparing and releasing are outside the timed launches
    groups = {}
    for i in range(nq):
        groups.setdefault((int(ls[i]), int(ks[i])), []).append(i)
    got = ids.cpu().numpy().view(np.uint32)
    same, t_plain_ms = True, 0.0
    for (L, k), idx in groups.items():
        idx = np.array(idx)
        qi = torch.from_numpy(queries[idx].view(np.uint8)).to(dev)
        s = pgb.Searcher(index, len(idx), pgb.QueryParams(k=k, beam_size=L,
                                                          exclude_query_id=False))
        oi = torch.empty((len(idx), k), dtype=torch.int32, device=dev)
        od = torch.empty_like(oi)
        t_plain_ms += sum(_timed_events(torch, stream, lambda: s.lanzar(qi, oi, od, None, sp),
                                        1, 1))
        same = same and np.array_equal(oi.cpu().numpy().view(np.uint32), got[idx, :k])
        s.liberar()
    b.close()
    qb = nq * len(tb) / (sum(tb) / 1e3)
    qp = nq / (t_plain_ms / 1e3)
    return {"batched_qps": qb, "plain_qps": qp, "plain_launches_per_step": len(groups),
            "batched_over_plain": qb / qp, "batched_ms": sum(tb) / len(tb),
            "plain_timing": "sum of per-group launch times (events), L2 warm",
            "identical_neighbours": bool(same), "batched_config": tuned,
            "l2": "flushed before every timed batched step"}


def run_mixed(args, local, kind="vamana"):
    """The mixed-beam batch (mixed_leg) on the Vamana graph, or (kind "hnsw") on the HNSW
    model (its beams above 256 use the (epoch, id) filter, whose epochs come from a device
    word, so the graph replays with fresh ones)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pgb = ge.load_package()
    if kind == "hnsw":
        base, h = load_hnsw(pgb)
        queries = rank_queries(0, MIXED_NQ)
        index = pgb.Index.hnsw(base, h, device=local)
    else:
        base, queries, graph = load_workload(pgb, 0, lambda: None, "vamana", MIXED_NQ)
        index = pgb.Index.flat(base, graph, device=local)
    steps = max(3, args.steps // 20)
    row = mixed_leg(pgb, torch, dev, index, queries, steps)
    print(json.dumps({
        "metric": "QPS, 100k queries of uneven Ls and k, batched (one launch) vs plain",
        "value": row["batched_qps"], "unit": "queries/s", "n_gpus": 1, "steps": steps, "warmup": 2,
        "ms_per_step": row["batched_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8", "data": "synthetic",
        "config": dict({"workload": "1M int8 d=100 %s, 100000 queries, Ls log-uniform [10,500], "
                                    "k in {10,50,100}" % ("HNSW M32 efc128" if kind == "hnsw"
                                                          else "Vamana R64")}, **row),
        "gpu_launches": _TIMED_LAUNCHES[0]}), flush=True)


def serve_rate(pgb, index, queries, gt_ids, gt_d, rate, seconds, rng):
    """One offered rate through the request loop for `seconds`: Poisson arrival events,
    half single queries and half bursts of 2-256, per-request Ls in {20,50,100,300} and k
    in {10,100}; sustained QPS, the server's p50/p99 submit-to-completion latency, the
    refused fraction and recall@10 of the completed requests."""
    srv = pgb.Server(index, max_beam=300, max_k=100, max_batch=2048, max_inflight=4)
    # arrival events: half single queries, half bursts uniform in 2..256
    mean_burst = 0.5 * 1 + 0.5 * 129
    n_events = max(1, int(rate * seconds / mean_burst))
    gaps = rng.exponential(mean_burst / rate, n_events)
    sizes = np.where(rng.random(n_events) < 0.5, 1, rng.integers(2, 257, n_events))
    t_evt = np.cumsum(gaps)
    # every request's query, beam and k drawn before the clock starts: event e submits
    # rows off[e]:off[e+1] of these arrays (contiguous views, no copies in the loop)
    off = np.concatenate([[0], np.cumsum(sizes)])
    sel_all = rng.integers(0, N_QUERIES, int(off[-1]))
    q_all = np.ascontiguousarray(queries[sel_all])
    L_all = rng.choice(np.array([20, 50, 100, 300], np.uint32), int(off[-1]))
    k_all = rng.choice(np.array([10, 100], np.uint32), int(off[-1]))
    # outstanding tickets in submission order; each pass polls the oldest POLL_HEAD of
    # them (batches complete roughly in launch order), so the client's own work stays
    # bounded when the server is saturated and the pool holds thousands of requests
    out_t, out_q = np.empty(0, np.uint64), np.empty(0, np.int64)
    new_t, new_q = [], []
    issued, done_q, recalls = 0, 0, []
    t0 = time.perf_counter()
    ev = 0
    while ev < n_events or len(out_t) or new_t:
        now = time.perf_counter() - t0
        while ev < n_events and t_evt[ev] <= now:
            a, b = int(off[ev]), int(off[ev + 1])
            t = srv.submit_many(q_all[a:b], L_all[a:b], k_all[a:b])
            if len(t):
                new_t.append(t)
                new_q.append(sel_all[a:a + len(t)])
            issued += len(t)
            ev += 1
        if new_t:
            out_t = np.concatenate([out_t] + new_t)
            out_q = np.concatenate([out_q] + new_q)
            new_t, new_q = [], []
        if len(out_t):
            head_t, head_q = out_t[:POLL_HEAD], out_q[:POLL_HEAD]
            done, oi, _, _ = srv.poll_many(head_t)
            if done.any():
                rec = pgb.recall(gt_ids[head_q[done]], gt_d[head_q[done]], oi[done][:, :K], K)
                recalls.append((rec, int(done.sum())))
                done_q += int(done.sum())
                out_t = np.concatenate([head_t[~done], out_t[POLL_HEAD:]])
                out_q = np.concatenate([head_q[~done], out_q[POLL_HEAD:]])
        if now > 20 * seconds:
            break
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    rec = sum(r * n for r, n in recalls) / max(1, sum(n for _, n in recalls))
    return {"offered_qps": rate, "sustained_qps": done_q / wall, "p50_us": st["p50_us"],
            "p99_us": st["p99_us"], "rejected": st["rejected"],
            "refused_frac": st["rejected"] / max(1, st["rejected"] + issued),
            "launches": st["launches"], "mean_batch": st["mean_batch"], "recall_at_10": rec}


def run_serving(args, local, kind="vamana"):
    """Poisson arrivals of single queries and bursts (1-256) at offered rates from 10k to
    2M QPS through the request loop; per-request Ls in {20,50,100,300}, k in {10,100}; on
    the Vamana graph or (kind "hnsw") the HNSW model of the same base."""
    import torch
    torch.cuda.set_device(local)
    pgb = ge.load_package()
    if kind == "hnsw":
        base, h = load_hnsw(pgb)
        queries = rank_queries(0)
        index = pgb.Index.hnsw(base, h, device=local)
    else:
        base, queries, graph = load_workload(pgb, 0, lambda: None, "vamana")
        index = pgb.Index.flat(base, graph, device=local)
    gt_ids, gt_d = ground_truth(base, queries, 0, local)
    rng = np.random.default_rng(1)
    rates = [int(r) for r in os.environ.get("PGB_SERVE_RATES",
                                            "10000,100000,500000,1000000,2000000").split(",")]
    seconds = float(os.environ.get("PGB_SERVE_SECONDS", "1.5"))
    rows = []
    for rate in rates:
        rows.append(serve_rate(pgb, index, queries, gt_ids, gt_d, rate, seconds, rng))
        log(rows[-1])
    best = max(rows, key=lambda r: r["sustained_qps"])
    print(json.dumps({
        "metric": "serving p50/p99 latency and sustained QPS, Poisson bursts, 1 B200",
        "value": best["sustained_qps"], "unit": "queries/s", "n_gpus": 1, "steps": len(rows),
        "warmup": 0, "ms_per_step": seconds * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8", "data": "synthetic",
        "config": {"workload": "1M int8 d=100 %s, per-request Ls in {20,50,100,300}, k in "
                               "{10,100}, bursts of 1-256" % ("HNSW M32 efc128" if kind == "hnsw"
                                                               else "Vamana R64"), "rates": rows},
        "gpu_launches": int(sum(r["launches"] for r in rows))}), flush=True)


if __name__ == "__main__":
    main()
