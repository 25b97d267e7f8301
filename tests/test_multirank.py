"""The multi-GPU bench path's host logic on CPU ranks (gloo, world size 2): each rank
searches its own query shard against its own replica of the index (no collective on the
data path), and the whole job's time is the slowest rank's, taken with one MAX
all-reduce that every rank joins."""
import multiprocessing as mp
import os
import socket

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime

    import torch
    import torch.distributed as dist

    import __graft_entry__ as ge
    import bench
    ge.load_package()
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, world, rank)
        q = bench.rank_queries(rank, 64)
        # every rank sees every shard's fingerprint to compare them
        fp = torch.tensor(np.frombuffer(q.tobytes()[:64], np.uint8).astype(np.int64))
        fps = [torch.zeros_like(fp) for _ in range(world)]
        dist.all_gather(fps, fp)
        # rank r "took" 10 + 5 r ms: the job's time is the slowest rank's
        worst = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu", world)
        out.put((rank, q.shape, [f.tolist() for f in fps], worst))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_queries_and_take_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, shape, fps, worst = out.get(timeout=240)
        res[rank] = (shape, fps, worst)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in range(world):
        shape, fps, worst = res[rank]
        assert shape == (64, 100)
        assert fps[0] != fps[1], "two ranks drew the same query shard"
        assert worst == 15.0  # the slower rank's time, on every rank
    assert res[0][1] == res[1][1]


def test_whole_job_rate_counts_every_rank():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    # 2 ranks x 29316 queries x 10 steps over the slowest rank's 0.5 s
    assert bench.whole_job_rate(29316, 2, 10, 0.5) == 2 * 29316 * 10 / 0.5
    assert bench.max_over_ranks(3.5, "cpu", 1) == 3.5
