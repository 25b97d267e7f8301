"""Serving loop: every request gets the same neighbours alone and in a concurrent mix
(and the oracle's answer for its own Ls and k); a full pool refuses admission."""
import threading

import numpy as np
import pytest

from conftest import assert_same

pytestmark = pytest.mark.gpu


def oracle_one(oracle, base, g, q, Ls, k):
    o = oracle.flat_search(base, g.degrees, g.edges, q[None], k, Ls, exclude_query_id=False)
    return o[0][0], o[1][0]


def drain(server, tickets, ks):
    out = {}
    for i, t in tickets.items():
        r = None
        while r is None:
            r = server.poll(t, ks[i], timeout_us=200_000)
        out[i] = r
    return out


def test_alone_and_in_the_mix_are_identical(pgb, oracle, golden, gpu):
    base, queries = golden.vectors_for("vamana")
    g = golden.graphs["vamana"]
    index = pgb.Index.flat(base, g)
    rng = np.random.default_rng(5)
    nq = len(queries)
    ls = rng.choice([20, 50, 100, 300], size=nq)
    ks = rng.choice([10, 100], size=nq)
    server = pgb.Server(index, max_beam=300, max_k=100, max_batch=32, max_inflight=3)
    # alone: one request on the GPU at a time
    alone = {}
    for i in range(nq):
        t = server.submit(queries[i], int(ls[i]), int(ks[i]))
        alone[i] = drain(server, {i: t}, ks)[i]
    # in the mix: everything at once, from two submitting threads
    tickets = {}
    lock = threading.Lock()

    def submit_range(lo, hi):
        for i in range(lo, hi):
            t = None
            while t is None:
                t = server.submit(queries[i], int(ls[i]), int(ks[i]))
            with lock:
                tickets[i] = t

    th = [threading.Thread(target=submit_range, args=(0, nq // 2)),
          threading.Thread(target=submit_range, args=(nq // 2, nq))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    mix = drain(server, tickets, ks)
    st = server.stats()
    for i in range(nq):
        assert_same(f"ids q{i}", mix[i][0], alone[i][0])
        assert_same(f"dists q{i}", mix[i][1], alone[i][1])
        oi, od = oracle_one(oracle, base, g, queries[i], int(ls[i]), int(ks[i]))
        assert_same(f"oracle q{i}", alone[i][0], oi)
    assert st["completed"] == 2 * nq and st["p99_us"] >= st["p50_us"] > 0
    assert st["launches"] < 2 * nq  # the mix was batched
    server.close()
    index.close()


def test_full_pool_refuses(pgb, golden, gpu):
    base, queries = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    server = pgb.Server(index, max_beam=40, max_k=10, max_batch=4, max_inflight=1)
    slots = server.stats()["pool_slots"]
    assert slots == 8
    tickets = [server.submit(queries[i], 40, 10) for i in range(slots)]
    assert all(t is not None for t in tickets)
    assert server.submit(queries[0], 40, 10) is None  # busy: admission refused
    for t in tickets:
        r = None
        while r is None:
            r = server.poll(t, 10, timeout_us=100_000)
    assert server.submit(queries[0], 40, 10) is not None  # slots freed
    assert server.stats()["rejected"] == 1
    with pytest.raises(pgb.PgbError):
        server.poll(123456789, 10)
    server.close()


def test_server_rejects_bad_requests(pgb, golden, gpu):
    base, queries = golden.vectors_for("vamana")
    index = pgb.Index.flat(base, golden.graphs["vamana"])
    server = pgb.Server(index, max_beam=40, max_k=10, max_batch=4, max_inflight=1)
    with pytest.raises(pgb.PgbError):
        server.submit(queries[0], 41, 10)
    with pytest.raises(pgb.PgbError):
        server.submit(queries[0], 40, 11)
    server.close()


def test_hnsw_requests_match_oracle_in_the_mix(pgb, oracle, golden, gpu):
    """HNSW serving: a batch runs as one launch with each query at its own (Ls, k), on
    tables prepared for max_beam (300: the global (epoch, id) filter) -- every request
    still gets the oracle's answer for its own Ls and k."""
    base, queries = golden.vectors_for("hnsw")
    h = golden.hnsw["hnsw"]
    index = pgb.Index.hnsw(base, h)
    rng = np.random.default_rng(11)
    nq = len(queries)
    ls = rng.choice([10, 50, 100, 300], size=nq)
    ks = rng.choice([10, 20], size=nq)
    server = pgb.Server(index, max_beam=300, max_k=20, max_batch=48, max_inflight=2)
    tickets = {}
    for i in range(nq):
        t = None
        while t is None:
            t = server.submit(queries[i], int(ls[i]), int(ks[i]))
        tickets[i] = t
    got = drain(server, tickets, ks)
    st = server.stats()
    for i in range(nq):
        oi, od, *_ = oracle.hnsw_search(base, h, queries[i][None], int(ks[i]), int(ls[i]))
        assert_same(f"ids q{i}", got[i][0], oi[0])
        assert_same(f"dists q{i}", got[i][1], od[0])
    assert st["completed"] == nq and st["launches"] < nq
    server.close()
    index.close()
