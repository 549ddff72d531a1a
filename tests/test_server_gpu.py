"""Serving engine (bw_server_*): continuous batching, admission by device
bytes, resident tables; every result bit-exact against GMP and identical
whether the request ran alone or inside a mix of concurrent requests."""
import threading
import time

import numpy as np
import pytest

import birdwing_b200 as bw
from birdwing_b200 import workloads
from oracle import gmp_ref

pytestmark = pytest.mark.gpu


def rand_words(n, rng):
    return workloads.rand_operand(rng, n)


def make_requests(count, seed, max_bits=1 << 20):
    rng = np.random.default_rng(seed)
    reqs = []
    for la, lb, sq in workloads.serving_sizes(count, seed=seed,
                                              hi_log=max_bits.bit_length() - 1):
        a = rand_words(la, rng)
        reqs.append((a, a if sq else rand_words(lb, rng)))
    return reqs


def test_alone_and_in_the_mix_are_identical():
    reqs = make_requests(300, seed=1)
    with bw.Server() as srv:
        alone = []
        for a, b in reqs:
            out, info = srv.wait(srv.submit(a, b))
            assert info["status"] == 0 and info["group_size"] == 1
            alone.append(out.copy())
        # all at once: they are admitted together and batched
        tickets = [srv.submit(a, b) for a, b in reqs]
        mixed = [srv.wait(t)[0] for t in tickets]
        st = srv.stats()
    assert st["max_group_size"] > 1
    assert st["completed"] == 600 and st["failed"] == 0
    for (a, b), x, y in zip(reqs, alone, mixed):
        assert (x == y).all()
        assert (x == gmp_ref.mul(a, b)).all(), (len(a), len(b))


@pytest.mark.parametrize("K,path", [(2, 32), (3, 64), (3, 32)])
def test_paths_and_prime_counts(K, path):
    reqs = make_requests(120, seed=2 + K + path, max_bits=1 << 18)
    with bw.Server(num_primes=K, path=path) as srv:
        tickets = [srv.submit(a, b) for a, b in reqs]
        outs = [srv.wait(t)[0] for t in tickets]
    for (a, b), o in zip(reqs, outs):
        assert (o == gmp_ref.mul(a, b)).all()


def test_admission_by_device_bytes():
    rng = np.random.default_rng(3)
    budget = 64 << 20
    reqs = [(rand_words(40000, rng), rand_words(30000, rng)) for _ in range(24)]
    with bw.Server(hbm_budget=budget, lanes=4) as srv:
        tickets = [srv.submit(a, b) for a, b in reqs]
        # a request that alone needs more than the budget is rejected up front
        big = rand_words(1 << 21, rng)
        with pytest.raises(bw.BwError) as ei:
            srv.submit(big, big)
        assert ei.value.code == bw._lib.BW_EREJECT
        outs = [srv.wait(t)[0] for t in tickets]
        st = srv.stats()
    assert st["peak_bytes_in_flight"] <= budget
    assert st["rejected"] == 1 and st["completed"] == 24
    for (a, b), o in zip(reqs, outs):
        assert (o == gmp_ref.mul(a, b)).all()


def test_poisson_arrivals_from_threads():
    reqs = make_requests(400, seed=4, max_bits=1 << 22)
    rng = np.random.default_rng(5)
    gaps = rng.exponential(1.0 / 4000.0, size=len(reqs))
    tickets = [None] * len(reqs)
    with bw.Server() as srv:
        srv.prewarm(18)

        def feeder(lo, hi):
            t_next = time.perf_counter()
            for i in range(lo, hi):
                t_next += 2 * gaps[i]
                while time.perf_counter() < t_next:
                    pass
                tickets[i] = srv.submit(*reqs[i])

        th = [threading.Thread(target=feeder, args=(0, 200)),
              threading.Thread(target=feeder, args=(200, 400))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        srv.drain()
        infos = {d["ticket"]: d for d in srv.harvest(1000)}
        st = srv.stats()
    assert len(infos) == len(reqs) and st["queue_depth"] == 0
    for (a, b), t in zip(reqs, tickets):
        d = infos[t]
        assert d["status"] == 0
        assert d["submit_us"] <= d["admit_us"] <= d["launch_us"] <= d["done_us"]
        assert (d["out"] == gmp_ref.mul(a, b)).all()


def test_destroy_with_requests_outstanding():
    reqs = make_requests(200, seed=6)
    srv = bw.Server(max_groups=1, lanes=1)
    for a, b in reqs:
        srv.submit(a, b)
    srv.close()        # waiting ones fail with BW_EBUSY, admitted ones finish
    with bw.Server() as srv2:
        a, b = reqs[0]
        out, _ = srv2.wait(srv2.submit(a, b))
        assert (out == gmp_ref.mul(a, b)).all()


def test_wait_poll_and_errors():
    rng = np.random.default_rng(7)
    with bw.Server() as srv:
        a = rand_words(1000, rng)
        t = srv.submit(a, a)
        out, info = srv.wait(t, timeout_ms=-1)
        assert (out == gmp_ref.mul(a, a)).all()
        with pytest.raises(bw.BwError):
            srv.wait(t, timeout_ms=0)          # released already
        with pytest.raises(bw.BwError):
            srv.submit(a, a, out=np.zeros(10, dtype=np.uint32))
        # many results per call as numpy columns
        ops = [(rand_words(n, rng), rand_words(n // 3 + 1, rng)) for n in (10, 5000, 40000)]
        tickets = [srv.submit(x, y) for x, y in ops]
        srv.drain()
        rec, outs = srv.harvest_arrays()
        assert sorted(rec["ticket"].tolist()) == sorted(tickets)
        assert (rec["status"] == 0).all() and (rec["done_us"] >= rec["submit_us"]).all()
        by_ticket = dict(zip(rec["ticket"].tolist(), outs))
        for t, (x, y) in zip(tickets, ops):
            assert (by_ticket[t] == gmp_ref.mul(x, y)).all()


def test_pinned_buffers_move_by_dma():
    # operands and results in pinned host memory (large ones move by DMA
    # straight to and from the device), mixed with pageable ones in the same
    # groups; squarings included
    import torch

    def pinned(x):
        return torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)

    rng = np.random.default_rng(9)
    reqs = []
    for i, (la, lb) in enumerate([(20000, 17000), (40000, 40000), (3000, 200), (70000, 9000),
                                  (16384, 16384), (50000, 1), (100, 100), (33000, 33000)]):
        a = rand_words(la, rng)
        b = a if i % 4 == 1 else rand_words(lb, rng)
        if i % 2 == 0:
            a = pinned(a)
            b = a if i % 4 == 1 else pinned(b)
        out = np.zeros(len(a) + len(b), dtype=np.uint32)
        if i % 3 != 2:
            out = pinned(out)
        reqs.append((a, b, out))
    with bw.Server() as srv:
        for rep in range(2):
            tickets = [srv.submit(a, b, out=o) for a, b, o in reqs]   # together: batched
            for t in tickets:
                srv.wait(t)
            for a, b, o in reqs:
                assert (o == gmp_ref.mul(a, b)).all(), (rep, len(a), len(b))
                o[:] = 0
