"""Batched products (bw_batch_*) through the C ABI: bit-exact against GMP and
the oracle, for both kernel forms (one CTA per product, and the 4-step
kernels with a product grid dimension), both prime paths, squarings,
replays of the captured graph, tuning, and the uneven-size mix the batched
benchmark runs."""
import json

import numpy as np
import pytest

import birdwing_b200 as bw
from birdwing_b200 import workloads
from oracle import gmp_ref, oracle

pytestmark = pytest.mark.gpu


def rand_words(n, rng):
    return workloads.rand_operand(rng, n)


def log_n_of(path, la, lb):
    cpw = 2 if path == 32 else 1
    m = (la + lb) * cpw - 1
    return max(4, (m - 1).bit_length())


def default_small(ln):
    """The library's default kernel form: one CTA per product up to 2^12 points."""
    return ln <= 12


def run_batch(items, K=2):
    """items: [(path, a, b)]; returns outputs in order."""
    with bw.Batch(num_primes=K) as bt:
        outs = [bt.add(a, b, path=p) for p, a, b in items]
        bt.run()
        return [o.copy() for o in outs], bt.info()


@pytest.mark.parametrize("K", [2, 3])
def test_mixed_sizes_vs_oracle(K):
    rng = np.random.default_rng(11 + K)
    shapes = [(1, 1), (1, 2), (3, 5), (8, 8), (9, 8), (16, 16), (31, 33), (100, 3),
              (255, 256), (256, 256), (1000, 1), (1023, 1025), (2048, 2048), (3000, 700),
              (4095, 4097), (8192, 8191), (16000, 5000)]
    items = []
    for path in (64, 32):
        for la, lb in shapes:
            if path == 32 and (la + lb) * 2 > (1 << 17):
                continue
            items.append((path, rand_words(la, rng), rand_words(lb, rng)))
    outs, info = run_batch(items, K)
    assert info["products"] == len(items)
    assert info["small_buckets"] >= 1 and info["buckets"] > info["small_buckets"]
    for (p, a, b), got in zip(items, outs):
        if len(a) + len(b) <= 4096:
            want = oracle.multiply(a, b, p, K)
        else:
            want = gmp_ref.mul(a, b)
        assert (got == want).all(), (p, len(a), len(b))


@pytest.mark.parametrize("path", [64, 32])
@pytest.mark.parametrize("small", [True, False])
def test_power_of_two_product_length(path, small):
    # la + lb - 1 coefficients filling the transform exactly: the final carry
    # lands in the word just past the n-th coefficient word
    rng = np.random.default_rng(5)
    cases = [(16, 1), (1 << 12, 1), (1, 1 << 11), (1 << 10, 1 << 10 | 1)]
    if not small:
        cases.append((1 << 16, 1) if path == 64 else (1 << 15, 1))
    items = []
    for la, lb in cases:
        a = np.full(la, 0xFFFFFFFF, dtype=np.uint32)
        b = rand_words(lb, rng)
        items.append((path, a, b))
        items.append((path, rand_words(la, rng), b))
    for p, a, b in items:
        bw.set_tune_entry(p, 2, log_n_of(p, len(a), len(b)), small and
                          log_n_of(p, len(a), len(b)) <= (13 if p == 64 else 14))
    try:
        outs, _ = run_batch(items)
    finally:
        for p, a, b in items:
            ln = log_n_of(p, len(a), len(b))
            bw.set_tune_entry(p, 2, ln, default_small(ln))
    for (p, a, b), got in zip(items, outs):
        assert (got == gmp_ref.mul(a, b)).all(), (p, len(a), len(b))


@pytest.mark.parametrize("small", [True, False])
def test_forms_agree_on_the_same_products(small):
    # the same bucket in both kernel forms gives identical words
    rng = np.random.default_rng(21)
    items = [(64, rand_words(700, rng), rand_words(300, rng)) for _ in range(5)]
    items += [(32, rand_words(600, rng), rand_words(600, rng)) for _ in range(5)]
    keys = {(p, log_n_of(p, len(a), len(b))) for p, a, b in items}
    for p, ln in keys:
        bw.set_tune_entry(p, 2, ln, small)
    try:
        outs, info = run_batch(items)
    finally:
        for p, ln in keys:
            bw.set_tune_entry(p, 2, ln, default_small(ln))
    assert info["small_buckets"] == (len(keys) if small else 0)
    for (p, a, b), got in zip(items, outs):
        assert (got == gmp_ref.mul(a, b)).all()


def test_squares_in_batch():
    rng = np.random.default_rng(8)
    items = []
    for path in (64, 32):
        for n in (1, 7, 64, 1000, 2048, 5000, 20000):
            if path == 32 and 4 * n > (1 << 17):
                continue
            a = rand_words(n, rng)
            items.append((path, a, a))
        a = np.full(3000, 0xFFFFFFFF, dtype=np.uint32)
        items.append((path, a, a))
    outs, _ = run_batch(items)
    for (p, a, b), got in zip(items, outs):
        assert (got == gmp_ref.mul(a, a)).all(), (p, len(a))


def test_graph_replay_with_new_values():
    rng = np.random.default_rng(9)
    sizes = [(64, 500, 100), (32, 500, 100), (64, 6000, 6000), (32, 12000, 3000),
             (64, 3, 3)]
    ops = [(p, rand_words(la, rng), rand_words(lb, rng)) for p, la, lb in sizes]
    with bw.Batch() as bt:
        outs = [bt.add(a, b, path=p) for p, a, b in ops]
        for rep in range(3):
            for _, a, b in ops:
                a[:] = rand_words(len(a), rng)
                b[:] = rand_words(len(b), rng)
            t = bt.run(timing=True)
            assert t["mul_ms"] > 0
            for (p, a, b), got in zip(ops, outs):
                assert (got == gmp_ref.mul(a, b)).all(), (rep, p, len(a))
        nodes = bt.info()["graph_nodes"]
        assert nodes > 0
        # adding a product rebuilds the layout
        a2 = rand_words(77, rng)
        o2 = bt.add(a2, a2)
        bt.run()
        assert (o2 == gmp_ref.mul(a2, a2)).all()
        for (p, a, b), got in zip(ops, outs):
            assert (got == gmp_ref.mul(a, b)).all()
        bt.clear()
        assert bt.info()["products"] == 0
        bt.run()  # empty batch is a no-op


def test_upload_compute_download_split():
    rng = np.random.default_rng(10)
    a, b = rand_words(4000, rng), rand_words(1000, rng)
    with bw.Batch() as bt:
        out = bt.add(a, b)
        bt.run(bw._lib.BW_BATCH_UPLOAD)
        bt.run(bw._lib.BW_BATCH_COMPUTE)
        out[:] = 0
        bt.run(bw._lib.BW_BATCH_DOWNLOAD)
        assert (out == gmp_ref.mul(a, b)).all()


def test_rejects_oversize_and_short_output():
    with bw.Batch() as bt:
        a = np.ones((1 << 25) + 1, dtype=np.uint32)
        with pytest.raises(bw.BwError):
            bt.add(a, a)            # n = 2^27 > 2^26
        small = np.ones(4, dtype=np.uint32)
        with pytest.raises(bw.BwError):
            bt.add(small, small, out=np.zeros(7, dtype=np.uint32))


def test_autotune_and_tune_table_roundtrip():
    rng = np.random.default_rng(12)
    items = [(64, rand_words(3000, rng), rand_words(900, rng)) for _ in range(8)]
    items += [(32, rand_words(2500, rng), rand_words(2500, rng)) for _ in range(8)]
    with bw.Batch() as bt:
        outs = [bt.add(a, b, path=p) for p, a, b in items]
        bt.autotune(reps=2)
        table = bw.tune_table()
        keys = {(p, log_n_of(p, len(a), len(b))) for p, a, b in items}
        tuned = {(e["path"], e["log_n"]) for e in table if e["ms"] > 0}
        assert keys <= tuned
        json.loads(json.dumps(table))
        bt.run()
        for (p, a, b), got in zip(items, outs):
            assert (got == gmp_ref.mul(a, b)).all()
    assert all(e["row_radix"] in (0, 8, 16) for e in table)
    bw.load_tune_table(table)
    # restore defaults for the other tests
    for p, ln in keys:
        bw.set_tune_entry(p, 2, ln, default_small(ln))


@pytest.mark.parametrize("row_radix", [8, 16])
def test_forced_row_radix_exact(row_radix):
    # the 4-step groups with row rounds of either radix on both paths (the
    # autotuner's candidates), rows from 2^6 to 2^12 points
    rng = np.random.default_rng(13 + row_radix)
    items = []
    for p in (64, 32):
        for words in (700, 3000, 20000, 60000):
            items += [(p, rand_words(words, rng), rand_words(words // 3 + 1, rng))
                      for _ in range(3)]
    keys = {(p, log_n_of(p, len(a), len(b))) for p, a, b in items}
    try:
        for p, ln in keys:
            bw.set_tune_entry(p, 2, ln, False, 0, row_radix)
        with bw.Batch() as bt:
            outs = [bt.add(a, b, path=p) for p, a, b in items]
            bt.run()
            for (p, a, b), got in zip(items, outs):
                assert (got == gmp_ref.mul(a, b)).all(), (p, len(a), len(b), row_radix)
    finally:
        for p, ln in keys:
            bw.set_tune_entry(p, 2, ln, default_small(ln))


def test_uneven_mix_vs_gmp():
    # the batched benchmark's mix (4096 products, 2^12..2^20 bits, 1/8x..1x,
    # half on each prime path), every product against GMP
    mix = workloads.batch_mix(4096, seed=3)
    outs, info = run_batch(mix)
    assert info["products"] == 4096
    for (p, a, b), got in zip(mix, outs):
        assert (got == gmp_ref.mul(a, b)).all(), (p, len(a), len(b))


def test_lookback_wait_fault_is_reported_and_recoverable():
    # the 4-step groups' carry look-back waits are bounded: with the fault
    # injected (every wait looks for a record nobody writes) the run reports
    # BW_ETIMEOUT, and the same batch is correct once it is switched off
    rng = np.random.default_rng(44)
    items = [(64, rand_words(30000, rng), rand_words(9000, rng)) for _ in range(3)]
    items += [(32, rand_words(20000, rng), rand_words(20000, rng)) for _ in range(3)]
    with bw.Batch() as bt:
        outs = [bt.add(a, b, path=p) for p, a, b in items]
        bt.set_wait_limit(2000)
        bt.inject_wait_fault(True)
        with pytest.raises(bw.BwError) as ei:
            bt.run()
        assert ei.value.code == bw._lib.BW_ETIMEOUT
        bt.inject_wait_fault(False)
        bt.set_wait_limit(1 << 22)
        bt.run()
        for (p, a, b), got in zip(items, outs):
            assert (got == gmp_ref.mul(a, b)).all()


@pytest.mark.parametrize("K", [2, 3])
def test_persistent_small_products_exact(K):
    """BW_BATCH_PERSISTENT: the small buckets of both paths run as one
    persistent kernel per path pulling work items from a device queue; every
    product of a mixed batch (small and 4-step buckets, squarings) is
    bit-exact against GMP, on the first run and on graph replays."""
    rng = np.random.default_rng(41 + K)
    items = []
    for path in (64, 32):
        for la, lb in [(1, 1), (2, 1), (7, 9), (64, 64), (100, 13), (511, 512), (1000, 999),
                       (2047, 5), (3000, 3000), (20000, 7000)]:
            a = rand_words(la, rng)
            items.append((path, a, a if la == 64 else rand_words(lb, rng)))
    with bw.Batch(num_primes=K, persistent=True) as bt:
        outs = [bt.add(a, b, path=p) for p, a, b in items]
        for rep in range(3):
            for o in outs:
                o[:] = 0
            bt.run()
            for (p, a, b), got in zip(items, outs):
                assert (got == gmp_ref.mul(a, b)).all(), (rep, p, len(a), len(b))
        info = bt.info()
    assert info["small_buckets"] >= 2 and info["buckets"] > info["small_buckets"]


def test_persistent_matches_graph_of_grids_on_the_mix():
    """The benchmark's uneven mix (512 products) gives the same outputs in the
    persistent form and in the default graph of per-bucket grids."""
    items = workloads.batch_mix(512, seed=9)
    res = {}
    for persistent in (False, True):
        with bw.Batch(num_primes=2, persistent=persistent) as bt:
            outs = [bt.add(a, b, path=p) for p, a, b in items]
            bt.run()
            res[persistent] = [o.copy() for o in outs]
    for x, y, (p, a, b) in zip(res[False], res[True], items):
        assert (x == y).all()
    for j in range(0, len(items), 37):
        _, a, b = items[j]
        assert (res[True][j] == gmp_ref.mul(a, b)).all()
