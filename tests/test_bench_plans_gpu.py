"""Parity of the exact plans the benchmark times, at the benchmark's sizes.

Every plain workload in birdwing_b200.workloads.PLAIN is built here with the
same bw_plan_create arguments bench.py passes (the table is shared), its
resolved algorithm is checked against the table's `expect` entry, and its
product -- through host buffers and through the device-pointer graph replay
the benchmark times -- is compared bit for bit with GMP mpz_mul on the
benchmark's seeded operands.  The reference's own full-size check is the GMP
comparison of tests/test_full_multiply.cpp:551-556."""
import numpy as np
import pytest

import birdwing_b200 as bw
from birdwing_b200 import workloads
from oracle import gmp_ref, mt64

pytestmark = pytest.mark.gpu


def bench_operands(name):
    w = workloads.PLAIN[name]
    a = mt64.random_words_top_fast(w["words_a"], w["seeds"][0])
    b = a if w["square"] else mt64.random_words_top_fast(w["words_b"], w["seeds"][1])
    return a, b


def device_product(c, a, b, square, reps=2):
    """The benchmark's timed call: device pointers, graph replay, twice."""
    import torch
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = da if square else torch.from_numpy(b.view(np.int32)).cuda()
    dc = torch.empty(a.size + b.size, dtype=torch.int32, device="cuda")
    outs = []
    for _ in range(reps):
        dc.fill_(-1)
        torch.cuda.synchronize()
        c.multiply_device(da.data_ptr(), a.size, db.data_ptr(), b.size, dc.data_ptr(),
                          dc.numel())
        c.sync()
        outs.append(dc.cpu().numpy().view(np.uint32).copy())
    return outs


def plans_of(name):
    """The benchmarked plan and, if different, the workload as the reference
    states it (its coefficient width and prime count)."""
    w = workloads.PLAIN[name]
    return (["plan"] + (["literal"] if w["literal"] != w["plan"] else []) +
            (["other"] if w.get("other") else []))


@pytest.mark.parametrize("name,which", [(n, k) for n in ("1", "2", "2sq", "prof", "prof32")
                                        for k in plans_of(n)])
def test_benchmarked_plan_bit_exact(name, which):
    w = workloads.PLAIN[name]
    la, lb, path, k, flags = workloads.plain_plan_args(name, which)
    a, b = bench_operands(name)
    want = gmp_ref.mul(a, b)
    with bw.Plan(la, lb, path, k, flags=flags) as p, bw.Context(p) as c:
        if which == "plan":
            for key, v in w["expect"].items():
                assert p.info[key] == v, (key, p.info[key], v)
        if which == "other":
            for key, v in workloads.OTHER_EXPECT.items():
                assert p.info[key] == v, (key, p.info[key], v)
        got = c.square(a) if w["square"] else c.multiply(a, b)
        assert (got == want).all()
        for out in device_product(c, a, b, w["square"]):
            assert (out == want).all()


def test_config4_plans_bit_exact():
    # 2^33-bit operands (1 GiB each): the benchmarked plan and the reference's
    # statement (32-bit coefficients, n = 2^29, three primes), both checked
    # by residues mod 2^64 and three random 61-bit primes, then against one
    # GMP product (minutes of host CPU)
    name = "4"
    w = workloads.PLAIN[name]
    a, b = bench_operands(name)
    got = {}
    for which in plans_of(name):
        la, lb, path, k, flags = workloads.plain_plan_args(name, which)
        with bw.Plan(la, lb, path, k, flags=flags) as p, bw.Context(p) as c:
            if which == "plan":
                for key, v in w["expect"].items():
                    assert p.info[key] == v, (key, p.info[key], v)
            got[which] = c.multiply(a, b)
    A = int.from_bytes(a.tobytes(), "little")
    B = int.from_bytes(b.tobytes(), "little")
    rng = np.random.default_rng(61)
    mods = [1 << 64]
    while len(mods) < 4:
        m = int(rng.integers(1 << 60, 1 << 61)) | 1
        if pow(3, m - 1, m) == 1:  # probable prime
            mods.append(m)
    for which, out in got.items():
        C = int.from_bytes(out.tobytes(), "little")
        for m in mods:
            assert C % m == (A % m) * (B % m) % m, (which, m)
        del C
    del A, B
    want = gmp_ref.mul(a, b)
    for which, out in got.items():
        assert (out == want).all(), which
