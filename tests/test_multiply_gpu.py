"""Parity of the CUDA path (through the C ABI) with the oracle and GMP.

Bit-exact everywhere: this is integer arithmetic.  Small and medium sizes
are checked against the oracle (the CPU restatement of the reference's
algorithm) and GMP; the benchmark sizes against GMP and through
size-independent properties (squaring == self-product, linearity in one
operand, products mod small primes)."""
import os

import numpy as np
import pytest

import birdwing_b200 as bw
from oracle import gmp_ref, mt64, oracle

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "fixtures.npz"))
PATHS = [(64, 2), (64, 3), (32, 2), (32, 3)]


def as_int(w):
    return int.from_bytes(np.ascontiguousarray(w).view(np.uint8).tobytes(), "little")


def gpu_mul(a, b, path=64, K=2):
    with bw.Plan(len(a), len(b), path, K) as p, bw.Context(p) as c:
        return c.multiply(a, b)


def rand_words(n, rng, top=True):
    w = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    if top:
        w[-1] |= np.uint32(0x80000000)
    return w


@pytest.mark.parametrize("path,K", PATHS)
def test_golden_reference_pattern_u32(path, K):
    # tests/test_full_multiply.cpp:245-265 (test_full_pipeline sizes)
    for L in (4, 8, 16, 64, 128, 2048, 10000):
        a, b, c = GOLD[f"ref32_{L}_a"], GOLD[f"ref32_{L}_b"], GOLD[f"ref32_{L}_c"]
        assert (gpu_mul(a, b, path, K) == c).all(), L


@pytest.mark.parametrize("path,K", PATHS)
def test_golden_reference_pattern_u64(path, K):
    # tests/test_full_multiply.cpp:482-518 (64-bit limbs incl. UINT64_MAX)
    for L in (4, 16, 64, 256, 1024, 4096):
        a, b, c = GOLD[f"ref64_{L}_a"], GOLD[f"ref64_{L}_b"], GOLD[f"ref64_{L}_c"]
        got = gpu_mul(a.view(np.uint32), b.view(np.uint32), path, K)
        assert (got.view(np.uint64) == c).all(), L


@pytest.mark.parametrize("path,K", PATHS)
def test_golden_unbalanced(path, K):
    for stem in ("top_1000x125", "top_4096x4096", "top_777x3001"):
        a, b, c = GOLD[stem + "_a"], GOLD[stem + "_b"], GOLD[stem + "_c"]
        assert (gpu_mul(a, b, path, K) == c).all(), stem


def test_reference_simple_cases():
    # tests/test_full_multiply.cpp:268-287
    one = np.array([1, 0, 0, 0], dtype=np.uint32)
    z = np.zeros(4, dtype=np.uint32)
    f = np.array([42, 0, 0, 0], dtype=np.uint32)
    for path, K in PATHS:
        assert as_int(gpu_mul(one, one, path, K)) == 1
        assert as_int(gpu_mul(z, f, path, K)) == 0
        # root-of-unity probe, L = 8 (:307-351): A[1] = 1, B[0] = 1
        a = np.zeros(8, dtype=np.uint32)
        b = np.zeros(8, dtype=np.uint32)
        a[1] = 1
        b[0] = 1
        c = gpu_mul(a, b, path, K)
        assert c[1] == 1 and as_int(c) == 1 << 32


def test_identities_large():
    # tests/test_full_multiply.cpp:289-305 at L = 2^20
    L = 1 << 20
    Z = np.zeros(L, dtype=np.uint32)
    O = np.ones(L, dtype=np.uint32)
    for path, K in ((64, 2), (32, 3)):
        assert not gpu_mul(Z, Z, path, K).any()
        assert not gpu_mul(O, Z, path, K).any()
        r = gpu_mul(O, O, path, K)
        assert r[0] == 1
        assert (r == gmp_ref.mul(O, O)).all()


@pytest.mark.parametrize("path,K", PATHS)
def test_sizes_sweep_vs_oracle(path, K):
    rng = np.random.default_rng(100 + path + K)
    shapes = [(1, 1), (1, 2), (2, 1), (3, 5), (7, 7), (8, 8), (9, 8), (15, 17), (16, 16),
              (31, 33), (100, 3), (3, 100), (255, 256), (256, 256), (257, 255), (1000, 1),
              (1023, 1025), (2048, 2048), (4095, 4097), (5000, 300)]
    for la, lb in shapes:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        want = oracle.multiply(a, b, path, K)
        assert (gpu_mul(a, b, path, K) == want).all(), (la, lb)


def test_sizes_sweep_vs_gmp_medium():
    rng = np.random.default_rng(7)
    for la, lb in [(1 << 14, 1 << 14), ((1 << 16) + 3, (1 << 15) - 5), (1 << 17, 1 << 10),
                   (123457, 98765), (1 << 19, 1 << 19)]:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        want = gmp_ref.mul(a, b)
        for path, K in ((64, 2), (64, 3), (32, 2)):
            assert (gpu_mul(a, b, path, K) == want).all(), (la, lb, path, K)


@pytest.mark.parametrize("path,K", PATHS)
def test_carry_stress_all_ones(path, K):
    # (2^(32m) - 1)^2 and (2^(32m)-1)(2^(32m)+1): long runs of 0xFFFFFFFF words
    # force propagate chains through many carry tiles
    for m in (1, 7, 2048, 2049, 1 << 15):
        a = np.full(m, 0xFFFFFFFF, dtype=np.uint32)
        assert (gpu_mul(a, a, path, K) == gmp_ref.mul(a, a)).all(), m
        b = np.zeros(m + 1, dtype=np.uint32)
        b[0] = 1
        b[m] = 1
        if (m + m + 1) * (2 if path == 32 else 1) <= (1 << 24):
            got = gpu_mul(a, b, path, K)
            assert (got == gmp_ref.mul(a, b)).all(), m


@pytest.mark.parametrize("path,K", [(64, 2), (32, 3)])
def test_square_paths(path, K):
    rng = np.random.default_rng(11)
    for L in (1, 5, 64, 1000, 4096, 1 << 16):
        a = rand_words(L, rng)
        want = gmp_ref.mul(a, a)
        with bw.Plan(L, L, path, K) as p, bw.Context(p) as c:
            assert (c.square(a) == want).all(), L
            assert (c.multiply(a, a) == want).all(), L   # same array: squaring schedule
            b = a.copy()
            assert (c.multiply(a, b) == want).all(), L   # distinct arrays: full schedule


def test_context_reuse_and_timing():
    rng = np.random.default_rng(3)
    L = 1 << 12
    with bw.Plan(L, L, 64) as p, bw.Context(p) as c:
        for _ in range(5):
            a, b = rand_words(L, rng), rand_words(L, rng)
            out, t = c.multiply(a, b, timing=True)
            assert (out == gmp_ref.mul(a, b)).all()
            assert t["total_ms"] > 0 and t["fwd_ms"] >= 0


@pytest.mark.parametrize("path,K", PATHS)
def test_crt_coefficient_dump(path, K):
    # the reference's CRT dump (src/gpu_ntt.cu:843-884): convolution
    # coefficients before carry, compared with the oracle's per-prime
    # convolutions joined by the oracle's Garner
    rng = np.random.default_rng(5)
    for la, lb in ((3, 5), (100, 77), (1000, 1000)):
        a, b = rand_words(la, rng), rand_words(lb, rng)
        with bw.Plan(la, lb, path, K) as p, bw.Context(p) as c:
            got = c.coeffs(a, b)
            n = p.N
        per = 2 if path == 32 else 1
        ca = [int(x) for x in (a.view(np.uint16) if per == 2 else a)]
        cb = [int(x) for x in (b.view(np.uint16) if per == 2 else b)]
        primes, roots, logs = oracle.path_basis(path)
        log_n = n.bit_length() - 1
        res = []
        for k in range(K):
            w = oracle.lib.oracle_root_for(primes[k], roots[k], logs[k], log_n)
            res.append(oracle.conv_mod(ca, cb, primes[k], w, n))
        want = [oracle.garner([int(r[i]) for r in res], primes[:K]) for i in range(n)]
        assert got == want
        # and the coefficients are the exact linear convolution
        lin = [0] * n
        for i, x in enumerate(ca):
            if x:
                for j, y in enumerate(cb):
                    lin[i + j] += x * y
        assert got == lin


def test_device_pointers_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    la, lb = 50000, 30001
    a, b = rand_words(la, rng), rand_words(lb, rng)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dc = torch.zeros(la + lb + 5, dtype=torch.int32, device="cuda")
    with bw.Plan(la, lb, 64) as p, bw.Context(p) as c:
        c.multiply_device(da.data_ptr(), la, db.data_ptr(), lb, dc.data_ptr() + 4, la + lb)
        c.sync()
        got = dc.cpu().numpy().view(np.uint32)
    assert got[0] == 0 and (got[1:1 + la + lb] == gmp_ref.mul(a, b)).all()
    assert not got[1 + la + lb:].any()


def test_wrong_sizes_are_rejected():
    with bw.Plan(8, 8, 64) as p, bw.Context(p) as c:
        with pytest.raises(bw.BwError) as e:
            c.multiply(np.ones(9, dtype=np.uint32), np.ones(8, dtype=np.uint32))
        assert e.value.code == -1
        # the context still works afterwards
        a = np.arange(1, 9, dtype=np.uint32)
        assert (c.multiply(a, a) == gmp_ref.mul(a, a)).all()


def test_lookback_wait_fault_is_reported_and_recoverable():
    # inject a look-back flag that nothing sets: every bounded wait runs out,
    # the call returns BW_ETIMEOUT instead of hanging, the context survives
    import ctypes
    rng = np.random.default_rng(4)
    L = 1 << 16
    a, b = rand_words(L, rng), rand_words(L, rng)
    want = gmp_ref.mul(a, b)
    with bw.Plan(L, L, 64) as p, bw.Context(p) as c:
        assert (c.multiply(a, b) == want).all()
        assert bw.lib.bw_ctx_set_wait_limit(c._h, 200) == 0
        assert bw.lib.bw_ctx_inject_wait_fault(c._h, 1) == 0
        with pytest.raises(bw.BwError) as e:
            c.multiply(a, b)
        assert e.value.code == -4
        assert bw.lib.bw_ctx_inject_wait_fault(c._h, 0) == 0
        assert bw.lib.bw_ctx_set_wait_limit(c._h, 1 << 22) == 0
        assert (c.multiply(a, b) == want).all()
        del ctypes


def test_config1_plain_small():
    # the 2^20-bit workload: 2^20-bit operands (2^15 words), 16-bit
    # coefficients, n = 2^17, three 30-bit primes
    a = mt64.random_words_top(1 << 15, 1234)
    b = mt64.random_words_top(1 << 15, 5678)
    with bw.Plan(a.size, b.size, 32, 3) as p, bw.Context(p) as c:
        assert p.info["log_n"] == 17 and p.info["num_primes"] == 3
        assert (c.multiply(a, b) == gmp_ref.mul(a, b)).all()


def test_config2_three_primes_properties():
    # size-independent checks at the full size: residues of the product mod
    # small primes and mod 2^64 equal the products of the operands' residues
    a = mt64.random_words_top_fast(1 << 23, 42)
    b = mt64.random_words_top_fast(1 << 23, 43)
    got = gpu_mul(a, b, 64, 3)
    A, B, C = as_int(a), as_int(b), as_int(got)
    for m in (2 ** 64, 2 ** 61 - 1, 1000000007, 998244353, (1 << 31) - 1):
        assert C % m == (A % m) * (B % m) % m
    assert C.bit_length() <= 64 * (1 << 23)


@pytest.mark.parametrize("path,K", PATHS)
def test_three_pass_schedule_vs_oracle(path, K):
    # the n = R * R2 * C schedule (used beyond n = 2^26), forced at small sizes
    flags = bw._lib.BW_PLAN_THREE_PASS
    rng = np.random.default_rng(200 + path + K)
    for la, lb in [(1, 1), (8, 8), (9, 8), (100, 77), (1000, 1000), (4096, 3000), (5000, 1)]:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        with bw.Plan(la, lb, path, K, flags=flags) as p, bw.Context(p) as c:
            assert p.info["log_rows"] >= 1
            got = c.multiply(a, b)
            sq = c.square(a) if la == lb else None
        assert (got == oracle.multiply(a, b, path, K)).all(), (la, lb)
        if sq is not None:
            assert (sq == oracle.multiply(a, a, path, K)).all(), la


def test_three_pass_schedule_vs_gmp_medium():
    flags = bw._lib.BW_PLAN_THREE_PASS
    rng = np.random.default_rng(17)
    for la, lb, path, K in [(1 << 16, 1 << 16, 64, 2), ((1 << 19) + 5, (1 << 18) - 3, 64, 3),
                            (1 << 18, 1 << 18, 32, 2), (1 << 20, 1 << 20, 64, 2)]:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        with bw.Plan(la, lb, path, K, flags=flags) as p, bw.Context(p) as c:
            got = c.multiply(a, b)
        assert (got == gmp_ref.mul(a, b)).all(), (la, lb, path, K)


def test_async_host_mode_two_contexts():
    # BW_PTR_HOST_ASYNC: two contexts of one plan used in turn, pinned buffers
    import torch
    rng = np.random.default_rng(31)
    la, lb = 50000, 30001
    pairs = [(rand_words(la, rng), rand_words(lb, rng)) for _ in range(6)]

    def pinned(x):
        return torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)

    ins = [(pinned(a), pinned(b)) for a, b in pairs]
    outs = [pinned(np.zeros(la + lb, dtype=np.uint32)) for _ in pairs]
    with bw.Plan(la, lb, 64, 2) as p, bw.Context(p) as c0, bw.Context(p) as c1:
        ctxs = [c0, c1]
        for i, ((a, b), o) in enumerate(zip(ins, outs)):
            c = ctxs[i % 2]
            if i >= 2:
                c.sync()
            c.multiply_async(a, b, o)
        c0.sync()
        c1.sync()
        # timing cannot be asked for in this mode
        import ctypes
        t = bw._lib.bw_timing()
        rc = bw.lib.bw_multiply(c0._h, bw.api._ptr(ins[0][0]), la, bw.api._ptr(ins[0][1]), lb,
                                bw.api._ptr(outs[0]), la + lb, bw._lib.BW_PTR_HOST_ASYNC,
                                ctypes.byref(t))
        assert rc == bw._lib.BW_EINVAL
    for (a, b), o in zip(pairs, outs):
        assert (o == gmp_ref.mul(a, b)).all()


@pytest.mark.gpu
def test_stage_order_across_contexts():
    """Three contexts of one plan form an ordered copy-in / kernels / copy-out
    pipeline: products issued in turn (asynchronous, blocking with timing, and
    squarings) stay exact, and a context whose events the plan's order
    refers to can be destroyed while the others keep going."""
    import torch
    rng = np.random.default_rng(37)
    la, lb = 70001, 65536

    def pinned(x):
        return torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)

    pairs = [(rand_words(la, rng), rand_words(lb, rng)) for _ in range(9)]
    ins = [(pinned(a), pinned(b)) for a, b in pairs]
    outs = [pinned(np.zeros(la + lb, dtype=np.uint32)) for _ in pairs]
    with bw.Plan(la, lb, 64, 2) as p:
        ctxs = [bw.Context(p) for _ in range(3)]
        for i, ((a, b), o) in enumerate(zip(ins[:6], outs[:6])):
            c = ctxs[i % 3]
            if i >= 3:
                c.sync()
            c.multiply_async(a, b, o)
        # the last issuer owns the plan's stage events: destroy it mid-stream
        ctxs[2].close()
        for i in range(6, 9):
            c = ctxs[i % 2]
            c.sync()
            c.multiply_async(ins[i][0], ins[i][1], outs[i])
        for c in ctxs[:2]:
            c.sync()
        # blocking calls with stage times, alternating contexts
        for i in range(2):
            got, t = ctxs[i].multiply(pairs[i][0], pairs[i][1], timing=True)
            assert (got == gmp_ref.mul(*pairs[i])).all()
            assert t["total_ms"] > 0
        for c in ctxs[:2]:
            c.close()
    for (a, b), o in zip(pairs, outs):
        assert (o == gmp_ref.mul(a, b)).all()
    with bw.Plan(la, la, 32, 3) as p, bw.Context(p) as c0, bw.Context(p) as c1:
        sq = [pinned(rand_words(la, rng)) for _ in range(4)]
        so = [pinned(np.zeros(2 * la, dtype=np.uint32)) for _ in sq]
        for i, (x, o) in enumerate(zip(sq, so)):
            c = (c0, c1)[i % 2]
            if i >= 2:
                c.sync()
            c.multiply_async(x, x, o)
        c0.sync()
        c1.sync()
        for x, o in zip(sq, so):
            assert (o == gmp_ref.mul(x, x)).all()


@pytest.mark.parametrize("path,K,la,lb", [(64, 2, 70000, 50000), (32, 3, 3000, 2999),
                                          (64, 3, 5000, 1)])
def test_device_pointer_graph_replay(path, K, la, lb):
    # device-pointer products replay one captured graph while the pointers
    # stay the same; new values every time, direct (timed) launches in
    # between, and a pointer change recaptures
    import torch
    rng = np.random.default_rng(41 + la)
    with bw.Plan(la, lb, path, K) as p, bw.Context(p) as c:
        da = torch.empty(la, dtype=torch.int32, device="cuda")
        db = torch.empty(lb, dtype=torch.int32, device="cuda")
        dc = torch.empty(la + lb, dtype=torch.int32, device="cuda")
        dc2 = torch.empty(la + lb, dtype=torch.int32, device="cuda")
        for it in range(5):
            a, b = rand_words(la, rng), rand_words(lb, rng)
            da.copy_(torch.from_numpy(a.view(np.int32)))
            db.copy_(torch.from_numpy(b.view(np.int32)))
            torch.cuda.synchronize()
            out = dc2 if it == 3 else dc
            c.multiply_device(da.data_ptr(), la, db.data_ptr(), lb, out.data_ptr(), la + lb,
                              timing=(it == 2))
            c.sync()
            got = out.cpu().numpy().view(np.uint32)
            assert (got == gmp_ref.mul(a, b)).all(), it


def test_p32_longest_transform_vs_gmp():
    # the 32-bit path at its longest transform (2^25 points, K = 2): two
    # 2^28-bit operands split into 16-bit coefficients, against GMP
    a = mt64.random_words_top_fast(1 << 23, 99)
    b = mt64.random_words_top_fast(1 << 23, 98)
    with bw.Plan(a.size, b.size, 32, 2) as p, bw.Context(p) as c:
        assert p.info["log_n"] == 25
        got = c.multiply(a, b)
    assert (got == gmp_ref.mul(a, b)).all()


def test_automatic_path_choice():
    # num_primes 0: the 32-bit path with 16-bit coefficients while its
    # transform has at most 2^21 points, then the 32-bit path with 64-bit
    # coefficients (six primes) up to 2^23 points, then the 64-bit path with
    # 64-bit coefficients
    for la, lb, want, bits, k in [(1, 1, 32, 16, 2), (1000, 700, 32, 16, 2),
                                  (1 << 19, 1 << 19, 32, 16, 2),
                                  (1 << 19, (1 << 19) + 1, 32, 64, 6),
                                  (1 << 22, 1 << 22, 32, 64, 6), (1 << 23, 1 << 23, 32, 64, 6),
                                  ((1 << 23) + 2, (1 << 23) + 2, 64, 64, 3)]:
        with bw.Plan(la, lb) as p:
            got = (p.info["path"], p.info["coeff_bits"], p.info["num_primes"])
            assert got == (want, bits, k), (la, lb, p.info)
    # the 64-bit path below the 64-bit-coefficient threshold keeps 32-bit ones
    with bw.Plan(1 << 18, 1 << 18, 64) as p:
        assert p.info["coeff_bits"] == 32 and p.info["num_primes"] == 2
    # explicit num_primes: the reference's coefficients, the 32-bit path up to
    # 2^24 points
    for la, lb, want in [(1 << 22, 1 << 22, 32), (1 << 22, (1 << 22) + 1, 64)]:
        with bw.Plan(la, lb, bw.BW_PATH_AUTO, 2) as p:
            assert p.info["path"] == want and p.info["coeff_bits"] in (16, 32), (la, lb)


@pytest.mark.gpu
@pytest.mark.parametrize("path,K", [(64, 2), (32, 3), (32, 2)])
def test_chunked_host_copies(path, K):
    """Copy-in by column blocks under K1 and copy-out by word ranges under K4,
    for every chunk count: exact against GMP for ragged sizes (partial last
    rows, an operand shorter than one row, unbalanced operands), squarings,
    the three-pass schedule, pageable and pinned buffers."""
    import torch
    rng = np.random.default_rng(41 + path + K)

    def pinned(x):
        return torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)

    cases = [(300001, 299999, 0), (262144, 262144, 0), (500000, 7, 0), (123457, 65536, 0),
             (40001, 39999, bw._lib.BW_PLAN_THREE_PASS)]
    for la, lb, flags in cases:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        want = gmp_ref.mul(a, b)
        pa, pb = pinned(a), pinned(b)
        with bw.Plan(la, lb, path, K, flags=flags) as p, bw.Context(p) as c:
            for chunks in (1, 2, 4, 8, 16):
                c.set_copy_chunks(chunks)
                assert (c.multiply(a, b) == want).all(), (la, lb, flags, chunks)
                out = pinned(np.zeros(la + lb, dtype=np.uint32))
                assert (c.multiply(pa, pb, out=out) == want).all(), (la, lb, flags, chunks)
            c.set_copy_chunks(0)
            assert (c.multiply(a, b) == want).all()
        if la == lb or flags:
            with bw.Plan(la, la, path, K, flags=flags) as p, bw.Context(p) as c:
                for chunks in (1, 4, 16):
                    c.set_copy_chunks(chunks)
                    assert (c.square(a) == gmp_ref.mul(a, a)).all(), (la, flags, chunks)
    with bw.Plan(1000, 1000, path, K) as p, bw.Context(p) as c:
        with pytest.raises(bw.BwError):
            c.set_copy_chunks(17)
        with pytest.raises(bw.BwError):
            c.set_copy_chunks(-1)


@pytest.mark.gpu
def test_chunked_copies_in_the_ordered_ring():
    """Chunked copies on three contexts used in turn (stage order), with a
    context reconfigured to whole copies in the middle of the stream."""
    import torch
    rng = np.random.default_rng(43)
    la, lb = 1 << 20, (1 << 20) + 3

    def pinned(x):
        return torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)

    pairs = [(rand_words(la, rng), rand_words(lb, rng)) for _ in range(4)]
    ins = [(pinned(a), pinned(b)) for a, b in pairs]
    outs = [pinned(np.zeros(la + lb, dtype=np.uint32)) for _ in range(9)]
    with bw.Plan(la, lb, 64, 2) as p:
        ctxs = [bw.Context(p) for _ in range(3)]
        for i in range(9):
            c = ctxs[i % 3]
            if i >= 3:
                c.sync()
            if i == 4:
                c.set_copy_chunks(1)
            c.multiply_async(ins[i % 4][0], ins[i % 4][1], outs[i])
        for c in ctxs:
            c.sync()
        for c in ctxs:
            c.close()
    for i in range(9):
        assert (outs[i] == gmp_ref.mul(*pairs[i % 4])).all(), i


@pytest.mark.gpu
def test_one_shot_cache():
    """One-shot products keep the plan and context of recent sizes: repeated,
    interleaved and concurrent calls stay exact, a small limit evicts, and a
    zero limit frees everything and turns the cache off."""
    import threading
    rng = np.random.default_rng(47)
    sizes = [(5000, 4000), (70000, 3), (1 << 16, 1 << 16), (5000, 4000)]
    ops = [(rand_words(la, rng), rand_words(lb, rng)) for la, lb in sizes]
    try:
        for _ in range(2):
            for a, b in ops:
                assert (bw.multiply(a, b) == gmp_ref.mul(a, b)).all()
                c, ms = bw.host_multiply_merge(a, b)
                assert (c == gmp_ref.mul(a, b)).all() and ms > 0
        # one size from four threads at once
        a, b = ops[2]
        want = gmp_ref.mul(a, b)
        bad = []

        def work():
            for _ in range(5):
                if not (bw.multiply(a, b) == want).all():
                    bad.append(1)

        th = [threading.Thread(target=work) for _ in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not bad
        # a limit below one context: every call builds and frees its own
        bw.host_once_cache_limit(1 << 20)
        for a, b in ops:
            assert (bw.multiply(a, b) == gmp_ref.mul(a, b)).all()
        bw.host_once_cache_limit(0)
        for a, b in ops[:2]:
            assert (bw.multiply(a, b) == gmp_ref.mul(a, b)).all()
    finally:
        bw.host_once_cache_limit(4 << 30)


COEF64 = bw._lib.BW_PLAN_COEF64


@pytest.mark.gpu
def test_coef64_vs_gmp():
    """64-bit coefficients with three primes (BW_PLAN_COEF64): exact against
    GMP over odd word counts (the last coefficient without a high word),
    single words, unbalanced operands, power-of-two boundaries, long carry
    chains, squarings and the three-pass schedule."""
    rng = np.random.default_rng(53)
    shapes = [(1, 1), (1, 2), (2, 1), (3, 3), (7, 9), (8, 8), (31, 33), (64, 64), (65, 63),
              (1000, 1), (1, 1000), (1023, 1025), (4096, 4096), (4097, 4095), (12345, 678),
              (1 << 16, 1 << 16), ((1 << 16) + 1, (1 << 16) - 1), (300001, 299999),
              (1 << 19, 3), (1 << 20, 1 << 20)]
    for la, lb in shapes:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        with bw.Plan(la, lb, 64, 0, flags=COEF64) as p, bw.Context(p) as c:
            assert p.info["coeff_bits"] == 64 and p.info["num_primes"] == 3
            assert (c.multiply(a, b) == gmp_ref.mul(a, b)).all(), (la, lb)
    for m in (1, 2, 7, 2048, 2049, 1 << 15, (1 << 18) + 1):
        ones = np.full(m, 0xFFFFFFFF, dtype=np.uint32)
        with bw.Plan(m, m, 64, 0, flags=COEF64) as p, bw.Context(p) as c:
            assert (c.square(ones) == gmp_ref.mul(ones, ones)).all(), m
        b = np.zeros(m + 1, dtype=np.uint32)
        b[0] = 1
        b[m] = 1
        with bw.Plan(m, m + 1, 64, 0, flags=COEF64) as p, bw.Context(p) as c:
            assert (c.multiply(ones, b) == gmp_ref.mul(ones, b)).all(), m
    for la, lb in [(1, 1), (9, 8), (100, 77), (1000, 1000), (4096, 3000), (5000, 1),
                   (40001, 39999)]:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        flags = COEF64 | bw._lib.BW_PLAN_THREE_PASS
        with bw.Plan(la, lb, 64, 3, flags=flags) as p, bw.Context(p) as c:
            assert (c.multiply(a, b) == gmp_ref.mul(a, b)).all(), (la, lb)
        with bw.Plan(la, la, 64, 3, flags=flags) as p, bw.Context(p) as c:
            assert (c.square(a) == gmp_ref.mul(a, a)).all(), la


@pytest.mark.gpu
def test_coef64_copies_pointers_and_choice():
    """64-bit coefficients through chunked host copies, device pointers with
    graph replay, and the automatic choice (num_primes 0 on the 64-bit path);
    explicit num_primes keeps the reference's 32-bit coefficients and the
    coefficient dump refuses 64-bit plans."""
    import torch
    rng = np.random.default_rng(59)
    la, lb = 300001, 262144
    a, b = rand_words(la, rng), rand_words(lb, rng)
    want = gmp_ref.mul(a, b)
    with bw.Plan(la, lb, 64) as p, bw.Context(p) as c:
        assert p.info["coeff_bits"] == 64
        for chunks in (1, 2, 8, 16):
            c.set_copy_chunks(chunks)
            assert (c.multiply(a, b) == want).all(), chunks
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(b.view(np.int32)).cuda()
        dc = torch.zeros(la + lb, dtype=torch.int32, device="cuda")
        for _ in range(3):
            c.multiply_device(da.data_ptr(), la, db.data_ptr(), lb, dc.data_ptr(), la + lb)
            c.sync()
            assert (dc.cpu().numpy().view(np.uint32) == want).all()
        # operand b at an odd word offset of a device buffer
        buf = torch.zeros(lb + 1, dtype=torch.int32, device="cuda")
        buf[1:] = db
        c.multiply_device(da.data_ptr(), la, buf.data_ptr() + 4, lb, dc.data_ptr(), la + lb)
        c.sync()
        assert (dc.cpu().numpy().view(np.uint32) == want).all()
        with pytest.raises(bw.BwError):
            c.coeffs(a, b)
    for K in (2, 3):
        with bw.Plan(la, lb, 64, K) as p:
            assert p.info["coeff_bits"] == 32 and p.info["num_primes"] == K
    # 64-bit coefficients take 3 primes on the 64-bit path, 6 on the 32-bit one
    with pytest.raises(bw.BwError):
        bw.Plan(100, 100, 32, 2, flags=COEF64)
    with pytest.raises(bw.BwError):
        bw.Plan(100, 100, 64, 2, flags=COEF64)


@pytest.mark.gpu
def test_radix_switches_exact():
    """The round-radix tuning switches of single products on the 64-bit path
    (radix-8 column passes, radix-16 rows) keep products exact."""
    L = bw._lib
    rng = np.random.default_rng(61)
    for la, lb in [(1000, 999), (65537, 4097), (300001, 299999)]:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        want = gmp_ref.mul(a, b)
        for K, fl in ((0, COEF64), (2, 0)):
            for sw in (L.BW_PLAN_COL_RADIX8, L.BW_PLAN_RADIX16,
                       L.BW_PLAN_COL_RADIX8 | L.BW_PLAN_THREE_PASS):
                with bw.Plan(la, lb, 64, K, flags=fl | sw) as p, bw.Context(p) as c:
                    assert (c.multiply(a, b) == want).all(), (la, lb, K, sw)


def test_tma_inverse_columns_exact():
    """The inverse column pass with tensor-copy tiles (BW_PLAN_TMA_COLS) and
    with per-element cp.async (BW_PLAN_NO_TMA_COLS) give the same exact
    products on both paths, for every coefficient width, squarings and
    device pointers at an odd word offset (graph replay)."""
    import torch
    L = bw._lib
    rng = np.random.default_rng(71)
    for la, lb in [(1, 1), (3000, 1777), (65537, 4097), ((1 << 19) + 3, (1 << 18) - 5)]:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        want = gmp_ref.mul(a, b)
        for path, K in ((64, 0), (64, 2), (32, 2), (32, 3), (32, 6)):
            for fl in (L.BW_PLAN_TMA_COLS, L.BW_PLAN_NO_TMA_COLS):
                if K == 6:
                    fl |= L.BW_PLAN_COEF64
                with bw.Plan(la, lb, path, K, flags=fl) as p, bw.Context(p) as c:
                    assert (c.multiply(a, b) == want).all(), (la, lb, path, K, fl)
                    if la == lb:
                        assert (c.square(a) == gmp_ref.mul(a, a)).all()
    # device pointers, the operand at an odd word offset, graph replay twice
    la = lb = (1 << 20) + 1
    a, b = rand_words(la, rng), rand_words(lb, rng)
    want = gmp_ref.mul(a, b)
    buf = torch.from_numpy(np.concatenate([[7], a, b]).astype(np.uint32).view(np.int32)).cuda()
    dc = torch.empty(la + lb, dtype=torch.int32, device="cuda")
    for fl in (L.BW_PLAN_TMA_COLS, L.BW_PLAN_NO_TMA_COLS):
        with bw.Plan(la, lb, 64, 0, flags=fl) as p, bw.Context(p) as c:
            for _ in range(2):
                dc.fill_(-1)
                c.multiply_device(buf.data_ptr() + 4, la, buf.data_ptr() + 4 * (1 + la), lb,
                                  dc.data_ptr(), la + lb)
                c.sync()
                assert (dc.cpu().numpy().view(np.uint32) == want).all(), fl


def test_shuffle_row_exchange_exact():
    """The warp-shuffle exchange of the 32-bit path's 2^12-point rows
    (BW_PLAN_SHFL_ROWS) gives the products of the shared-memory exchange;
    squarings keep the shared-memory path."""
    L = bw._lib
    rng = np.random.default_rng(73)
    for la, lb in [((1 << 21) - 7, (1 << 21) + 5), (1 << 22, (1 << 21) + 1), (1 << 21, 1 << 21)]:
        a, b = rand_words(la, rng), rand_words(lb, rng)
        want = gmp_ref.mul(a, b)
        with bw.Plan(la, lb, 32, 2, flags=L.BW_PLAN_SHFL_ROWS) as p, bw.Context(p) as c:
            assert p.info["log_cols"] == 12
            assert (c.multiply(a, b) == want).all(), (la, lb)
            if la == lb:
                assert (c.square(a) == gmp_ref.mul(a, a)).all()


@pytest.mark.gpu
def test_coef64_squaring_chunks_and_ring():
    """64-bit coefficients: squarings through every chunk count, and products
    on three contexts of one plan used in turn (stage order, whole copies)
    then on one context (chunked copies)."""
    import torch
    rng = np.random.default_rng(67)

    def pinned(x):
        return torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)

    la = (1 << 20) + 5
    a = rand_words(la, rng)
    want = gmp_ref.mul(a, a)
    with bw.Plan(la, la, 64) as p, bw.Context(p) as c:
        assert p.info["coeff_bits"] == 64
        for chunks in (1, 2, 4, 8, 16):
            c.set_copy_chunks(chunks)
            assert (c.square(a) == want).all(), chunks
    lb = (1 << 20) - 3
    pairs = [(rand_words(la, rng), rand_words(lb, rng)) for _ in range(3)]
    ins = [(pinned(x), pinned(y)) for x, y in pairs]
    outs = [pinned(np.zeros(la + lb, dtype=np.uint32)) for _ in range(7)]
    with bw.Plan(la, lb, 64) as p:
        ctxs = [bw.Context(p) for _ in range(3)]
        for i in range(6):
            c = ctxs[i % 3]
            if i >= 3:
                c.sync()
            c.multiply_async(ins[i % 3][0], ins[i % 3][1], outs[i])
        for c in ctxs:
            c.sync()
        for c in ctxs[1:]:
            c.close()
        ctxs[0].multiply_async(ins[0][0], ins[0][1], outs[6])   # alone again: chunked
        ctxs[0].sync()
        ctxs[0].close()
    for i in range(7):
        assert (outs[i] == gmp_ref.mul(*pairs[i % 3])).all(), i
