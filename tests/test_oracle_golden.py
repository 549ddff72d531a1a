"""The oracle (oracle/bw_oracle.c) pinned against the reference's own golden
vectors and known-answer tests, and against GMP on the reference's seeded
inputs (tests/golden/fixtures.npz).  CPU only."""
import os

import numpy as np
import pytest

from oracle import gmp_ref, mt64, oracle

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "fixtures.npz"))


def as_int(w):
    return int.from_bytes(np.ascontiguousarray(w).view(np.uint8).tobytes(), "little")


# scripts/full_mul.py:103-124 -- [1,2,3,4] x [5,6,7,8] with three 31-bit
# primes and primitive 8th roots; CRT result [5,16,34,60,61,52,32,0]
FULL_MUL_PRIMES = [2013265921, 1811939329, 469762049]
FULL_MUL_ROOTS8 = [1592366214, 1452317833, 129701348]


def test_full_mul_py_golden():
    res = []
    for p, w in zip(FULL_MUL_PRIMES, FULL_MUL_ROOTS8):
        assert pow(w, 8, p) == 1 and pow(w, 4, p) != 1  # primitive 8th roots
        res.append(oracle.conv_mod([1, 2, 3, 4], [5, 6, 7, 8], p, w, 8))
    out = [oracle.garner([int(r[i]) for r in res], FULL_MUL_PRIMES) for i in range(8)]
    assert out == [5, 16, 34, 60, 61, 52, 32, 0]


def test_ntt_roundtrip_and_definition():
    primes, roots, logs = oracle.path_basis(64)
    p = primes[0]
    w = oracle.lib.oracle_root_for(primes[0], roots[0], logs[0], 4)
    x = list(range(1, 17))
    X = oracle.ntt(x, w, p)
    assert [int(v) for v in X] == [sum(x[i] * pow(w, i * k, p) for i in range(16)) % p
                                   for k in range(16)]
    assert [int(v) for v in oracle.intt(X, w, p)] == x


def test_crt_cpp_kats():
    # tests/test_crt.cpp:19-103
    p1, p2, p3 = 2013265921, 1811939329, 469762049
    x = 12345678901234567890 % (p1 * p2)
    assert oracle.garner([x % p1, x % p2], [p1, p2]) == x
    P = p1 * p2 * p3
    x = ((123456789123 << 64) ^ 987654321) % P
    assert oracle.garner([x % p1, x % p2, x % p3], [p1, p2, p3]) == x


@pytest.mark.parametrize("primes", [
    [0x23800001, 0x26800001, 0x2d000001],         # tests/test_crt_gpu.cu:509 (32-bit)
    [0x400002600000001, 0x400004200000001],       # :506 (hybrid)
    [0x400002600000001, 0x400004200000001, 0x400001100000001],  # :492-496 (native)
])
def test_crt_gpu_cu_values(primes):
    # tests/test_crt_gpu.cu:159-265 and 403-485
    M = 1
    for p in primes:
        M *= p
    vals = [0, 1, 12, 255, 65535, 0xFFFFFFFF, 1 << 89, 1 << 128, (1 << 160) - 1,
            (1 << 159) + 12345, (1 << 63) - 1, (1 << 64) - 1]
    for x in vals:
        if x >= M:
            continue  # the reference skips values beyond the modulus product
        assert oracle.garner([x % p for p in primes], primes) == x
    # residues (i*7 + j*13 + 1) mod p_j, N=64, against a direct CRT
    for i in range(64):
        r = [(i * 7 + j * 13 + 1) % p for j, p in enumerate(primes)]
        x = oracle.garner(r, primes)
        assert x < M and all(x % p == rj for p, rj in zip(primes, r))


def _carry_ref(coeffs, bits, m):
    v = sum(c << (bits * i) for i, c in enumerate(coeffs))
    return [(v >> (32 * j)) & 0xFFFFFFFF for j in range(m)]


def test_carry_patterns():
    # tests/test_carry_prop.cu:331-390 (128-bit coefficients -> 32-bit words)
    M32 = 0xFFFFFFFF
    pats = {
        "zeros": [0] * 64,
        "small": list(range(1, 65)),
        "single_overflow": [M32 + 1] + [0] * 63,
        "max_limbs": [M32] * 1024,
        "wide": [(1 << 70) + 12345] + [0] * 15,
        "cross_segment": [0] * 1023 + [M32 + 1] + [0] * 1024,
        "u160_max": [(1 << 160) - 1] * 8,
        "u160_wide": [12345 + (1 << 159)] + [0] * 15,
    }
    big = []
    for i in range(1 << 12):
        big.append([i * 12345 + 1, (1 << 70) + (i % 1000), M32,
                    ((i % 17) << 64) + i * 99991][i % 4])
    pats["large_random"] = big
    for name, cs in pats.items():
        for bits in (32, 16):
            m = len(cs) * bits // 32 + 6
            got = [int(v) for v in oracle.carry(cs, bits, m)]
            assert got == _carry_ref(cs, bits, m), (name, bits)


def test_limits_helpers_match_reference_constants():
    # tests/test_ntt_limits.cpp:63-111
    v2 = oracle.lib.oracle_v2
    ro = oracle.lib.oracle_root_order_log
    assert v2(0x2d000001 - 1) == 24 and v2(0x23800001 - 1) == 23 and v2(0x26800001 - 1) == 23
    assert v2(0x400002600000001 - 1) == 33 and v2(0x400004200000001 - 1) == 33
    assert v2(0x400001100000001 - 1) == 32
    assert ro(663, 0x2d000001) == 23 and ro(721, 0x23800001) == 23 and ro(19, 0x26800001) == 23
    assert ro(273765203699653965, 0x400002600000001) == 33
    assert ro(26231613454922890, 0x400004200000001) == 33
    assert ro(144261359744151243, 0x400001100000001) == 32


def test_reference_primes_product():
    # the reference's own bases multiply correctly in the oracle (limbs < 2^30
    # for its 32-bit pipeline, tests/test_full_multiply.cpp:69-70)
    a = GOLD["ref32_128_a"]
    b = GOLD["ref32_128_b"]
    primes = [0x2d000001, 0x23800001, 0x26800001]
    roots = [663, 721, 19]
    logs = [23, 23, 23]
    c = oracle.multiply_basis(a, b, 32, primes, roots, logs)
    assert (c == GOLD["ref32_128_c"]).all()


@pytest.mark.parametrize("path,K", [(64, 2), (64, 3), (32, 2), (32, 3)])
def test_oracle_vs_fixtures(path, K):
    for key in GOLD.files:
        if not key.endswith("_a"):
            continue
        stem = key[:-2]
        a, b, c = GOLD[stem + "_a"], GOLD[stem + "_b"], GOLD[stem + "_c"]
        if a.size > 4096 and not (path == 64 and K == 2):
            continue
        got = oracle.multiply(a, b, path, K)
        assert (got == c.view(np.uint32)).all(), stem


def test_schoolbook_vs_gmp():
    for L in (4, 8, 16, 64, 128, 2048):
        a, b, c = GOLD[f"ref32_{L}_a"], GOLD[f"ref32_{L}_b"], GOLD[f"ref32_{L}_c"]
        assert (oracle.schoolbook(a, b) == c).all()


def test_mt64_matches_std():
    for seed in (1234, 5678):
        g = mt64.MT64(seed)
        assert [g() for _ in range(64)] == [int(x) for x in GOLD[f"mt_raw_{seed}"]]
    # the C++ standard's check value for the default seed ([rand.predef])
    g = mt64.MT64()
    for _ in range(9999):
        g()
    assert g() == 9981545732273789042


def test_gmp_binding():
    a = np.array([0xFFFFFFFF] * 5, dtype=np.uint32)
    c = gmp_ref.mul(a, a)
    assert as_int(c) == as_int(a) ** 2
