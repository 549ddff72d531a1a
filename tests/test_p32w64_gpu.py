"""The 32-bit prime path with 64-bit coefficients (BW_PLAN_COEF64 on
BW_PATH_P32): six primes below 2^30, transforms of up to 2^23 points.

Products are compared bit for bit with GMP mpz_mul (the reference's own
full-size check, tests/test_full_multiply.cpp:551-556) at ragged, odd,
squaring, carry-heavy and full sizes, through host buffers (whole and
chunked copies) and device pointers, in both forms of the forward column
pass (one prime per CTA, and the six-prime loop)."""
import numpy as np
import pytest

import birdwing_b200 as bw
from birdwing_b200 import _lib as L
from oracle import gmp_ref, mt64

pytestmark = pytest.mark.gpu

PRIMES6 = [595591169, 645922817, 754974721, 880803841, 897581057, 998244353]


def plan(la, lb, flags=0):
    return bw.Plan(la, lb, L.BW_PATH_P32, 0, flags=L.BW_PLAN_COEF64 | flags)


def test_plan_resolves_six_primes():
    with plan(1 << 20, 1 << 20) as p:
        assert p.info["path"] == 32
        assert p.info["coeff_bits"] == 64
        assert p.info["num_primes"] == 6
        assert p.info["primes"] == PRIMES6
        assert p.info["log_n"] == 20


def test_limits_and_arguments():
    # 2^23-word operands are the largest square product (n = 2^23)
    with plan(1 << 23, 1 << 23) as p:
        assert p.info["log_n"] == 23
    with pytest.raises(bw.BwError) as e:
        plan((1 << 23) + 2, (1 << 23) + 2)
    assert e.value.code == L.BW_ESIZE
    with pytest.raises(bw.BwError) as e:
        bw.Plan(1024, 1024, L.BW_PATH_P32, 3, flags=L.BW_PLAN_COEF64)
    assert e.value.code == L.BW_EINVAL
    with bw.Plan(1024, 1024, L.BW_PATH_P32, 6, flags=L.BW_PLAN_COEF64) as p:
        assert p.info["num_primes"] == 6


@pytest.mark.parametrize("la,lb", [(1, 1), (2, 1), (3, 5), (17, 4), (255, 256), (1000, 777),
                                   (4096, 4096), (65535, 1), (1 << 16, (1 << 16) + 1),
                                   (300001, 123457), ((1 << 20) + 3, (1 << 19) - 5)])
def test_products_exact(la, lb):
    a = mt64.random_words_top_fast(la, 11 + la)
    b = mt64.random_words_top_fast(lb, 29 + lb)
    with plan(la, lb) as p, bw.Context(p) as c:
        assert (c.multiply(a, b) == gmp_ref.mul(a, b)).all()


@pytest.mark.parametrize("la,lb", [(5, 3), (4096, 4095), ((1 << 20) + 3, (1 << 19) - 5)])
def test_one_prime_per_cta_form_exact(la, lb):
    # BW_PLAN_K1_ONE_PRIME: the forward column pass runs one prime per CTA
    # instead of looping over the six primes in one CTA
    a = mt64.random_words_top_fast(la, 71 + la)
    b = mt64.random_words_top_fast(lb, 83 + lb)
    with plan(la, lb, L.BW_PLAN_K1_ONE_PRIME) as p, bw.Context(p) as c:
        assert (c.multiply(a, b) == gmp_ref.mul(a, b)).all()


@pytest.mark.parametrize("la", [1, 7, 4097, 1 << 18])
def test_squaring_exact(la):
    a = mt64.random_words_top_fast(la, 101 + la)
    with plan(la, la) as p, bw.Context(p) as c:
        assert (c.square(a) == gmp_ref.mul(a, a)).all()


@pytest.mark.parametrize("words", [1 << 12, 1 << 21])
def test_all_ones_operands(words):
    # every coefficient at its maximum (2^64 - 1): the largest convolution
    # values (min(na, nb) (2^64 - 1)^2) and the longest carry chains
    a = np.full(words, 0xFFFFFFFF, dtype=np.uint32)
    with plan(words, words) as p, bw.Context(p) as c:
        assert (c.multiply(a, a.copy()) == gmp_ref.mul(a, a)).all()


def test_chunked_host_copies_exact():
    # 2^21-word operands: the host call splits the copy-in under K1 and the
    # copy-out under the look-back carry into pieces
    la = lb = 1 << 21
    a = mt64.random_words_top_fast(la, 1234)
    b = mt64.random_words_top_fast(lb, 5678)
    want = gmp_ref.mul(a, b)
    with plan(la, lb) as p, bw.Context(p) as c:
        for _ in range(2):
            assert (c.multiply(a, b) == want).all()


def test_full_size_device_pointers_exact():
    # the largest square product: 2^28-bit operands, n = 2^23, through the
    # device-pointer graph replay and through host buffers
    import torch
    la = lb = 1 << 23
    a = mt64.random_words_top_fast(la, 1234)
    b = mt64.random_words_top_fast(lb, 5678)
    want = gmp_ref.mul(a, b)
    with plan(la, lb) as p, bw.Context(p) as c:
        assert p.info["log_n"] == 23 and p.info["log_cols"] == 12
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(b.view(np.int32)).cuda()
        dc = torch.empty(la + lb, dtype=torch.int32, device="cuda")
        for _ in range(2):
            dc.fill_(-1)
            torch.cuda.synchronize()
            c.multiply_device(da.data_ptr(), la, db.data_ptr(), lb, dc.data_ptr(), dc.numel())
            c.sync()
            assert (dc.cpu().numpy().view(np.uint32) == want).all()
        assert (c.multiply(a, b) == want).all()
        assert (c.square(a) == gmp_ref.mul(a, a)).all()


def test_odd_word_offsets_exact():
    # operands at odd word offsets of a device buffer: the forward pass stages
    # each 64-bit coefficient as two 4-byte copies instead of one 8-byte copy
    import torch
    la, lb = 300001, 262147
    a = mt64.random_words_top_fast(la, 9)
    b = mt64.random_words_top_fast(lb, 10)
    want = gmp_ref.mul(a, b)
    buf = torch.from_numpy(np.concatenate([[7], a, b]).astype(np.uint32).view(np.int32)).cuda()
    dc = torch.empty(la + lb, dtype=torch.int32, device="cuda")
    for flags in (0, L.BW_PLAN_K1_ONE_PRIME):
        with plan(la, lb, flags) as p, bw.Context(p) as c:
            for _ in range(2):
                dc.fill_(-1)
                torch.cuda.synchronize()
                c.multiply_device(buf.data_ptr() + 4, la, buf.data_ptr() + 4 * (1 + la), lb,
                                  dc.data_ptr(), la + lb)
                c.sync()
                assert (dc.cpu().numpy().view(np.uint32) == want).all(), flags
