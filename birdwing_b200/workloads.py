"""Seeded synthetic operand mixes for the batched and served forms.

Values are uniform random words with the top bit of each operand set, as in
the reference's own benchmark operands (tests/test_full_multiply.cpp, the
mt19937_64 fills); sizes follow the two mixes the batched and serving
benchmarks are quoted on:

* ``batch_mix``: bit lengths log-uniform in [2^12, 2^20], the second operand
  1/8x to 1x the first (log-uniform), half the products on the 32-bit prime
  path and half on the 64-bit path;
* ``serving_sizes``: bit lengths log-uniform in [2^10, 2^24], 20% squarings,
  the same length ratio for the rest.
"""
import numpy as np

from ._lib import BW_PATH_P32, BW_PATH_P64


def rand_operand(rng, words):
    w = rng.integers(0, 1 << 32, size=words, dtype=np.uint64).astype(np.uint32)
    w[-1] |= np.uint32(0x80000000)
    return w


def _loguniform_bits(rng, lo_log, hi_log, size):
    return np.exp2(rng.uniform(lo_log, hi_log, size=size))


def batch_sizes(count, seed=3, lo_log=12, hi_log=20):
    """[(path, la, lb)] for `count` products (lengths in 32-bit words)."""
    rng = np.random.default_rng(seed)
    bits_a = _loguniform_bits(rng, lo_log, hi_log, count)
    ratio = np.exp2(rng.uniform(-3.0, 0.0, size=count))
    paths = np.where(rng.permutation(count) < count // 2, BW_PATH_P32, BW_PATH_P64)
    out = []
    for i in range(count):
        ba = int(bits_a[i])
        bb = max(1, int(ba * ratio[i]))
        out.append((int(paths[i]), (ba + 31) // 32, (bb + 31) // 32))
    return out


def batch_mix(count, seed=3, lo_log=12, hi_log=20):
    """[(path, a, b)] with operand arrays (uint32 words)."""
    rng = np.random.default_rng(seed + 1000)
    return [(p, rand_operand(rng, la), rand_operand(rng, lb))
            for p, la, lb in batch_sizes(count, seed, lo_log, hi_log)]


def serving_sizes(count, seed=5, lo_log=10, hi_log=24, square_frac=0.2):
    """[(la, lb, square)] for `count` requests (lengths in 32-bit words)."""
    rng = np.random.default_rng(seed)
    bits_a = _loguniform_bits(rng, lo_log, hi_log, count)
    ratio = np.exp2(rng.uniform(-3.0, 0.0, size=count))
    sq = rng.uniform(size=count) < square_frac
    out = []
    for i in range(count):
        ba = int(bits_a[i])
        la = (ba + 31) // 32
        if sq[i]:
            out.append((la, la, True))
        else:
            out.append((la, (max(1, int(ba * ratio[i])) + 31) // 32, False))
    return out
