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

from ._lib import BW_PATH_P32, BW_PATH_P64, BW_PLAN_COEF64


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


# ---------------------------------------------------------------- plain products
# The single-product workloads the benchmark times, with the exact plan
# arguments it passes to bw_plan_create.  The parity tests build their plans
# from the same entries, so the algorithm that is timed and the one that is
# tested cannot drift apart.  Fields:
#   words_a, words_b  operand lengths in u32 words (uniform random, top bit set)
#   seeds             mt19937_64 seeds of the two operands (the reference's
#                     1234 / 5678, tests/test_full_multiply.cpp:61-73)
#   square            the second operand is the first (one forward transform)
#   plan              (path, num_primes, flags) given to bw_plan_create; the
#                     library's own choice where num_primes is 0
#   expect            what that plan must resolve to (bw_plan_info fields)
#   ref               (path, num_primes) of the reference's algorithm for the
#                     same product, which the CPU restatement runs
#   literal           (path, num_primes, flags) of the workload as the
#                     reference states it (its coefficient width and prime
#                     count), timed beside the library's choice
#   other             (optional) the same product on the other prime path,
#                     timed beside it: the 32-bit path with 64-bit
#                     coefficients (six primes) for the 2^28-bit workloads
PLAIN = {
    "2": dict(
        words_a=1 << 23, words_b=1 << 23, seeds=(1234, 5678), square=False,
        plan=(BW_PATH_P64, 0, 0),
        expect=dict(path=64, coeff_bits=64, num_primes=3, log_n=23, log_cols=12),
        ref=(64, 2), literal=(BW_PATH_P64, 2, 0),
        other=(BW_PATH_P32, 0, BW_PLAN_COEF64),
        desc="plain 2^28-bit x 2^28-bit product"),
    "2sq": dict(
        words_a=1 << 23, words_b=1 << 23, seeds=(1234, 1234), square=True,
        plan=(BW_PATH_P64, 0, 0),
        expect=dict(path=64, coeff_bits=64, num_primes=3, log_n=23, log_cols=12),
        ref=(64, 2), literal=(BW_PATH_P64, 2, 0),
        other=(BW_PATH_P32, 0, BW_PLAN_COEF64),
        desc="squaring of a 2^28-bit integer"),
    "1": dict(
        words_a=1 << 15, words_b=1 << 15, seeds=(1234, 5678), square=False,
        plan=(BW_PATH_P32, 3, 0),
        expect=dict(path=32, coeff_bits=16, num_primes=3, log_n=17),
        ref=(32, 3), literal=(BW_PATH_P32, 3, 0),
        desc="plain 2^20-bit x 2^20-bit product, 16-bit coefficients, n=2^17, "
             "3 x 30-bit primes"),
    "4": dict(
        words_a=1 << 28, words_b=1 << 28, seeds=(1234, 5678), square=False,
        plan=(BW_PATH_P64, 0, 0),
        expect=dict(path=64, coeff_bits=64, num_primes=3, log_n=28),
        ref=(64, 3), literal=(BW_PATH_P64, 3, 0),
        desc="plain huge 2^33-bit x 2^33-bit product (1 GiB operands), three-pass schedule"),
    # a smaller product of the same kernels, for ncu captures (working set > L2)
    "prof": dict(
        words_a=1 << 21, words_b=1 << 21, seeds=(1234, 5678), square=False,
        plan=(BW_PATH_P64, 0, 0),
        expect=dict(path=64, coeff_bits=64, num_primes=3, log_n=21),
        ref=(64, 2), literal=(BW_PATH_P64, 2, 0),
        desc="plain 2^26-bit x 2^26-bit product (profiling size)"),
    # the same size on the 32-bit path (16-bit coefficients, two primes)
    "prof32": dict(
        words_a=1 << 21, words_b=1 << 21, seeds=(1234, 5678), square=False,
        plan=(BW_PATH_P32, 2, 0),
        expect=dict(path=32, coeff_bits=16, num_primes=2, log_n=23, log_cols=12),
        ref=(32, 2), literal=(BW_PATH_P32, 2, 0),
        desc="plain 2^26-bit x 2^26-bit product on the 32-bit path (profiling size)"),
}


def plain_plan_args(name, which="plan"):
    """(la, lb, path, num_primes, flags) of a plain workload's plan: the
    benchmarked one (which="plan") or the reference's literal statement of
    the workload (which="literal")."""
    w = PLAIN[name]
    path, k, flags = w[which]
    return w["words_a"], w["words_b"], path, k, flags


# what the `other` plans resolve to (bw_plan_info fields)
OTHER_EXPECT = dict(path=32, coeff_bits=64, num_primes=6)


def algorithm_of(info):
    """One-line description of what a plan runs, from bw_plan_info fields."""
    prime_bits = 58 if info["path"] == 64 else 30
    return (f"{info['coeff_bits']}-bit coefficients, n=2^{info['log_n']}, "
            f"{info['num_primes']} x {prime_bits}-bit primes ({info['path']}-bit prime path)")
