"""64-bit Mersenne Twister (MT19937-64, Matsumoto & Nishimura 2000) with the
parameters of C++ std::mt19937_64, so that the reference's seeded inputs
(tests/test_full_multiply.cpp:61-73, 431-441 use std::mt19937_64) can be
regenerated without a compiler.  Checked against std::mt19937_64 output by
tests/golden/gen_golden.py.  Test infrastructure only.
"""
import numpy as np

_NN, _MM = 312, 156
_A = 0xB5026F5AA96619E9
_UM = 0xFFFFFFFF80000000
_LM = 0x7FFFFFFF
_M64 = (1 << 64) - 1


class MT64:
    def __init__(self, seed=5489):
        mt = [0] * _NN
        mt[0] = seed & _M64
        for i in range(1, _NN):
            mt[i] = (6364136223846793005 * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i) & _M64
        self.mt = mt
        self.i = _NN

    def _twist(self):
        mt = self.mt
        for i in range(_NN):
            x = (mt[i] & _UM) | (mt[(i + 1) % _NN] & _LM)
            xa = x >> 1
            if x & 1:
                xa ^= _A
            mt[i] = mt[(i + _MM) % _NN] ^ xa
        self.i = 0

    def __call__(self):
        if self.i >= _NN:
            self._twist()
        x = self.mt[self.i]
        self.i += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        return x & _M64


def random_limbs_ref32(n, seed):
    """tests/test_full_multiply.cpp:61-73: word i is 0 if i%8==0, 1 if i%8==1,
    else (uint32_t)rng() % 2^30."""
    rng = MT64(seed)
    out = np.zeros(n, dtype=np.uint32)
    for i in range(n):
        if i % 8 == 0:
            out[i] = 0
        elif i % 8 == 1:
            out[i] = 1
        else:
            out[i] = (rng() & 0xFFFFFFFF) % (1 << 30)
    return out


def random_limbs_ref64(n, seed):
    """tests/test_full_multiply.cpp:431-441: u64 limb i is 0, 1, UINT64_MAX
    for i%8 == 0, 1, 2, else rng()."""
    rng = MT64(seed)
    out = np.zeros(n, dtype=np.uint64)
    for i in range(n):
        r = i % 8
        out[i] = 0 if r == 0 else 1 if r == 1 else _M64 if r == 2 else rng()
    return out


def random_words_top(nwords, seed):
    """Uniform random u32 words from successive 64-bit outputs (low word
    first), top bit of the top word set: the operands of the throughput
    configurations."""
    rng = MT64(seed)
    out = np.zeros(nwords + (nwords & 1), dtype=np.uint64)
    half = out.size // 2
    v = np.array([rng() for _ in range(half)], dtype=np.uint64)
    w = v.view(np.uint32)[:nwords].copy()
    w[-1] |= np.uint32(0x80000000)
    return w


def random_words_top_fast(nwords, seed):
    """Same distribution for large operands via numpy's PCG64 (seeded), used
    where regenerating with MT19937-64 in Python would be slow."""
    rng = np.random.default_rng(seed)
    w = rng.integers(0, 1 << 32, size=nwords, dtype=np.uint64).astype(np.uint32)
    w[-1] |= np.uint32(0x80000000)
    return w
