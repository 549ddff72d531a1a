"""Generate tests/golden/fixtures.npz.

Inputs come from C++ std::mt19937_64 in the reference's patterns
(tests/test_full_multiply.cpp:61-73 and 431-441 of nikitaborisov/birdwing),
products from GMP mpz_mul, each product cross-checked with Python's own
integer multiplication.  The same run checks oracle/mt64.py against
std::mt19937_64.  Run from the repo root:  python tests/golden/gen_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import gmp_ref, mt64  # noqa: E402


def mt(tool, kind, n, seed, dtype):
    out = subprocess.run([tool, kind, str(n), str(seed)], check=True, capture_output=True).stdout
    return np.frombuffer(out, dtype=dtype).copy()


def as_int(w):
    return int.from_bytes(np.ascontiguousarray(w).view(np.uint8).tobytes(), "little")


def main():
    tmp = tempfile.mkdtemp()
    tool = os.path.join(tmp, "mt_limbs")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", tool, os.path.join(HERE, "mt_limbs.cpp")],
                   check=True)
    fx = {}
    # MT19937-64 self-check: C++ vs Python for two seeds
    for seed in (1234, 5678):
        raw = mt(tool, "raw", 2000, seed, np.uint64)
        g = mt64.MT64(seed)
        py = np.array([g() for _ in range(2000)], dtype=np.uint64)
        assert (raw == py).all(), "mt64.py disagrees with std::mt19937_64"
        fx[f"mt_raw_{seed}"] = raw[:64]
    # reference pattern, 32-bit words (test_full_pipeline sizes)
    for L in (4, 8, 16, 64, 128, 2048, 10000):
        a = mt(tool, "ref32", L, 1234, np.uint32)
        b = mt(tool, "ref32", L, 5678, np.uint32)
        assert (a == mt64.random_limbs_ref32(L, 1234)).all()
        c = gmp_ref.mul(a, b)
        assert as_int(c) == as_int(a) * as_int(b)
        fx[f"ref32_{L}_a"], fx[f"ref32_{L}_b"], fx[f"ref32_{L}_c"] = a, b, c
    # reference pattern, 64-bit limbs (test_native_pipeline sizes)
    for L in (4, 16, 64, 256, 1024, 4096):
        a = mt(tool, "ref64", L, 1234, np.uint64)
        b = mt(tool, "ref64", L, 5678, np.uint64)
        assert (a == mt64.random_limbs_ref64(L, 1234)).all()
        c = gmp_ref.mul(a.view(np.uint32), b.view(np.uint32))
        assert as_int(c) == as_int(a) * as_int(b)
        fx[f"ref64_{L}_a"], fx[f"ref64_{L}_b"], fx[f"ref64_{L}_c"] = a, b, c.view(np.uint64)
    # uniform words with the top bit set, unbalanced shapes
    for (la, lb, sa, sb) in ((1000, 125, 11, 12), (4096, 4096, 13, 14), (777, 3001, 15, 16)):
        a = mt64.random_words_top(la, sa)
        b = mt64.random_words_top(lb, sb)
        c = gmp_ref.mul(a, b)
        assert as_int(c) == as_int(a) * as_int(b)
        fx[f"top_{la}x{lb}_a"], fx[f"top_{la}x{lb}_b"], fx[f"top_{la}x{lb}_c"] = a, b, c
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **fx)
    print(f"wrote {len(fx)} arrays; GMP {gmp_ref.version}")


if __name__ == "__main__":
    main()
