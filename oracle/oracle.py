"""ctypes binding of liboracle.so, the CPU restatement of the reference's
multiply algorithm (bw_oracle.c).  Test infrastructure only."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build(force=False):
    src = os.path.join(HERE, "bw_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(src) > os.path.getmtime(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "-B", "liboracle.so"], check=True)
    return LIB_PATH


def _load():
    build()
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    SZ = ctypes.c_size_t
    U64 = ctypes.c_uint64
    I = ctypes.c_int
    sig = {
        "oracle_v2": (I, [U64]),
        "oracle_root_order_log": (I, [U64, U64]),
        "oracle_root_for": (U64, [U64, U64, I, I]),
        "oracle_ntt": (None, [P, SZ, U64, U64]),
        "oracle_intt": (None, [P, SZ, U64, U64]),
        "oracle_conv_mod": (I, [U64, U64, P, SZ, P, SZ, P, SZ]),
        "oracle_garner": (I, [I, P, P, P]),
        "oracle_carry": (I, [P, SZ, I, P, SZ]),
        "oracle_schoolbook": (I, [P, SZ, P, SZ, P]),
        "oracle_multiply_basis": (I, [I, I, P, P, P, P, SZ, P, SZ, P]),
        "oracle_path_basis": (I, [I, P, P, P]),
        "oracle_multiply": (I, [I, I, P, SZ, P, SZ, P]),
        "oracle_set_threads": (None, [I]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _u32(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.uint64 else a.astype(np.uint32, copy=False)


def multiply(a, b, path=64, num_primes=2):
    a, b = _u32(a), _u32(b)
    out = np.zeros(a.size + b.size, dtype=np.uint32)
    rc = lib.oracle_multiply(path, num_primes, _p(a), a.size, _p(b), b.size, _p(out))
    if rc:
        raise RuntimeError(f"oracle_multiply rc={rc}")
    return out


def multiply_basis(a, b, coeff_bits, primes, roots_max, max_logs):
    a, b = _u32(a), _u32(b)
    K = len(primes)
    pr = np.array(primes, dtype=np.uint64)
    ro = np.array(roots_max, dtype=np.uint64)
    ml = np.array(max_logs, dtype=np.int32)
    out = np.zeros(a.size + b.size, dtype=np.uint32)
    rc = lib.oracle_multiply_basis(coeff_bits, K, _p(pr), _p(ro), _p(ml), _p(a), a.size, _p(b),
                                   b.size, _p(out))
    if rc:
        raise RuntimeError(f"oracle_multiply_basis rc={rc}")
    return out


def schoolbook(a, b):
    a, b = _u32(a), _u32(b)
    out = np.zeros(a.size + b.size, dtype=np.uint32)
    lib.oracle_schoolbook(_p(a), a.size, _p(b), b.size, _p(out))
    return out


def conv_mod(a, b, p, omega_n, n):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.zeros(n, dtype=np.uint64)
    rc = lib.oracle_conv_mod(p, omega_n, _p(a), a.size, _p(b), b.size, _p(out), n)
    if rc:
        raise RuntimeError(f"oracle_conv_mod rc={rc}")
    return out


def ntt(a, omega, p):
    a = np.array(a, dtype=np.uint64)
    lib.oracle_ntt(_p(a), a.size, omega, p)
    return a


def intt(a, omega, p):
    a = np.array(a, dtype=np.uint64)
    lib.oracle_intt(_p(a), a.size, omega, p)
    return a


def garner(residues, primes):
    """Python int reconstructed (mod 2^192) from residues mod primes."""
    r = np.array(residues, dtype=np.uint64)
    pr = np.array(primes, dtype=np.uint64)
    x = np.zeros(3, dtype=np.uint64)
    rc = lib.oracle_garner(len(primes), _p(pr), _p(r), _p(x))
    if rc:
        raise RuntimeError(f"oracle_garner rc={rc}")
    return int(x[0]) | (int(x[1]) << 64) | (int(x[2]) << 128)


def carry(coeffs, coeff_bits, m):
    """Words of sum c_i 2^(coeff_bits i) (coeffs: Python ints < 2^192)."""
    c3 = np.zeros(3 * len(coeffs), dtype=np.uint64)
    mask = (1 << 64) - 1
    for i, c in enumerate(coeffs):
        c3[3 * i] = c & mask
        c3[3 * i + 1] = (c >> 64) & mask
        c3[3 * i + 2] = (c >> 128) & mask
    out = np.zeros(m, dtype=np.uint32)
    rc = lib.oracle_carry(_p(c3), len(coeffs), coeff_bits, _p(out), m)
    if rc:
        raise RuntimeError(f"oracle_carry rc={rc}")
    return out


def path_basis(path):
    pr = np.zeros(3, dtype=np.uint64)
    ro = np.zeros(3, dtype=np.uint64)
    ml = np.zeros(3, dtype=np.int32)
    lib.oracle_path_basis(path, _p(pr), _p(ro), _p(ml))
    return [int(x) for x in pr], [int(x) for x in ro], [int(x) for x in ml]
