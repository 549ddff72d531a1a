"""GMP mpz_mul through ctypes (libgmp.so.10), for checking products bit-exact.

No gmp.h is installed, so the documented mpz API is declared here by hand:
an mpz_t is {int alloc; int size; mp_limb_t *d} and the public mpz_*
functions are exported as __gmpz_*.  Test infrastructure only.
"""
import ctypes
import ctypes.util
import time

import numpy as np


class _mpz(ctypes.Structure):
    _fields_ = [("alloc", ctypes.c_int), ("size", ctypes.c_int), ("d", ctypes.c_void_p)]


def _find():
    for name in ("libgmp.so.10", ctypes.util.find_library("gmp")):
        if not name:
            continue
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    raise OSError("libgmp not found")


_g = _find()
_P = ctypes.POINTER(_mpz)
for _n, _r, _a in [
    ("__gmpz_init", None, [_P]),
    ("__gmpz_clear", None, [_P]),
    ("__gmpz_import", None, [_P, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t, ctypes.c_int,
                             ctypes.c_size_t, ctypes.c_void_p]),
    ("__gmpz_export", ctypes.c_void_p, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.c_int, ctypes.c_size_t, ctypes.c_int,
                                        ctypes.c_size_t, _P]),
    ("__gmpz_mul", None, [_P, _P, _P]),
]:
    _f = getattr(_g, _n)
    _f.restype = _r
    _f.argtypes = _a

# module-level names (a leading "__" inside a class body would be mangled)
z_init = _g.__gmpz_init
z_clear = _g.__gmpz_clear
z_import = _g.__gmpz_import
z_export = _g.__gmpz_export
z_mul = _g.__gmpz_mul

version = ctypes.c_char_p.in_dll(_g, "__gmp_version").value.decode()


class Mpz:
    def __init__(self, words=None):
        self.z = _mpz()
        z_init(ctypes.byref(self.z))
        if words is not None:
            self.set_words(words)

    def set_words(self, words):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        z_import(ctypes.byref(self.z), w.size, -1, 4, 0, 0, w.ctypes.data)

    def words(self, n):
        out = np.zeros(n, dtype=np.uint32)
        need = (abs(self.z.size) * 8 + 3) // 4
        buf = np.zeros(max(n, need) + 2, dtype=np.uint32)
        cnt = ctypes.c_size_t(0)
        z_export(buf.ctypes.data, ctypes.byref(cnt), -1, 4, 0, 0, ctypes.byref(self.z))
        if np.any(buf[n:]):
            raise ValueError("product does not fit")
        out[:] = buf[:n]
        return out

    def __del__(self):
        try:
            z_clear(ctypes.byref(self.z))
        except Exception:
            pass


def mul(a, b):
    """a * b for little-endian u32 word arrays; returns len(a)+len(b) words."""
    a = np.ascontiguousarray(a).view(np.uint32) if np.asarray(a).dtype == np.uint64 else a
    b = np.ascontiguousarray(b).view(np.uint32) if np.asarray(b).dtype == np.uint64 else b
    za, zb, zc = Mpz(a), Mpz(b), Mpz()
    z_mul(ctypes.byref(zc.z), ctypes.byref(za.z), ctypes.byref(zb.z))
    return zc.words(len(a) + len(b))


def time_mul(a, b, reps=1):
    """Seconds per mpz_mul (import/export excluded), single thread."""
    za, zb, zc = Mpz(a), Mpz(b), Mpz()
    t0 = time.perf_counter()
    for _ in range(reps):
        z_mul(ctypes.byref(zc.z), ctypes.byref(za.z), ctypes.byref(zb.z))
    return (time.perf_counter() - t0) / reps
