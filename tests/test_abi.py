"""The C-ABI library loads, exports every function include/birdwing.h
declares, and its host-side admission logic behaves like the reference's
ntt_limits (no GPU calls here)."""
import ctypes
import os
import re

import pytest

import birdwing_b200 as bw
from birdwing_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "birdwing.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bw_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 15
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, n


def test_abi_version():
    assert bw.lib.bw_abi_version() == 2


def test_limits():
    l64 = bw.limits(bw.BW_PATH_P64)
    l32 = bw.limits(bw.BW_PATH_P32)
    assert l64["max_log_n"] == 32 and l64["num_primes"] == 2
    assert l32["max_log_n"] == 25
    assert l32["max_square_words"] == (1 << 24) // 2
    assert bw.limits(bw.BW_PATH_P32, 3)["max_log_n"] == 24
    assert bw.limits(bw.BW_PATH_P64, 3)["num_primes"] == 3


@pytest.mark.parametrize("la,lb,path,K,ok", [
    (1, 1, 64, 0, True), (1 << 23, 1 << 23, 64, 0, True), (1 << 28, 1 << 28, 64, 0, True),
    (1 << 31, 1 << 31, 64, 2, True), (1 << 32, 1 << 32, 64, 2, False),
    (1 << 32, 1 << 32, 64, 0, True),    # 64-bit coefficients: n = 2^32
    (1 << 33, 1 << 33, 64, 0, False),   # n = 2^33 > v2(p - 1) = 32
    (1 << 15, 1 << 15, 32, 0, True),
    (1 << 23, 1 << 23, 32, 0, True),    # 2^24 16-bit coefficients each -> n = 2^25
    (1 << 24, 1 << 23, 32, 0, False),   # n = 2^26 is beyond the 32-bit path
    (0, 5, 64, 0, False), (5, 0, 32, 0, False),
])
def test_size_supported(la, lb, path, K, ok):
    good, why = bw.size_supported(la, lb, path, K)
    assert good == ok
    if not ok:
        assert why


def test_bad_arguments_are_reported_not_fatal():
    h = ctypes.c_void_p()
    assert bw.lib.bw_plan_create(ctypes.byref(h), 17, 4, 4, 0, 0) == _lib.BW_EINVAL
    assert "path" in _lib.last_error()
    assert bw.lib.bw_plan_create(ctypes.byref(h), 64, 4, 4, 5, 0) == _lib.BW_EINVAL
    assert bw.lib.bw_plan_create(ctypes.byref(h), 64, 0, 4, 0, 0) == _lib.BW_ESIZE
    assert bw.lib.bw_plan_create(None, 64, 4, 4, 0, 0) == _lib.BW_EINVAL
    with pytest.raises(bw.BwError) as e:
        bw.Plan(1 << 32, 1 << 32, bw.BW_PATH_P64, 2)   # n = 2^33 > v2(p - 1) = 32
    assert e.value.code == _lib.BW_ESIZE
    # 64-bit coefficients halve n: 2^33-word operands need n = 2^33
    with pytest.raises(bw.BwError) as e:
        bw.Plan(1 << 33, 1 << 33, bw.BW_PATH_P64)
    assert e.value.code == _lib.BW_ESIZE


def test_limb_conversions():
    import numpy as np
    x = (1 << 200) + 12345
    w = bw.int_to_limbs(x)
    assert w.dtype == np.uint32 and bw.limbs_to_int(w) == x
    assert bw.limbs_to_int(bw.int_to_limbs(7, 4)) == 7
    assert bw.limbs_to_int(np.array([1, 2], dtype=np.uint64)) == 1 + (2 << 64)


def test_tune_table_entries():
    # host-side table (no GPU): an entry with the row radix round-trips through
    # the JSON export, and a radix other than 0, 8 or 16 is refused
    bw.set_tune_entry(64, 2, 30, False, 15, 16)
    bw.set_tune_entry(32, 2, 30, True)
    table = {(e["path"], e["log_n"]): e for e in bw.tune_table()}
    assert table[(64, 30)]["log_cols"] == 15 and table[(64, 30)]["row_radix"] == 16
    assert table[(32, 30)]["small"] == 1 and table[(32, 30)]["row_radix"] == 0
    with pytest.raises(bw.BwError) as e:
        bw.set_tune_entry(64, 2, 30, False, 15, 32)
    assert e.value.code == _lib.BW_EINVAL
    bw.load_tune_table([table[(64, 30)]])
    assert {(e["path"], e["log_n"]): e for e in bw.tune_table()}[(64, 30)]["row_radix"] == 16
