"""Python mirror of the reference's host API for the multiply path.

Names follow the reference (nikitaborisov/birdwing):

  * ``host_multiply_merge(A, B)``   -- include/multiply.h:9-23, one-shot product
  * ``Plan``   ~ NTTPrecomputed      -- precompute_ntt + upload_ntt_precomputed
  * ``Context`` ~ NTTContext          -- allocate_ntt_context
  * ``Context.execute``               -- execute_ntt_multiply (incl. the CRT dump)

Operands are little-endian arrays of 32-bit words (numpy uint32); a u64 limb
array (the reference's NATIVE_HOST_LIMBS pipeline) is the same memory viewed
as twice as many u32 words.  Every call goes through libbirdwing.so; errors
raise BwError (the reference prints and calls exit(1) instead,
src/ntt_limits.cpp:256-280).
"""
import ctypes

import numpy as np

from . import _lib as L
from ._lib import BwError, check, lib

__all__ = [
    "Plan", "Context", "host_multiply_merge", "host_multiply_merge_native", "multiply",
    "square", "limits", "size_supported", "int_to_limbs", "limbs_to_int", "BwError", "Batch",
    "tune_table", "set_tune_entry", "load_tune_table", "Server", "host_once_cache_limit",
]


def int_to_limbs(x, n=None):
    """Python int -> little-endian uint32 array (of length n if given)."""
    if x < 0:
        raise ValueError("negative")
    nbytes = max(1, (x.bit_length() + 7) // 8)
    if n is not None:
        nbytes = max(nbytes, 4 * n)
    nbytes = (nbytes + 3) // 4 * 4
    a = np.frombuffer(x.to_bytes(nbytes, "little"), dtype="<u4").copy()
    if n is not None:
        if np.any(a[n:]):
            raise ValueError("value does not fit in n words")
        a = a[:n]
    return a


def limbs_to_int(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.uint32)
    return int.from_bytes(np.ascontiguousarray(a, dtype="<u4").tobytes(), "little")


def _as_u32(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return a.view(np.uint32)
    if a.dtype != np.uint32:
        raise TypeError(f"limbs must be uint32 or uint64, got {a.dtype}")
    return a


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def limits(path=L.BW_PATH_P64, num_primes=0):
    info = L.bw_limits_info()
    check(lib.bw_limits(path, num_primes, ctypes.byref(info)))
    return {"path": info.path, "num_primes": info.num_primes, "max_log_n": info.max_log_n,
            "max_square_words": info.max_square_words}


def size_supported(la, lb, path=L.BW_PATH_AUTO, num_primes=0):
    """(ok, why) -- reference: multiply_size_supported(L_A, L_B, &why)."""
    rc = lib.bw_size_supported(path, num_primes, la, lb)
    return rc == L.BW_OK, ("" if rc == L.BW_OK else L.last_error())


class Plan:
    """Per-size tables on the device (twiddles, Garner constants)."""

    def __init__(self, la, lb, path=L.BW_PATH_AUTO, num_primes=0, log_cols=0, flags=0):
        h = ctypes.c_void_p()
        flags = flags | ((log_cols & 0x1F) << 8)
        check(lib.bw_plan_create(ctypes.byref(h), path, la, lb, num_primes, flags))
        self._h = h
        info = L.bw_plan_info()
        check(lib.bw_plan_get_info(self._h, ctypes.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in L.bw_plan_info._fields_ if f != "primes"}
        self.info["primes"] = [int(p) for p in info.primes[: info.num_primes]]
        self.la, self.lb = la, lb
        self.N = 1 << info.log_n
        self.logN = info.log_n

    def close(self):
        if self._h:
            lib.bw_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Context:
    """Device scratch + stream for products of one plan's size."""

    def __init__(self, plan, stream=None):
        h = ctypes.c_void_p()
        check(lib.bw_ctx_create(ctypes.byref(h), plan._h, ctypes.c_void_p(stream or 0)))
        self._h = h
        self.plan = plan

    @property
    def stream(self):
        return lib.bw_ctx_stream(self._h)

    def close(self):
        if self._h:
            lib.bw_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def multiply(self, a, b, out=None, timing=False):
        """Host arrays in, host array out (copies and synchronises)."""
        a = _as_u32(a)
        b = _as_u32(b)
        lc = a.size + b.size
        if out is None:
            out = np.empty(lc, dtype=np.uint32)
        t = L.bw_timing()
        same = a is b
        check(lib.bw_multiply(self._h, _ptr(a), a.size, _ptr(a) if same else _ptr(b), b.size,
                              _ptr(out), out.size, L.BW_PTR_HOST,
                              ctypes.byref(t) if timing else None))
        return (out, t.as_dict()) if timing else out

    def square(self, a, out=None, timing=False):
        a = _as_u32(a)
        if out is None:
            out = np.empty(2 * a.size, dtype=np.uint32)
        t = L.bw_timing()
        check(lib.bw_square(self._h, _ptr(a), a.size, _ptr(out), out.size, L.BW_PTR_HOST,
                            ctypes.byref(t) if timing else None))
        return (out, t.as_dict()) if timing else out

    def multiply_async(self, a, b, out):
        """Host arrays (pinned for real overlap): enqueue copy-in, product and
        copy-out and return at once; the arrays must stay alive and unchanged
        until sync()."""
        a = _as_u32(a)
        b = a if b is a else _as_u32(b)
        check(lib.bw_multiply(self._h, _ptr(a), a.size, _ptr(b), b.size, _ptr(out), out.size,
                              L.BW_PTR_HOST_ASYNC, None))
        return out

    def multiply_device(self, a_ptr, la, b_ptr, lb, c_ptr, lc, timing=False):
        """Device pointers (ints); enqueues on the context stream."""
        t = L.bw_timing()
        check(lib.bw_multiply(self._h, ctypes.c_void_p(a_ptr), la, ctypes.c_void_p(b_ptr), lb,
                              ctypes.c_void_p(c_ptr), lc, L.BW_PTR_DEVICE,
                              ctypes.byref(t) if timing else None))
        return t.as_dict() if timing else None

    def sync(self):
        check(lib.bw_ctx_sync(self._h))

    def set_copy_chunks(self, chunks):
        """Chunks of host copies overlapped with the first and last kernels
        (0: automatic, 1: whole copies)."""
        check(lib.bw_ctx_set_copy_chunks(self._h, chunks))

    def coeffs(self, a, b):
        """Convolution coefficients after Garner, as Python ints (length n)."""
        a = _as_u32(a)
        b = _as_u32(b)
        n = self.plan.N
        w = np.empty(3 * n, dtype=np.uint32)
        same = a is b
        check(lib.bw_multiply_coeffs(self._h, _ptr(a), a.size, _ptr(a) if same else _ptr(b),
                                     b.size, _ptr(w), w.size))
        w = w.reshape(n, 3).astype(object)
        return [int(r[0]) | (int(r[1]) << 32) | (int(r[2]) << 64) for r in w]

    # reference spelling: execute_ntt_multiply(ctx, a, b, C_out, timing)
    def execute(self, a, b, timing=False):
        return self.multiply(a, b, timing=timing)


def multiply(a, b, path=L.BW_PATH_AUTO):
    """One-shot product of two uint32 arrays (plan and context cached per size)."""
    a = _as_u32(a)
    b = _as_u32(b)
    out = np.empty(a.size + b.size, dtype=np.uint32)
    ms = ctypes.c_float()
    check(lib.bw_multiply_host_once(_ptr(a), a.size, _ptr(b), b.size, _ptr(out), out.size, path,
                                    ctypes.byref(ms)))
    return out


def host_once_cache_limit(nbytes):
    """Device memory kept by the one-shot calls' plan/context cache
    (``multiply``, ``host_multiply_merge``); 0 frees it and turns it off."""
    check(lib.bw_host_once_cache_limit(int(nbytes)))


def square(a, path=L.BW_PATH_AUTO):
    with Plan(len(a), len(a), path) as p, Context(p) as c:
        return c.square(a)


def host_multiply_merge(A, B):
    """Reference: host_multiply_merge (src/host_multiply.cpp:27-86).  Returns
    (C, duration_ms) with C of length len(A) + len(B)."""
    A = np.asarray(A, dtype=np.uint32)
    B = np.asarray(B, dtype=np.uint32)
    out = np.empty(A.size + B.size, dtype=np.uint32)
    ms = ctypes.c_float()
    check(lib.bw_multiply_host_once(_ptr(A), A.size, _ptr(B), B.size, _ptr(out), out.size,
                                    L.BW_PATH_AUTO, ctypes.byref(ms)))
    return out, ms.value


def host_multiply_merge_native(A, B):
    """Reference: host_multiply_merge_native (src/host_multiply.cpp:90-134):
    u64 limbs in, u64 limbs out."""
    A = np.ascontiguousarray(A, dtype=np.uint64)
    B = np.ascontiguousarray(B, dtype=np.uint64)
    out, ms = host_multiply_merge(A.view(np.uint32), B.view(np.uint32))
    return out.view(np.uint64), ms


class Batch:
    """Many independent products of uneven sizes run together (bw_batch_*).

    ``add`` keeps references to the host arrays: every ``run`` re-reads the
    operands and rewrites the outputs, so a caller can refill the same arrays
    and run again (the captured graph is replayed while the list of products
    is unchanged).  The reference has no batched form; its unit is one
    host_multiply_merge call per product.
    """

    def __init__(self, num_primes=2, stream=None, persistent=False):
        h = ctypes.c_void_p()
        flags = L.BW_BATCH_THREE_PRIMES if num_primes == 3 else 0
        if persistent:
            flags |= L.BW_BATCH_PERSISTENT
        check(lib.bw_batch_create(ctypes.byref(h), ctypes.c_void_p(stream or 0), flags))
        self._h = h
        self._keep = []
        self.outputs = []

    def add(self, a, b, out=None, path=L.BW_PATH_AUTO):
        """Append a * b; returns the output array (len(a) + len(b) words)."""
        a = _as_u32(a)
        b = a if b is a else _as_u32(b)
        if out is None:
            out = np.zeros(a.size + b.size, dtype=np.uint32)
        check(lib.bw_batch_add(self._h, path, _ptr(a), a.size, _ptr(b), b.size, _ptr(out),
                               out.size))
        self._keep.append((a, b, out))
        self.outputs.append(out)
        return out

    def clear(self):
        check(lib.bw_batch_clear(self._h))
        self._keep = []
        self.outputs = []

    def run(self, what=0, timing=False):
        t = L.bw_timing()
        check(lib.bw_batch_run(self._h, what, ctypes.byref(t) if timing else None))
        return t.as_dict() if timing else None

    def info(self):
        i = L.bw_batch_info()
        check(lib.bw_batch_get_info(self._h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in L.bw_batch_info._fields_}

    def autotune(self, reps=3):
        check(lib.bw_batch_autotune(self._h, reps))

    def set_wait_limit(self, polls):
        """Test hook: polls a look-back wait may take before BW_ETIMEOUT."""
        check(lib.bw_batch_set_wait_limit(self._h, polls))

    def inject_wait_fault(self, enable=True):
        """Test hook: make every look-back wait of the 4-step groups run out."""
        check(lib.bw_batch_inject_wait_fault(self._h, 1 if enable else 0))

    def close(self):
        if self._h:
            lib.bw_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def tune_table():
    """The process-wide batch tune table (list of dicts)."""
    import json
    need = ctypes.c_size_t()
    check(lib.bw_tune_table_export(None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(need.value)
    check(lib.bw_tune_table_export(buf, need.value, ctypes.byref(need)))
    return json.loads(buf.value.decode())


def set_tune_entry(path, num_primes, log_n, small, log_cols=0, row_radix=0):
    """One tune-table entry: one CTA per product (small), or the 4-step
    kernels with 2^log_cols columns (0: automatic) and row rounds of radix
    row_radix (8 or 16; 0: the path's default)."""
    check(lib.bw_tune_table_set(path, num_primes, log_n, 1 if small else 0, log_cols,
                                row_radix))


def load_tune_table(entries):
    """Install entries as produced by tune_table() (e.g. read back from JSON)."""
    for e in entries:
        set_tune_entry(e["path"], e["num_primes"], e["log_n"], e["small"], e["log_cols"],
                       e.get("row_radix", 0))


class Server:
    """Request loop with continuous batching (bw_server_*).

    ``submit`` queues a product and returns a ticket at once; the library's
    own threads admit requests by device bytes, batch the ones that wait
    together, and finish them asynchronously.  The operand and output arrays
    are kept referenced here until the request is waited for or harvested.
    """

    def __init__(self, hbm_budget=0, pinned=0, lanes=0, max_groups=0, num_primes=2,
                 path=L.BW_PATH_AUTO):
        cfg = L.bw_server_config(hbm_budget, pinned, lanes, max_groups, num_primes, path)
        h = ctypes.c_void_p()
        check(lib.bw_server_create(ctypes.byref(h), ctypes.byref(cfg)))
        self._h = h
        self._live = {}

    def prewarm(self, max_log_n, path=L.BW_PATH_AUTO):
        check(lib.bw_server_prewarm(self._h, path, max_log_n))

    def submit(self, a, b, out=None, path=L.BW_PATH_AUTO):
        a = _as_u32(a)
        b = a if b is a else _as_u32(b)
        if out is None:
            out = np.zeros(a.size + b.size, dtype=np.uint32)
        t = ctypes.c_uint64()
        check(lib.bw_server_submit(self._h, path, _ptr(a), a.size, _ptr(b), b.size, _ptr(out),
                                   out.size, ctypes.byref(t)))
        self._live[t.value] = (a, b, out)
        return t.value

    @staticmethod
    def _info(i):
        return {f: getattr(i, f) for f, _ in L.bw_request_info._fields_}

    def wait(self, ticket, timeout_ms=-1):
        """(out, info) of one request; raises BwError if it failed or, with a
        timeout, has not finished (it then stays queued)."""
        info = L.bw_request_info()
        rc = lib.bw_server_wait(self._h, ticket, timeout_ms, ctypes.byref(info))
        if rc != L.BW_OK and info.ticket == 0:
            raise L.BwError(rc, L.last_error())
        _, _, out = self._live.pop(ticket, (None, None, None))
        check(rc)
        return out, self._info(info)

    def harvest(self, max_items=4096):
        """Finished requests (any order) as info dicts, each with its 'out'."""
        buf = (L.bw_request_info * max_items)()
        n = ctypes.c_size_t()
        check(lib.bw_server_harvest(self._h, buf, max_items, ctypes.byref(n)))
        res = []
        for i in range(n.value):
            d = self._info(buf[i])
            d["out"] = self._live.pop(d["ticket"], (None, None, None))[2]
            res.append(d)
        return res

    def harvest_arrays(self, max_items=8192):
        """Finished requests as numpy columns (ticket, status, submit_us,
        admit_us, launch_us, done_us, group_size) plus their output arrays,
        for clients that handle many results per call."""
        buf = (L.bw_request_info * max_items)()
        n = ctypes.c_size_t()
        check(lib.bw_server_harvest(self._h, buf, max_items, ctypes.byref(n)))
        dt = np.dtype({"names": [f for f, _ in L.bw_request_info._fields_],
                       "formats": ["<u8", "<i4", "<f8", "<f8", "<f8", "<f8", "<u8", "<u8",
                                   "<u8", "<u8"],
                       "offsets": [getattr(L.bw_request_info, f).offset
                                   for f, _ in L.bw_request_info._fields_],
                       "itemsize": ctypes.sizeof(L.bw_request_info)})
        rec = np.frombuffer(buf, dtype=dt, count=n.value).copy()
        outs = [self._live.pop(int(t), (None, None, None))[2] for t in rec["ticket"]]
        return rec, outs

    def drain(self, timeout_ms=-1):
        check(lib.bw_server_drain(self._h, timeout_ms))

    def stats(self):
        st = L.bw_server_stats()
        check(lib.bw_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in L.bw_server_stats._fields_}

    def close(self):
        if self._h:
            lib.bw_server_destroy(self._h)
            self._h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
