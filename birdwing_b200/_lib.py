"""ctypes binding of libbirdwing.so (the C ABI declared in include/birdwing.h).

Importing this module loads the in-tree shared library.  There is no
fallback: if the library is missing the import fails with a message that
says how to build it.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbirdwing.so")

BW_OK = 0
BW_EINVAL = -1
BW_ENOMEM = -2
BW_ECUDA = -3
BW_ETIMEOUT = -4
BW_EREJECT = -5
BW_ESIZE = -6
BW_ECHECK = -7
BW_EBUSY = -8

BW_PATH_AUTO = 0
BW_PATH_P32 = 32
BW_PATH_P64 = 64

BW_PTR_HOST = 0
BW_PTR_DEVICE = 1
BW_PTR_HOST_ASYNC = 2

BW_PLAN_RADIX8 = 1 << 16
BW_PLAN_TW_SMEM = 1 << 17
BW_PLAN_THREE_PASS = 1 << 18
BW_PLAN_WIDE_COLS = 1 << 19
BW_PLAN_COEF64 = 1 << 20
BW_PLAN_RADIX16 = 1 << 21
BW_PLAN_COL_RADIX8 = 1 << 22
BW_PLAN_TMA_COLS = 1 << 23
BW_PLAN_NO_TMA_COLS = 1 << 24
BW_PLAN_SHFL_ROWS = 1 << 25
BW_PLAN_K1_ONE_PRIME = 1 << 26

BW_BATCH_THREE_PRIMES = 1
BW_BATCH_PERSISTENT = 2
BW_BATCH_UPLOAD = 1
BW_BATCH_COMPUTE = 2
BW_BATCH_DOWNLOAD = 4

_NAMES = {
    BW_EINVAL: "BW_EINVAL", BW_ENOMEM: "BW_ENOMEM", BW_ECUDA: "BW_ECUDA",
    BW_ETIMEOUT: "BW_ETIMEOUT", BW_EREJECT: "BW_EREJECT", BW_ESIZE: "BW_ESIZE",
    BW_ECHECK: "BW_ECHECK", BW_EBUSY: "BW_EBUSY",
}


class BwError(RuntimeError):
    """A negative status from the C ABI, with bw_last_error()'s message."""

    def __init__(self, code, msg):
        super().__init__(f"{_NAMES.get(code, code)}: {msg}")
        self.code = code


class bw_timing(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in
                ("h2d_ms", "fwd_ms", "mul_ms", "intt_ms", "crt_carry_ms", "d2h_ms", "total_ms")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class bw_plan_info(ctypes.Structure):
    _fields_ = [
        ("path", ctypes.c_int), ("num_primes", ctypes.c_int), ("log_n", ctypes.c_int),
        ("log_rows", ctypes.c_int), ("log_cols", ctypes.c_int), ("coeff_bits", ctypes.c_int),
        ("la", ctypes.c_size_t), ("lb", ctypes.c_size_t), ("lc", ctypes.c_size_t),
        ("plan_device_bytes", ctypes.c_size_t), ("ctx_device_bytes", ctypes.c_size_t),
        ("primes", ctypes.c_uint64 * 6),
    ]


class bw_limits_info(ctypes.Structure):
    _fields_ = [("path", ctypes.c_int), ("num_primes", ctypes.c_int),
                ("max_log_n", ctypes.c_int), ("max_square_words", ctypes.c_size_t)]


class bw_batch_info(ctypes.Structure):
    _fields_ = [(n, ctypes.c_size_t) for n in
                ("products", "buckets", "small_buckets", "graph_nodes", "device_bytes",
                 "kernel_nodes")]


class bw_server_config(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("pinned_bytes", ctypes.c_size_t),
                ("lanes", ctypes.c_int), ("max_groups_in_flight", ctypes.c_int),
                ("num_primes", ctypes.c_int), ("path", ctypes.c_int)]


class bw_request_info(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("status", ctypes.c_int),
                ("submit_us", ctypes.c_double), ("admit_us", ctypes.c_double),
                ("launch_us", ctypes.c_double), ("done_us", ctypes.c_double),
                ("group_size", ctypes.c_size_t), ("device_bytes", ctypes.c_size_t),
                ("la", ctypes.c_size_t), ("lb", ctypes.c_size_t)]


class bw_server_stats(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_uint64) for n in ("submitted", "completed", "rejected", "failed",
                                                  "groups", "kernel_launches")] +
                [(n, ctypes.c_size_t) for n in ("max_group_size", "bytes_in_flight",
                                                 "peak_bytes_in_flight", "resident_plan_bytes",
                                                 "queue_depth", "groups_in_flight",
                                                 "budget_bytes")])


# symbol -> (restype, argtypes)
_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_I = ctypes.c_int
_U = ctypes.c_uint
SIGNATURES = {
    "bw_abi_version": (_I, []),
    "bw_last_error": (ctypes.c_char_p, []),
    "bw_limits": (_I, [_I, _I, ctypes.POINTER(bw_limits_info)]),
    "bw_size_supported": (_I, [_I, _I, _SZ, _SZ]),
    "bw_plan_create": (_I, [ctypes.POINTER(_P), _I, _SZ, _SZ, _I, _U]),
    "bw_plan_destroy": (_I, [_P]),
    "bw_plan_get_info": (_I, [_P, ctypes.POINTER(bw_plan_info)]),
    "bw_ctx_create": (_I, [ctypes.POINTER(_P), _P, _P]),
    "bw_ctx_destroy": (_I, [_P]),
    "bw_ctx_stream": (_P, [_P]),
    "bw_ctx_sync": (_I, [_P]),
    "bw_multiply": (_I, [_P, _P, _SZ, _P, _SZ, _P, _SZ, _U, ctypes.POINTER(bw_timing)]),
    "bw_square": (_I, [_P, _P, _SZ, _P, _SZ, _U, ctypes.POINTER(bw_timing)]),
    "bw_multiply_coeffs": (_I, [_P, _P, _SZ, _P, _SZ, _P, _SZ]),
    "bw_garner_carry_noalloc": (_I, [_I, _I, _P, _SZ, _P, _SZ, _P]),
    "bw_ctx_set_wait_limit": (_I, [_P, _I]),
    "bw_ctx_set_copy_chunks": (_I, [_P, _I]),
    "bw_ctx_inject_wait_fault": (_I, [_P, _I]),
    "bw_multiply_host_once": (_I, [_P, _SZ, _P, _SZ, _P, _SZ, _I,
                                   ctypes.POINTER(ctypes.c_float)]),
    "bw_host_once_cache_limit": (_I, [_SZ]),
    "bw_batch_create": (_I, [ctypes.POINTER(_P), _P, _U]),
    "bw_batch_destroy": (_I, [_P]),
    "bw_batch_clear": (_I, [_P]),
    "bw_batch_add": (_I, [_P, _I, _P, _SZ, _P, _SZ, _P, _SZ]),
    "bw_batch_run": (_I, [_P, _U, ctypes.POINTER(bw_timing)]),
    "bw_batch_get_info": (_I, [_P, ctypes.POINTER(bw_batch_info)]),
    "bw_batch_autotune": (_I, [_P, _I]),
    "bw_batch_set_wait_limit": (_I, [_P, _I]),
    "bw_batch_inject_wait_fault": (_I, [_P, _I]),
    "bw_tune_table_export": (_I, [ctypes.c_char_p, _SZ, ctypes.POINTER(_SZ)]),
    "bw_tune_table_set": (_I, [_I, _I, _I, _I, _I, _I]),
    "bw_server_create": (_I, [ctypes.POINTER(_P), ctypes.POINTER(bw_server_config)]),
    "bw_server_destroy": (_I, [_P]),
    "bw_server_prewarm": (_I, [_P, _I, _I]),
    "bw_server_submit": (_I, [_P, _I, _P, _SZ, _P, _SZ, _P, _SZ,
                              ctypes.POINTER(ctypes.c_uint64)]),
    "bw_server_wait": (_I, [_P, ctypes.c_uint64, _I, ctypes.POINTER(bw_request_info)]),
    "bw_server_harvest": (_I, [_P, ctypes.POINTER(bw_request_info), _SZ,
                               ctypes.POINTER(_SZ)]),
    "bw_server_drain": (_I, [_P, _I]),
    "bw_server_get_stats": (_I, [_P, ctypes.POINTER(bw_server_stats)]),
    "bw_butterfly_rate": (_I, [_I, _I, _I, ctypes.POINTER(ctypes.c_float),
                               ctypes.POINTER(ctypes.c_double)]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python birdwing_b200/build.py` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error():
    return lib.bw_last_error().decode(errors="replace")


def check(rc):
    if rc != BW_OK:
        raise BwError(rc, last_error())
    return rc
