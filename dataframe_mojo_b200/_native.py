"""ctypes binding of libdfcuda.so (include/dfcuda.h).

The library is loaded from this package directory only; when it is missing the
import of any provider entry point that needs it raises.  There is no CPU
fallback anywhere in the provider.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libdfcuda.so"

ABI_VERSION = 1

# dfc_status
OK, UNSUPPORTED, INVALID, DATA_OVERFLOW, DATA_FAULT, CAPACITY, OOM, TIMEOUT, DEVICE, NO_DEVICE = range(10)

# dfc_dtype
INT8, INT16, INT32, INT64, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64 = range(1, 11)

# predicate kinds / comparisons
PRED_CMP, PRED_IS_NULL, PRED_IS_NOT_NULL, PRED_AND, PRED_OR, PRED_NOT, PRED_TRUE = range(1, 8)
LT, LE, GT, GE, EQ, NE = range(1, 7)

# aggregations
AGG_COUNT, AGG_SUM, AGG_MEAN, AGG_MIN, AGG_MAX, AGG_VAR, AGG_STD, AGG_LEN, AGG_NULL_COUNT = range(1, 10)
AGG_FIRST, AGG_LAST, AGG_N_UNIQUE = 10, 11, 12

# query flags
Q_MAINTAIN_ORDER = 1
Q_FORCE_GLOBAL = 2
Q_FORCE_SHARED = 4
Q_FORCE_PARTITIONED = 16
Q_FLOAT32_COMPENSATED = 8

COLUMN_HOST = 0
COLUMN_DEVICE = 1


class Lit(C.Union):
    _fields_ = [("i", C.c_int64), ("u", C.c_uint64), ("f", C.c_double)]


class PredOp(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("column", C.c_int32),
        ("cmp", C.c_int32),
        ("reserved", C.c_int32),
        ("lit", Lit),
    ]


class Agg(C.Structure):
    _fields_ = [("op", C.c_int32), ("column", C.c_int32), ("ddof", C.c_int32), ("min_count", C.c_int32)]


class Query(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("flags", C.c_uint32),
        ("n_inputs", C.c_int32),
        ("n_keys", C.c_int32),
        ("inputs", C.POINTER(C.c_void_p)),
        ("keys", C.POINTER(C.c_int32)),
        ("n_pred", C.c_int32),
        ("n_aggs", C.c_int32),
        ("pred", C.POINTER(PredOp)),
        ("aggs", C.POINTER(Agg)),
        ("stream", C.c_void_p),
    ]


class DeviceInfo(C.Structure):
    _fields_ = [
        ("ordinal", C.c_int32),
        ("sm_count", C.c_int32),
        ("cc_major", C.c_int32),
        ("cc_minor", C.c_int32),
        ("total_bytes", C.c_uint64),
        ("budget_bytes", C.c_int64),
        ("name", C.c_char * 96),
    ]


class Timings(C.Structure):
    _fields_ = [
        ("scan_ns", C.c_double),
        ("finish_ns", C.c_double),
        ("total_ns", C.c_double),
        ("groups", C.c_uint64),
        ("table_slots", C.c_uint64),
        ("regime", C.c_int32),
        ("retries", C.c_int32),
        ("launches", C.c_int32),
        ("partitions", C.c_int32),
        ("aggregate_ns", C.c_double),
        ("cluster_ctas", C.c_int32),
        ("compensated", C.c_int32),
        ("count_ns", C.c_double),
        ("place_ns", C.c_double),
        ("kept_rows", C.c_uint64),
        ("placed_row_bytes", C.c_uint64),
        ("direct_slots", C.c_uint64),
    ]


class ByteCostC(C.Structure):
    """dfc_byte_cost."""

    _fields_ = [("fixed_ns", C.c_double), ("ns_per_byte", C.c_double)]


class DeviceColumnDesc(C.Structure):
    """dfc_device_column: a column in device memory, read in place."""

    _fields_ = [("dtype", C.c_int32), ("reserved", C.c_int32), ("values", C.c_void_p), ("validity", C.c_void_p)]


class DeviceOutput(C.Structure):
    """dfc_device_output: caller-owned device buffers of one output column."""

    _fields_ = [("values", C.c_void_p), ("validity", C.c_void_p), ("dtype", C.c_int32), ("has_nulls", C.c_int32)]


class Completion(C.Structure):
    """dfc_completion: one finished served request."""

    _fields_ = [
        ("tag", C.c_uint64),
        ("status", C.c_int32),
        ("reserved", C.c_int32),
        ("result", C.c_void_p),
        ("latency_ns", C.c_double),
        ("queue_ns", C.c_double),
        ("message", C.c_char * 160),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("pending", C.c_uint64),
        ("inflight", C.c_uint64),
        ("max_inflight_seen", C.c_int64),
        ("bytes_held", C.c_int64),
        ("budget", C.c_int64),
    ]


# Bytes of the fixed working-memory array behind dfc_groupby_noalloc.
NOALLOC_SCRATCH_BYTES = 64 << 20


# (name, restype, argtypes) of every entry point include/dfcuda.h declares.
SIGNATURES = [
    ("dfc_version", C.c_uint32, []),
    ("dfc_installed", C.c_int32, []),
    ("dfc_device_count", C.c_int32, []),
    ("dfc_device_info_get", C.c_int, [C.c_int32, C.POINTER(DeviceInfo)]),
    ("dfc_set_memory_limit", C.c_int, [C.c_int32, C.c_int64]),
    (
        "dfc_column_register",
        C.c_int,
        [C.c_int32, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(C.c_void_p)],
    ),
    ("dfc_column_release", C.c_int, [C.c_void_p]),
    ("dfc_column_rows", C.c_uint64, [C.c_void_p]),
    ("dfc_column_null_count", C.c_int32, [C.c_void_p]),
    ("dfc_groupby", C.c_int, [C.POINTER(Query), C.POINTER(C.c_void_p)]),
    (
        "dfc_groupby_noalloc",
        C.c_int,
        [C.POINTER(Query), C.c_int32, C.c_uint64, C.POINTER(DeviceColumnDesc), C.c_uint64, C.POINTER(DeviceOutput),
         C.POINTER(C.c_uint64)],
    ),
    ("dfc_groupby_batch", C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int)]),
    ("dfc_batch_error", C.c_char_p, [C.c_int32]),
    ("dfc_server_create", C.c_int, [C.c_int32, C.c_int32, C.c_int64, C.POINTER(C.c_void_p)]),
    ("dfc_server_submit", C.c_int, [C.c_void_p, C.POINTER(Query), C.c_uint64]),
    ("dfc_server_poll", C.c_int32, [C.c_void_p, C.POINTER(Completion), C.c_int32, C.c_int32]),
    ("dfc_server_stats_get", C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    ("dfc_server_destroy", None, [C.c_void_p]),
    ("dfc_result_rows", C.c_uint64, [C.c_void_p]),
    ("dfc_result_columns", C.c_int32, [C.c_void_p]),
    (
        "dfc_result_column",
        C.c_int,
        [C.c_void_p, C.c_int32, C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)],
    ),
    ("dfc_result_copy_to_host", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    ("dfc_result_copy_to_device", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    ("dfc_measure_transfer", C.c_int, [C.c_int32, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("dfc_result_free", None, [C.c_void_p]),
    ("dfc_result_residence", C.c_void_p, [C.c_void_p, C.c_int32]),
    ("dfc_result_validity_residence", C.c_void_p, [C.c_void_p, C.c_int32]),
    ("dfc_residence_to_host", C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64]),
    ("dfc_residence_release", None, [C.c_void_p]),
    ("dfc_last_timings", C.c_int, [C.POINTER(Timings)]),
    ("dfc_set_thread_stream", C.c_int, [C.c_int32, C.c_void_p]),
    ("dfc_last_error", C.c_char_p, []),
    ("dfc_status_name", C.c_char_p, [C.c_int]),
]

_lock = threading.Lock()
_lib = None


def library_present() -> bool:
    return LIB_PATH.exists()


def lib() -> C.CDLL:
    """The loaded library; raises when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m dataframe_mojo_b200.build` "
                    "(the provider has no CPU fallback)"
                )
            handle = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
            for name, res, args in SIGNATURES:
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            if handle.dfc_version() != ABI_VERSION:
                raise RuntimeError("libdfcuda.so ABI version mismatch")
            _lib = handle
    return _lib


def last_error() -> str:
    msg = lib().dfc_last_error()
    return msg.decode() if msg else ""
