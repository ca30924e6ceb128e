"""ctypes binding of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The provider package never
imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from dataframe_mojo_b200 import _native as N
from dataframe_mojo_b200.frame import Bound, DataFrame, Plan, Series, bind, decode_outputs, np_dtype, pack_validity

LIB_PATH = Path(__file__).resolve().parent / "_build" / "liboracle.so"


class OrcColumn(C.Structure):
    _fields_ = [
        ("dtype", C.c_int32),
        ("rows", C.c_uint64),
        ("values", C.c_void_p),
        ("validity", C.c_void_p),
        ("bit_offset", C.c_uint64),
    ]


class OrcQuery(C.Structure):
    _fields_ = [
        ("flags", C.c_uint32),
        ("n_inputs", C.c_int32),
        ("n_keys", C.c_int32),
        ("inputs", C.POINTER(OrcColumn)),
        ("keys", C.POINTER(C.c_int32)),
        ("n_pred", C.c_int32),
        ("n_aggs", C.c_int32),
        ("pred", C.POINTER(N.PredOp)),
        ("aggs", C.POINTER(N.Agg)),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from dataframe_mojo_b200.build import build_oracle

            build_oracle()
        h = C.CDLL(str(LIB_PATH))
        h.orc_groupby.restype = C.c_int32
        h.orc_groupby.argtypes = [C.POINTER(OrcQuery), C.POINTER(C.c_void_p)]
        h.orc_groupby_parallel.restype = C.c_int32
        h.orc_groupby_parallel.argtypes = [C.POINTER(OrcQuery), C.c_int32, C.POINTER(C.c_void_p)]
        h.orc_result_rows.restype = C.c_uint64
        h.orc_result_rows.argtypes = [C.c_void_p]
        h.orc_result_columns.restype = C.c_int32
        h.orc_result_columns.argtypes = [C.c_void_p]
        h.orc_result_dtype.restype = C.c_int32
        h.orc_result_dtype.argtypes = [C.c_void_p, C.c_int32]
        h.orc_result_values.restype = C.c_void_p
        h.orc_result_values.argtypes = [C.c_void_p, C.c_int32]
        h.orc_result_valid.restype = C.c_void_p
        h.orc_result_valid.argtypes = [C.c_void_p, C.c_int32]
        h.orc_result_first_rows.restype = C.c_void_p
        h.orc_result_first_rows.argtypes = [C.c_void_p]
        h.orc_result_free.restype = None
        h.orc_result_free.argtypes = [C.c_void_p]
        h.orc_error.restype = C.c_char_p
        h.orc_error.argtypes = []
        _lib = h
    return _lib


class OracleError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def run(plan_or_bound, threads: int | None = None):
    """Runs the oracle: sequential when `threads` is None, else the
    multithreaded restatement with that many workers (0 = all).
    Returns (DataFrame, first_rows)."""
    bound = plan_or_bound if isinstance(plan_or_bound, Bound) else bind(
        plan_or_bound.plan if hasattr(plan_or_bound, "plan") else plan_or_bound
    )
    h = lib()
    n = len(bound.series)
    cols = (OrcColumn * n)()
    keep = []
    for i, s in enumerate(bound.series):
        bits = pack_validity(s.valid)
        keep.append(bits)
        cols[i].dtype = N_dtype(s)
        cols[i].rows = len(s)
        cols[i].values = s.values.ctypes.data if len(s) else None
        cols[i].validity = bits.ctypes.data if bits is not None else None
        cols[i].bit_offset = 0
    keys = (C.c_int32 * len(bound.keys))(*bound.keys)
    pred = (N.PredOp * max(1, len(bound.pred)))()
    for i, (kind, column, cmp, (lk, lv)) in enumerate(bound.pred):
        pred[i].kind, pred[i].column, pred[i].cmp = kind, column, cmp
        if lk == "f":
            pred[i].lit.f = lv
        elif lk == "u":
            pred[i].lit.u = lv
        else:
            pred[i].lit.i = lv
    aggs = (N.Agg * max(1, len(bound.aggs)))()
    for i, (op, column, ddof, min_count) in enumerate(bound.aggs):
        aggs[i].op, aggs[i].column, aggs[i].ddof, aggs[i].min_count = op, column, ddof, min_count
    q = OrcQuery()
    q.flags = N.Q_MAINTAIN_ORDER if bound.maintain_order else 0
    q.n_inputs = n
    q.n_keys = len(bound.keys)
    q.inputs = C.cast(cols, C.POINTER(OrcColumn))
    q.keys = C.cast(keys, C.POINTER(C.c_int32))
    q.n_pred = len(bound.pred)
    q.n_aggs = len(bound.aggs)
    q.pred = C.cast(pred, C.POINTER(N.PredOp))
    q.aggs = C.cast(aggs, C.POINTER(N.Agg))
    out = C.c_void_p()
    if threads is None:
        st = h.orc_groupby(C.byref(q), C.byref(out))
    else:
        st = h.orc_groupby_parallel(C.byref(q), threads, C.byref(out))
    if st != 0:
        raise OracleError(st, h.orc_error().decode())
    try:
        rows = int(h.orc_result_rows(out))
        series = []
        for i, name in enumerate(bound.out_names):
            dt = np_dtype(h.orc_result_dtype(out, i))
            vals = np.ctypeslib.as_array(C.cast(h.orc_result_values(out, i), C.POINTER(C.c_uint8)), (rows * dt.itemsize,)) if rows else np.empty(0, np.uint8)
            vals = vals.view(dt).copy()
            valid = np.ctypeslib.as_array(C.cast(h.orc_result_valid(out, i), C.POINTER(C.c_uint8)), (rows,)).astype(bool) if rows else np.empty(0, bool)
            series.append(Series(name, vals, valid.copy()))
        first = (
            np.ctypeslib.as_array(C.cast(h.orc_result_first_rows(out), C.POINTER(C.c_uint64)), (rows,)).copy()
            if rows
            else np.empty(0, np.uint64)
        )
    finally:
        h.orc_result_free(out)
    return decode_outputs(bound, DataFrame(series)), first


def N_dtype(s: Series) -> int:
    from dataframe_mojo_b200.frame import dfc_dtype

    return dfc_dtype(s.dtype)
