"""The provider interface, mirrored: the thirteen functions the reference core
calls through dataframe/_accel_provider.mojo:10-27, with the behaviour the
contract gives them (docs/design/accelerator-contract.md:22-70), backed by
libdfcuda.so.

    installed execute describe execute_profiled
    handoff_supports handoff_execute handoff_estimate
    devices transfer_model pipeline_supports pipeline_estimate pipeline_costs run_pipeline

Plus the resident-table form (columns registered once, queried many times),
which is what `run_pipeline` over device-resident inputs means for a
discrete device (dataframe/storage/residence.mojo:33-147).

Errors: unsupported work raises ``UnsupportedError`` before anything is
submitted; checked-sum overflow raises ``ProviderError`` with the CPU
provider's exact text; a data fault (``DataFaultError``) asks the caller to
let the CPU adjudicate, as the reference's data-fault marker does
(dataframe_metal/accelerator/faults.mojo:1-18).  The provider itself never
runs anything on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .frame import (Bound, DataFrame, LazyFrame, Plan, Series, bind, bits_all_set, decode_outputs, dfc_dtype,
                    np_dtype, unpack_validity)

BACKEND = "cuda"
MEMORY_DISCRETE = 1
MEMORY_UNIFIED = 2


class ProviderError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class UnsupportedError(ProviderError):
    pass


class DataFaultError(ProviderError):
    pass


def _error(status: int, msg: str) -> ProviderError:
    msg = msg or N.lib().dfc_status_name(status).decode()
    if status in (N.UNSUPPORTED, N.INVALID):
        return UnsupportedError(status, msg)
    if status == N.DATA_FAULT:
        return DataFaultError(status, msg)
    return ProviderError(status, msg)


def _check(status: int) -> None:
    if status == N.OK:
        return
    raise _error(status, N.last_error())


def _device_from_env() -> int:
    """DATAFRAME_ACCEL_DEVICE, the name the reference's providers read
    (docs/design/accelerator-contract.md:168-171); a bad value raises."""
    raw = os.environ.get("DATAFRAME_ACCEL_DEVICE", "")
    if raw == "":
        return 0
    try:
        dev = int(raw)
    except ValueError:
        raise ValueError(f"DATAFRAME_ACCEL_DEVICE={raw!r} is not a device ordinal") from None
    if dev < 0:
        raise ValueError(f"DATAFRAME_ACCEL_DEVICE={raw!r} is negative")
    return dev


def _memory_limit() -> int:
    raw = os.environ.get("DATAFRAME_ACCEL_MEMORY_LIMIT", "")
    if raw == "":
        return -1
    try:
        v = int(raw)
    except ValueError:
        raise ValueError(f"DATAFRAME_ACCEL_MEMORY_LIMIT={raw!r} is not a byte count") from None
    if v <= 0:
        raise ValueError(f"DATAFRAME_ACCEL_MEMORY_LIMIT={raw!r} must be positive")
    return v


_REGIMES = {"": 0, "auto": 0, "global": N.Q_FORCE_GLOBAL, "shared": N.Q_FORCE_SHARED,
            "partitioned": N.Q_FORCE_PARTITIONED}


_FLOAT32 = {"": 0, "fp64": 0, "compensated": N.Q_FLOAT32_COMPENSATED}


def _regime_flags() -> int:
    """DATAFRAME_ACCEL_REGIME: auto (default; chosen from the estimated group
    count), global, shared or partitioned.  DATAFRAME_ACCEL_FLOAT32: fp64
    (default; Float32 sums and variances accumulate in FP64) or compensated
    (compensated FP32 partials in the shared-memory tables, merged in FP64).
    A bad value raises."""
    raw = os.environ.get("DATAFRAME_ACCEL_REGIME", "").strip().lower()
    if raw not in _REGIMES:
        raise ValueError(f"DATAFRAME_ACCEL_REGIME={raw!r} is not one of auto, global, shared, partitioned")
    f32 = os.environ.get("DATAFRAME_ACCEL_FLOAT32", "").strip().lower()
    if f32 not in _FLOAT32:
        raise ValueError(f"DATAFRAME_ACCEL_FLOAT32={f32!r} is not one of fp64, compensated")
    return _REGIMES[raw] | _FLOAT32[f32]


# ---------------------------------------------------------------------------
# Device columns and results.
# ---------------------------------------------------------------------------
class DeviceColumn:
    """A column resident in HBM (values + normalised validity bitmap)."""

    def __init__(self, series: Series, device: int = 0, *, device_pointer: int | None = None):
        lib = N.lib()
        self.name = series.name
        self.dtype = series.dtype
        self.rows = len(series)
        self.device = device
        bits = series.validity_bits()
        handle = C.c_void_p()
        if device_pointer is None:
            values = series.values
            _check(
                lib.dfc_column_register(
                    device,
                    dfc_dtype(values.dtype),
                    self.rows,
                    values.ctypes.data if self.rows else None,
                    bits.ctypes.data if bits is not None else None,
                    0,
                    N.COLUMN_HOST,
                    C.byref(handle),
                )
            )
        else:
            if bits is not None:
                raise UnsupportedError(N.UNSUPPORTED, "device columns take a device validity pointer")
            _check(
                lib.dfc_column_register(
                    device, dfc_dtype(series.dtype), self.rows, device_pointer, None, 0, N.COLUMN_DEVICE, C.byref(handle)
                )
            )
        self.handle = handle

    @classmethod
    def from_host_pointer(cls, name: str, dtype, rows: int, values_ptr: int, validity_ptr: int | None = None,
                          bit_offset: int = 0, device: int = 0) -> "DeviceColumn":
        """Registers host memory (pinned or pageable) without a numpy copy."""
        self = cls.__new__(cls)
        self.name, self.dtype, self.rows, self.device = name, np.dtype(dtype), rows, device
        handle = C.c_void_p()
        _check(
            N.lib().dfc_column_register(
                device, dfc_dtype(dtype), rows, values_ptr, validity_ptr, bit_offset, N.COLUMN_HOST, C.byref(handle)
            )
        )
        self.handle = handle
        return self

    @classmethod
    def from_resident(cls, series: "ResidentSeries", device: int | None = None) -> "DeviceColumn":
        """A resident result column as the input of a following query, read
        in place on the device (no host round trip); the column keeps the
        series, and so its device buffers, alive."""
        self = cls.__new__(cls)
        self.name, self.dtype, self.rows = series.name, series.dtype, len(series)
        self.device = series.device if device is None else device
        self._keep = series
        handle = C.c_void_p()
        _check(
            N.lib().dfc_column_register(
                self.device, dfc_dtype(series.dtype), self.rows, series.device_values if self.rows else None,
                series.device_validity, 0, N.COLUMN_DEVICE, C.byref(handle)
            )
        )
        self.handle = handle
        return self

    @property
    def null_count(self) -> int:
        return int(N.lib().dfc_column_null_count(self.handle)) if self.handle else 0

    def release(self) -> None:
        if self.handle:
            N.lib().dfc_column_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class ResidentSeries(Series):
    """A result column left in device memory, the shape of the reference's
    `_DeviceResidence` (dataframe/storage/residence.mojo:20-72): an opaque
    handle with C-ABI callbacks (dfc_residence_to_host / _release).  The
    first host read of values or validity copies them once, under a lock;
    the device buffers stay until the series is released, so a following
    device query reads them in place (DeviceColumn.from_resident)."""

    def __init__(self, name: str, result: "DeviceResult", i: int):
        lib = N.lib()
        dtype, vals, valid = result.column_info(i)
        self.name = name
        self.categories = None
        self.device = result.device
        self._dtype = np.dtype(dtype)
        self._rows = result.rows
        self.device_values = vals
        self.device_validity = valid
        self._ctx = lib.dfc_result_residence(result.handle, i)
        self._vctx = lib.dfc_result_validity_residence(result.handle, i) if valid else None
        self._lock = threading.Lock()
        self._host = None
        self._bits = None
        self._valid = None

    def on_host(self) -> bool:
        return self._host is not None

    def _copy(self) -> None:
        with self._lock:
            if self._host is not None:
                return
            lib = N.lib()
            values = np.empty(self._rows, dtype=self._dtype)
            if self._rows and lib.dfc_residence_to_host(self._ctx, values.ctypes.data, values.nbytes) != 0:
                raise ProviderError(N.DEVICE, "copying a device result column to the host failed")
            if self._vctx:
                bits = np.empty((self._rows + 7) // 8, dtype=np.uint8)
                if self._rows and lib.dfc_residence_to_host(self._vctx, bits.ctypes.data, bits.nbytes) != 0:
                    raise ProviderError(N.DEVICE, "copying a device validity bitmap to the host failed")
                if not bits_all_set(bits, self._rows):
                    self._bits = bits
            self._host = values

    @property
    def values(self) -> np.ndarray:
        self._copy()
        return self._host

    @property
    def valid(self) -> np.ndarray | None:
        self._copy()
        if self._bits is not None:
            self._valid = unpack_validity(self._bits, self._rows)
            self._bits = None
        return self._valid

    @property
    def dtype(self) -> np.dtype:
        return self._dtype

    def __len__(self) -> int:
        return self._rows

    def release(self) -> None:
        lib = N.lib()
        for attr in ("_ctx", "_vctx"):
            ctx = getattr(self, attr, None)
            if ctx:
                lib.dfc_residence_release(ctx)
                setattr(self, attr, None)

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class DeviceResult:
    """A query result resident on the device: key columns then one column per
    aggregation.  ``to_frame`` copies it to the host."""

    def __init__(self, handle: C.c_void_p, names: list[str], device: int = 0):
        self.handle = handle
        self.names = names
        self.device = device
        self.rows = int(N.lib().dfc_result_rows(handle))

    def column_info(self, i: int) -> tuple[np.dtype, int, int | None]:
        dt = C.c_int()
        vals = C.c_void_p()
        valid = C.c_void_p()
        _check(N.lib().dfc_result_column(self.handle, i, C.byref(dt), C.byref(vals), C.byref(valid)))
        return np_dtype(dt.value), vals.value, valid.value

    def to_resident(self) -> DataFrame:
        """The result as a frame of ResidentSeries: nothing is copied until a
        column is read on the host."""
        return DataFrame([ResidentSeries(name, self, i) for i, name in enumerate(self.names)])

    def to_frame(self, into: dict | None = None) -> DataFrame:
        """Copies the result to host memory.  `into` maps column names to
        (values, bits) host arrays of at least rows elements / ceil(rows/8)
        bytes (pinned memory copies at full speed); the frame then views them."""
        lib = N.lib()
        cols = []
        for i, name in enumerate(self.names):
            dtype, _, dvalid = self.column_info(i)
            if into is not None:
                vbuf, bbuf = into[name]
                if vbuf.dtype != dtype or len(vbuf) < self.rows or len(bbuf) < (self.rows + 7) // 8:
                    raise ValueError(f"buffer for {name!r} is too small or of the wrong type")
                values = vbuf[: self.rows]
                bits = bbuf[: (self.rows + 7) // 8] if dvalid else None
            else:
                values = np.empty(self.rows, dtype=dtype)
                bits = np.empty((self.rows + 7) // 8, dtype=np.uint8) if dvalid else None
            _check(
                lib.dfc_result_copy_to_host(
                    self.handle,
                    i,
                    values.ctypes.data if self.rows else None,
                    bits.ctypes.data if bits is not None and self.rows else None,
                )
            )
            cols.append(Series.from_bits(name, values, bits))
        return DataFrame(cols)

    def free(self) -> None:
        if self.handle:
            N.lib().dfc_result_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _query_struct(bound: Bound, handles: list, stream: int | None, flags: int = 0):
    n = len(handles)
    inputs = (C.c_void_p * n)(*[h.value for h in handles])
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
    q = N.Query()
    q.abi_version = N.ABI_VERSION
    q.flags = flags | (N.Q_MAINTAIN_ORDER if bound.maintain_order else 0)
    q.n_inputs = n
    q.n_keys = len(bound.keys)
    q.inputs = C.cast(inputs, C.POINTER(C.c_void_p))
    q.keys = C.cast(keys, C.POINTER(C.c_int32))
    q.n_pred = len(bound.pred)
    q.n_aggs = len(bound.aggs)
    q.pred = C.cast(pred, C.POINTER(N.PredOp))
    q.aggs = C.cast(aggs, C.POINTER(N.Agg))
    q.stream = stream
    # Keep the arrays alive with the struct.
    q._keep = (inputs, keys, pred, aggs)
    return q


def run_bound(bound: Bound, columns: list[DeviceColumn], stream: int | None = None, flags: int = 0) -> DeviceResult:
    """Runs a bound region over registered columns; the result stays on the device."""
    q = _query_struct(bound, [c.handle for c in columns], stream, flags)
    out = C.c_void_p()
    _check(N.lib().dfc_groupby(C.byref(q), C.byref(out)))
    return DeviceResult(out, bound.out_names, getattr(columns[0], "device", 0) if columns else 0)


def run_batch(jobs: list, stream: int | None = None, flags: int = 0) -> list:
    """Runs many bound regions in one submission (dfc_groupby_batch).  `jobs`
    is a list of (Bound, [DeviceColumn]); returns, per job, a DeviceResult or
    the ProviderError that query raised."""
    qs = [_query_struct(b, [c.handle for c in cols], stream, flags) for b, cols in jobs]
    n = len(qs)
    ptrs = (C.c_void_p * max(1, n))(*[C.cast(C.pointer(q), C.c_void_p) for q in qs])
    outs = (C.c_void_p * max(1, n))()
    sts = (C.c_int * max(1, n))()
    _check(N.lib().dfc_groupby_batch(ptrs, n, outs, sts))
    res = []
    for i, (b, _) in enumerate(jobs):
        if sts[i] == N.OK:
            res.append(DeviceResult(C.c_void_p(outs[i]), b.out_names))
        else:
            res.append(_error(sts[i], N.lib().dfc_batch_error(i).decode()))
    return res


class Server:
    """The served form (dfc_server_*): submit bound regions over registered
    columns; a native worker admits them as in-flight slots and memory allow
    and overlaps their work on the device; poll() returns completions as
    (tag, DeviceResult or ProviderError, latency_ns, queue_ns)."""

    def __init__(self, device: int = 0, max_inflight: int = 64, memory_budget: int = -1):
        h = C.c_void_p()
        _check(N.lib().dfc_server_create(device, max_inflight, memory_budget, C.byref(h)))
        self.handle = h
        self._names: dict[int, list[str]] = {}
        self._buf = (N.Completion * 256)()

    def submit(self, bound: Bound, columns: list, tag: int, flags: int = 0) -> None:
        q = _query_struct(bound, [c.handle for c in columns], None, flags)
        self._names[tag] = bound.out_names
        _check(N.lib().dfc_server_submit(self.handle, C.byref(q), tag))

    def poll(self, wait_ms: int = 0) -> list:
        n = N.lib().dfc_server_poll(self.handle, self._buf, len(self._buf), wait_ms)
        out = []
        for i in range(n):
            c = self._buf[i]
            names = self._names.pop(int(c.tag))
            if c.status == N.OK:
                res = DeviceResult(C.c_void_p(c.result), names)
            else:
                res = _error(c.status, c.message.decode())
            out.append((int(c.tag), res, c.latency_ns, c.queue_ns))
        return out

    def stats(self) -> dict:
        s = N.ServerStats()
        _check(N.lib().dfc_server_stats_get(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.ServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            N.lib().dfc_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def last_timings() -> dict:
    t = N.Timings()
    _check(N.lib().dfc_last_timings(C.byref(t)))
    return {
        "scan_ns": t.scan_ns,
        "finish_ns": t.finish_ns,
        "total_ns": t.total_ns,
        "groups": int(t.groups),
        "table_slots": int(t.table_slots),
        "regime": int(t.regime),
        "retries": int(t.retries),
        "launches": int(t.launches),
        "partitions": int(t.partitions),
        "aggregate_ns": t.aggregate_ns,
        "cluster_ctas": int(t.cluster_ctas),
        "compensated": int(t.compensated),
        "count_ns": t.count_ns,
        "place_ns": t.place_ns,
        "kept_rows": int(t.kept_rows),
        "placed_row_bytes": int(t.placed_row_bytes),
        "direct_slots": int(t.direct_slots),
    }


def set_thread_stream(device: int, stream: int | None) -> None:
    """Routes this thread's library calls on `device` through `stream`."""
    _check(N.lib().dfc_set_thread_stream(device, stream))


class ResidentTable:
    """Columns of a DataFrame registered once and kept resident in HBM, so
    repeated queries move no input bytes (config 5's tables)."""

    def __init__(self, frame: DataFrame, device: int | None = None):
        self.device = _device_from_env() if device is None else device
        self.frame = frame
        self.columns = {name: DeviceColumn(frame.column(name), self.device) for name in frame.columns}

    def run(self, lazy: LazyFrame | Plan, stream: int | None = None, flags: int = 0) -> DeviceResult:
        plan = lazy.plan if isinstance(lazy, LazyFrame) else lazy
        bound = bind(plan)
        return run_bound(bound, [self.columns[n] for n in bound.names], stream, flags)

    def release(self) -> None:
        for c in self.columns.values():
            c.release()
        self.columns = {}


def _region_plan(plan) -> Plan:
    return plan.plan if isinstance(plan, LazyFrame) else plan


def _execute_plan(plan: Plan, device: int) -> DataFrame:
    bound = bind(plan)
    flags = _regime_flags()
    # DATAFRAME_ACCEL_MEMORY_LIMIT bounds each query's device memory: a query
    # that would need more is rejected before submission (DFC_UNSUPPORTED).
    _check(N.lib().dfc_set_memory_limit(device, max(_memory_limit(), 0)))
    cols = [DeviceColumn(s, device) for s in bound.series]
    try:
        result = run_bound(bound, cols, flags=flags)
        _record_run(plan, last_timings()["total_ns"], bound)
        try:
            return decode_outputs(bound, result.to_frame())
        finally:
            result.free()
    finally:
        for c in cols:
            c.release()


def _unsupported_reason(plan: Plan) -> str | None:
    if plan.keys is None:
        return "the region has no aggregation"
    try:
        bound = bind(plan)
    except (TypeError, ValueError, KeyError) as e:
        return str(e)
    if len(bound.keys) > 4:
        return "more than four keys"
    if len(bound.names) > 16:
        return "more than sixteen input columns"
    if len(bound.aggs) > 32:
        return "more than thirty-two aggregations"
    if plan.source.height >= 0xFFFFFFFF:
        return "more than 2^32-2 rows"
    return None


# ---------------------------------------------------------------------------
# The thirteen provider functions.
# ---------------------------------------------------------------------------
def installed() -> bool:
    """Whether the backend could run here; opens no driver and creates no context."""
    if not N.library_present():
        return False
    try:
        return bool(N.lib().dfc_installed())
    except OSError:
        return False


def describe(plan) -> str:
    """``ENGINE accel: ...`` text for explain; never raises and never touches a device."""
    try:
        p = _region_plan(plan)
        reason = _unsupported_reason(p)
        if reason:
            return f"ENGINE accel: rejected ({reason})"
        return f"ENGINE accel: {BACKEND} filtered hash group-by: {p.describe()}"
    except Exception as e:  # describe does not raise
        return f"ENGINE accel: rejected ({e})"


def execute(plan) -> tuple[DataFrame, DataFrame]:
    """Runs the whole plan; returns (result, report).  Unsupported plans raise
    before anything is submitted."""
    p = _region_plan(plan)
    reason = _unsupported_reason(p)
    if reason:
        raise UnsupportedError(N.UNSUPPORTED, f"accelerator cannot run this plan: {reason}")
    device = _device_from_env()
    _memory_limit()
    t0 = time.perf_counter_ns()
    result = _execute_plan(p, device)
    wall = time.perf_counter_ns() - t0
    t = last_timings()
    report = DataFrame(
        [
            Series("engine", np.array([0], np.int32)),
            Series("device", np.array([device], np.int32)),
            Series("groups", np.array([t["groups"]], np.int64)),
            Series("scan_ns", np.array([t["scan_ns"]], np.float64)),
            Series("finish_ns", np.array([t["finish_ns"]], np.float64)),
            Series("wall_ns", np.array([wall], np.float64)),
        ]
    )
    return result, report


def execute_profiled(plan) -> tuple[DataFrame, DataFrame]:
    return execute(plan)


def handoff_supports(region) -> bool:
    """False: the contract asks a provider for a discrete device to decline
    node hand-off (docs/design/accelerator-contract.md:31); whole plans go
    through `execute` and placed pipelines through `run_pipeline`."""
    return False


def handoff_execute(region) -> DataFrame:
    p = _region_plan(region)
    reason = _unsupported_reason(p)
    if reason:
        raise UnsupportedError(N.UNSUPPORTED, f"accelerator cannot run this region: {reason}")
    return _execute_plan(p, _device_from_env())


def handoff_estimate(region, rows: int) -> tuple[str, float]:
    """(calibration key, estimated ns for `rows` input rows, moves included); -1: not measured."""
    p = _region_plan(region)
    key = "cuda:groupby:v1:" + describe(p)
    return key, -1.0


@dataclass
class DeviceInfo:
    backend: str
    ordinal: int
    name: str
    memory: int
    budget_bytes: int
    total_bytes: int
    sm_count: int


@dataclass
class ByteCost:
    """`fixed_ns + ns_per_byte * bytes` nanoseconds; negative: not measured
    (dataframe/devices.mojo:44-56)."""

    fixed_ns: float = -1.0
    ns_per_byte: float = -1.0

    def measured(self) -> bool:
        return self.fixed_ns >= 0 and self.ns_per_byte >= 0

    def cost(self, nbytes: int) -> float:
        return self.fixed_ns + self.ns_per_byte * nbytes


@dataclass
class TransferModel:
    """Host <-> device copy costs measured on this machine
    (dataframe/devices.mojo:59-80); startup_ns is not measured here."""

    to_device: ByteCost = field(default_factory=ByteCost)
    to_host: ByteCost = field(default_factory=ByteCost)
    startup_ns: float = -1.0

    def measured(self) -> bool:
        return self.to_device.measured() and self.to_host.measured()


@dataclass
class PipelineFeatures:
    rows: int = 0
    input_bytes: int = 0
    groups: int = -1


def devices() -> list[DeviceInfo]:
    """Each sm_100 device; reads driver metadata only, creates no context."""
    if not installed():
        return []
    lib = N.lib()
    out = []
    for i in range(lib.dfc_device_count()):
        info = N.DeviceInfo()
        if lib.dfc_device_info_get(i, C.byref(info)) != N.OK:
            continue
        budget = _memory_limit()
        out.append(
            DeviceInfo(
                BACKEND,
                info.ordinal,
                info.name.decode(),
                MEMORY_DISCRETE,
                budget if budget > 0 else int(info.budget_bytes),
                int(info.total_bytes),
                int(info.sm_count),
            )
        )
    return out


_transfer: dict[int, TransferModel] = {}


def calibrate_transfer(device: int, nbytes: int = 1 << 28) -> TransferModel:
    """Measures pinned host <-> device copies once (dfc_measure_transfer) and
    keeps the model for transfer_model()."""
    to_dev, to_host = N.ByteCostC(), N.ByteCostC()
    _check(N.lib().dfc_measure_transfer(device, nbytes, C.byref(to_dev), C.byref(to_host)))
    m = TransferModel(ByteCost(to_dev.fixed_ns, to_dev.ns_per_byte), ByteCost(to_host.fixed_ns, to_host.ns_per_byte))
    _transfer[device] = m
    return m


def transfer_model(device: int) -> TransferModel:
    return _transfer.get(device, TransferModel())


def pipeline_supports(pipeline, device: int) -> bool:
    try:
        return installed() and _unsupported_reason(_region_plan(pipeline)) is None
    except Exception:
        return False


# Device-time calibration, per layout (the region with its literals left
# out): nanoseconds per input byte, from this provider's own timed queries
# (dfc_last_timings total).  Before a layout has run, the model measured for
# this provider on B200: the 100M-row filtered group-by (2.0125 GB of input
# columns) took 7.3 ms, and a query's fixed cost (planning, statistics,
# launches, result) is about 0.3 ms.
_DEFAULT_NS_PER_BYTE = 7.0e6 / 2.0125e9
_FIXED_NS = 3.0e5
_calibration: dict[str, list[float]] = {}
_calibration_lock = threading.Lock()


def _layout_key(plan: Plan) -> str:
    src = plan.source
    cols = sorted({f.column for f in plan.filters if getattr(f, "column", None)} | set(plan.keys or [])
                  | {a.column for a in plan.aggs or []})
    types = ",".join(f"{c}:{src.column(c).dtype}" for c in cols)
    def shape(f) -> str:
        return f.kind + (f.op or "") + "(" + ",".join(shape(a) for a in f.args) + ")"

    filt = ";".join(shape(f) for f in plan.filters)
    aggs = ",".join(f"{a.op}:{a.column}" for a in plan.aggs or [])
    return f"cuda:groupby:v2:{types}|{filt}|{plan.keys}|{aggs}"


def _input_bytes(plan: Plan, rows: int | None = None, bound: Bound | None = None) -> int:
    bound = bound or bind(plan)
    n = len(bound.series[0]) if rows is None and bound.series else (rows or 0)
    per_row = sum(s.dtype.itemsize + (0.125 if s.has_nulls else 0.0) for s in bound.series)
    return int(n * per_row)


def _record_run(plan: Plan, device_ns: float, bound: Bound | None = None) -> None:
    nbytes = _input_bytes(plan, bound=bound)
    if nbytes <= 0 or device_ns <= _FIXED_NS:
        return
    rate = (device_ns - _FIXED_NS) / nbytes
    with _calibration_lock:
        old = _calibration.get(_layout_key(plan))
        _calibration[_layout_key(plan)] = [rate if old is None else 0.5 * old[0] + 0.5 * rate,
                                           1.0 if old is None else old[1] + 1.0]


def pipeline_estimate(pipeline, device: int, features: PipelineFeatures | None = None) -> float:
    """Estimated device nanoseconds of the pipeline's region, input and
    output moves excluded (those are transfer_model's): fixed cost plus the
    layout's calibrated ns per input byte; -1 when the region is not one this
    provider runs."""
    try:
        p = _region_plan(pipeline)
        if _unsupported_reason(p) is not None:
            return -1.0
        nbytes = features.input_bytes if features and features.input_bytes > 0 else _input_bytes(
            p, features.rows if features and features.rows > 0 else None)
        with _calibration_lock:
            cal = _calibration.get(_layout_key(p))
        return _FIXED_NS + nbytes * (cal[0] if cal else _DEFAULT_NS_PER_BYTE)
    except Exception:
        return -1.0


def pipeline_costs(pipeline, device: int, features: PipelineFeatures | None = None) -> tuple[float, float]:
    """(matched CPU ns, device ns): -1 for the CPU keeps the core's generic
    calibration (dataframe/lazy_api.mojo:2537-2541)."""
    return -1.0, pipeline_estimate(pipeline, device, features)


def run_pipeline(pipeline, device: int) -> DataFrame:
    """Runs the region and leaves its result on the device: a frame of
    ResidentSeries, copied to the host column by column when first read
    (the reference's device-resident pipeline output,
    dataframe/storage/residence.mojo:33-147).  Columns decoded from
    dictionary codes are read on the host at once."""
    p = _region_plan(pipeline)
    reason = _unsupported_reason(p)
    if reason:
        raise UnsupportedError(N.UNSUPPORTED, f"accelerator cannot run this pipeline: {reason}")
    bound = bind(p)
    _check(N.lib().dfc_set_memory_limit(device, max(_memory_limit(), 0)))
    cols = [DeviceColumn(s, device) for s in bound.series]
    try:
        result = run_bound(bound, cols, flags=_regime_flags())
        t = last_timings()
        try:
            frame = result.to_resident()
        finally:
            result.free()  # the resident columns hold their own references
    finally:
        for c in cols:
            c.release()
    _record_run(p, t["total_ns"], bound)
    return decode_outputs(bound, frame)
