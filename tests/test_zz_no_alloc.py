"""dfc_groupby_noalloc against dfc_groupby, through the C ABI.

The no-allocation entry point is for callers that cannot call cudaMalloc:
code whose device heap belongs to another allocator (a framework's caching
pool, a fixed memory budget) or that must not allocate on its request path.
They hand in device inputs and device output buffers; the library's working
memory comes from one fixed array shared by every call.  These tests run it
several times in a row, so a call that left state behind in the array would
corrupt the next, and compare each result with the allocating entry point's
on the same device data: keys, integer results, validity and group order bit
for bit; floating sums and means within the tolerance of the other parity
tests (relative 1e-12 of the summands' magnitude), variances within
1e-10 * (1 + |value|).

This file is collected last on purpose: it adds nothing the other GPU tests
need, and a run that stops at its first failure has then run all of them.
"""
import ctypes as C

import numpy as np
import pytest

from casegen import config1, config1_plan, config2
from dataframe_mojo_b200 import _native as N
from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, bind, col, dfc_dtype, np_dtype

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-12
VAR_RTOL = 1e-10


def _torch():
    import torch

    return torch


def device_bytes(arr: np.ndarray):
    """A cuda byte tensor holding `arr` (torch allocations are 256-byte aligned)."""
    torch = _torch()
    raw = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
    if raw.size == 0:
        raw = np.zeros(16, np.uint8)
    return torch.from_numpy(raw.copy()).cuda()


def device_columns(frame: DataFrame, names: list[str]):
    """Device copies of the named columns: values, and validity as LSB-first
    32-bit words at bit offset 0 (None when the column has no nulls)."""
    keep, descs = [], (N.DeviceColumnDesc * len(names))()
    for i, name in enumerate(names):
        s = frame[name]
        vals = device_bytes(s.values)
        keep.append(vals)
        descs[i].dtype = dfc_dtype(s.values.dtype)
        descs[i].values = vals.data_ptr()
        descs[i].validity = None
        if s.valid is not None:
            bits = np.packbits(s.valid.astype(np.uint8), bitorder="little")
            words = np.zeros(((len(s) + 31) // 32) * 4, np.uint8)
            words[: bits.size] = bits
            valid = device_bytes(words)
            keep.append(valid)
            descs[i].validity = valid.data_ptr()
    return descs, keep


def run_noalloc(plan, capacity: int, flags: int = 0, stream=None) -> DataFrame:
    """The plan through dfc_groupby_noalloc; `stream` (a torch stream) is
    passed as the query's stream when given."""
    torch = _torch()
    bound = bind(plan.plan if hasattr(plan, "plan") else plan)
    frame = DataFrame(bound.series)
    descs, keep = device_columns(frame, [s.name for s in bound.series])
    q = provider._query_struct(bound, [C.c_void_p(None)] * len(bound.names),
                               stream.cuda_stream if stream is not None else None, flags)
    n_out = len(bound.out_names)
    outs = (N.DeviceOutput * n_out)()
    bufs = []
    for i in range(n_out):
        v = torch.empty(max(1, capacity) * 8, dtype=torch.uint8, device="cuda")
        m = torch.empty(max(1, (capacity + 31) // 32) * 4, dtype=torch.uint8, device="cuda")
        bufs += [v, m]
        outs[i].values, outs[i].validity = v.data_ptr(), m.data_ptr()
    groups = C.c_uint64(0)
    torch.cuda.synchronize()
    st = N.lib().dfc_groupby_noalloc(C.byref(q), 0, len(bound.series[0]), descs, capacity, outs, C.byref(groups))
    if st != N.OK:
        raise provider.ProviderError(st, N.last_error())
    if stream is not None:
        stream.synchronize()
    g = groups.value
    cols = []
    for i, name in enumerate(bound.out_names):
        dt = np_dtype(outs[i].dtype)
        vals = bufs[2 * i][: g * dt.itemsize].cpu().numpy().view(dt).copy()
        words = bufs[2 * i + 1][: ((g + 31) // 32) * 4].cpu().numpy()
        valid = np.unpackbits(words, bitorder="little")[:g].astype(bool)
        assert bool(outs[i].has_nulls) == (not valid.all()), name
        cols.append(Series(name, vals, valid if not valid.all() else None))
    del keep
    return DataFrame(cols)


def assert_same(a: DataFrame, b: DataFrame, label: str, floats=(), var_cols=(), scales=None):
    assert a.columns == b.columns, label
    assert a.height == b.height, (label, a.height, b.height)
    for c in a.columns:
        x, y = a[c], b[c]
        vx = np.ones(len(x), bool) if x.valid is None else x.valid
        vy = np.ones(len(y), bool) if y.valid is None else y.valid
        assert np.array_equal(vx, vy), (label, c, "validity")
        assert x.values.dtype == y.values.dtype, (label, c)
        if c in floats or c in var_cols:
            xv, yv = x.values.astype(np.float64)[vx], y.values.astype(np.float64)[vx]
            if c in var_cols:
                bound = VAR_RTOL * (1 + np.abs(yv))
            else:
                bound = SUM_RTOL * np.maximum(np.abs(yv), scales[c][vx] if scales and c in scales else 0.0)
            ok = (np.abs(xv - yv) <= bound) | (xv == yv) | (np.isnan(xv) & np.isnan(yv))
            assert ok.all(), (label, c, np.nonzero(~ok)[0][:5])
        else:
            assert np.array_equal(x.values[vx], y.values[vx]), (label, c)


def config2_small():
    frame = config2(rows=1_000_000, distinct=1_000)
    plan = (
        frame.lazy()
        .filter(col("p") < 50)
        .group_by(["k1", "k2"], maintain_order=True)
        .agg([col("v").sum().alias("sum"), col("v").mean().alias("mean"), col("v").min().alias("min"),
              col("v").max().alias("max"), col("v").count().alias("count"), col("v").var().alias("var")])
    )
    return plan


def config2_scales(ref: DataFrame):
    n = ref["count"].values.astype(np.float64)
    m = np.maximum(np.abs(ref["min"].values), np.abs(ref["max"].values)).astype(np.float64)
    m = np.where(np.isfinite(m), m, 0.0)
    return {"sum": n * m, "mean": m}


def test_noalloc_matches_groupby_on_calls_in_a_row():
    """Three calls back to back: few groups (shared-memory tables), then
    about 60K groups with nulls and floats (the global table fills much of
    the array), then the first query again over what the second left."""
    small = config1_plan(config1())
    big = config2_small()
    ref_small, _ = provider.execute(small)
    ref_big, _ = provider.execute(big)

    first = run_noalloc(small, capacity=1024)
    assert_same(first, ref_small, "call 1")
    second = run_noalloc(big, capacity=100_000)
    assert second.height > 10_000
    assert_same(second, ref_big, "call 2", floats=("sum", "mean"), var_cols=("var",), scales=config2_scales(ref_big))
    third = run_noalloc(small, capacity=1024)
    assert_same(third, ref_small, "call 3")


def test_noalloc_rejects_what_the_array_cannot_hold():
    plan = config1_plan(config1(rows=1_000_000))
    with pytest.raises(provider.ProviderError) as ei:
        run_noalloc(plan, capacity=10_000_000)
    assert ei.value.status == N.CAPACITY
    assert "fixed scratch array holds" in str(ei.value)


def test_noalloc_reports_more_groups_than_capacity():
    keys = np.arange(5000, dtype=np.int64)
    frame = DataFrame([Series("k", keys), Series("v", np.ones(5000, np.int64))])
    plan = frame.lazy().group_by("k").agg(col("v").sum())
    with pytest.raises(provider.ProviderError) as ei:
        run_noalloc(plan, capacity=100)
    assert ei.value.status == N.CAPACITY
    # The next call is unaffected.
    out = run_noalloc(plan, capacity=5000)
    assert out.height == 5000 and int(out["v"].values.sum()) == 5000


def test_noalloc_compensated_out_of_range_reruns_in_fp64():
    """Float32 partials that leave the FP32 range: the entry point reruns the
    query in FP64 inside its own array, as dfc_groupby does, and the second
    call in a row (same array) agrees again."""
    rows = 4096
    keys = (np.arange(rows) % 4).astype(np.int32)
    frame = DataFrame([Series("k", keys), Series("v", np.full(rows, 3.0e38, np.float32))])
    plan = frame.lazy().group_by("k", maintain_order=True).agg([col("v").sum().alias("s"), col("v").var().alias("var")])
    for call in range(2):
        out = run_noalloc(plan, capacity=64, flags=N.Q_FLOAT32_COMPENSATED)
        assert np.allclose(out["s"].values, 1024 * float(np.float32(3.0e38)), rtol=1e-12), call
        assert np.all(out["var"].values == 0.0), call
        t = provider.last_timings()
        assert t["retries"] == 1 and t["compensated"] == 0, t


def test_noalloc_compensated_in_range_matches_groupby():
    rng = np.random.default_rng(71)
    rows = 200_000
    frame = DataFrame([
        Series("k", rng.integers(0, 300, rows).astype(np.int32)),
        Series("v", (rng.standard_normal(rows) * 1e3).astype(np.float32)),
    ])
    plan = frame.lazy().group_by("k", maintain_order=True).agg(
        [col("v").sum().alias("s"), col("v").mean().alias("m"), col("v").var().alias("var")])
    ref, _ = provider.execute(plan)
    out = run_noalloc(plan, capacity=1024, flags=N.Q_FLOAT32_COMPENSATED)
    assert provider.last_timings()["compensated"] != 0
    # Compensated FP32 partials against dfc_groupby's FP64 accumulation:
    # 1e-9 of the summands' magnitude (sum |x| per group), the bound the
    # compensated tests hold against the oracle; variances 1e-8 relative.
    order = {int(k): i for i, k in enumerate(ref["k"].values)}
    idx = np.array([order[int(k)] for k in frame["k"].values])
    mags = {"s": np.bincount(idx, weights=np.abs(frame["v"].values.astype(np.float64)), minlength=ref.height)}
    mags["m"] = mags["s"] / np.bincount(idx, minlength=ref.height)
    assert out.columns == ref.columns and out.height == ref.height
    assert np.array_equal(out["k"].values, ref["k"].values)
    for c in ("s", "m"):
        assert np.all(np.abs(out[c].values - ref[c].values) <= 1e-9 * mags[c]), c
    assert np.all(np.abs(out["var"].values - ref["var"].values) <= 1e-8 * (1 + np.abs(ref["var"].values)))


def ticket_frame(rows: int, seed: int) -> DataFrame:
    """Three nullable Int64 keys (wider than one 64-bit key word together, so
    keys are hashed and checked at the claiming row) and a nullable value."""
    rng = np.random.default_rng(seed)
    cols = []
    for i in range(3):
        cols.append(Series(f"k{i}", rng.integers(-3, 3, rows).astype(np.int64) * (1 << 40),
                           rng.random(rows) > 0.1))
    cols.append(Series("v", rng.integers(-1000, 1000, rows).astype(np.int64), rng.random(rows) > 0.05))
    cols.append(Series("p", rng.integers(0, 10, rows).astype(np.int32)))
    return DataFrame(cols)


def ticket_plan(frame: DataFrame):
    return (frame.lazy().filter(col("p") >= 2).group_by(["k0", "k1", "k2"], maintain_order=True)
            .agg([col("v").sum().alias("s"), col("v").min().alias("lo"), col("v").max().alias("hi"),
                  col("v").count().alias("n"), col("v").null_count().alias("nulls"), col("v").len().alias("len")]))


def test_noalloc_ticket_keys_with_nulls_against_oracle():
    """A 3-key nullable Int64 query (ticket keys) against the CPU oracle
    directly, bit for bit: every output here is an integer."""
    from oracle import binding

    plan = ticket_plan(ticket_frame(300_000, 72))
    ref, _ = binding.run(plan)
    assert ref.height > 200
    for call in range(2):
        out = run_noalloc(plan, capacity=4096)
        assert_same(out, ref, f"ticket call {call}")


def test_noalloc_empty_input():
    frame = DataFrame([Series("k", np.zeros(0, np.int64)), Series("v", np.zeros(0, np.float64))])
    plan = frame.lazy().group_by("k", maintain_order=True).agg([col("v").sum().alias("s"), col("v").count().alias("n")])
    ref, _ = provider.execute(plan)
    out = run_noalloc(plan, capacity=16)
    assert out.height == 0 == ref.height
    assert out.columns == ref.columns


def test_noalloc_on_a_caller_stream():
    torch = _torch()
    plan = ticket_plan(ticket_frame(100_000, 73))
    ref, _ = provider.execute(plan)
    s = torch.cuda.Stream()
    out = run_noalloc(plan, capacity=4096, stream=s)
    assert_same(out, ref, "caller stream")
