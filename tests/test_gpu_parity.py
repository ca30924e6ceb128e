"""Parity of the CUDA path with the CPU oracle (which the golden tests pin to
the reference), through the C ABI.  Integers, keys, nulls and group order are
bit-exact; floating results carry the tolerance written beside each check."""
import math
import os

import numpy as np
import pytest

from casegen import (
    aggregate_model,
    aggregate_reductions,
    assert_frames_match,
    case_plan,
    config1,
    config1_plan,
    config2,
    config2_plan,
    expected_frame,
    load_cases,
)
from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding

pytestmark = pytest.mark.gpu

CASES = load_cases()

# Float tolerances.  Sums and means: the device adds in a different order
# than the CPU's input order, so they agree within the reference's own
# cross-worker budget (tests/execution_modes/test_aggregate_table_modes.mojo:
# 8-11: relative 1e-12), measured on the sum-of-magnitudes scale.  Variances:
# the public moments tolerance |gpu - cpu| <= 1e-10 * (1 + |cpu|)
# (docs/design/metal-moments.md:108-110).
SUM_RTOL = 1e-12
VAR_RTOL = 1e-10


def run_device(plan):
    return provider.execute(plan)[0]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_fixture(case):
    plan = case_plan(case)
    if "expected_error" in case:
        with pytest.raises(provider.ProviderError) as ei:
            run_device(plan)
        assert str(ei.value) == case["expected_error"]
        return
    if case.get("device_expect") == "data_fault":
        with pytest.raises(provider.DataFaultError):
            run_device(plan)
        return
    actual = run_device(plan)
    assert_frames_match(actual, expected_frame(case), rtol=1e-15, label=case["name"])


def magnitude(ref, count, lo, hi):
    """Per-group bound of sum |x|: count * max(|min|, |max|), from the oracle."""
    n = ref[count].values.astype(np.float64)
    m = np.maximum(np.abs(ref[lo].values.astype(np.float64)), np.abs(ref[hi].values.astype(np.float64)))
    m = np.where(np.isfinite(m), m, 0.0)
    return n * m, m


def compare_with_oracle(plan, label, float_cols=(), var_cols=(), scales=None):
    """Exact columns bit for bit; `float_cols` (sums, means) within SUM_RTOL of
    the summands' magnitude: `scales[c]` per group (sum |x| for a sum, max |x|
    for a mean) when given, else |oracle value|."""
    dev = run_device(plan)
    ref, _ = binding.run(plan)
    if callable(scales):
        scales = scales(ref)
    exact = [c for c in ref.columns if c not in float_cols and c not in var_cols]
    assert dev.columns == ref.columns
    assert dev.height == ref.height, (label, dev.height, ref.height)
    for c in exact:
        assert_frames_match(DataFrame([dev[c]]), DataFrame([ref[c]]), label=f"{label}:{c}")
    for c in float_cols:
        a, b = dev[c], ref[c]
        va = np.ones(len(b), bool) if b.valid is None else b.valid
        vd = np.ones(len(a), bool) if a.valid is None else a.valid
        assert np.array_equal(va, vd), (label, c, "validity")
        x, y = a.values.astype(np.float64), b.values.astype(np.float64)
        scale = np.abs(y) if scales is None or c not in scales else np.maximum(np.abs(y), scales[c])
        ok = (np.abs(x - y) <= SUM_RTOL * scale) | (np.isnan(x) & np.isnan(y)) | (x == y) | ~va
        assert ok.all(), (label, c, np.nonzero(~ok)[0][:5], x[~ok][:5], y[~ok][:5])
    for c in var_cols:
        a, b = dev[c], ref[c]
        assert (a.valid is None) == (b.valid is None) or np.array_equal(
            a.valid if a.valid is not None else np.ones(len(a), bool),
            b.valid if b.valid is not None else np.ones(len(b), bool),
        )
        va = b.valid if b.valid is not None else np.ones(len(b), bool)
        x, y = a.values[va], b.values[va]
        ok = (np.abs(x - y) <= VAR_RTOL * (1 + np.abs(y))) | (np.isnan(x) & np.isnan(y))
        assert ok.all(), (label, c, np.nonzero(~ok)[0][:5])
    return dev, ref


def test_config1_bit_exact():
    """1M rows, 16 Int64 keys, filter amount > 0, sum + count, maintain_order."""
    compare_with_oracle(config1_plan(config1()), "config1")


def test_config2_reduced_against_oracle():
    frame = config2(rows=2_000_000, distinct=100_000)
    dev, ref = compare_with_oracle(
        config2_plan(frame), "config2-2M", float_cols=("sum", "mean"), var_cols=("var",),
        scales=lambda ref: dict(zip(("sum", "mean"), magnitude(ref, "count", "min", "max"))),
    )
    assert dev.height > 100_000


def test_aggregate_table_generator():
    rows, groups, start = 36_000, 5_000, 1_001
    frame, _ = aggregate_model(rows, groups, start)
    plan = frame.lazy().filter(col("r") >= start).group_by(["i", "f"], maintain_order=True).agg(aggregate_reductions())
    # |y| <= 13.5 by the generator (tests/support/aggregate_table_reference.mojo:88-89).
    compare_with_oracle(plan, "aggregate_table", float_cols=("x_mean", "y_mean"), var_cols=("y_std",),
                        scales=lambda ref: {"x_mean": magnitude(ref, "x_count", "x_min", "x_max")[1], "y_mean": 13.5})


DTYPES = [np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32, np.uint64, np.float32, np.float64]


def random_frame(rng, rows, key_dtypes, val_dtypes, null_rate):
    cols = []
    for i, dt in enumerate(key_dtypes):
        if np.dtype(dt).kind == "f":
            pool = np.array([0.0, -0.0, np.nan, 1.5, -2.25, 1e300, -np.inf], dtype=dt)
            vals = pool[rng.integers(0, len(pool), rows)]
        else:
            info = np.iinfo(dt)
            pool = rng.integers(info.min, info.max, size=37, dtype=dt, endpoint=True)
            pool[:2] = [info.min, info.max]
            vals = pool[rng.integers(0, len(pool), rows)]
        valid = rng.random(rows) >= null_rate if null_rate else None
        cols.append(Series(f"k{i}", vals, valid))
    for i, dt in enumerate(val_dtypes):
        if np.dtype(dt).kind == "f":
            vals = (rng.standard_normal(rows) * 10.0 ** rng.integers(-3, 4, rows)).astype(dt)
            vals[rng.random(rows) < 0.01] = np.nan
            vals[rng.random(rows) < 0.01] = 0.0
            vals[rng.random(rows) < 0.01] = -0.0
        else:
            info = np.iinfo(dt)
            lo, hi = (info.min, info.max) if np.dtype(dt).itemsize <= 2 else (-1000, 1000) if info.min < 0 else (0, 2000)
            vals = rng.integers(lo, hi, size=rows, dtype=dt, endpoint=True)
        valid = rng.random(rows) >= null_rate if null_rate else None
        cols.append(Series(f"v{i}", vals, valid))
    cols.append(Series("p", rng.integers(0, 100, rows, dtype=np.int32), rng.random(rows) >= 0.02))
    return DataFrame(cols)


@pytest.mark.parametrize("seed", range(12))
def test_random_dtypes_against_oracle(seed):
    rng = np.random.default_rng(1000 + seed)
    nk = 1 + seed % 3
    key_dtypes = [DTYPES[(seed * 3 + i) % len(DTYPES)] for i in range(nk)]
    val_dtypes = [DTYPES[(seed * 5 + i) % len(DTYPES)] for i in range(2)]
    rows = int(rng.integers(1, 60_000))
    frame = random_frame(rng, rows, key_dtypes, val_dtypes, null_rate=0.1 if seed % 2 else 0.0)
    aggs = []
    floats, vars_ = [], []
    for i, dt in enumerate(val_dtypes):
        v = col(f"v{i}")
        aggs += [v.sum().alias(f"s{i}"), v.count().alias(f"n{i}"), v.min().alias(f"lo{i}"), v.max().alias(f"hi{i}"),
                 v.mean().alias(f"m{i}"), v.var().alias(f"var{i}"), v.std(ddof=0).alias(f"sd{i}"),
                 v.null_count().alias(f"nul{i}"), v.len().alias(f"len{i}")]
        floats.append(f"m{i}")
        vars_ += [f"var{i}", f"sd{i}"]
        if np.dtype(dt).kind == "f":
            floats.append(f"s{i}")
    pred = (col("p") < 70) | col("p").is_null() if seed % 3 == 0 else (col("p") >= 10)
    plan = frame.lazy().filter(pred).group_by([f"k{i}" for i in range(nk)], maintain_order=True).agg(aggs)
    try:
        def scales(ref):
            out = {}
            for i in range(len(val_dtypes)):
                total, single = magnitude(ref, f"n{i}", f"lo{i}", f"hi{i}")
                out[f"s{i}"], out[f"m{i}"] = total, single
            return out

        compare_with_oracle(plan, f"random{seed}", float_cols=floats, var_cols=vars_, scales=scales)
    except provider.DataFaultError:
        pytest.skip("moments adjudicated by the CPU (data fault)")


def test_empty_and_fully_filtered():
    frame = DataFrame([Series("k", np.arange(1000, dtype=np.int64)), Series("v", np.ones(1000))])
    out = run_device(frame.lazy().filter(col("k") < 0).group_by("k").agg(col("v").sum()))
    assert out.height == 0 and out.columns == ["k", "v"]
    empty = DataFrame([Series("k", np.zeros(0, np.int32)), Series("v", np.zeros(0))])
    out = run_device(empty.lazy().group_by("k").agg(col("v").mean()))
    assert out.height == 0 and out["v"].dtype == np.float64


def test_all_ones_key_word_and_extremes():
    """Keys whose packed word is all ones (Int64 -1, UInt64 max) use the
    table's reserved entry."""
    k = np.array([-1, 5, -1, 7, 5, -1], dtype=np.int64)
    v = np.arange(6, dtype=np.int64)
    out = run_device(DataFrame([Series("k", k), Series("v", v)]).lazy().group_by("k", maintain_order=True).agg(col("v").sum()))
    assert out["k"].values.tolist() == [-1, 5, 7]
    assert out["v"].values.tolist() == [0 + 2 + 5, 1 + 4, 3]
    ku = np.array([2**64 - 1, 0, 2**64 - 1], dtype=np.uint64)
    out = run_device(DataFrame([Series("k", ku), Series("v", v[:3])]).lazy().group_by("k", maintain_order=True).agg(col("v").len()))
    assert out["k"].values.tolist() == [2**64 - 1, 0] and out["v"].values.tolist() == [2, 1]


def test_integer_results_repeatable():
    frame = config2(rows=1_000_000, distinct=50_000)
    plan = frame.lazy().filter(col("p") < 50).group_by(["k1", "k2"], maintain_order=True).agg(
        [col("p").sum().alias("s"), col("v").count().alias("n"), col("v").min().alias("lo")]
    )
    a = run_device(plan)
    b = run_device(plan)
    assert a.equals(b)


def test_capacity_regrowth_after_small_learned_estimate():
    rng = np.random.default_rng(7)
    rows = 400_000
    keys = rng.integers(0, 2**40, rows, dtype=np.int64)
    frame = DataFrame([Series("k", keys), Series("v", np.ones(rows, np.int64)), Series("p", np.arange(rows, dtype=np.int64))])
    table = provider.ResidentTable(frame)
    try:
        small = table.run(frame.lazy().filter(col("p") < 100).group_by("k").agg(col("v").sum()))
        assert small.rows == 100
        small.free()
        # The first estimate for a new query shape comes from column
        # statistics; pin it to 100 groups so the table must regrow.
        os.environ["DFC_GROUPS_ESTIMATE"] = "100"
        try:
            big = table.run(frame.lazy().group_by("k", maintain_order=True).agg(col("v").sum()))
        finally:
            del os.environ["DFC_GROUPS_ESTIMATE"]
        t = provider.last_timings()
        assert t["retries"] >= 1
        out = big.to_frame()
        big.free()
        _, idx = np.unique(keys, return_index=True)
        assert np.array_equal(out["k"].values, keys[np.sort(idx)])
    finally:
        table.release()


@pytest.mark.slow
def test_config2_full_size_properties():
    """100M rows: group set, first-appearance order and counts exact; the sum
    of the group sums equals the total within the summation bound."""
    import torch

    frame = config2()
    dev = run_device(config2_plan(frame))
    k1, k2, p = frame["k1"].values, frame["k2"].values, frame["p"].values
    v, vv = frame["v"].values, frame["v"].valid
    sel = p < 50
    packed = torch.from_numpy((k1.astype(np.int64) << 32) | k2.astype(np.int64))[torch.from_numpy(sel)].cuda()
    uniq, inverse = torch.unique(packed, return_inverse=True)
    n = packed.numel()
    first = torch.full((uniq.numel(),), n, dtype=torch.int64, device="cuda")
    first.scatter_reduce_(0, inverse, torch.arange(n, device="cuda"), reduce="amin")
    order = uniq[torch.argsort(first)].cpu().numpy()
    got = (dev["k1"].values.astype(np.int64) << 32) | dev["k2"].values.astype(np.int64)
    assert np.array_equal(got, order)
    assert int(dev["count"].values.sum()) == int((sel & vv).sum())
    total = v[sel & vv].sum()
    assert abs(dev["sum"].values.sum() - total) <= 1e-9 * np.abs(v[sel & vv]).sum()
