"""Ungrouped filtered reductions: SCAN_FRAME -> FILTER* -> SELECT(reductions),
the reference's filtered reduction region (dataframe_metal/filter_plan.mojo:
149-200, kernels dataframe_metal/accelerator/gpu/filter_sum.mojo:1-20).  One
output row, also when the filter keeps no row: the reductions of nothing
(sum 0 unless min_count > 0; count, len and null_count 0; mean, min, max,
var and std null).

The CPU tests pin the oracle's restatement with hand-computed answers; the
GPU tests compare the CUDA path with the oracle (integers bit for bit,
floats within the parity tolerances of test_gpu_parity)."""
import math

import numpy as np
import pytest

from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding


def small_frame():
    return DataFrame([
        Series("x", np.array([5, -3, 0, 10, 7], np.int64), np.array([True, True, False, True, True])),
        Series("p", np.array([1, 0, 1, 1, 0], np.int32)),
        Series("f", np.array([1.5, np.nan, -0.0, 2.5, 4.0], np.float32)),
    ])


def reductions():
    x = col("x")
    return [x.sum().alias("s"), x.count().alias("n"), x.len().alias("len"), x.null_count().alias("nulls"),
            x.mean().alias("mean"), x.min().alias("lo"), x.max().alias("hi"), x.var().alias("var"),
            x.sum(min_count=1).alias("s1")]


def row(frame: DataFrame) -> dict:
    assert frame.height == 1
    return {c: (frame[c].values[0].item() if frame[c].is_valid(0) else None) for c in frame.columns}


def test_oracle_filtered_known_answer():
    out, _ = binding.run(small_frame().lazy().filter(col("p") == 1).select(reductions()))
    # Kept rows 0, 2, 3: x = 5, null, 10.
    assert row(out) == {"s": 15, "n": 2, "len": 3, "nulls": 1, "mean": 7.5, "lo": 5, "hi": 10, "var": 12.5, "s1": 15}


def test_oracle_empty_selection_is_one_identity_row():
    out, _ = binding.run(small_frame().lazy().filter(col("p") > 5).select(reductions()))
    assert row(out) == {"s": 0, "n": 0, "len": 0, "nulls": 0, "mean": None, "lo": None, "hi": None, "var": None,
                        "s1": None}


def test_oracle_no_filter_and_float_column():
    f = col("f")
    out, _ = binding.run(small_frame().lazy().select(
        [f.sum().alias("s"), f.min().alias("lo"), f.max().alias("hi"), f.count().alias("n")]))
    r = row(out)
    assert math.isnan(r["s"]) and r["n"] == 5
    assert r["lo"] == 0.0 and math.copysign(1.0, r["lo"]) < 0 and r["hi"] == 4.0  # NaN skipped; -0.0 kept


def test_select_rejects_an_empty_list():
    with pytest.raises(ValueError):
        small_frame().lazy().select([])


@pytest.mark.gpu
@pytest.mark.parametrize("pred", ["p==1", "p>5", "none"])
def test_gpu_known_cases_match_oracle(pred):
    from dataframe_mojo_b200 import provider

    lf = small_frame().lazy()
    if pred == "p==1":
        lf = lf.filter(col("p") == 1)
    elif pred == "p>5":
        lf = lf.filter(col("p") > 5)
    plan = lf.select(reductions())
    dev = provider.execute(plan)[0]
    ref, _ = binding.run(plan)
    assert dev.equals(ref), (row(dev), row(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(6))
def test_gpu_random_ungrouped_against_oracle(seed):
    from test_gpu_parity import DTYPES, compare_with_oracle

    rng = np.random.default_rng(9000 + seed)
    rows = int(rng.integers(1, 3_000_000)) if seed < 4 else int(rng.integers(0, 40))
    cols = [Series("p", rng.integers(0, 100, rows).astype(np.int32))]
    aggs, floats, vars_ = [], [], []
    for i in range(2):
        dt = DTYPES[(seed * 3 + i) % len(DTYPES)]
        if np.dtype(dt).kind == "f":
            vals = (rng.standard_normal(rows) * 100).astype(dt)
        else:
            info = np.iinfo(dt)  # |x| < 100: sums of 3M rows fit every sum type (Int32 stays Int32)
            vals = rng.integers(max(info.min, -100), min(info.max, 100), rows).astype(dt)
        cols.append(Series(f"v{i}", vals, rng.random(rows) > 0.1 if seed % 2 else None))
        v = col(f"v{i}")
        aggs += [v.sum().alias(f"s{i}"), v.count().alias(f"n{i}"), v.min().alias(f"lo{i}"), v.max().alias(f"hi{i}"),
                 v.mean().alias(f"m{i}"), v.var().alias(f"var{i}"), v.len().alias(f"len{i}")]
        floats.append(f"m{i}")
        vars_.append(f"var{i}")
        if np.dtype(dt).kind == "f":
            floats.append(f"s{i}")
    frame = DataFrame(cols)
    plan = frame.lazy().filter(col("p") < 37).select(aggs)

    def scales(ref):
        out = {}
        for i in range(2):
            n = ref[f"n{i}"].values.astype(np.float64)
            m = np.maximum(np.abs(ref[f"lo{i}"].values.astype(np.float64)), np.abs(ref[f"hi{i}"].values.astype(np.float64)))
            m = np.where(np.isfinite(m), m, 0.0)
            out[f"s{i}"], out[f"m{i}"] = n * m, m
        return out

    compare_with_oracle(plan, f"ungrouped{seed}", float_cols=floats, var_cols=vars_, scales=scales)


@pytest.mark.gpu
def test_gpu_ungrouped_int32_overflow_message():
    from dataframe_mojo_b200 import provider

    frame = DataFrame([Series("x", np.full(3, 2**30, np.int32))])
    with pytest.raises(provider.ProviderError) as ei:
        provider.execute(frame.lazy().select(col("x").sum()))
    with pytest.raises(binding.OracleError) as eo:
        binding.run(frame.lazy().select(col("x").sum()))
    assert str(ei.value) == str(eo.value)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["int32", "float32", "int64"])
def test_gpu_published_filtered_sum_workload(dtype):
    """bench.py's handoff form: the reference's published filtered sum
    (benchmarks/bench_handoff.mojo) on 5M rows, equal to the oracle (the
    values are small integers, so every sum is exact)."""
    import bench
    from dataframe_mojo_b200 import provider

    x = bench.handoff_values(dtype, 5_000_000, "cpu").numpy()
    frame = DataFrame([Series("x", x)])
    plan = bench.handoff_plan(frame)
    dev = provider.execute(plan)[0]
    ref, _ = binding.run(plan)
    assert dev.equals(ref), (row(dev), row(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("columns", [1, 2, 3])
def test_gpu_register_path_and_fallback(columns):
    """Up to two value columns run in registers (regime 3: per-thread states
    folded per warp and per CTA); a third value column takes the per-row
    shared-memory path (regime 1).  NaN, signed zeros, nulls and a
    far-from-zero mean (shifted moments re-centred across threads) against
    the oracle."""
    from dataframe_mojo_b200 import provider
    from test_gpu_parity import compare_with_oracle

    rng = np.random.default_rng(9100 + columns)
    rows = 4_000_000
    cols = [Series("p", rng.integers(0, 100, rows).astype(np.int32))]
    aggs, floats, vars_ = [], [], []
    for i in range(columns):
        if i == 0:
            x = 1e6 + rng.standard_normal(rows)
            x[rng.random(rows) < 1e-6] = np.nan
            x[rng.random(rows) < 0.001] = -0.0
            vals = x
        elif i == 1:
            vals = rng.integers(-(2**40), 2**40, rows).astype(np.int64)
        else:
            vals = rng.standard_normal(rows).astype(np.float32)
        cols.append(Series(f"v{i}", vals, rng.random(rows) > 0.05))
        v = col(f"v{i}")
        aggs += [v.sum().alias(f"s{i}"), v.count().alias(f"n{i}"), v.min().alias(f"lo{i}"), v.max().alias(f"hi{i}"),
                 v.mean().alias(f"m{i}"), v.var().alias(f"var{i}"), v.first().alias(f"f{i}"), v.last().alias(f"l{i}")]
        floats.append(f"m{i}")
        vars_.append(f"var{i}")
        if vals.dtype.kind == "f":
            floats.append(f"s{i}")
    plan = DataFrame(cols).lazy().filter(col("p") < 61).select(aggs + [col("v0").len().alias("len")])

    def scales(ref):
        out = {}
        for i in range(columns):
            n = ref[f"n{i}"].values.astype(np.float64)
            m = np.maximum(np.abs(ref[f"lo{i}"].values.astype(np.float64)), np.abs(ref[f"hi{i}"].values.astype(np.float64)))
            m = np.where(np.isfinite(m), m, 0.0)
            out[f"s{i}"], out[f"m{i}"] = n * m, m
        return out

    compare_with_oracle(plan, f"register{columns}", float_cols=floats, var_cols=vars_, scales=scales)
    provider.execute(plan)
    assert provider.last_timings()["regime"] == (3 if columns <= 2 else 1)


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [0, 1, 1025, 4099])
def test_gpu_register_path_edges(rows):
    """The register path on tiny and ragged inputs (a partial last tile, a
    partial quad), all-null values, NaN-only floats and a filter that keeps
    nothing, against the oracle."""
    from dataframe_mojo_b200 import provider

    rng = np.random.default_rng(rows + 3)
    f = np.full(rows, np.nan, np.float32)
    x = rng.integers(-9, 9, rows).astype(np.int32)
    frame = DataFrame([Series("x", x, np.zeros(rows, bool)), Series("f", f),
                       Series("p", rng.integers(0, 10, rows).astype(np.int32))])
    for pred in (col("p") < 6, col("p") > 50, None):
        lf = frame.lazy() if pred is None else frame.lazy().filter(pred)
        plan = lf.select([col("x").sum().alias("s"), col("x").count().alias("n"), col("x").min().alias("lo"),
                          col("f").sum().alias("fs"), col("f").max().alias("fh"), col("f").var().alias("fv"),
                          col("f").len().alias("len")])
        dev = provider.execute(plan)[0]
        ref, _ = binding.run(plan)
        assert dev.equals(ref), (rows, pred, row(dev), row(ref))
