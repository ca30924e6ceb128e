"""FIRST, LAST and N_UNIQUE (dataframe/aggregation/function.mojo:134-158).

FIRST / LAST: the value at the group's first / last row among the rows the
filter kept, null when that row's value is null (the reference keeps the
row's value and its validity, function.mojo:997-1013, 1586-1600, 2637-2650).
N_UNIQUE: the group's distinct values under key equality: null is one value,
every NaN one value, -0.0 == 0.0 (tests/public_contracts/
test_approx_n_unique.mojo:60-80).  On the device N_UNIQUE runs as two
group-bys (the distinct (keys, value) tuples, then their count per key
tuple).  CPU tests pin the oracle with hand-computed answers; GPU tests
compare every regime with the oracle bit for bit (all outputs here are exact)."""
import numpy as np
import pytest

from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding


def frame():
    nan = float("nan")
    return DataFrame([
        Series("k", np.array([1, 2, 1, 2, 1, 3, 3], np.int64)),
        Series("x", np.array([10, 0, 30, 40, 10, 7, 8], np.int32),
               np.array([True, False, True, True, True, True, False])),
        Series("f", np.array([nan, -0.0, nan, 0.0, 1.5, 0.0, 2.0], np.float64),
               np.array([True, True, True, True, True, False, False])),
        Series("p", np.array([1, 1, 1, 1, 1, 0, 1], np.int32)),
    ])


def aggs():
    return [col("x").first().alias("xf"), col("x").last().alias("xl"), col("x").n_unique().alias("xu"),
            col("f").first().alias("ff"), col("f").n_unique().alias("fu"), col("x").sum().alias("s")]


def cells(df: DataFrame, name: str) -> list:
    s = df[name]
    return [s.values[i].item() if s.is_valid(i) else None for i in range(df.height)]


def test_oracle_known_answers():
    out, _ = binding.run(frame().lazy().filter(col("p") == 1).group_by("k", maintain_order=True).agg(aggs()))
    assert cells(out, "k") == [1, 2, 3]
    assert cells(out, "xf") == [10, None, None]   # group 2's first row has a null x; group 3 keeps row 6 only
    assert cells(out, "xl") == [10, 40, None]
    assert cells(out, "xu") == [2, 2, 1]           # {10, 30}; {null, 40}; {null}
    ff = cells(out, "ff")
    assert np.isnan(ff[0]) and ff[1] == 0.0 and np.signbit(ff[1]) and ff[2] is None
    assert cells(out, "fu") == [2, 1, 1]           # {NaN, 1.5}; {-0.0 == 0.0}; {null}
    assert cells(out, "s") == [50, 40, 0]           # an all-null group sums to 0 (min_count 0)


def test_oracle_ungrouped_and_empty():
    lf = frame().lazy()
    out, _ = binding.run(lf.select([col("x").n_unique().alias("u"), col("x").first().alias("a"),
                                    col("x").last().alias("b")]))
    # x = 10, null, 30, 40, 10, 7, null: {10, 30, 40, 7, null}
    assert cells(out, "u") == [5] and cells(out, "a") == [10] and cells(out, "b") == [None]
    out, _ = binding.run(lf.filter(col("p") > 9).select([col("x").n_unique().alias("u"), col("x").first().alias("a")]))
    assert cells(out, "u") == [0] and cells(out, "a") == [None]


@pytest.mark.gpu
@pytest.mark.parametrize("regime", ["auto", "global", "shared", "partitioned"])
def test_gpu_known_answers_every_regime(regime, monkeypatch):
    from dataframe_mojo_b200 import provider

    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", regime)
    plan = frame().lazy().filter(col("p") == 1).group_by("k", maintain_order=True).agg(aggs())
    dev = provider.execute(plan)[0]
    ref, _ = binding.run(plan)
    assert dev.equals(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("regime", ["auto", "global", "partitioned"])
@pytest.mark.parametrize("seed", range(3))
def test_gpu_random_against_oracle(regime, seed, monkeypatch):
    from dataframe_mojo_b200 import provider

    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", regime)
    rng = np.random.default_rng(4100 + seed)
    rows = int(rng.integers(1, 600_000))
    groups = [50, 20_000, 300_000][seed]
    k = rng.integers(0, groups, rows).astype(np.int64)
    k[rng.random(rows) < 0.3] = 7  # a hot key
    v = rng.integers(-20, 20, rows).astype(np.int32)
    f = np.where(rng.random(rows) < 0.1, np.nan, rng.integers(-3, 3, rows) * 0.5)
    f[rng.random(rows) < 0.05] = -0.0
    fr = DataFrame([Series("k", k), Series("v", v, rng.random(rows) > 0.1), Series("f", f, rng.random(rows) > 0.05),
                    Series("p", rng.integers(0, 10, rows).astype(np.int32))])
    plan = fr.lazy().filter(col("p") >= 3).group_by("k", maintain_order=True).agg(
        [col("v").first().alias("vf"), col("v").last().alias("vl"), col("v").n_unique().alias("vu"),
         col("f").first().alias("ff"), col("f").last().alias("fl"), col("f").n_unique().alias("fu"),
         col("k").n_unique().alias("ku"), col("v").count().alias("n")])
    dev = provider.execute(plan)[0]
    ref, _ = binding.run(plan)
    assert dev.equals(ref)


@pytest.mark.gpu
def test_gpu_ungrouped_n_unique():
    from dataframe_mojo_b200 import provider

    rng = np.random.default_rng(4200)
    rows = 1_000_000
    fr = DataFrame([Series("x", rng.integers(0, 5000, rows).astype(np.int64), rng.random(rows) > 0.01),
                    Series("p", rng.integers(0, 10, rows).astype(np.int32))])
    for pred in (col("p") < 5, col("p") > 20):
        plan = fr.lazy().filter(pred).select([col("x").n_unique().alias("u"), col("x").first().alias("a"),
                                              col("x").last().alias("b"), col("x").sum().alias("s")])
        dev = provider.execute(plan)[0]
        ref, _ = binding.run(plan)
        assert dev.equals(ref)
