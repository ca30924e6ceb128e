"""Case builders shared by the tests: golden fixtures (tests/golden/), the
reference's test generators restated, and seeded synthetic workloads."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

from dataframe_mojo_b200.frame import DataFrame, Series, col

GOLDEN = Path(__file__).resolve().parent / "golden" / "fixtures.json"

_NP = {
    "int8": np.int8, "int16": np.int16, "int32": np.int32, "int64": np.int64,
    "uint8": np.uint8, "uint16": np.uint16, "uint32": np.uint32, "uint64": np.uint64,
    "float32": np.float32, "float64": np.float64,
}


def load_cases() -> list[dict]:
    return json.loads(GOLDEN.read_text())["cases"]


def series_from_json(name: str, spec: dict) -> Series:
    dt = _NP[spec["dtype"]]
    vals, valid = [], []
    for v in spec["values"]:
        if v is None:
            vals.append(0)
            valid.append(False)
        else:
            vals.append(float.fromhex(v) if isinstance(v, str) else v)
            valid.append(True)
    if dt in (np.uint64,):
        arr = np.array([int(v) for v in vals], dtype=np.uint64)
    elif np.dtype(dt).kind in "iu":
        arr = np.array(vals, dtype=object).astype(dt)
    else:
        arr = np.array(vals, dtype=dt)
    return Series(name, arr, np.array(valid, bool) if not all(valid) else None)


def frame_from_json(cols: dict) -> DataFrame:
    return DataFrame([series_from_json(n, s) for n, s in cols.items()])


def _pred(spec):
    kind = spec[0]
    if kind == "cmp":
        _, c, op, lit = spec
        x = col(c)
        return {"<": x.__lt__, "<=": x.__le__, ">": x.__gt__, ">=": x.__ge__, "==": x.__eq__, "!=": x.__ne__}[op](lit)
    if kind == "is_null":
        return col(spec[1]).is_null()
    if kind == "is_not_null":
        return col(spec[1]).is_not_null()
    if kind == "and":
        return _pred(spec[1]) & _pred(spec[2])
    if kind == "or":
        return _pred(spec[1]) | _pred(spec[2])
    if kind == "not":
        return ~_pred(spec[1])
    raise ValueError(kind)


def _agg(spec):
    op, c, name = spec[0], spec[1], spec[2]
    opts = spec[3] if len(spec) > 3 else {}
    x = col(c)
    e = {
        "sum": lambda: x.sum(min_count=opts.get("min_count", 0)),
        "mean": x.mean, "min": x.min, "max": x.max, "count": x.count, "len": x.len,
        "null_count": x.null_count,
        "var": lambda: x.var(ddof=opts.get("ddof", 1)),
        "std": lambda: x.std(ddof=opts.get("ddof", 1)),
    }[op]()
    return e.alias(name)


def case_plan(case: dict):
    lf = frame_from_json(case["columns"]).lazy()
    for f in case["filters"]:
        lf = lf.filter(_pred(f))
    return lf.group_by(case["keys"], maintain_order=case["maintain_order"]).agg([_agg(a) for a in case["aggs"]])


def expected_frame(case: dict) -> DataFrame:
    return frame_from_json(case["expected"])


def assert_frames_match(actual: DataFrame, expected: DataFrame, rtol: float = 0.0, atol: float = 0.0,
                        ordered: bool = True, label: str = "") -> None:
    """Same columns, dtypes, nulls and values; floats within rtol/atol
    (0 = bit-exact up to NaN == NaN; -0.0 vs 0.0 is checked by sign)."""
    assert actual.columns == expected.columns, (label, actual.columns, expected.columns)
    assert actual.height == expected.height, (label, actual.height, expected.height)
    for name in expected.columns:
        a, e = actual.column(name), expected.column(name)
        assert a.dtype == e.dtype, (label, name, a.dtype, e.dtype)
        va = np.ones(len(a), bool) if a.valid is None else a.valid
        ve = np.ones(len(e), bool) if e.valid is None else e.valid
        bad = np.nonzero(va != ve)[0]
        assert bad.size == 0, (label, name, "validity differs at rows", bad[:10])
        x, y = a.values[ve], e.values[ve]
        if a.dtype.kind == "f":
            both_nan = np.isnan(x) & np.isnan(y)
            if rtol == 0 and atol == 0:
                same = (x == y) & (np.signbit(x) == np.signbit(y))
            else:
                with np.errstate(invalid="ignore"):
                    same = np.abs(x.astype(np.float64) - y.astype(np.float64)) <= atol + rtol * np.abs(y.astype(np.float64))
            ok = same | both_nan
            bad = np.nonzero(~ok)[0]
            assert bad.size == 0, (label, name, "values differ", bad[:5], x[bad[:5]], y[bad[:5]])
        else:
            bad = np.nonzero(x != y)[0]
            assert bad.size == 0, (label, name, "values differ", bad[:5], x[bad[:5]], y[bad[:5]])


# ---------------------------------------------------------------------------
# tests/support/aggregate_table_reference.mojo:1-120, restated: row r belongs
# to group (r * 7919) % groups; keys and values are functions of g and r.
# ---------------------------------------------------------------------------
def group_of(row, groups):
    return (row * 7919) % groups


def int_key_valid(g):
    string_valid = g % 29 != 5
    return not (g % 31 == 7 and string_valid)


def int_key(g):
    return g * 1_000_003 - 5_000_000


def float_key(g):
    g = np.asarray(g)
    out = (g % 5).astype(np.float64) - 2.5
    out = np.where(g % 6 == 4, 0.0, out)
    out = np.where(g % 6 == 1, -0.0, out)
    out = np.where(g % 7 == 3, np.nan, out)
    return out


def aggregate_frame(rows: int, groups: int) -> DataFrame:
    r = np.arange(rows, dtype=np.int64)
    g = group_of(r, groups)
    i = int_key(g).astype(np.int64)
    iv = np.array([int_key_valid(x) for x in g], bool)
    f = float_key(g)
    x = ((r * 104729) % 1999 - 1000).astype(np.int32)
    xv = r % 17 != 3
    w = (r % 977) * 1_000_000_007 - 400_000_000_000
    wv = r % 13 != 4
    y = (r % 211).astype(np.float64) / 8 - 13
    yv = r % 19 != 9
    return DataFrame(
        [
            Series("i", i, iv),
            Series("f", f),
            Series("x", x, xv),
            Series("w", w.astype(np.int64), wv),
            Series("y", y, yv),
            Series("r", r),
        ]
    )


def aggregate_reductions():
    """test_aggregate_table_modes.mojo:26-38, without the string key."""
    return [
        col("x").sum(min_count=1).alias("x_sum"),
        col("x").mean().alias("x_mean"),
        col("x").min().alias("x_min"),
        col("x").max().alias("x_max"),
        col("x").count().alias("x_count"),
        col("w").sum(min_count=1).alias("w_sum"),
        col("w").null_count().alias("w_nulls"),
        col("x").len().alias("rows"),
        col("y").mean().alias("y_mean"),
        col("y").std().alias("y_std"),
    ]


def aggregate_model(rows: int, groups: int, start: int):
    """GroupModel of tests/support/aggregate_table_reference.mojo:140-245 over
    rows >= start, merged by the (i, f) key pair (nulls equal, NaN one value,
    -0.0 == 0.0) in first-row order."""
    frame = aggregate_frame(rows, groups)
    i, iv = frame["i"].values, frame["i"].valid
    f = frame["f"].values
    x, xv = frame["x"].values, frame["x"].valid
    w, wv = frame["w"].values, frame["w"].valid
    y, yv = frame["y"].values, frame["y"].valid
    models: dict = {}
    order = []
    for r in range(start, rows):
        fk = "nan" if math.isnan(f[r]) else (0.0 if f[r] == 0 else float(f[r]))
        key = (int(i[r]) if iv[r] else None, fk)
        m = models.get(key)
        if m is None:
            m = models[key] = {"first": r, "rows": 0, "xs": [], "ws": [], "w_nulls": 0, "ys": [], "i": key[0], "f": f[r]}
            order.append(key)
        m["rows"] += 1
        if xv[r]:
            m["xs"].append(int(x[r]))
        if wv[r]:
            m["ws"].append(int(w[r]))
        else:
            m["w_nulls"] += 1
        if yv[r]:
            m["ys"].append(float(y[r]))
    return frame, [models[k] for k in order]


# ---------------------------------------------------------------------------
# Seeded synthetic workloads of the benchmark configurations.
# ---------------------------------------------------------------------------
def config1(rows: int = 1_000_000, seed: int = 1) -> DataFrame:
    """1M rows; key Int64 uniform over 16 distinct values; amount Int64
    uniform in [-100, 1000]."""
    rng = np.random.default_rng(seed)
    distinct = rng.integers(-(2**62), 2**62, size=16, dtype=np.int64)
    key = distinct[rng.integers(0, 16, size=rows)]
    amount = rng.integers(-100, 1001, size=rows, dtype=np.int64)
    return DataFrame([Series("key", key), Series("amount", amount)])


def config1_plan(frame: DataFrame):
    return (
        frame.lazy()
        .filter(col("amount") > 0)
        .group_by("key", maintain_order=True)
        .agg([col("amount").sum().alias("sum"), col("amount").count().alias("count")])
    )


def zipf_ranks(rng, n: int, distinct: int, s: float) -> np.ndarray:
    """Ranks in [0, distinct) with P(rank k) proportional to (k+1)^-s (inverse CDF)."""
    w = np.arange(1, distinct + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = rng.random(n)
    return np.minimum(np.searchsorted(cdf, u, side="right"), distinct - 1)


def config2(rows: int = 100_000_000, seed: int = 2, distinct: int = 1_000_000) -> DataFrame:
    """keys k1 = Int32 Zipf(s=1.1) over `distinct` values (ranks mapped through
    a fixed permutation), k2 = UInt32 codes of a 64-value dictionary; v
    Float64 ~ Normal(0, 1e3) with 5% nulls; p Int32 uniform in [0, 100)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(distinct).astype(np.int32)
    k1 = perm[zipf_ranks(rng, rows, distinct, 1.1)]
    k2 = rng.integers(0, 64, size=rows, dtype=np.uint32)
    v = rng.normal(0.0, 1e3, size=rows)
    vv = rng.random(rows) >= 0.05
    p = rng.integers(0, 100, size=rows, dtype=np.int32)
    return DataFrame([Series("k1", k1), Series("k2", k2), Series("v", v, vv), Series("p", p)])


def config2_plan(frame: DataFrame, maintain_order: bool = True):
    return (
        frame.lazy()
        .filter(col("p") < 50)
        .group_by(["k1", "k2"], maintain_order=maintain_order)
        .agg(
            [
                col("v").sum().alias("sum"),
                col("v").mean().alias("mean"),
                col("v").min().alias("min"),
                col("v").max().alias("max"),
                col("v").count().alias("count"),
                col("v").var().alias("var"),
            ]
        )
    )
