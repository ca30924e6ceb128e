"""The radix-partitioned regime (many groups) against the CPU oracle, through
the C ABI: pass A partitions the selected rows, pass B aggregates each
partition in an L2-resident cluster table, the finish is shared with the
other regimes.  The same bars as the other parity tests: integers, keys,
nulls and group order bit-exact; floats within the tolerances written in
test_gpu_parity."""
import numpy as np
import pytest

from casegen import assert_frames_match, case_plan, config2, config2_plan, expected_frame, load_cases
from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, col
from test_gpu_parity import DTYPES, compare_with_oracle, magnitude, random_frame, run_device

pytestmark = pytest.mark.gpu

CASES = load_cases()


@pytest.fixture
def partitioned(monkeypatch):
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "partitioned")


def regime():
    return provider.last_timings()["regime"]


def test_config2_reduced_partitioned(partitioned):
    frame = config2(rows=2_000_000, distinct=100_000)
    dev, _ = compare_with_oracle(
        config2_plan(frame), "config2-2M-partitioned", float_cols=("sum", "mean"), var_cols=("var",),
        scales=lambda ref: dict(zip(("sum", "mean"), magnitude(ref, "count", "min", "max"))),
    )
    t = provider.last_timings()
    assert t["regime"] == 2 and t["partitions"] >= 16
    assert dev.height > 100_000


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_fixture_partitioned(case, partitioned):
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


def test_config2_many_groups_partitioned(partitioned):
    """4M rows over 1M x 64 key pairs: about 1.5M groups in 512 partitions."""
    frame = config2(rows=4_000_000, distinct=1_000_000)
    compare_with_oracle(
        config2_plan(frame), "config2-4M-partitioned", float_cols=("sum", "mean"), var_cols=("var",),
        scales=lambda ref: dict(zip(("sum", "mean"), magnitude(ref, "count", "min", "max"))),
    )
    assert regime() == 2


@pytest.mark.parametrize("seed", range(8))
def test_random_dtypes_partitioned(seed, partitioned):
    rng = np.random.default_rng(5000 + seed)
    nk = 1 + seed % 2
    key_dtypes = [DTYPES[(seed * 3 + i) % len(DTYPES)] for i in range(nk)]
    val_dtypes = [DTYPES[(seed * 7 + i) % len(DTYPES)] for i in range(2)]
    rows = int(rng.integers(1, 80_000))
    frame = random_frame(rng, rows, key_dtypes, val_dtypes, null_rate=0.1 if seed % 2 else 0.0)
    aggs, floats, vars_ = [], [], []
    for i, dt in enumerate(val_dtypes):
        v = col(f"v{i}")
        aggs += [v.sum().alias(f"s{i}"), v.count().alias(f"n{i}"), v.min().alias(f"lo{i}"), v.max().alias(f"hi{i}"),
                 v.mean().alias(f"m{i}"), v.var().alias(f"var{i}"), v.null_count().alias(f"nul{i}"),
                 v.len().alias(f"len{i}")]
        floats.append(f"m{i}")
        vars_.append(f"var{i}")
        if np.dtype(dt).kind == "f":
            floats.append(f"s{i}")
    plan = frame.lazy().filter(col("p") >= 10).group_by([f"k{i}" for i in range(nk)], maintain_order=True).agg(aggs)

    def scales(ref):
        out = {}
        for i in range(len(val_dtypes)):
            out[f"s{i}"], out[f"m{i}"] = magnitude(ref, f"n{i}", f"lo{i}", f"hi{i}")
        return out

    try:
        compare_with_oracle(plan, f"partitioned{seed}", float_cols=floats, var_cols=vars_, scales=scales)
    except provider.DataFaultError:
        pytest.skip("moments adjudicated by the CPU (data fault)")


def test_hot_key_skew(partitioned):
    """Half the rows on one key (one partition takes them, its page list
    grows past the average share; warps collapse the key's rows), the rest
    over 200K distinct keys."""
    rng = np.random.default_rng(11)
    rows = 1_500_000
    keys = rng.integers(0, 200_000, rows, dtype=np.int64)
    keys[rng.random(rows) < 0.5] = 123_456_789
    v = rng.integers(-1000, 1000, rows, dtype=np.int64)
    f = rng.standard_normal(rows)
    frame = DataFrame([Series("k", keys), Series("v", v), Series("f", f)])
    plan = frame.lazy().group_by("k", maintain_order=True).agg(
        [col("v").sum().alias("s"), col("v").min().alias("lo"), col("v").max().alias("hi"), col("v").count().alias("n"),
         col("f").sum().alias("fs"), col("f").min().alias("flo"), col("f").max().alias("fhi"), col("f").var().alias("fv")]
    )
    compare_with_oracle(plan, "hot-key", float_cols=("fs",), var_cols=("fv",),
                        scales=lambda ref: {"fs": magnitude(ref, "n", "flo", "fhi")[0]})
    assert regime() == 2


def test_all_ones_key_word_partitioned(partitioned):
    k = np.array([-1, 5, -1, 7, 5, -1], dtype=np.int64)
    v = np.arange(6, dtype=np.int64)
    out = run_device(DataFrame([Series("k", k), Series("v", v)]).lazy().group_by("k", maintain_order=True).agg(col("v").sum()))
    assert out["k"].values.tolist() == [-1, 5, 7]
    assert out["v"].values.tolist() == [0 + 2 + 5, 1 + 4, 3]
    assert regime() == 2


def test_regimes_agree_on_integers(monkeypatch):
    frame = config2(rows=1_000_000, distinct=50_000)
    plan = frame.lazy().filter(col("p") < 50).group_by(["k1", "k2"], maintain_order=True).agg(
        [col("p").sum().alias("s"), col("v").count().alias("n"), col("v").min().alias("lo"), col("v").max().alias("hi")]
    )
    outs = {}
    for name in ("global", "partitioned"):
        monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", name)
        outs[name] = run_device(plan)
    assert outs["global"].equals(outs["partitioned"])


QUAD_FILTERS = [
    (np.int32, "<", -5), (np.int32, ">=", 2**31 - 1), (np.int64, ">", 2**63 - 1), (np.int64, "<", -(2**63)),
    (np.int64, "!=", 7), (np.uint32, "<", 0), (np.uint32, "!=", 2**32 - 1), (np.uint32, ">", 2**31),
    (np.uint64, "<=", 2**63), (np.uint64, "<", 0), (np.int8, "==", -2), (np.uint16, ">=", 40000),
    (np.float64, "<", float("-inf")), (np.float64, ">", float("inf")), (np.float64, "!=", float("nan")),
    (np.float64, "==", float("nan")), (np.float64, "<=", 0.0), (np.float32, ">", 0.1), (np.float32, "<", 1e39),
]


@pytest.mark.parametrize("dt,op,lit", QUAD_FILTERS, ids=[f"{np.dtype(d).name}{o}{l}" for d, o, l in QUAD_FILTERS])
def test_quad_filter_edges(dt, op, lit, partitioned):
    """The quad row path's range form of one comparison (integer keys,
    1024-row tiles): boundary literals, empty ranges, NaN and infinities,
    unsigned columns; a nullable filter column."""
    rng = np.random.default_rng(abs(hash((np.dtype(dt).name, op))) % 2**32)
    rows = 70_000  # several full tiles and a ragged one
    keys = rng.integers(0, 3000, rows, dtype=np.int64)
    if np.dtype(dt).kind == "f":
        pool = np.array([0.0, -0.0, np.nan, np.inf, -np.inf, 0.1, -7.5, 1e300 if dt == np.float64 else 3e38], dt)
        f = pool[rng.integers(0, len(pool), rows)]
    else:
        info = np.iinfo(dt)
        pool = np.array([info.min, info.max, 0, 1, 2, 7] + list(rng.integers(info.min, info.max, 10, dtype=dt,
                                                                               endpoint=True)), dtype=dt)
        f = pool[rng.integers(0, len(pool), rows)]
    frame = DataFrame([Series("k", keys), Series("f", f, rng.random(rows) > 0.05),
                       Series("v", rng.integers(-50, 50, rows, dtype=np.int64))])
    x = col("f")
    pred = {"<": x.__lt__, "<=": x.__le__, ">": x.__gt__, ">=": x.__ge__, "==": x.__eq__, "!=": x.__ne__}[op](lit)
    plan = frame.lazy().filter(pred).group_by("k", maintain_order=True).agg(
        [col("v").sum().alias("s"), col("v").count().alias("n"), col("v").min().alias("lo")])
    compare_with_oracle(plan, f"quad-{np.dtype(dt).name}{op}{lit}")
    assert regime() == 2
