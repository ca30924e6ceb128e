"""String and Categorical columns through their codes.

A Categorical column is UInt32 codes plus a dictionary (dataframe/
categorical.mojo:1-17): it groups by canonical codes (repeated labels are one
group), keeps its dictionary in the output, and answers == / != by code.  A
String column is dictionary-encoded on the host, grouped by code and decoded
back to strings, as the reference does for a dictionary-coded String key
(dataframe/aggregation/group_by.mojo:307-317, 344-356).  Aggregations that
need only equality or a row's value (count, len, null_count, n_unique,
first, last) read such a column; the others are rejected.

CPU tests check the binding against a plain-Python grouping of the strings;
GPU tests compare the device with the oracle (both decoded) bit for bit."""
from collections import OrderedDict

import numpy as np
import pytest

from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding


def words(rng, n, pool):
    return np.array([pool[i] for i in rng.integers(0, len(pool), n)], dtype=object)


def sample(rows=20_000, seed=3):
    rng = np.random.default_rng(seed)
    pool = ["alpha", "beta", "gamma", "", "delta", "alpha ", "Beta", "ε", "x" * 40]
    city = words(rng, rows, pool)
    labels = ["red", "green", "red", "blue", "green"]  # repeated labels: codes 0/2 and 1/4 are one value
    cat = rng.integers(0, len(labels), rows).astype(np.uint32)
    return DataFrame([
        Series("city", city, rng.random(rows) > 0.05),
        Series("cat", cat, rng.random(rows) > 0.02, categories=labels),
        Series("v", rng.integers(-50, 50, rows).astype(np.int64)),
        Series("p", rng.integers(0, 10, rows).astype(np.int32)),
    ])


def python_groupby(frame: DataFrame, key: str, keep) -> OrderedDict:
    """key string (None for null) -> [sum of v, count] in first-appearance order."""
    out: OrderedDict = OrderedDict()
    for i in range(frame.height):
        if not keep(i):
            continue
        k = frame[key].item(i)
        acc = out.setdefault(k, [0, 0])
        acc[0] += int(frame["v"].values[i])
        acc[1] += 1
    return out


def test_string_key_against_python():
    f = sample()
    out, _ = binding.run(f.lazy().filter(col("p") >= 3).group_by("city", maintain_order=True).agg(
        [col("v").sum().alias("s"), col("v").len().alias("n")]))
    want = python_groupby(f, "city", lambda i: f["p"].values[i] >= 3)
    assert out["city"].to_list() == list(want)
    assert out["s"].to_list() == [a for a, _ in want.values()]
    assert out["n"].to_list() == [b for _, b in want.values()]


def test_categorical_key_keeps_its_dictionary_and_merges_repeated_labels():
    f = sample()
    out, _ = binding.run(f.lazy().group_by("cat", maintain_order=True).agg(col("v").sum().alias("s")))
    assert out["cat"].is_categorical
    assert list(out["cat"].categories) == ["red", "green", "red", "blue", "green"]
    got = out["cat"].to_list()
    assert sorted(x for x in got if x is not None) == ["blue", "green", "red"] and len(got) == 4  # + the null group
    want = python_groupby(f, "cat", lambda i: True)
    assert dict(zip(got, out["s"].to_list())) == {k: v[0] for k, v in want.items()}


def test_string_equality_filter_and_missing_literal():
    f = sample()
    for lit, op in (("beta", "=="), ("nowhere", "=="), ("nowhere", "!=")):
        pred = col("city") == lit if op == "==" else col("city") != lit
        out, _ = binding.run(f.lazy().filter(pred).select([col("v").sum().alias("s"), col("v").len().alias("n")]))
        keep = [f["city"].is_valid(i) and ((f["city"].item(i) == lit) == (op == "==")) for i in range(f.height)]
        assert out["n"].to_list() == [sum(keep)]
        assert out["s"].to_list() == [int(f["v"].values[np.array(keep)].sum())]


def test_unsupported_reductions_and_orderings_are_rejected():
    f = sample(100)
    with pytest.raises(TypeError):
        binding.run(f.lazy().group_by("cat").agg(col("city").sum()))
    with pytest.raises(TypeError):
        binding.run(f.lazy().filter(col("city") < "b").group_by("cat").agg(col("v").sum()))


@pytest.mark.gpu
@pytest.mark.parametrize("regime", ["auto", "global", "partitioned"])
def test_gpu_coded_keys_against_oracle(regime, monkeypatch):
    from dataframe_mojo_b200 import provider

    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", regime)
    f = sample(300_000, seed=11)
    plans = [
        f.lazy().filter(col("p") >= 3).group_by(["city", "cat"], maintain_order=True).agg(
            [col("v").sum().alias("s"), col("city").first().alias("f"), col("cat").last().alias("l"),
             col("city").n_unique().alias("u")]),
        f.lazy().filter(col("cat") == "green").group_by("city", maintain_order=True).agg(col("v").count().alias("n")),
    ]
    for plan in plans:
        dev = provider.execute(plan)[0]
        ref, _ = binding.run(plan)
        assert dev.equals(ref)
