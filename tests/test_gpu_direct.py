"""Direct-addressed own tables (dataframe/aggregation/perfect_hash.mojo:1-50):
integer keys whose exact ranges together fit 12 bits take slot
sum((value - min + 1, 0 for null) << shift) in each CTA's shared-memory
table, with no hashing or probing.  Each case checks that the direct path
ran (dfc_timings.direct_slots) and that the result equals the oracle's bit
for bit (every output here is exact); a key domain too wide for 12 bits
falls back to hashed tables with the same result."""
import numpy as np
import pytest

from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding

pytestmark = pytest.mark.gpu


def frame(seed, rows, keys):
    rng = np.random.default_rng(seed)
    cols = []
    for name, dt, lo, hi, nulls in keys:
        v = rng.integers(lo, hi + 1, rows).astype(dt)
        cols.append(Series(name, v, rng.random(rows) > nulls if nulls else None))
    cols.append(Series("v", rng.integers(-1000, 1000, rows).astype(np.int64), rng.random(rows) > 0.05))
    cols.append(Series("p", rng.integers(0, 10, rows).astype(np.int32)))
    return DataFrame(cols)


def plan_of(f, keys):
    v = col("v")
    return f.lazy().filter(col("p") < 7).group_by(keys, maintain_order=True).agg(
        [v.sum().alias("s"), v.count().alias("n"), v.min().alias("lo"), v.max().alias("hi"),
         v.first().alias("f"), v.last().alias("l"), v.len().alias("len"), v.null_count().alias("z")])


CASES = {
    # name: (key specs (name, dtype, min, max, null share), expected direct bits)
    "int8_signed": ([("a", np.int8, -7, 5, 0.0)], 4),
    "int8_uint16_nulls": ([("a", np.int8, -3, 3, 0.1), ("b", np.uint16, 100, 140, 0.05)], 9),
    "int32_negative": ([("a", np.int32, -1010, -990, 0.02)], 5),
    "int64_offset": ([("a", np.int64, 10**12, 10**12 + 200, 0.0)], 8),
    "uint32_codes_int16": ([("a", np.uint32, 0, 63, 0.0), ("b", np.int16, -2, 2, 0.2)], 10),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("regime", ["auto", "shared"])
def test_direct_tables_match_oracle(case, regime, monkeypatch):
    from dataframe_mojo_b200 import provider

    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", regime)
    specs, bits = CASES[case]
    f = frame(sum(map(ord, case)), 400_000, specs)
    plan = plan_of(f, [s[0] for s in specs])
    dev = provider.execute(plan)[0]
    t = provider.last_timings()
    ref, _ = binding.run(plan)
    assert dev.equals(ref), case
    if regime == "shared":
        assert t["direct_slots"] == max(64, 1 << bits), (case, t)


def test_wide_domain_stays_hashed(monkeypatch):
    from dataframe_mojo_b200 import provider

    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "shared")
    rng = np.random.default_rng(3)
    k = rng.choice(np.array([-(2**40), 0, 5, 2**40], np.int64), 200_000)  # 4 keys over a 2^41 range
    f = DataFrame([Series("a", k), Series("v", rng.integers(0, 9, 200_000).astype(np.int64)),
                   Series("p", rng.integers(0, 10, 200_000).astype(np.int32))])
    plan = plan_of(f, ["a"])
    dev = provider.execute(plan)[0]
    assert provider.last_timings()["direct_slots"] == 0
    ref, _ = binding.run(plan)
    assert dev.equals(ref)


@pytest.mark.parametrize("rows", [0, 1, 37])
@pytest.mark.parametrize("regime", ["auto", "shared"])
def test_direct_edge_cases(rows, regime, monkeypatch):
    """Tiny inputs, all-null keys and a filter that keeps nothing."""
    from dataframe_mojo_b200 import provider

    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", regime)
    rng = np.random.default_rng(rows + 7)
    a = rng.integers(-3, 4, rows).astype(np.int8)
    b = rng.integers(0, 9, rows).astype(np.uint16)
    frame = DataFrame([Series("a", a, np.zeros(rows, bool)), Series("b", b, rng.random(rows) > 0.3),
                       Series("v", rng.integers(-5, 5, rows).astype(np.int64)),
                       Series("p", rng.integers(0, 10, rows).astype(np.int32))])
    for pred in (col("p") < 7, col("p") > 100):
        plan = frame.lazy().filter(pred).group_by(["a", "b"], maintain_order=True).agg(
            [col("v").sum().alias("s"), col("v").count().alias("n"), col("v").first().alias("f")])
        dev = provider.execute(plan)[0]
        ref, _ = binding.run(plan)
        assert dev.equals(ref), (rows, regime)
