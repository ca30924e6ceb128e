"""The batched form (dfc_groupby_batch) against the one-query-per-call path:
every query of a mixed batch must give the same result as when it runs
alone -- keys, integer results, validity and group order bit for bit; float
sums and means within the summation bound of the other parity tests
(relative 1e-12 of the summands' magnitude), variances within
1e-10 * (1 + |value|) -- and a failing query must fail alone, with the same
status and message."""
import numpy as np
import pytest

from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, bind, col
from test_gpu_parity import DTYPES, random_frame

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-12
VAR_RTOL = 1e-10


def make_jobs(rng, n):
    """n queries over a few resident frames: sizes from 0 to 400K rows, one
    to three keys, filters, nulls."""
    jobs, keep = [], []
    for i in range(n):
        nk = 1 + i % 3
        key_dtypes = [DTYPES[(i * 3 + j) % len(DTYPES)] for j in range(nk)]
        val_dtypes = [np.int64, np.float32] if i % 2 else [np.int32, np.float64]
        rows = int(rng.choice([0, 1, 37, 5_000, 60_000, 400_000]))
        frame = random_frame(rng, rows, key_dtypes, val_dtypes, null_rate=0.02 if i % 4 else 0.0)
        aggs = []
        for j in range(2):
            v = col(f"v{j}")
            aggs += [v.sum().alias(f"s{j}"), v.mean().alias(f"m{j}"), v.min().alias(f"lo{j}"), v.max().alias(f"hi{j}"),
                     v.count().alias(f"n{j}"), v.var().alias(f"var{j}")]
        plan = frame.lazy().filter(col("p") >= int(rng.integers(0, 60))).group_by(
            [f"k{j}" for j in range(nk)], maintain_order=bool(i % 5)).agg(aggs)
        bound = bind(plan.plan)
        cols = [provider.DeviceColumn(s) for s in bound.series]
        keep.append(cols)
        jobs.append((bound, cols))
    return jobs, keep


def canonical(frame, nkeys):
    """Rows ordered by their keys (validity, then bytes): the order of a
    query without maintain_order is the device's, not a contract."""
    parts = []
    for c in frame.columns[:nkeys]:
        s = frame[c]
        valid = np.ones(len(s), bool) if s.valid is None else s.valid
        raw = np.ascontiguousarray(s.values).view(np.uint8).reshape(len(s), s.values.dtype.itemsize)
        parts.append(np.concatenate([valid[:, None].astype(np.uint8), np.where(valid[:, None], raw, 0)], axis=1))
    keyb = np.concatenate(parts, axis=1) if parts else np.zeros((frame.height, 0), np.uint8)
    order = np.lexsort(keyb.T[::-1]) if keyb.shape[1] else np.arange(frame.height)
    cols = []
    for c in frame.columns:
        s = frame[c]
        cols.append(Series(c, s.values[order], None if s.valid is None else s.valid[order]))
    return DataFrame(cols)


def same(a, b, label):
    assert a.columns == b.columns and a.height == b.height, (label, a.height, b.height)
    for c in a.columns:
        x, y = a[c], b[c]
        vx = np.ones(len(x), bool) if x.valid is None else x.valid
        vy = np.ones(len(y), bool) if y.valid is None else y.valid
        assert np.array_equal(vx, vy), (label, c)
        xv, yv = x.values[vx], y.values[vx]
        if c.startswith(("m", "var")) or (c.startswith("s") and xv.dtype.kind == "f"):
            xf, yf = xv.astype(np.float64), yv.astype(np.float64)
            j = c[-1]
            scale = np.abs(yf)
            if c.startswith(("s", "m")):
                lo, hi = b[f"lo{j}"], b[f"hi{j}"]
                m = np.maximum(np.abs(lo.values.astype(np.float64)), np.abs(hi.values.astype(np.float64)))[vx]
                m = np.where(np.isfinite(m), m, 0.0)
                n = b[f"n{j}"].values.astype(np.float64)[vx]
                scale = np.maximum(scale, m * (n if c.startswith("s") else 1.0))
                tol = SUM_RTOL * scale
            else:
                tol = VAR_RTOL * (1 + np.abs(yf))
            ok = (np.abs(xf - yf) <= tol) | (xf == yf) | (np.isnan(xf) & np.isnan(yf))
            assert ok.all(), (label, c, np.nonzero(~ok)[0][:5])
        else:
            assert xv.tobytes() == yv.tobytes(), (label, c)  # bit for bit (NaN keys included)


def test_batch_matches_one_by_one():
    rng = np.random.default_rng(77)
    jobs, keep = make_jobs(rng, 40)
    batch = provider.run_batch(jobs)
    for i, ((bound, cols), got) in enumerate(zip(jobs, batch)):
        try:
            alone = provider.run_bound(bound, cols)
        except provider.ProviderError as e:
            assert isinstance(got, provider.ProviderError), (i, got)
            assert got.status == e.status and str(got) == str(e), (i, str(got), str(e))
            continue
        assert isinstance(got, provider.DeviceResult), (i, got)
        x, y = got.to_frame(), alone.to_frame()
        if not bound.maintain_order:
            x, y = canonical(x, len(bound.keys)), canonical(y, len(bound.keys))
        same(x, y, f"query {i}")
        got.free()
        alone.free()
    for cols in keep:
        for c in cols:
            c.release()


def test_batch_failures_stay_per_query():
    """An overflowing Int32 sum, an unsupported plan and a good query in one
    batch: only the first two fail, each with its own message."""
    big = np.full(10, 2**31 - 1, dtype=np.int32)
    f1 = DataFrame([Series("k", np.zeros(10, np.int64)), Series("v", big)])
    over = bind(f1.lazy().group_by("k").agg(col("v").sum()).plan)
    good_frame = DataFrame([Series("k", np.arange(1000, dtype=np.int64) % 7), Series("v", np.ones(1000, np.int64))])
    good = bind(good_frame.lazy().group_by("k", maintain_order=True).agg(col("v").sum()).plan)
    jobs = []
    for b in (over, good):
        jobs.append((b, [provider.DeviceColumn(s) for s in b.series]))
    # A query with five keys is rejected before anything runs.
    wide = DataFrame([Series(f"k{i}", np.zeros(4, np.int8)) for i in range(5)] + [Series("v", np.ones(4))])
    wb = bind(wide.lazy().group_by([f"k{i}" for i in range(5)]).agg(col("v").sum()).plan)
    jobs.append((wb, [provider.DeviceColumn(s) for s in wb.series]))
    out = provider.run_batch(jobs)
    assert isinstance(out[0], provider.ProviderError) and str(out[0]) == "int32 expression sum overflow"
    assert isinstance(out[1], provider.DeviceResult)
    r = out[1].to_frame()
    assert r["k"].values.tolist() == list(range(7)) and int(r["v"].values.sum()) == 1000
    out[1].free()
    assert isinstance(out[2], provider.UnsupportedError)
    for _, cols in jobs:
        for c in cols:
            c.release()
