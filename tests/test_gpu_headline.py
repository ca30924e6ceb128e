"""The 100M-row configuration the headline rows/s is quoted on, checked
against the CPU oracle at full size.

The data are exactly what bench.py times: its seeded generator (seed 2, run
on the device), copied to the host.  The query goes through the provider
(host columns registered, the query, the result copied back), once with the
automatic regime choice (the radix-partitioned regime for these 7.4M
groups) and once forced onto the global table; the oracle's multithreaded
restatement of the reference aggregate table checks both.  Bars, as in
test_gpu_parity: keys, group order, counts, min/max and validity bit for bit;
sums and means within 1e-12 of the summands' magnitude (count x max |x| per
group); variances within 1e-10 (1 + |var|)."""
import numpy as np
import pytest

from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series
from test_gpu_parity import SUM_RTOL, VAR_RTOL, magnitude

pytestmark = pytest.mark.gpu


def compare_frames(dev: DataFrame, ref: DataFrame, label: str, float_cols=(), var_cols=(), scales=None):
    from casegen import assert_frames_match

    assert dev.columns == ref.columns, label
    assert dev.height == ref.height, (label, dev.height, ref.height)
    for c in ref.columns:
        if c in float_cols or c in var_cols:
            continue
        assert_frames_match(DataFrame([dev[c]]), DataFrame([ref[c]]), label=f"{label}:{c}")
    for c in tuple(float_cols) + tuple(var_cols):
        a, b = dev[c], ref[c]
        va = np.ones(len(b), bool) if b.valid is None else b.valid
        vd = np.ones(len(a), bool) if a.valid is None else a.valid
        assert np.array_equal(va, vd), (label, c, "validity")
        x, y = a.values.astype(np.float64)[va], b.values.astype(np.float64)[va]
        if c in var_cols:
            bound = VAR_RTOL * (1 + np.abs(y))
        else:
            bound = SUM_RTOL * np.maximum(np.abs(y), scales[c][va])
        ok = (np.abs(x - y) <= bound) | (x == y) | (np.isnan(x) & np.isnan(y))
        assert ok.all(), (label, c, int((~ok).sum()), np.nonzero(~ok)[0][:5])


@pytest.fixture(scope="module")
def headline():
    import bench
    import torch

    cols = bench.generate(bench.ROWS, 2, "cuda")
    h = bench.host_numpy(cols)
    del cols
    torch.cuda.empty_cache()
    frame = DataFrame([Series("k1", h["k1"]), Series("k2", h["k2"]), Series("v", h["v"], h["v_valid"]),
                       Series("p", h["p"])])
    plan = bench.plan_for(frame)
    from oracle import binding

    ref, _ = binding.run(plan, threads=0)
    return plan, ref


def scales_of(ref):
    s, m = magnitude(ref, "count", "min", "max")
    return {"sum": s, "mean": m}


def test_headline_auto_regime_against_oracle(headline, monkeypatch):
    monkeypatch.delenv("DATAFRAME_ACCEL_REGIME", raising=False)
    plan, ref = headline
    assert ref.height > 7_000_000
    dev = provider.execute(plan)[0]
    t = provider.last_timings()
    compare_frames(dev, ref, "headline-auto", float_cols=("sum", "mean"), var_cols=("var",), scales=scales_of(ref))
    assert t["regime"] == 2, t  # the radix-partitioned regime takes 7.4M groups


def test_headline_global_table_against_oracle(headline, monkeypatch):
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "global")
    plan, ref = headline
    dev = provider.execute(plan)[0]
    assert provider.last_timings()["regime"] == 0
    compare_frames(dev, ref, "headline-global", float_cols=("sum", "mean"), var_cols=("var",), scales=scales_of(ref))
