"""Whole-pipeline placement (engine="auto"): pipeline_supports /
pipeline_estimate / pipeline_costs give the core's placement solver a device
cost for a region this provider runs (dataframe/lazy_api.mojo:2935-3110,
2537-2541), and run_pipeline leaves the result on the device, copied to the
host per column on first read (dataframe/storage/residence.mojo:33-147), so
a following device query reads it in place."""
import numpy as np
import pytest

from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding


def frame(rows=50_000, seed=5):
    rng = np.random.default_rng(seed)
    return DataFrame([Series("k", rng.integers(0, 500, rows).astype(np.int64)),
                      Series("v", rng.integers(-9, 9, rows).astype(np.int64), rng.random(rows) > 0.1),
                      Series("p", rng.integers(0, 10, rows).astype(np.int32))])


def region(f):
    return f.lazy().filter(col("p") < 6).group_by("k", maintain_order=True).agg(
        [col("v").sum().alias("s"), col("v").count().alias("n"), col("v").min().alias("lo")])


def test_estimates_scale_with_input_and_follow_calibration():
    small, large = region(frame(1_000)), region(frame(100_000))
    a, b = provider.pipeline_estimate(small, 0), provider.pipeline_estimate(large, 0)
    assert 0 < a < b
    assert provider.pipeline_costs(large, 0) == (-1.0, b)
    # A measured run of the layout replaces the built-in rate.
    provider._record_run(large.plan, 10 * b)
    assert provider.pipeline_estimate(large, 0) > b
    feats = provider.PipelineFeatures(rows=100_000, input_bytes=4_000_000)
    assert provider.pipeline_estimate(large, 0, feats) > 0


def test_unsupported_region_has_no_estimate():
    f = frame(100)
    lf = f.lazy().filter(col("p") < 6)  # no aggregation: not a region this provider runs
    assert provider.pipeline_estimate(lf, 0) == -1.0
    assert provider.pipeline_supports(lf, 0) is False


@pytest.mark.gpu
def test_run_pipeline_result_is_resident_and_feeds_a_device_query():
    f = frame()
    out = provider.run_pipeline(region(f), 0)
    assert all(isinstance(out[c], provider.ResidentSeries) for c in out.columns)
    assert not out["s"].on_host()
    ref, _ = binding.run(region(f))
    assert out.equals(ref)
    assert out["s"].on_host()
    # The resident result as the input of a second query, read in place.
    cols = {n: provider.DeviceColumn.from_resident(out[n]) for n in ("k", "s")}
    shape = DataFrame([Series("k", np.zeros(1, np.int64)), Series("s", np.zeros(1, np.int64))])
    from dataframe_mojo_b200.frame import bind

    second = shape.lazy().filter(col("s") > 0).group_by("k", maintain_order=True).agg(col("s").max().alias("m"))
    bound = bind(second.plan)
    res = provider.run_bound(bound, [cols[n] for n in bound.names])
    got = res.to_frame()
    res.free()
    host = DataFrame([ref["k"], ref["s"]])
    want, _ = binding.run(host.lazy().filter(col("s") > 0).group_by("k", maintain_order=True).agg(
        col("s").max().alias("m")))
    assert got.equals(want)
    for c in cols.values():
        c.release()


@pytest.mark.gpu
def test_transfer_model_is_measured():
    """dfc_measure_transfer: pinned copies fitted to the reference's ByteCost
    (fixed_ns + ns_per_byte x bytes, dataframe/devices.mojo:44-80); PCIe
    rates lie between 1 and 200 GB/s."""
    m = provider.calibrate_transfer(0, 1 << 26)
    assert m.measured() and provider.transfer_model(0) == m
    for c in (m.to_device, m.to_host):
        assert 1 / 200 <= c.ns_per_byte <= 1.0, c
        assert 0 <= c.fixed_ns < 1e6, c
        assert c.cost(1 << 30) > c.cost(1 << 20)
    with pytest.raises(provider.UnsupportedError):
        provider.calibrate_transfer(0, 1024)  # below 8 KiB: DFC_INVALID
