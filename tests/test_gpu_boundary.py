"""The provider boundary under failure, through the C ABI: the device memory
limit (DATAFRAME_ACCEL_MEMORY_LIMIT), borrowed pointers that are not device
memory of the query's device, host-side fault injection (DFCUDA_FAULT=alloc|
capacity|timeout|overflow) and the host's bounded wait (DFC_WAIT_TIMEOUT_S).
Every failure is made on the host: no kernel is broken and nothing waits on
the GPU without a bound.  After each failure the next query must run and
match the oracle (contract: unsupported work is rejected before submission,
errors after submission propagate, docs/design/accelerator-contract.md:
189-202)."""
import ctypes as C

import numpy as np
import pytest

from casegen import config1, config1_plan, config2, config2_plan
from dataframe_mojo_b200 import _native as N
from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding
from test_gpu_parity import compare_with_oracle, magnitude

pytestmark = pytest.mark.gpu


def small():
    return config1_plan(config1(rows=200_000))


def assert_recovers():
    plan = small()
    assert provider.execute(plan)[0].equals(binding.run(plan)[0])


def test_memory_limit_rejects_before_submission(monkeypatch):
    monkeypatch.setenv("DATAFRAME_ACCEL_MEMORY_LIMIT", "4096")
    with pytest.raises(provider.UnsupportedError) as ei:
        provider.execute(small())
    assert "memory limit" in str(ei.value)
    assert provider.devices()[0].budget_bytes == 4096
    monkeypatch.setenv("DATAFRAME_ACCEL_MEMORY_LIMIT", str(64 << 30))
    assert_recovers()
    monkeypatch.delenv("DATAFRAME_ACCEL_MEMORY_LIMIT")
    assert_recovers()


def test_device_column_must_be_device_memory():
    host = np.arange(1024, dtype=np.int64)
    h = C.c_void_p()
    st = N.lib().dfc_column_register(0, N.INT64, len(host), host.ctypes.data, None, 0, N.COLUMN_DEVICE, C.byref(h))
    assert st == N.INVALID
    assert "device memory" in N.last_error()
    assert_recovers()


def test_noalloc_rejects_host_inputs():
    from dataframe_mojo_b200.frame import bind

    plan = small()
    bound = bind(plan.plan)
    keep = [np.ascontiguousarray(s.values) for s in bound.series]
    descs = (N.DeviceColumnDesc * len(keep))()
    for i, (s, arr) in enumerate(zip(bound.series, keep)):
        descs[i].dtype = N.INT64 if arr.dtype == np.int64 else N.INT32
        descs[i].values = arr.ctypes.data
        descs[i].validity = None
    outs = (N.DeviceOutput * len(bound.out_names))()
    groups = C.c_uint64(0)
    q = provider._query_struct(bound, [C.c_void_p(None)] * len(bound.names), None, 0)
    st = N.lib().dfc_groupby_noalloc(C.byref(q), 0, len(bound.series[0]), descs, 0, outs, C.byref(groups))
    assert st == N.INVALID and "device memory" in N.last_error()


def test_injected_allocation_failure(monkeypatch):
    monkeypatch.setenv("DFCUDA_FAULT", "alloc")
    with pytest.raises(provider.ProviderError) as ei:
        provider.execute(small())
    assert ei.value.status == N.OOM and "DFCUDA_FAULT=alloc" in str(ei.value)
    monkeypatch.delenv("DFCUDA_FAULT")
    assert_recovers()


@pytest.mark.parametrize("regime", ["global", "partitioned"])
def test_injected_capacity_reruns_and_matches(monkeypatch, regime):
    monkeypatch.setenv("DFCUDA_FAULT", "capacity")
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", regime)
    frame = config2(rows=500_000, distinct=20_000)
    compare_with_oracle(config2_plan(frame), f"capacity-{regime}", float_cols=("sum", "mean"), var_cols=("var",),
                        scales=lambda ref: dict(zip(("sum", "mean"), magnitude(ref, "count", "min", "max"))))
    assert provider.last_timings()["retries"] >= 1


def test_injected_timeout(monkeypatch):
    monkeypatch.setenv("DFCUDA_FAULT", "timeout")
    with pytest.raises(provider.ProviderError) as ei:
        provider.execute(small())
    assert ei.value.status == N.TIMEOUT
    monkeypatch.delenv("DFCUDA_FAULT")
    assert_recovers()


def test_injected_overflow_gives_the_cpu_text(monkeypatch):
    monkeypatch.setenv("DFCUDA_FAULT", "overflow")
    frame = DataFrame([Series("k", np.arange(10, dtype=np.int64) % 3), Series("v", np.ones(10, np.int32))])
    with pytest.raises(provider.ProviderError) as ei:
        provider.execute(frame.lazy().group_by("k").agg(col("v").sum()))
    assert ei.value.status == N.DATA_OVERFLOW
    assert str(ei.value) == "int32 expression sum overflow"
    monkeypatch.delenv("DFCUDA_FAULT")
    assert_recovers()


def test_host_wait_limit_expires(monkeypatch):
    """A wait limit far shorter than the query: the host gives up with
    DFC_TIMEOUT while the kernels finish on their own (the working memory is
    released stream-ordered, after them); the next query is unaffected."""
    frame = config2(rows=20_000_000, distinct=100_000)
    plan = config2_plan(frame)
    monkeypatch.setenv("DFC_WAIT_TIMEOUT_S", "0.000001")
    with pytest.raises(provider.ProviderError) as ei:
        provider.execute(plan)
    assert ei.value.status == N.TIMEOUT
    monkeypatch.delenv("DFC_WAIT_TIMEOUT_S")
    assert_recovers()
