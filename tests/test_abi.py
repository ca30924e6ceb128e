"""The C ABI without a GPU: the library loads, exports every symbol
include/dfcuda.h declares, and the provider's host-side rules hold."""
import re
from pathlib import Path

import numpy as np
import pytest

from casegen import config1, config1_plan
from dataframe_mojo_b200 import _native as N
from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, bind, col

HEADER = Path(__file__).resolve().parent.parent / "include" / "dfcuda.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"DFC_API\s+[\w\s\*]+?\b(dfc_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "dfc_groupby" in names and "dfc_column_register" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    bound = {s[0] for s in N.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_version_and_status_names():
    lib = N.lib()
    assert lib.dfc_version() == N.ABI_VERSION
    assert lib.dfc_status_name(N.DATA_OVERFLOW) == b"data overflow"
    assert lib.dfc_status_name(N.OK) == b"ok"


def test_installed_and_describe_touch_no_device():
    assert provider.installed() in (True, False)
    plan = config1_plan(config1(rows=1000))
    text = provider.describe(plan)
    assert text.startswith("ENGINE accel:") and "SCAN_FRAME" in text


def test_discrete_device_declines_node_handoff():
    plan = config1_plan(config1(rows=100))
    assert provider.handoff_supports(plan) is False
    key, est = provider.handoff_estimate(plan, 100)
    assert key.startswith("cuda:groupby") and est == -1.0


def test_unsupported_plans_rejected_before_submission():
    frame = DataFrame([Series(f"k{i}", np.arange(4, dtype=np.int32)) for i in range(5)] + [Series("v", np.ones(4))])
    plan = frame.lazy().group_by([f"k{i}" for i in range(5)]).agg(col("v").sum())
    assert "rejected" in provider.describe(plan)
    with pytest.raises(provider.UnsupportedError):
        provider.execute(plan)
    assert provider.pipeline_supports(plan, 0) is False


def test_literal_binding_follows_column_type():
    frame = DataFrame([Series("k", np.zeros(3, np.int32)), Series("p", np.arange(3, dtype=np.int32))])
    with pytest.raises(TypeError):
        bind(frame.lazy().filter(col("p") > 2**40).group_by("k").agg(col("p").sum()).plan)
    with pytest.raises(TypeError):
        bind(frame.lazy().filter(col("p") > 1.5).group_by("k").agg(col("p").sum()).plan)
    b = bind(frame.lazy().filter((col("p") > 0) & ~col("p").is_null()).group_by("k").agg(col("p").sum()).plan)
    assert [op[0] for op in b.pred] == [N.PRED_CMP, N.PRED_IS_NULL, N.PRED_NOT, N.PRED_AND]


def test_env_settings_validated():
    import os

    old = os.environ.get("DATAFRAME_ACCEL_DEVICE")
    os.environ["DATAFRAME_ACCEL_DEVICE"] = "gpu0"
    try:
        with pytest.raises(ValueError):
            provider._device_from_env()
    finally:
        if old is None:
            del os.environ["DATAFRAME_ACCEL_DEVICE"]
        else:
            os.environ["DATAFRAME_ACCEL_DEVICE"] = old


def test_regime_setting(monkeypatch):
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "partitioned")
    assert provider._regime_flags() == N.Q_FORCE_PARTITIONED
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "Global")
    assert provider._regime_flags() == N.Q_FORCE_GLOBAL
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "")
    assert provider._regime_flags() == 0
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "radix")
    with pytest.raises(ValueError):
        provider._regime_flags()
    monkeypatch.setenv("DATAFRAME_ACCEL_REGIME", "shared")
    monkeypatch.setenv("DATAFRAME_ACCEL_FLOAT32", "compensated")
    assert provider._regime_flags() == N.Q_FORCE_SHARED | N.Q_FLOAT32_COMPENSATED
    monkeypatch.setenv("DATAFRAME_ACCEL_FLOAT32", "fp32")
    with pytest.raises(ValueError):
        provider._regime_flags()


def test_cpu_engine_is_not_part_of_the_provider():
    plan = config1_plan(config1(rows=10))
    with pytest.raises(ValueError):
        plan.collect(engine="cpu")


@pytest.mark.parametrize("rows", [0, 1, 7, 8, 9, 63, 64, 65, 1000, 4099])
def test_packed_validity_series(rows):
    """Result columns keep the packed bitmap they were copied into and unpack
    it on first use; an all-set bitmap means no nulls."""
    from dataframe_mojo_b200.frame import bits_all_set, pack_validity

    rng = np.random.default_rng(rows)
    values = rng.integers(0, 100, rows).astype(np.int64)
    all_set = np.full((rows + 7) // 8 + 3, 0xFF, np.uint8)  # longer than needed, tail bytes ignored
    s = Series.from_bits("x", values, all_set)
    assert not s.has_nulls and s.valid is None and s.validity_bits() is None
    assert bits_all_set(all_set, rows)

    valid = rng.random(rows) < 0.7
    if rows:
        valid[-1] = False  # a null in the last (possibly partial) byte
    bits = pack_validity(valid)
    padded = np.concatenate([bits, np.zeros(2, np.uint8)]) if rows else bits
    s = Series.from_bits("x", values, padded)
    assert s.has_nulls == (rows > 0)
    if rows:
        assert not bits_all_set(bits, rows)
        assert np.array_equal(s.validity_bits(), bits)  # kept packed, not repacked
        assert np.array_equal(s.valid, valid)
        assert s.equals(Series("x", values, valid))
        assert s.to_list() == [int(v) if ok else None for v, ok in zip(values, valid)]
    # Bits beyond `rows` in the last byte do not count.
    if rows % 8:
        tail = pack_validity(np.ones(rows, bool))
        tail[-1] &= (1 << (rows % 8)) - 1
        assert bits_all_set(tail, rows)
    with pytest.raises(ValueError):
        Series.from_bits("x", np.zeros(64, np.int64), np.zeros(7, np.uint8))
