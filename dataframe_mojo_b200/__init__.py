"""dataframe_mojo_b200 — a B200 (sm_100a) accelerator provider for
dataframe_mojo's filtered hash group-by:

    filter(predicate) -> group_by(keys, maintain_order) -> agg(sum/count/min/max/mean/var/std/len/null_count)

The compute is libdfcuda.so (csrc/, C ABI in include/dfcuda.h).  This Python
layer mirrors the reference's provider interface (provider.py) and the plan
shapes the core hands it (frame.py); it has no CPU execution path.
"""
from .frame import DataFrame, LazyFrame, Series, col, lit
from .provider import (
    DataFaultError,
    DeviceColumn,
    DeviceResult,
    ProviderError,
    ResidentTable,
    UnsupportedError,
    describe,
    devices,
    execute,
    execute_profiled,
    handoff_estimate,
    handoff_execute,
    handoff_supports,
    installed,
    pipeline_costs,
    pipeline_estimate,
    pipeline_supports,
    run_pipeline,
    transfer_model,
)

__all__ = [
    "DataFrame",
    "LazyFrame",
    "Series",
    "col",
    "lit",
    "DataFaultError",
    "DeviceColumn",
    "DeviceResult",
    "ProviderError",
    "ResidentTable",
    "UnsupportedError",
    "describe",
    "devices",
    "execute",
    "execute_profiled",
    "handoff_estimate",
    "handoff_execute",
    "handoff_supports",
    "installed",
    "pipeline_costs",
    "pipeline_estimate",
    "pipeline_supports",
    "run_pipeline",
    "transfer_model",
]
