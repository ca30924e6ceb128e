"""The sharded group-by with real device partials: the rows of one frame
split into 2-4 shards, each shard aggregated on the GPU with its result kept
on the device, the partial rows copied device to device into torch tensors
(dfc_result_copy_to_device), routed to their keys' owners by hash and merged
on the device, against the oracle over all rows (the bars of the CPU merge
tests).  One GPU stands in for the ranks, one after another; the exchange
across ranks is covered by the gloo test.  A world-size-1 NCCL group runs
execute_sharded end to end (all_to_all_single and all_gather on the device)."""
import socket

import numpy as np
import pytest

from casegen import config2
from dataframe_mojo_b200 import provider, shard
from dataframe_mojo_b200.frame import bind, col
from oracle import binding
from test_shard import check, make_frame, make_plan

pytestmark = pytest.mark.gpu


def device_partial(sub):
    bound = bind(sub)
    inputs = [provider.DeviceColumn(s, 0) for s in bound.series]
    try:
        return provider.run_bound(bound, inputs)
    finally:
        for c in inputs:
            c.release()


def merged(lazy, frame, world, owners=None):
    partials, spec, rows_name = [], None, None
    try:
        for part in shard.split_rows(frame, world):
            sub, spec, rows_name = shard.partial_plan(lazy.plan, part)
            partials.append(device_partial(sub))
        return shard.merge_partials(lazy.plan, partials, spec, rows_name, owners=owners)
    finally:
        for p in partials:
            p.free()


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("keys", [["k1"], ["k1", "k2"]])
def test_device_partials_merge_to_one_query(world, keys):
    frame = make_frame(31 + world, 200_000)
    lazy = make_plan(frame, keys)
    check(merged(lazy, frame, world), binding.run(lazy)[0], frame, keys)


def test_config2_shape_sharded():
    """2M rows of the 100M-row configuration's data over 200K Zipf keys x 64
    codes, in 4 shards hashed to 3 owners."""
    frame = config2(rows=2_000_000, distinct=200_000)
    lazy = frame.lazy().filter(col("p") < 50).group_by(["k1", "k2"], maintain_order=True).agg(
        [col("v").sum().alias("s_v"), col("v").mean().alias("m_v"), col("v").min().alias("lo_v"),
         col("v").max().alias("hi_v"), col("v").count().alias("n_v"), col("v").var().alias("var_v")])
    check(merged(lazy, frame, 4, owners=3), binding.run(lazy)[0], frame, ["k1", "k2"], p_below=50)


def test_execute_sharded_over_nccl_world_1():
    import datetime

    import torch
    import torch.distributed as dist

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        frame = make_frame(41, 300_000)
        lazy = make_plan(frame, ["k1", "k2"])
        got = shard.execute_sharded(lazy, 0, 1)
        check(got, binding.run(lazy)[0], frame, ["k1", "k2"])
    finally:
        dist.destroy_process_group()
