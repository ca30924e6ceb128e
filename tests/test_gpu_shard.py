"""The sharded group-by with real device partials: the rows of one frame
split into 2-4 shards, each shard aggregated on the GPU through the provider,
the partials merged on the host, against the oracle over all rows (the same
bars as the CPU merge tests).  One GPU stands in for the ranks, one after
another; the exchange itself is covered by the gloo test."""
import numpy as np
import pytest

from casegen import config2
from dataframe_mojo_b200 import provider, shard
from dataframe_mojo_b200.frame import col
from oracle import binding
from test_shard import check, make_frame, make_plan

pytestmark = pytest.mark.gpu


def device_run(plan):
    return provider.execute(plan)[0]


def merged(lazy, frame, world):
    parts = shard.split_rows(frame, world)
    partials, spec, rows_name = [], None, None
    for part in parts:
        sub, spec, rows_name = shard.partial_plan(lazy.plan, part)
        partials.append(device_run(sub))
    return shard.merge_partials(lazy.plan, partials, spec, rows_name)


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("keys", [["k1"], ["k1", "k2"]])
def test_device_partials_merge_to_one_query(world, keys):
    frame = make_frame(31 + world, 200_000)
    lazy = make_plan(frame, keys)
    check(merged(lazy, frame, world), binding.run(lazy)[0], frame, keys)


def test_config2_shape_sharded():
    """2M rows of the 100M-row configuration's data over 200K Zipf keys x 64
    codes, in 4 shards."""
    frame = config2(rows=2_000_000, distinct=200_000)
    lazy = frame.lazy().filter(col("p") < 50).group_by(["k1", "k2"], maintain_order=True).agg(
        [col("v").sum().alias("s_v"), col("v").mean().alias("m_v"), col("v").min().alias("lo_v"),
         col("v").max().alias("hi_v"), col("v").count().alias("n_v"), col("v").var().alias("var_v")])
    check(merged(lazy, frame, 4), binding.run(lazy)[0], frame, ["k1", "k2"], p_below=50)
