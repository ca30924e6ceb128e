"""The sharded group-by's host logic on CPU: rows split across ranks, each
rank's partial aggregations computed by the oracle (standing in for the rank's
GPU), the merge of the partials against the oracle over all rows -- keys,
integers, validity and group order bit-exact, sums and means within 1e-12 of
the summands' magnitude, variances within 1e-10 -- and the exchange over a
world-size-2 gloo process group."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from dataframe_mojo_b200 import shard
from dataframe_mojo_b200.frame import DataFrame, Series, col
from oracle import binding

SUM_RTOL = 1e-12
VAR_RTOL = 1e-10


def oracle_run(plan):
    return binding.run(plan)[0]


def make_frame(seed, rows):
    rng = np.random.default_rng(seed)
    k1 = rng.integers(0, 50, rows).astype(np.int32)
    k2 = rng.choice(np.array([0.0, -0.0, np.nan, 1.5, -2.0]), rows)
    vi = rng.integers(-10**9, 10**9, rows, dtype=np.int64)
    vf = (rng.standard_normal(rows) * 10.0 ** rng.integers(-3, 4, rows)).astype(np.float32)
    vf[rng.random(rows) < 0.02] = np.nan
    vf[rng.random(rows) < 0.02] = -0.0
    vd = rng.standard_normal(rows) * 1e3
    return DataFrame([
        Series("k1", k1, rng.random(rows) >= 0.05),
        Series("k2", k2, rng.random(rows) >= 0.05),
        Series("vi", vi, rng.random(rows) >= 0.1),
        Series("vf", vf, rng.random(rows) >= 0.1),
        Series("vd", vd, rng.random(rows) >= 0.1),
        Series("p", rng.integers(0, 100, rows).astype(np.int32)),
    ])


def make_plan(frame, keys):
    aggs = []
    for c in ("vi", "vf", "vd"):
        v = col(c)
        aggs += [v.sum().alias(f"s_{c}"), v.mean().alias(f"m_{c}"), v.count().alias(f"n_{c}"),
                 v.var().alias(f"var_{c}"), v.std(ddof=0).alias(f"sd_{c}"),
                 v.null_count().alias(f"z_{c}"), v.len().alias(f"l_{c}")]
    aggs += [col("vi").min().alias("lo_vi"), col("vd").max().alias("hi_vd"), col("vd").min().alias("lo_vd")]
    aggs += [col("vd").sum(min_count=3).alias("s3_vd")]
    return frame.lazy().filter(col("p") < 80).group_by(keys, maintain_order=True).agg(aggs)


def abs_sums(frame, keys, column, want, p_below=80):
    """Per output group of `want`: sum |x| over the rows the filter (p <
    p_below) keeps."""
    keep = frame["p"].values < p_below
    rows = [Series(k, frame[k].values[keep], None if frame[k].valid is None else frame[k].valid[keep]) for k in keys]
    kb = shard._key_bytes(rows)
    uniq, inv = np.unique(kb, return_inverse=True)
    v = frame[column]
    valid = (np.ones(frame.height, bool) if v.valid is None else v.valid)[keep]
    x = np.where(valid & ~np.isnan(v.values[keep].astype(np.float64)), np.abs(v.values[keep].astype(np.float64)), 0.0)
    tot = np.bincount(inv.ravel(), weights=x, minlength=len(uniq))
    out = shard._key_bytes([want[k] for k in keys])
    return tot[np.searchsorted(uniq, out)]


def check(got, want, frame, keys, p_below=80):
    assert got.columns == want.columns
    assert got.height == want.height
    for c in want.columns:
        a, b = got[c], want[c]
        va = np.ones(len(a), bool) if a.valid is None else a.valid
        vb = np.ones(len(b), bool) if b.valid is None else b.valid
        assert np.array_equal(va, vb), c
        x, y = a.values[vb], b.values[vb]
        assert x.dtype == y.dtype, (c, x.dtype, y.dtype)
        if c.startswith(("var_", "sd_")):
            ok = (np.abs(x - y) <= VAR_RTOL * (1 + np.abs(y))) | (np.isnan(x) & np.isnan(y))
            assert ok.all(), c
        elif x.dtype.kind == "f" and c.startswith(("s", "m_")):
            column = c.split("_", 1)[1]
            scale = abs_sums(frame, keys, column, want, p_below)[vb]
            if c.startswith("m_"):
                scale = scale / np.maximum(want[f"n_{column}"].values[vb], 1)
            # A Float32 sum is rounded to Float32 after the sum.
            eps = np.finfo(x.dtype).eps if x.dtype == np.float32 else 0.0
            tol = SUM_RTOL * scale + eps * np.abs(y.astype(np.float64))
            ok = (np.abs(x.astype(np.float64) - y) <= tol) | (np.isnan(x) & np.isnan(y)) | (x == y)
            assert ok.all(), (c, np.nonzero(~ok)[0][:5])
        else:
            assert x.tobytes() == y.tobytes(), c


@pytest.mark.parametrize("world", [1, 2, 3])
@pytest.mark.parametrize("keys", [["k1"], ["k1", "k2"]])
def test_merge_of_partials_matches_one_query(world, keys):
    frame = make_frame(11 + world, 20_000)
    lazy = make_plan(frame, keys)
    parts = shard.split_rows(frame, world)
    partials = []
    spec = rows_name = None
    for part in parts:
        sub, spec, rows_name = shard.partial_plan(lazy.plan, part)
        partials.append(oracle_run(sub))
    got = shard.merge_partials(lazy.plan, partials, spec, rows_name)
    check(got, oracle_run(lazy), frame, keys)


def test_empty_shards():
    frame = make_frame(5, 7)
    lazy = make_plan(frame, ["k1"])
    parts = shard.split_rows(frame, 4)
    partials, spec, rows_name = [], None, None
    for part in parts:
        sub, spec, rows_name = shard.partial_plan(lazy.plan, part)
        partials.append(oracle_run(sub))
    check(shard.merge_partials(lazy.plan, partials, spec, rows_name), oracle_run(lazy), frame, ["k1"])


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        frame = make_frame(21, 30_000)
        lazy = make_plan(frame, ["k1", "k2"])
        got = shard.execute_sharded(lazy, rank, world, run=oracle_run)
        if rank == 0:
            check(got, oracle_run(lazy), frame, ["k1", "k2"])
            out.put("ok")
    except Exception as e:  # reported to the test process
        out.put(f"rank {rank}: {e!r}")
        raise
    finally:
        dist.destroy_process_group()


def test_exchange_over_gloo_world_2():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert out.get(timeout=5) == "ok"
