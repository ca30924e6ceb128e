"""The sharded group-by on CPU: rows split across ranks, each rank's partial
aggregations computed by the oracle (standing in for the rank's GPU), the
partial rows routed to their keys' owners by hash, the owners' merge (torch
tensors, as on the device) against the oracle over all rows -- keys,
integers, validity and group order bit-exact, sums and means within 1e-12 of
the summands' magnitude, variances within 1e-10 -- in one process and over a
world-size-2 gloo process group (all_to_all_single + all_gather)."""
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


def key_bytes(cols: list[Series]) -> np.ndarray:
    """One fixed-width byte string per row: per key column a validity byte and
    the value bytes (0 when null; NaN canonical and -0.0 as 0.0 for floats)."""
    n = len(cols[0]) if cols else 0
    pieces = []
    for s in cols:
        valid = np.ones(n, bool) if s.valid is None else s.valid
        v = s.values.copy()
        if v.dtype.kind == "f":
            v = np.where(np.isnan(v), np.array(np.nan, v.dtype), v).astype(v.dtype)
            v = np.where(v == 0, np.zeros(1, v.dtype), v).astype(v.dtype)
        raw = np.ascontiguousarray(v).view(np.uint8).reshape(n, v.dtype.itemsize).copy()
        raw[~valid] = 0
        pieces += [valid[:, None].astype(np.uint8), raw]
    mat = np.ascontiguousarray(np.concatenate(pieces, axis=1))
    return mat.view(np.dtype((np.void, mat.shape[1]))).ravel()


def abs_sums(frame, keys, column, want, p_below=80):
    """Per output group of `want`: sum |x| over the rows the filter (p <
    p_below) keeps."""
    keep = frame["p"].values < p_below
    rows = [Series(k, frame[k].values[keep], None if frame[k].valid is None else frame[k].valid[keep]) for k in keys]
    kb = key_bytes(rows)
    uniq, inv = np.unique(kb, return_inverse=True)
    v = frame[column]
    valid = (np.ones(frame.height, bool) if v.valid is None else v.valid)[keep]
    x = np.where(valid & ~np.isnan(v.values[keep].astype(np.float64)), np.abs(v.values[keep].astype(np.float64)), 0.0)
    tot = np.bincount(inv.ravel(), weights=x, minlength=len(uniq))
    out = key_bytes([want[k] for k in keys])
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


def partials_of(lazy, frame, world):
    partials, spec, rows_name = [], None, None
    for part in shard.split_rows(frame, world):
        sub, spec, rows_name = shard.partial_plan(lazy.plan, part)
        partials.append(oracle_run(sub))
    return partials, spec, rows_name


@pytest.mark.parametrize("owners", [1, 2, 5])
def test_owner_routing_is_independent_of_owner_count(owners):
    """Every group lands on exactly one owner: the merged result does not
    depend on how many owners the rows are hashed to."""
    frame = make_frame(17, 15_000)
    lazy = make_plan(frame, ["k1", "k2"])
    partials, spec, rows_name = partials_of(lazy, frame, 3)
    got = shard.merge_partials(lazy.plan, partials, spec, rows_name, owners=owners)
    check(got, oracle_run(lazy), frame, ["k1", "k2"])


def test_owner_hash_treats_equal_keys_alike():
    """NaN payloads, -0.0 / 0.0 and the bits under a null key do not change a
    key's owner."""
    import torch

    vals = np.array([np.nan, -np.nan, 0.0, -0.0, 7.0, 1.0], np.float64)
    bits = vals.view(np.int64).copy()
    bits[1] |= 5  # another NaN payload
    valid = np.array([True, True, True, True, False, False])
    cols = shard._Cols()
    cols.add("k", torch.from_numpy(bits), torch.from_numpy(valid), np.float64)
    own = shard._owner(shard._key_matrix(cols, ["k"]), 1 << 20).tolist()
    assert own[0] == own[1] and own[2] == own[3] and own[4] == own[5]
    assert len({own[0], own[2], own[4]}) == 3


def test_unsigned_and_narrow_columns():
    rng = np.random.default_rng(8)
    rows = 6_000
    frame = DataFrame([
        Series("k", rng.integers(0, 40, rows).astype(np.uint16), rng.random(rows) > 0.05),
        Series("u", rng.integers(0, 2**62, rows, dtype=np.uint64) * np.uint64(3), rng.random(rows) > 0.1),
        Series("i", rng.integers(-2**31, 2**31 - 1, rows).astype(np.int32) // 100_000, rng.random(rows) > 0.1),
        Series("b", rng.integers(-128, 127, rows).astype(np.int8)),
        Series("f", rng.standard_normal(rows).astype(np.float32)),
        Series("p", rng.integers(0, 100, rows).astype(np.int32)),
    ])
    lazy = frame.lazy().filter(col("p") < 80).group_by("k", maintain_order=True).agg(
        [col("u").min().alias("lo_u"), col("u").max().alias("hi_u"), col("i").sum().alias("s_i"),
         col("b").sum().alias("s_b"), col("b").min().alias("lo_b"), col("f").max().alias("hi_f"),
         col("f").min().alias("lo_f"), col("i").mean().alias("m_i"), col("u").count().alias("n_u")])
    partials, spec, rows_name = partials_of(lazy, frame, 4)
    want = oracle_run(lazy)
    got = shard.merge_partials(lazy.plan, partials, spec, rows_name, owners=3)
    assert got.columns == want.columns
    for c in want.columns:
        if c == "m_i":
            assert np.allclose(got[c].values, want[c].values, rtol=1e-12, atol=0), c
        else:
            assert got[c].equals(want[c]), c


def test_sum_overflow_across_shards_raises_the_cpu_message():
    """Each shard's Int64 sum fits; the total does not: the merge raises the
    CPU provider's overflow error."""
    from dataframe_mojo_b200 import provider

    frame = DataFrame([Series("k", np.zeros(4, np.int64)), Series("v", np.full(4, 2**62, np.int64))])
    lazy = frame.lazy().group_by("k", maintain_order=True).agg(col("v").sum().alias("s"))
    partials, spec, rows_name = partials_of(lazy, frame, 4)
    with pytest.raises(provider.ProviderError) as got:
        shard.merge_partials(lazy.plan, partials, spec, rows_name)
    with pytest.raises(binding.OracleError) as want:
        oracle_run(lazy)
    assert str(got.value) == str(want.value)


def test_non_group_by_and_string_keys_are_rejected():
    frame = make_frame(3, 10)
    with pytest.raises(ValueError):
        shard.execute_sharded(frame.lazy().select(col("vi").sum()), 0, 1, run=oracle_run)
    strs = DataFrame([Series("s", np.array(["a", "b"], dtype=object)), Series("v", np.arange(2))])
    with pytest.raises(ValueError):
        shard.merge_partials(strs.lazy().group_by("s").agg(col("v").count()).plan, [], {}, "__rows")


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
