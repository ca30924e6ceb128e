"""The served form: requests submitted to the native server (continuous
batching, memory admission) give the same results as each query run alone
-- keys, integers, validity and group order bit for bit, floats within the
summation and moments bounds of the other parity tests -- and errors stay
with their request."""
import time

import numpy as np
import pytest

from dataframe_mojo_b200 import provider
from test_gpu_batch import canonical, make_jobs, same

pytestmark = pytest.mark.gpu


def serve_all(server, jobs, gap_s=0.0):
    for i, (bound, cols) in enumerate(jobs):
        server.submit(bound, cols, i)
        if gap_s:
            time.sleep(gap_s)
    got = {}
    deadline = time.time() + 120
    while len(got) < len(jobs) and time.time() < deadline:
        for tag, res, lat, queue in server.poll(wait_ms=50):
            assert lat >= queue >= 0
            got[tag] = res
    assert len(got) == len(jobs)
    return got


def check_against_alone(jobs, got):
    for i, (bound, cols) in enumerate(jobs):
        try:
            alone = provider.run_bound(bound, cols)
        except provider.ProviderError as e:
            assert isinstance(got[i], provider.ProviderError), (i, got[i])
            assert got[i].status == e.status and str(got[i]) == str(e)
            continue
        assert isinstance(got[i], provider.DeviceResult), (i, got[i])
        x, y = got[i].to_frame(), alone.to_frame()
        if not bound.maintain_order:
            x, y = canonical(x, len(bound.keys)), canonical(y, len(bound.keys))
        same(x, y, f"request {i}")
        got[i].free()
        alone.free()


def test_served_requests_match_alone():
    rng = np.random.default_rng(91)
    jobs, keep = make_jobs(rng, 48)
    server = provider.Server(max_inflight=16)
    try:
        got = serve_all(server, jobs, gap_s=0.0005)
        assert server.stats()["completed"] == len(jobs)
    finally:
        server.close()
    check_against_alone(jobs, got)
    for cols in keep:
        for c in cols:
            c.release()


def test_memory_admission_one_at_a_time():
    """A budget below any request's working memory admits one request at a
    time (the server never starves): every result still arrives, in order of
    admission, and matches the query alone."""
    rng = np.random.default_rng(5)
    jobs, keep = make_jobs(rng, 10)
    server = provider.Server(max_inflight=8, memory_budget=1)
    try:
        got = serve_all(server, jobs)
        assert server.stats()["max_inflight_seen"] <= 1
    finally:
        server.close()
    check_against_alone(jobs, got)
    for cols in keep:
        for c in cols:
            c.release()


def test_full_grid_requests_two_in_flight():
    """Requests whose scans fill every SM (2M rows each): the server keeps at
    most two of them in flight, reuses finished requests' working memory, and
    every result matches the query run alone."""
    rng = np.random.default_rng(17)
    jobs, keep = [], []
    from dataframe_mojo_b200.frame import bind, col
    from test_gpu_parity import random_frame

    frames = [random_frame(rng, 2_000_000, [np.int32], [np.int64, np.float64], null_rate=0.02) for _ in range(2)]
    for i in range(12):
        frame = frames[i % 2]
        plan = frame.lazy().filter(col("p") >= int(rng.integers(0, 60))).group_by("k0", maintain_order=True).agg(
            [col("v0").sum().alias("s0"), col("v0").min().alias("lo0"), col("v0").max().alias("hi0"),
             col("v0").count().alias("n0"), col("v1").mean().alias("m1"), col("v1").var().alias("var1"),
             col("v1").min().alias("lo1"), col("v1").max().alias("hi1"), col("v1").count().alias("n1")])
        bound = bind(plan.plan)
        cols = [provider.DeviceColumn(s) for s in bound.series]
        keep.append(cols)
        jobs.append((bound, cols))
    server = provider.Server(max_inflight=16)
    try:
        got = serve_all(server, jobs)
        stats = server.stats()
        assert stats["completed"] == len(jobs)
        assert stats["max_inflight_seen"] <= 2, stats
    finally:
        server.close()
    check_against_alone(jobs, got)
    for cols in keep:
        for c in cols:
            c.release()
