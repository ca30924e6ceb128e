"""Benchmark of the filtered hash group-by on B200.

Workload (the 100M-row configuration): 100,000,000 rows; keys k1 = Int32
Zipf(s=1.1) over 1,000,000 values and k2 = UInt32 codes of a 64-value
dictionary; v Float64 ~ Normal(0, 1e3) with 5% random nulls; filter on a
second Int32 column p uniform in [0, 100) < 50; aggregations sum, mean, min,
max, count, var of v; groups in first-appearance order (maintain_order=True).
Synthetic and seeded (seed 2 + rank).

One step = one whole query (scan + finish, result columns on the device) over
inputs already resident in HBM; `value` = rows all ranks processed per second,
timed with CUDA events on the query's stream, max over ranks.  Inputs are
2.01 GB per rank (> 126 MB L2), so no L2 flush is needed between steps.
`e2e` = the same query through the C ABI with host buffers: every step
registers the inputs from pinned host memory (host->device copies), runs the
query and copies every result column back (device->host), timed by CUDA
events on the library's stream; `e2e.phases_ms` splits one further, untimed
step by the host clock into upload, query, download and release.

`--impl reference` times the CPU restatement of the reference's parallel
aggregate table (oracle/, all host threads) on a bounded sample of the same
workload; rank 0 only.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ROWS = 100_000_000
DISTINCT = 1_000_000
ZIPF_S = 1.1
CODES = 64
BYTES_PER_ROW = 4 + 4 + 8 + 4 + 1 / 8  # k1, k2, v, p, v's validity bit
COUNT_BYTES_PER_ROW = 4 + 4 + 4  # the counting pass reads the keys and the filter column
METRIC = "group-by rows/s"
WORKLOAD = (
    "100M-row filtered group-by: keys (Int32 Zipf s=1.1 over 1M, UInt32 codes of 64), "
    "v Float64 N(0,1e3) 5% nulls, filter p<50 (p Int32 uniform [0,100)), "
    "aggs sum/mean/min/max/count/var, maintain_order=True"
)
FALLBACK_HBM_GBS = 6650.0


def measured_hbm_gbs() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def generate(rows: int, seed: int, device: str):
    """Seeded synthetic columns of the workload, generated on `device`."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    ranks = torch.arange(1, DISTINCT + 1, dtype=torch.float64, device=device)
    cdf = torch.cumsum(ranks.pow(-ZIPF_S), 0)
    cdf /= cdf[-1].clone()
    perm = torch.randperm(DISTINCT, generator=g, device=device).to(torch.int32)
    out = {}
    chunk = 1 << 24
    k1 = torch.empty(rows, dtype=torch.int32, device=device)
    for s in range(0, rows, chunk):
        e = min(rows, s + chunk)
        u = torch.rand(e - s, generator=g, dtype=torch.float64, device=device)
        r = torch.searchsorted(cdf, u, right=True).clamp_(max=DISTINCT - 1)
        k1[s:e] = perm[r]
    out["k1"] = k1
    out["k2"] = torch.randint(0, CODES, (rows,), generator=g, device=device, dtype=torch.int64).to(torch.int32)
    out["v"] = torch.randn(rows, generator=g, dtype=torch.float64, device=device) * 1e3
    out["v_valid"] = torch.rand(rows, generator=g, device=device) >= 0.05
    out["p"] = torch.randint(0, 100, (rows,), generator=g, device=device, dtype=torch.int64).to(torch.int32)
    return out


def pack_bits_torch(valid):
    """LSB-first packed validity bytes of a bool tensor (on its device)."""
    import torch

    n = valid.numel()
    pad = (-n) % 8
    v = torch.cat([valid, torch.zeros(pad, dtype=torch.bool, device=valid.device)]) if pad else valid
    w = (v.view(-1, 8).to(torch.uint8) << torch.arange(8, device=valid.device, dtype=torch.uint8)).sum(1, dtype=torch.uint8)
    return w


def plan_for(frame_like):
    from dataframe_mojo_b200.frame import col

    return (
        frame_like.lazy()
        .filter(col("p") < 50)
        .group_by(["k1", "k2"], maintain_order=True)
        .agg(
            [
                col("v").sum().alias("sum"),
                col("v").mean().alias("mean"),
                col("v").min().alias("min"),
                col("v").max().alias("max"),
                col("v").count().alias("count"),
                col("v").var().alias("var"),
            ]
        )
    )


class Clocks:
    """nvidia-smi clock and throttle samples during the timed region."""

    def __init__(self, index: int):
        self.path = Path(tempfile.gettempdir()) / f"dfc_clocks_{os.getpid()}.csv"
        self.proc = None
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                [
                    "nvidia-smi",
                    f"--id={index}",
                    "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                    "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                    "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                    "--format=csv,noheader,nounits",
                    "-lms",
                    "100",
                ],
                stdout=self.f,
                stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(mx)) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def traffic_per_launch(kernel: str) -> float | None:
    """DRAM bytes of one full-size launch of `kernel` from the committed ncu
    summaries (a smaller capture scaled by rows), if any."""
    p = ROOT / "profiles" / "kernel_traffic.json"
    try:
        return float(json.loads(p.read_text())[kernel]["dram_bytes_per_full_launch"])
    except Exception:
        return None


def roofline_of(step_t: list[dict], rows: int) -> dict:
    """HBM roofline from the library's CUDA-event timings of the timed steps.

    Radix-partitioned regime, per pass (algorithmic bytes per launch):
    counting pass rows x 12 B (keys and filter column); placement (pass A)
    rows x 20.125 B read + kept rows x placed row bytes written; aggregation
    (pass B) kept rows x placed row bytes read (the groups' records, about
    groups x 64 B, left out).  The dominant pass is the roofline's kernel;
    "query" is the single-pass minimum (rows x 20.125 B) over the query's
    whole device time.  Table regimes: one scan kernel, rows x 20.125 B."""
    peak, peak_kind = measured_hbm_gbs()

    def mean_s(k):
        return float(np.mean([t[k] for t in step_t])) * 1e-9

    last = step_t[-1]
    in_bytes = rows * BYTES_PER_ROW
    if last["regime"] == 2:
        kept, rb = last["kept_rows"], last["placed_row_bytes"]
        passes = {
            "partition_count": (rows * COUNT_BYTES_PER_ROW, mean_s("count_ns")),
            "partition_kernel": (in_bytes + kept * rb, mean_s("place_ns")),
            "partition_aggregate": (kept * rb, mean_s("aggregate_ns")),
        }
        extra = {"kept_rows": kept, "placed_row_bytes": rb, "partitions": last["partitions"]}
    else:
        passes = {"scan_kernel": (in_bytes, mean_s("scan_ns"))}
        extra = {}
    dominant = max(passes, key=lambda k: passes[k][1])
    b, s = passes[dominant]
    achieved = b / s / 1e9
    query_s = mean_s("scan_ns") + mean_s("aggregate_ns") + mean_s("finish_ns")
    return {
        "bound": "hbm",
        "kernel": dominant,
        "achieved": achieved,
        "peak": peak,
        "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
        "unit": "GB/s",
        "frac": achieved / peak,
        "traffic": traffic_per_launch(dominant),
        "algorithmic_bytes": b,
        "kernel_ms": s * 1e3,
        "regime": ["global table", "shared-memory tables", "radix-partitioned", "ungrouped in registers"][last["regime"]],
        "passes": {k: {"algorithmic_bytes": pb, "ms": ps * 1e3, "gbs": pb / ps / 1e9, "frac": pb / ps / 1e9 / peak,
                       "traffic": traffic_per_launch(k)} for k, (pb, ps) in passes.items()},
        "finish_ms": mean_s("finish_ns") * 1e3,
        "query": {"single_pass_bytes": in_bytes, "device_ms": query_s * 1e3, "gbs": in_bytes / query_s / 1e9,
                  "frac": in_bytes / query_s / 1e9 / peak},
        **extra,
    }


def cpu_baseline(frame_np, sample_rows: int, threads: int) -> dict:
    """The oracle's parallel restatement of the reference CPU aggregate table
    on the first `sample_rows` rows, all host threads."""
    from dataframe_mojo_b200.frame import DataFrame, Series
    from oracle import binding

    sub = DataFrame(
        [
            Series("k1", frame_np["k1"][:sample_rows]),
            Series("k2", frame_np["k2"][:sample_rows]),
            Series("v", frame_np["v"][:sample_rows], frame_np["v_valid"][:sample_rows]),
            Series("p", frame_np["p"][:sample_rows]),
        ]
    )
    plan = plan_for(sub)
    binding.run(plan, threads=threads)  # warm caches
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        binding.run(plan, threads=threads)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    return {
        "value": sample_rows / t,
        "unit": "rows/s",
        "cores": threads,
        "physical_cores": physical_cores(),
        "kind": "port",
        "sample": f"first {sample_rows:,} rows of the workload, median of 3 runs, {t:.3f} s each",
    }


def physical_cores() -> int | None:
    """Physical cores of the host (the threads used may count SMT siblings)."""
    try:
        import psutil

        return psutil.cpu_count(logical=False)
    except Exception:
        return None


def host_numpy(cols):
    return {
        "k1": cols["k1"].cpu().numpy(),
        "k2": cols["k2"].cpu().numpy().view(np.uint32),
        "v": cols["v"].cpu().numpy(),
        "v_valid": cols["v_valid"].cpu().numpy(),
        "p": cols["p"].cpu().numpy(),
    }


def run_reference(args, rank: int, world: int) -> int:
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    rows = args.sample_rows
    import torch

    cols = generate(rows, 2, "cpu")
    frame_np = {
        "k1": cols["k1"].numpy(),
        "k2": cols["k2"].numpy().view(np.uint32),
        "v": cols["v"].numpy(),
        "v_valid": cols["v_valid"].numpy(),
        "p": cols["p"].numpy(),
    }
    from dataframe_mojo_b200.frame import DataFrame, Series
    from oracle import binding

    sub = DataFrame(
        [Series("k1", frame_np["k1"]), Series("k2", frame_np["k2"]), Series("v", frame_np["v"], frame_np["v_valid"]),
         Series("p", frame_np["p"])]
    )
    plan = plan_for(sub)
    for _ in range(args.warmup):
        binding.run(plan, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        binding.run(plan, threads=threads)
    dt = time.perf_counter() - t0
    value = rows * args.steps / dt
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "rows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded generator, seed 2)",
        "config": {"workload": WORKLOAD, "rows_per_step": rows, "full_rows": ROWS},
        "cpu_baseline": {
            "value": value,
            "unit": "rows/s",
            "cores": threads,
            "physical_cores": physical_cores(),
            "kind": "port",
            "sample": f"{rows:,} rows of the workload per step (the full 100M-row query does not fit a few-minute run)",
        },
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _register(tensor, dtype_code, rows, valid_bytes=None):
    """A device column over a torch tensor (kept alive by the caller)."""
    import ctypes as C

    from dataframe_mojo_b200 import _native as native

    h = C.c_void_p()
    st = native.lib().dfc_column_register(0, dtype_code, rows, tensor.data_ptr(),
                                          valid_bytes.data_ptr() if valid_bytes is not None else None, 0,
                                          native.COLUMN_DEVICE, C.byref(h))
    if st != native.OK:
        raise RuntimeError(native.last_error())
    return type("DeviceHandle", (), {"handle": h})()


def batched_specs(nq: int) -> list[dict]:
    """The batched configuration's query shapes, in order: rows log-uniform
    1K-20M; one Int64 key of cardinality log-uniform 1-2M, uniform or Zipf
    s=1.2; a filter on the Int64 value against a random threshold."""
    rng = np.random.default_rng(4)
    specs = []
    for _ in range(nq):
        rows = int(math.exp(rng.uniform(math.log(1e3), math.log(2e7))))
        card = max(1, int(math.exp(rng.uniform(0.0, math.log(2e6)))))
        zipf = bool(rng.integers(0, 2))
        thr = int(rng.integers(-1000, 1000))
        specs.append({"rows": rows, "card": card, "zipf": zipf, "thr": thr})
    return specs


def batched_columns(q: int, spec: dict, device: str) -> dict:
    """Query q's columns (seed 4 + q): key k, Int64 value a and Float32 value
    b with 2% nulls each (validity as packed LSB-first bytes)."""
    import torch

    rows, card = spec["rows"], spec["card"]
    g = torch.Generator(device=device)
    g.manual_seed(4 + q)
    if spec["zipf"]:
        w = torch.arange(1, card + 1, device=device, dtype=torch.float64).pow(-1.2)
        cdf = torch.cumsum(w, 0)
        cdf /= cdf[-1].clone()
        u = torch.rand(rows, generator=g, device=device, dtype=torch.float64)
        k = torch.searchsorted(cdf, u).clamp_(max=card - 1)
    else:
        k = torch.randint(0, card, (rows,), generator=g, device=device)
    a = torch.randint(-1000, 1001, (rows,), generator=g, device=device)
    b = torch.randn(rows, generator=g, device=device, dtype=torch.float32)
    va = torch.rand(rows, generator=g, device=device) >= 0.02
    vb = torch.rand(rows, generator=g, device=device) >= 0.02
    return {"k": k, "a": a, "b": b, "va": va, "vb": vb}


def batched_plan(frame_like, thr: int):
    from dataframe_mojo_b200.frame import col

    return frame_like.lazy().filter(col("a") > thr).group_by("k", maintain_order=True).agg(
        [col("a").sum().alias("sa"), col("b").mean().alias("mb"), col("a").min().alias("lo"),
         col("b").max().alias("hi"), col("b").count().alias("n")])


def batched_jobs(device: str, nq: int):
    """The batched configuration's queries (batched_specs, batched_columns):
    the jobs (bound plan, registered columns), what keeps their buffers
    alive, the total rows and per query (rows, cardinality, zipf)."""
    import torch
    from dataframe_mojo_b200 import _native as native
    from dataframe_mojo_b200.frame import bind
    from dataframe_mojo_b200.frame import DataFrame, Series

    shape = DataFrame([Series("k", np.zeros(1, np.int64)), Series("a", np.zeros(1, np.int64)),
                       Series("b", np.zeros(1, np.float32))])
    jobs, keep, total, info = [], [], 0, []
    for q, spec in enumerate(batched_specs(nq)):
        c = batched_columns(q, spec, device)
        rows = spec["rows"]
        va, vb = pack_bits_torch(c["va"]), pack_bits_torch(c["vb"])
        bound = bind(batched_plan(shape, spec["thr"]).plan)
        hs = {"k": _register(c["k"], native.INT64, rows), "a": _register(c["a"], native.INT64, rows, va),
              "b": _register(c["b"], native.FLOAT32, rows, vb)}
        keep.append((c, va, vb, hs))
        jobs.append((bound, [hs[n] for n in bound.names]))
        info.append((rows, spec["card"], spec["zipf"]))
        total += rows
    torch.cuda.synchronize()
    return jobs, keep, total, info


def batched_form(device: str, nq: int) -> dict:
    """The batched configuration (batched_jobs): times the plain path (one
    dfc_groupby per query) and the batched one (dfc_groupby_batch), both
    after a warm-up pass of each."""
    import torch
    from dataframe_mojo_b200 import _native as native
    from dataframe_mojo_b200 import provider

    jobs, keep, total, info = batched_jobs(device, nq)
    # Where the plain path's time goes, by query size: the library's device
    # time (scan, aggregation and finish events) and the host's per query.
    account = {k: {"queries": 0, "rows": 0, "device_ms": 0.0, "wall_ms": 0.0}
               for k in ("over_1M_rows", "1M_rows_or_fewer")}

    def plain():
        for (bd, cl), (rows, _, _) in zip(jobs, info):
            t0 = time.perf_counter()
            r = provider.run_bound(bd, cl)
            t = provider.last_timings()
            r.free()
            a = account["over_1M_rows" if rows > 1_000_000 else "1M_rows_or_fewer"]
            a["queries"] += 1
            a["rows"] += rows
            a["device_ms"] += (t["scan_ns"] + t["aggregate_ns"] + t["finish_ns"]) * 1e-6
            a["wall_ms"] += (time.perf_counter() - t0) * 1e3

    def batched():
        for r in provider.run_batch(jobs):
            if isinstance(r, Exception):
                raise r
            r.free()

    times = {}
    for name, fn in (("plain", plain), ("batched", batched), ("plain", plain), ("batched", batched)):
        if name == "plain":
            for a in account.values():
                a.update(queries=0, rows=0, device_ms=0.0, wall_ms=0.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        times[name] = time.perf_counter() - t0  # the second (warm) pass counts
    for *_, hs in keep:
        for h in hs.values():
            native.lib().dfc_column_release(h.handle)
    return {
        "config": "batched: %d queries, rows log-uniform 1K-20M (%d rows), Int64 key cardinality log-uniform 1-2M "
                  "(uniform or Zipf 1.2), Int64 + Float32 values 2%% nulls, filter on the Int64 value" % (nq, total),
        "queries": nq,
        "rows": total,
        "plain_ms": times["plain"] * 1e3,
        "batched_ms": times["batched"] * 1e3,
        "plain_rows_per_s": total / times["plain"],
        "batched_rows_per_s": total / times["batched"],
        "speedup": times["plain"] / times["batched"],
        "plain_account": account,
    }


def served_sizes() -> list[int]:
    """Rows of the served configuration's 8 resident tables (seeds 5 + table id)."""
    return [int(x) for x in np.geomspace(1e7, 2e8, 8)]


SERVED_AGGS = ("sum", "mean", "min", "max", "count", "var")


def served_requests(nreq: int, rate: float = 2000.0):
    """The served configuration's requests, in order: table, key subset
    ({k1}, {k2} or {k1, k2}), aggregation list and threshold (p < t); and
    their Poisson arrival times at `rate` per second."""
    rng = np.random.default_rng(5)
    specs = []
    for _ in range(nreq):
        t = int(rng.integers(0, len(served_sizes())))
        keys = [["k1"], ["k2"], ["k1", "k2"]][int(rng.integers(0, 3))]
        pick = [a for a in SERVED_AGGS if rng.random() < 0.5] or [SERVED_AGGS[0]]
        specs.append({"table": t, "keys": keys, "aggs": pick, "thr": int(rng.integers(1, 100))})
    return specs, np.cumsum(rng.exponential(1.0 / rate, nreq))


def served_plan(frame_like, spec: dict):
    from dataframe_mojo_b200.frame import col

    return frame_like.lazy().filter(col("p") < spec["thr"]).group_by(spec["keys"], maintain_order=True).agg(
        [getattr(col("v"), n)().alias(n) for n in spec["aggs"]])


def served_form(device: str, nreq: int, rate: float = 2000.0, inflight: int = 32) -> dict:
    """The served configuration: 8 resident tables of 10M-200M rows (the
    100M-row workload's schema, seeds 5 + table id), nreq requests arriving
    as a Poisson process at `rate` per second, each a group-by with a random
    threshold (p < t), key subset ({k1}, {k2} or {k1, k2}) and aggregation
    list.  The plain path serves them first-in first-out with one
    dfc_groupby at a time; the served path submits them to the native server
    (continuous batching).  Latency = completion - arrival."""
    import torch
    from dataframe_mojo_b200 import _native as native
    from dataframe_mojo_b200 import provider
    from dataframe_mojo_b200.frame import bind
    from dataframe_mojo_b200.frame import DataFrame, Series, col

    sizes = served_sizes()
    tables = []
    for t, n in enumerate(sizes):
        c = generate(n, 5 + t, device)
        vb = pack_bits_torch(c["v_valid"])
        hs = {"k1": _register(c["k1"], native.INT32, n), "k2": _register(c["k2"], native.UINT32, n),
              "v": _register(c["v"], native.FLOAT64, n, vb), "p": _register(c["p"], native.INT32, n)}
        tables.append((c, vb, hs))
    torch.cuda.synchronize()
    shape = DataFrame([Series("k1", np.zeros(1, np.int32)), Series("k2", np.zeros(1, np.uint32)),
                       Series("v", np.zeros(1)), Series("p", np.zeros(1, np.int32))])
    specs, arrivals = served_requests(nreq, rate)
    reqs = []
    for t, plan in ((sp["table"], served_plan(shape, sp)) for sp in specs):
        bound = bind(plan.plan)
        reqs.append((bound, [tables[t][2][n] for n in bound.names]))

    # Warm-up: every table once (statistics, learned group counts).
    for bound, cl in reqs[: min(nreq, 16)]:
        try:
            provider.run_bound(bound, cl).free()
        except provider.DataFaultError:
            pass

    def plain(arrivals, n):
        lat = []
        t0 = time.perf_counter()
        for (bound, cl), at in zip(reqs[:n], arrivals[:n]):
            while time.perf_counter() - t0 < at:
                pass
            try:
                provider.run_bound(bound, cl).free()
            except provider.DataFaultError:
                pass  # answered: the core adjudicates such a query on the CPU
            lat.append(time.perf_counter() - t0 - at)
        return np.array(lat), time.perf_counter() - t0

    def served(arrivals, n):
        server = provider.Server(max_inflight=inflight)
        lat = {}
        t0 = time.perf_counter()
        i = 0
        while len(lat) < n:
            now = time.perf_counter() - t0
            while i < n and arrivals[i] <= now:
                server.submit(reqs[i][0], reqs[i][1], i)
                i += 1
            # Wait briefly for completions once every request is submitted.
            for tag, res, _, _ in server.poll(wait_ms=0 if i < n else 2):
                if isinstance(res, provider.DataFaultError):
                    pass  # answered: the core adjudicates such a query on the CPU
                elif isinstance(res, Exception):
                    raise res
                else:
                    res.free()
                lat[tag] = time.perf_counter() - t0 - arrivals[tag]
        span = time.perf_counter() - t0
        server.close()
        return np.array([lat[j] for j in range(n)]), span

    def pct(lat):
        return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}

    lp, sp_ = plain(arrivals, nreq)
    ls, ss = served(arrivals, nreq)
    # Latency under load: the first requests again, their Poisson arrivals
    # rescaled to 50%, 80% and 100% of the served path's saturated rate.
    capacity = nreq / ss
    n_load = min(nreq, 150)
    loads = {}
    for frac in (0.5, 0.8, 1.0):
        arr = np.asarray(arrivals[:n_load]) * (rate / (frac * capacity))
        lpl, _ = plain(arr, n_load)
        lsl, _ = served(arr, n_load)
        loads[f"{int(frac * 100)}%"] = {"arrivals_per_s": frac * capacity, "requests": n_load,
                                        "plain": pct(lpl), "served": pct(lsl)}
    for c, vb, hs in tables:
        for h in hs.values():
            native.lib().dfc_column_release(h.handle)
    return {
        "config": "served: 8 resident tables of 10M-200M rows (%d rows), %d requests, Poisson arrivals at %.0f/s, "
                  "random threshold, key subset and aggregation list" % (sum(sizes), nreq, rate),
        "requests": nreq,
        "plain": {"p50_ms": float(np.percentile(lp, 50) * 1e3), "p99_ms": float(np.percentile(lp, 99) * 1e3),
                  "queries_per_s": nreq / sp_},
        "served": {"p50_ms": float(np.percentile(ls, 50) * 1e3), "p99_ms": float(np.percentile(ls, 99) * 1e3),
                   "queries_per_s": nreq / ss},
        "throughput_ratio": (nreq / ss) / (nreq / sp_),
        "latency_under_load": loads,
    }


# The reference's published filtered sums (benchmarks/bench_handoff.mojo,
# docs/apple-metal.md:453-457): 50M rows on an M1 Mac mini, best of 5 warm
# collects, (CPU executor on 8 threads, Metal hand-off reading the column in
# place) in ms.
HANDOFF_PUBLISHED_MS = {"int32": (23.2, 9.4), "float32": (14.0, 9.7), "int64": (17.1, 16.5)}


def handoff_values(dtype: str, rows: int, device: str):
    """bench_handoff's column: x = (row * 7919) % spread - spread // 2, spread
    7 for Int32 (so the filtered sum of any size fits Int32) and 2001 else."""
    import torch

    spread = 7 if dtype == "int32" else 2001
    r = torch.arange(rows, dtype=torch.int64, device=device)
    x = (r * 7919) % spread - spread // 2
    return x.to({"int32": torch.int32, "float32": torch.float32, "int64": torch.int64}[dtype])


def handoff_plan(frame_like):
    from dataframe_mojo_b200.frame import col

    return frame_like.lazy().filter(col("x") > 0).select(col("x").sum())


def handoff_form(device: str, rows: int = 50_000_000, reps: int = 20) -> dict:
    """The reference's published workload: filter(x > 0).select(x.sum()) over
    one 50M-row column of each type.  `ms`: one query over the column
    resident in HBM (the discrete-GPU form of reading it in place), CUDA
    events around `reps` queries after 3 warm-ups; `e2e_ms`: the same from a
    pinned host buffer (registration copy, query, result copy).  Best of the
    reps, as the reference reports; the mean beside it."""
    import torch

    from dataframe_mojo_b200 import _native as native
    from dataframe_mojo_b200 import provider
    from dataframe_mojo_b200.frame import DataFrame, Series, bind

    out = {}
    codes = {"int32": (native.INT32, np.int32), "float32": (native.FLOAT32, np.float32),
             "int64": (native.INT64, np.int64)}
    stream = torch.cuda.Stream()
    for name, (code, npdt) in codes.items():
        x = handoff_values(name, rows, device)
        torch.cuda.synchronize()
        h = _register(x, code, rows)
        bound = bind(handoff_plan(DataFrame([Series("x", np.zeros(1, npdt))])).plan)
        cols = [h]
        for _ in range(3):
            provider.run_bound(bound, cols, stream=stream.cuda_stream).free()
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = provider.run_bound(bound, cols, stream=stream.cuda_stream)
            e1.record(stream)
            r.free()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        host = x.cpu().pin_memory()
        e2e = []
        for i in range(reps // 2 + 1):
            t0 = time.perf_counter()
            dc = provider.DeviceColumn.from_host_pointer("x", npdt, rows, host.data_ptr(), None, 0, 0)
            r = provider.run_bound(bound, [dc])
            total = r.to_frame().column(r.names[0]).values[0]
            r.free()
            dc.release()
            if i:
                e2e.append((time.perf_counter() - t0) * 1e3)
        native.lib().dfc_column_release(h.handle)
        cpu_ms, metal_ms = HANDOFF_PUBLISHED_MS[name]
        best = float(min(times))
        out[name] = {"ms": best, "mean_ms": float(np.mean(times)), "e2e_ms": float(min(e2e)),
                     "gbs": rows * np.dtype(npdt).itemsize / best / 1e6, "sum": float(total),
                     "published_m1_cpu_ms": cpu_ms, "published_m1_metal_ms": metal_ms,
                     "vs_published_metal": metal_ms / best, "vs_published_cpu": cpu_ms / best}
        del x, host
        torch.cuda.empty_cache()
    return {"config": f"filter(x > 0).select(x.sum()), {rows:,} rows per column (benchmarks/bench_handoff.mojo)",
            "by_dtype": out}


def precision_form(device: str, rows: int, reps: int = 5) -> dict:
    """The precision configuration: `rows` rows, Int32 keys uniform over 10K
    groups, Float32 values with log-uniform magnitudes in [1e-6, 1e6] and
    random signs (seed 3); group_by(k).agg(sum, mean, var) accumulated in
    FP64 (the default) and as compensated FP32 partials merged in FP64.  Per
    arm: device-resident time per query (best of `reps`, each a full
    dfc_groupby with its readback) and the per-group maximum errors against
    an extended-precision (long double) oracle on the host: sums relative to
    sum |x|, variances relative to the variance.  A Float32 column's sum is a
    Float32 result, so the accumulated sum is read through the Float64 mean
    (mean x count)."""
    import torch
    from dataframe_mojo_b200 import _native as native
    from dataframe_mojo_b200 import provider
    from dataframe_mojo_b200.frame import bind
    from dataframe_mojo_b200.frame import DataFrame, Series, col

    g = torch.Generator(device=device)
    g.manual_seed(3)
    keys = torch.randint(0, 10_000, (rows,), generator=g, device=device, dtype=torch.int32)
    mags = torch.pow(10.0, torch.rand(rows, generator=g, device=device, dtype=torch.float64) * 12.0 - 6.0)
    sign = torch.where(torch.rand(rows, generator=g, device=device) < 0.5, -1.0, 1.0).to(torch.float64)
    vals = (sign * mags).to(torch.float32)
    del mags, sign
    torch.cuda.synchronize()
    hs = {"k": _register(keys, native.INT32, rows), "v": _register(vals, native.FLOAT32, rows)}
    shape = DataFrame([Series("k", np.zeros(1, np.int32)), Series("v", np.zeros(1, np.float32))])
    plan = shape.lazy().group_by("k").agg([col("v").sum().alias("s"), col("v").mean().alias("m"),
                                           col("v").var().alias("var")])
    bound = bind(plan.plan)
    cl = [hs[n] for n in bound.names]

    # Extended-precision oracle on the host.
    k_h = keys.cpu().numpy()
    v_h = vals.cpu().numpy()
    order = np.argsort(k_h, kind="stable")
    ks = k_h[order]
    starts = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]])
    counts = np.diff(np.r_[starts, rows])
    x = v_h[order].astype(np.longdouble)
    del order
    gsum = np.add.reduceat(x, starts)
    gabs = np.add.reduceat(np.abs(x), starts)
    d = x - np.repeat(gsum / counts, counts)
    gvar = np.add.reduceat(d * d, starts) / (counts - 1)
    del x, d
    gkeys = ks[starts]

    arms = {}
    for name, flags in (("fp64", 0), ("compensated_fp32", native.Q_FLOAT32_COMPENSATED)):
        provider.run_bound(bound, cl, flags=flags).free()  # warm-up (learned group count)
        best, t, r = float("inf"), None, None
        for rep in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = provider.run_bound(bound, cl, flags=flags)
            dt = time.perf_counter() - t0
            if dt < best:
                best, t = dt, provider.last_timings()
            if rep < reps - 1:
                r.free()
        out = r.to_frame()
        r.free()
        o = np.argsort(out["k"].values)
        if not np.array_equal(out["k"].values[o], gkeys):
            raise RuntimeError("precision form: group keys differ from the oracle")
        s = out["m"].values[o].astype(np.longdouble) * counts
        v = out["var"].values[o].astype(np.longdouble)
        arms[name] = {
            "ms": best * 1e3,
            "rows_per_s": rows / best,
            "scan_ms": t["scan_ns"] / 1e6,
            "algorithmic_gbs": rows * 8 / (t["scan_ns"] / 1e9) / 1e9,
            "cluster_ctas": t["cluster_ctas"],
            "compensated_fields": t["compensated"],
            "max_sum_err_over_sum_abs": float(np.max(np.abs(s - gsum) / gabs)),
            "max_sum_rel_err": float(np.max(np.abs(s - gsum) / np.maximum(np.abs(gsum), np.finfo(np.float64).tiny))),
            "max_var_rel_err": float(np.max(np.abs(v - gvar) / gvar)),
        }
    for h in hs.values():
        native.lib().dfc_column_release(h.handle)
    return {
        "config": "precision: %d rows, Int32 keys uniform over 10K groups, Float32 log-uniform |x| in [1e-6, 1e6] "
                  "with random signs; sum/mean/var; errors against a long-double oracle; 8 algorithmic bytes/row" % rows,
        "rows": rows,
        "groups": int(len(gkeys)),
        **arms,
    }


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dfcuda")
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--sample-rows", type=int, default=10_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-queries", type=int, default=512, help="batched form: queries (0: skip)")
    ap.add_argument("--served-requests", type=int, default=400, help="served form: requests (0: skip)")
    ap.add_argument("--served-inflight", type=int, default=32, help="served form: requests in flight at most")
    ap.add_argument("--precision-rows", type=int, default=100_000_000, help="precision form: rows (0: skip)")
    ap.add_argument("--handoff-rows", type=int, default=50_000_000,
                    help="the reference's published filtered sums: rows per column (0: skip)")
    ap.add_argument("--only", choices=["precision", "batched", "served", "handoff"],
                    help="run one configuration form alone and print its JSON object (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("at least 3 warm-up steps")
    if args.only:
        import torch

        torch.cuda.set_device(0)
        if args.only == "precision":
            out = precision_form("cuda:0", args.precision_rows)
        elif args.only == "batched":
            out = batched_form("cuda:0", args.batch_queries)
        elif args.only == "handoff":
            out = handoff_form("cuda:0", args.handoff_rows)
        else:
            out = served_form("cuda:0", args.served_requests, inflight=args.served_inflight)
        print(json.dumps(out), flush=True)
        return 0

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device(f"cuda:{local}"))

    from dataframe_mojo_b200 import provider
    from dataframe_mojo_b200.frame import Bound, bind

    device = local
    rows = args.rows
    cols = generate(rows, 2 + rank, f"cuda:{local}")
    vbits = pack_bits_torch(cols["v_valid"])
    torch.cuda.synchronize()

    # Device-resident inputs (registered as borrowed device columns; the
    # validity bitmap is normalised into the library's own buffer).
    lib = provider.N.lib()
    import ctypes as C

    handles = {}
    for name in ("k1", "k2", "v", "p"):
        h = C.c_void_p()
        t = cols[name]
        dt = {"k1": provider.N.INT32, "k2": provider.N.UINT32, "v": provider.N.FLOAT64, "p": provider.N.INT32}[name]
        validity = vbits.data_ptr() if name == "v" else None
        st = lib.dfc_column_register(device, dt, rows, t.data_ptr(), validity, 0, provider.N.COLUMN_DEVICE, C.byref(h))
        provider._check(st)
        handles[name] = h

    class _Shape:
        """Plan builder over the workload's schema (values never read)."""

        def lazy(self):
            from dataframe_mojo_b200.frame import DataFrame, LazyFrame, Series

            df = DataFrame(
                [
                    Series("k1", np.zeros(1, np.int32)),
                    Series("k2", np.zeros(1, np.uint32)),
                    Series("v", np.zeros(1, np.float64)),
                    Series("p", np.zeros(1, np.int32)),
                ]
            )
            return df.lazy()

    bound = bind(plan_for(_Shape()).plan)
    stream = torch.cuda.Stream()
    col_list = [type("H", (), {"handle": handles[n]})() for n in bound.names]

    def step():
        res = provider.run_bound(bound, col_list, stream=stream.cuda_stream)
        return res

    for _ in range(args.warmup):
        r = step()
        groups = r.rows
        r.free()
    torch.cuda.synchronize()

    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    step_t = []
    launches = 0
    start.record(stream)
    for _ in range(args.steps):
        # Each step's result is complete on the device when run_bound
        # returns; releasing it, as a caller does once it has read it, keeps
        # the memory pool at a steady size.
        r = step()
        t = provider.last_timings()
        step_t.append(t)
        launches += t["launches"]
        r.free()
    end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = start.elapsed_time(end) / args.steps
    ms_t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = rows * world / (ms_max * 1e-3)

    roofline = roofline_of(step_t, rows)

    # End to end through the C ABI with host buffers (pinned).
    host = {n: cols[n].cpu().pin_memory() for n in ("k1", "k2", "v", "p")}
    host_bits = vbits.cpu().pin_memory()
    torch.cuda.synchronize()
    e2e_stream = torch.cuda.Stream()
    provider.set_thread_stream(device, e2e_stream.cuda_stream)
    dtypes = {"k1": np.int32, "k2": np.uint32, "v": np.float64, "p": np.int32}
    h2d = sum(host[n].numel() * host[n].element_size() for n in host) + host_bits.numel()

    # Result buffers in pinned host memory too, sized from the device-resident
    # run's group count with a margin.
    out_cap = int(groups * 1.25) + 4096
    out_types = {"k1": np.int32, "k2": np.uint32, "sum": np.float64, "mean": np.float64, "min": np.float64,
                 "max": np.float64, "count": np.int64, "var": np.float64}
    pinned_out = {
        n: (torch.empty(out_cap * np.dtype(t).itemsize, dtype=torch.uint8, pin_memory=True).numpy().view(t),
            torch.empty((out_cap + 7) // 8, dtype=torch.uint8, pin_memory=True).numpy())
        for n, t in out_types.items()
    }

    def e2e_step(marks=None):
        # `marks`: host clock readings after each phase (upload, query,
        # download, release), each after a device synchronisation.
        def mark():
            if marks is not None:
                torch.cuda.synchronize()
                marks.append(time.perf_counter())

        mark()
        dcols = {}
        for n in ("k1", "k2", "v", "p"):
            dcols[n] = provider.DeviceColumn.from_host_pointer(
                n, dtypes[n], rows, host[n].data_ptr(), host_bits.data_ptr() if n == "v" else None, 0, device
            )
        mark()
        res = provider.run_bound(bound, [dcols[n] for n in bound.names])
        mark()
        frame = res.to_frame(into=pinned_out)
        out_bytes = sum(frame.column(c).values.nbytes + (len(frame.column(c)) + 7) // 8 for c in frame.columns)
        mark()
        res.free()
        for c in dcols.values():
            c.release()
        mark()
        return out_bytes

    for _ in range(1):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(e2e_stream)
    d2h = 0
    step_host_ms, step_retries = [], []
    for _ in range(args.e2e_steps):
        # Each step ends synchronised (its result copied to the host), so the
        # host clock around it reads the step; the retries are the library's.
        t0 = time.perf_counter()
        d2h = e2e_step()
        step_host_ms.append(round((time.perf_counter() - t0) * 1e3, 3))
        step_retries.append(provider.last_timings()["retries"])
    e1.record(e2e_stream)
    torch.cuda.synchronize()
    # Two more steps, after the timed ones and not part of them, read by the
    # host clock phase by phase (the faster of the two): what an end-to-end
    # step is made of.
    phases = None
    for _ in range(2):
        marks = []
        e2e_step(marks)
        ph = {k: (b - a) * 1e3 for k, a, b in zip(("upload", "query", "download", "release"), marks, marks[1:])}
        if phases is None or sum(ph.values()) < sum(phases.values()):
            phases = ph
    provider.set_thread_stream(device, None)
    e2e_ms = e0.elapsed_time(e1) / args.e2e_steps
    et = torch.tensor([e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e = {
        "value": rows * world / (float(et.item()) * 1e-3),
        "unit": "rows/s",
        "h2d_bytes_per_step": int(h2d),
        "d2h_bytes_per_step": int(d2h),
        "steps": args.e2e_steps,
        "ms_per_step": float(et.item()),
        "phases_ms": {k: round(v, 3) for k, v in phases.items()},
        "step_host_ms": step_host_ms,
        "step_retries": step_retries,
    }

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sample = min(args.sample_rows, rows)
        frame_np = {
            "k1": cols["k1"][:sample].cpu().numpy(),
            "k2": cols["k2"][:sample].cpu().numpy().view(np.uint32),
            "v": cols["v"][:sample].cpu().numpy(),
            "v_valid": cols["v_valid"][:sample].cpu().numpy(),
            "p": cols["p"][:sample].cpu().numpy(),
        }
        cpu = cpu_baseline(frame_np, sample, os.cpu_count() or 1)

    for h in handles.values():
        lib.dfc_column_release(h)
    del cols
    torch.cuda.empty_cache()
    batched = served = precision = handoff = None
    if world == 1 and args.precision_rows > 0:
        precision = precision_form(f"cuda:{local}", args.precision_rows)
        torch.cuda.empty_cache()
    if world == 1 and args.batch_queries > 0:
        batched = batched_form(f"cuda:{local}", args.batch_queries)
        torch.cuda.empty_cache()
    if world == 1 and args.served_requests > 0:
        served = served_form(f"cuda:{local}", args.served_requests, inflight=args.served_inflight)
        torch.cuda.empty_cache()
    if world == 1 and args.handoff_rows > 0:
        handoff = handoff_form(f"cuda:{local}", args.handoff_rows)
        torch.cuda.empty_cache()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "rows/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded torch generator, seed 2 + rank)",
            "config": {
                "workload": WORKLOAD,
                "rows_per_gpu": rows,
                "groups": int(groups),
                "parallelism": f"replicas x{world} (independent row partitions, no collective)",
                "l2": "inputs 2.01 GB per GPU > 126 MB L2 (no flush needed)",
            },
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        if precision is not None:
            line["precision"] = precision
        if batched is not None:
            line["batched"] = batched
        if served is not None:
            line["served"] = served
        if handoff is not None:
            line["handoff"] = handoff
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
