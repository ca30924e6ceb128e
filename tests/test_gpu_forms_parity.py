"""The batched and served workloads bench.py times, checked against the CPU
oracle query by query.

Batched (512 queries): the largest query (about 20M rows), the Zipf query
with the largest key cardinality and four more picked by a seeded draw,
rebuilt with bench.py's own generator (batched_specs, batched_columns),
submitted together through dfc_groupby_batch.  Served (400 requests over 8
resident tables): the first requests that address the two smallest tables
(10M and 15M rows), rebuilt with bench.py's served_requests and submitted to
the native request server.  Every result is compared with the oracle on host
copies of the same data: keys, order, counts, min/max and validity bit for
bit, sums and means within 1e-12 of the summands' magnitude, variances within
1e-10 (1 + |var|) (the bars of test_gpu_parity)."""
import numpy as np
import pytest

from dataframe_mojo_b200 import _native as N
from dataframe_mojo_b200 import provider
from dataframe_mojo_b200.frame import DataFrame, Series, bind, col
from oracle import binding
from test_gpu_headline import compare_frames

pytestmark = pytest.mark.gpu


def unpack(mask_tensor) -> np.ndarray:
    return mask_tensor.cpu().numpy().astype(bool)


def scales_of(frame: DataFrame, keys, pred, value: str, ref_names) -> dict:
    """Per-group sum |x| bound (count * max |x|) and max |x|, from the oracle."""
    lf = frame.lazy().filter(pred).group_by(keys, maintain_order=True).agg(
        [col(value).min().alias("_lo"), col(value).max().alias("_hi"), col(value).count().alias("_n")])
    ref, _ = binding.run(lf, threads=0)
    m = np.maximum(np.abs(ref["_lo"].values.astype(np.float64)), np.abs(ref["_hi"].values.astype(np.float64)))
    m = np.where(np.isfinite(m), m, 0.0)
    out = {}
    for name in ref_names:
        out[name] = ref["_n"].values.astype(np.float64) * m if name.startswith("s") or name == "sum" else m
    return out


def test_batched_sample_against_oracle():
    import bench
    import torch

    specs = bench.batched_specs(512)
    rows = np.array([s["rows"] for s in specs])
    zipf_cards = [(s["card"], q) for q, s in enumerate(specs) if s["zipf"]]
    picks = [int(rows.argmax()), max(zipf_cards)[1]]
    rng = np.random.default_rng(44)
    picks += [int(q) for q in rng.choice(len(specs), 4, replace=False) if q not in picks]
    shape = DataFrame([Series("k", np.zeros(1, np.int64)), Series("a", np.zeros(1, np.int64)),
                       Series("b", np.zeros(1, np.float32))])
    jobs, frames, keep = [], [], []
    for q in picks:
        spec = specs[q]
        c = bench.batched_columns(q, spec, "cuda")
        va, vb = bench.pack_bits_torch(c["va"]), bench.pack_bits_torch(c["vb"])
        n = spec["rows"]
        hs = {"k": bench._register(c["k"], N.INT64, n), "a": bench._register(c["a"], N.INT64, n, va),
              "b": bench._register(c["b"], N.FLOAT32, n, vb)}
        bound = bind(bench.batched_plan(shape, spec["thr"]).plan)
        jobs.append((bound, [hs[x] for x in bound.names]))
        keep.append((c, va, vb, hs))
        frames.append(DataFrame([Series("k", c["k"].cpu().numpy()),
                                 Series("a", c["a"].cpu().numpy(), unpack(c["va"])),
                                 Series("b", c["b"].cpu().numpy(), unpack(c["vb"]))]))
    torch.cuda.synchronize()
    try:
        results = provider.run_batch(jobs)
        for q, frame, res in zip(picks, frames, results):
            if isinstance(res, Exception):
                raise res
            dev = res.to_frame()
            res.free()
            plan = bench.batched_plan(frame, specs[q]["thr"])
            ref, _ = binding.run(plan, threads=0)
            sc = scales_of(frame, ["k"], col("a") > specs[q]["thr"], "b", ["mb"])
            compare_frames(dev, ref, f"batched query {q} ({specs[q]})", float_cols=("mb",), scales=sc)
    finally:
        for *_, hs in keep:
            for h in hs.values():
                N.lib().dfc_column_release(h.handle)


def test_served_requests_against_oracle():
    import bench
    import torch

    specs, _ = bench.served_requests(400)
    chosen = [(i, s) for i, s in enumerate(specs) if s["table"] in (0, 1)][:6]
    assert len(chosen) >= 4
    sizes = bench.served_sizes()
    tables = {}
    for t in sorted({s["table"] for _, s in chosen}):
        c = bench.generate(sizes[t], 5 + t, "cuda")
        vb = bench.pack_bits_torch(c["v_valid"])
        n = sizes[t]
        hs = {"k1": bench._register(c["k1"], N.INT32, n), "k2": bench._register(c["k2"], N.UINT32, n),
              "v": bench._register(c["v"], N.FLOAT64, n, vb), "p": bench._register(c["p"], N.INT32, n)}
        h = bench.host_numpy(c)
        frame = DataFrame([Series("k1", h["k1"]), Series("k2", h["k2"]), Series("v", h["v"], h["v_valid"]),
                           Series("p", h["p"])])
        tables[t] = (c, vb, hs, frame)
    torch.cuda.synchronize()
    shape = DataFrame([Series("k1", np.zeros(1, np.int32)), Series("k2", np.zeros(1, np.uint32)),
                       Series("v", np.zeros(1)), Series("p", np.zeros(1, np.int32))])
    server = provider.Server(max_inflight=8)
    try:
        for i, s in chosen:
            bound = bind(bench.served_plan(shape, s).plan)
            server.submit(bound, [tables[s["table"]][2][x] for x in bound.names], i)
        done = {}
        while len(done) < len(chosen):
            for tag, res, _, _ in server.poll(wait_ms=50):
                if isinstance(res, Exception):
                    raise res
                done[tag] = res.to_frame()
                res.free()
        for i, s in chosen:
            frame = tables[s["table"]][3]
            ref, _ = binding.run(bench.served_plan(frame, s), threads=0)
            floats = tuple(a for a in ("sum", "mean") if a in s["aggs"])
            vars_ = ("var",) if "var" in s["aggs"] else ()
            sc = scales_of(frame, s["keys"], col("p") < s["thr"], "v", floats) if floats else None
            compare_frames(done[i], ref, f"served request {i} ({s})", float_cols=floats, var_cols=vars_, scales=sc)
    finally:
        server.close()
        for c, vb, hs, _ in tables.values():
            for h in hs.values():
                N.lib().dfc_column_release(h.handle)
