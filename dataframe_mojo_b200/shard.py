"""Sharded group-by: the rows split across ranks (one process per GPU), each
rank aggregating its own rows on its own GPU, one exchange of the partial
groups, and a merge that restores the result of one query over all rows.

Order: every rank's result is in first-appearance order of its own rows, and
rank r's rows all come after rank r-1's.  Concatenating the partial results
in rank order therefore puts each group's first occurrence at its global
first appearance, so the merged groups are ordered by the position of their
first occurrence in that concatenation (maintain_order=True; without it the
order is not part of the result).

Partial states: each rank runs the query with aggregations a merge can
combine -- counts, rows, null counts, integer sums (sum types are exact),
means (a Float column's sum is rebuilt as mean x count in FP64, since a
Float32 sum is a Float32 result), population variances (M2 = var0 x n, merged
by Chan et al.'s pairwise update), minima and maxima -- and the merge
finishes the requested aggregations from them, with the same null, NaN,
signed-zero and overflow rules as the single-GPU path.

The exchange is one all-gather of the partial results
(`torch.distributed.all_gather_object`), which works on the NCCL and gloo
backends alike; the merge runs on the host.  Partial results hold one row
per group and rank, far fewer bytes than the rows the ranks aggregated.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from .frame import AggExpr, DataFrame, LazyFrame, Plan, Series


@dataclass
class _Partial:
    """The partial aggregations of one value column."""

    column: str
    count: str
    mean: str | None = None
    isum: str | None = None
    var0: str | None = None
    lo: str | None = None
    hi: str | None = None
    nulls: str | None = None


def partial_plan(plan: Plan, part: DataFrame) -> tuple[Plan, dict, str]:
    """The plan a rank runs over its rows `part` (same filters and keys,
    maintain_order=True), the partial aggregations per value column and the
    name of the rows-per-group column."""
    if plan.keys is None or plan.aggs is None:
        raise ValueError("a sharded query is a group-by")
    src = plan.source
    parts: dict[str, _Partial] = {}
    aggs: list[AggExpr] = []

    def add(op, column, name, ddof=1):
        aggs.append(AggExpr(op, column, name, ddof=ddof, min_count=0))
        return name

    rows_name = add(N.AGG_LEN, plan.aggs[0].column if plan.aggs else plan.keys[0], "__rows")
    for a in plan.aggs:
        c = a.column
        p = parts.get(c)
        if p is None:
            p = parts[c] = _Partial(c, add(N.AGG_COUNT, c, f"__n_{c}"))
        is_float = src.column(c).dtype.kind == "f"
        if a.op in (N.AGG_SUM, N.AGG_MEAN, N.AGG_VAR, N.AGG_STD):
            if is_float or a.op in (N.AGG_VAR, N.AGG_STD, N.AGG_MEAN):
                p.mean = p.mean or add(N.AGG_MEAN, c, f"__m_{c}")
            if not is_float and a.op in (N.AGG_SUM, N.AGG_MEAN):
                p.isum = p.isum or add(N.AGG_SUM, c, f"__s_{c}")
        if a.op in (N.AGG_VAR, N.AGG_STD):
            p.var0 = p.var0 or add(N.AGG_VAR, c, f"__v_{c}", ddof=0)
        if a.op == N.AGG_MIN:
            p.lo = p.lo or add(N.AGG_MIN, c, f"__lo_{c}")
        if a.op == N.AGG_MAX:
            p.hi = p.hi or add(N.AGG_MAX, c, f"__hi_{c}")
        if a.op == N.AGG_NULL_COUNT:
            p.nulls = p.nulls or add(N.AGG_NULL_COUNT, c, f"__z_{c}")
    sub = Plan(part, list(plan.filters), list(plan.keys), aggs, True)
    return sub, parts, rows_name


def _key_bytes(cols: list[Series]) -> np.ndarray:
    """One fixed-width byte string per row: per key column a validity byte and
    the value bytes (0 when null; NaN canonical and -0.0 as 0.0 for floats,
    the keys' equality)."""
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
        pieces.append(valid[:, None].astype(np.uint8))
        pieces.append(raw)
    mat = np.ascontiguousarray(np.concatenate(pieces, axis=1)) if pieces else np.zeros((n, 1), np.uint8)
    return mat.view(np.dtype((np.void, mat.shape[1]))).ravel()


def _cat(parts: list[DataFrame], name: str) -> Series:
    vals = np.concatenate([p[name].values for p in parts])
    if all(p[name].valid is None for p in parts):
        return Series(name, vals)
    valid = np.concatenate([np.ones(p.height, bool) if p[name].valid is None else p[name].valid for p in parts])
    return Series(name, vals, valid)


def _valid(s: Series) -> np.ndarray:
    return np.ones(len(s), bool) if s.valid is None else s.valid


def merge_partials(plan: Plan, parts: list[DataFrame], spec: dict, rows_name: str) -> DataFrame:
    """The query's result from the ranks' partial results, `parts` in rank
    order."""
    from .provider import DataFaultError, ProviderError

    keys = [_cat(parts, k) for k in plan.keys]
    total = sum(p.height for p in parts)
    kb = _key_bytes(keys)
    _, first, inv = np.unique(kb, return_index=True, return_inverse=True)
    inv = inv.ravel()
    # Groups in order of their first occurrence; rows sorted by group, rank order kept.
    order_groups = np.argsort(first, kind="stable")
    rank_of = np.empty_like(order_groups)
    rank_of[order_groups] = np.arange(len(order_groups))
    gid = rank_of[inv] if total else inv
    rows = np.argsort(gid, kind="stable")
    gsorted = gid[rows]
    starts = np.flatnonzero(np.r_[True, gsorted[1:] != gsorted[:-1]]) if total else np.zeros(0, np.int64)
    G = len(starts)
    firsts = rows[starts]

    def red_add(a):
        return np.add.reduceat(a[rows], starts) if G else np.zeros(0, a.dtype)

    out_cols = [Series(k.name, k.values[firsts], None if k.valid is None else k.valid[firsts]) for k in keys]
    merged = {}
    for c, p in spec.items():
        n = red_add(_cat(parts, p.count).values.astype(np.int64))
        d = {"n": n}
        if p.mean is not None:
            m = _cat(parts, p.mean)
            ni = _cat(parts, p.count).values.astype(np.float64)
            mv = np.where(_valid(m), m.values, 0.0)
            d["fsum"] = red_add(mv * ni)
            if p.var0 is not None:
                v0 = _cat(parts, p.var0)
                mean = np.divide(d["fsum"], n, out=np.zeros(G), where=n > 0)
                dev = mv - mean[gid]
                m2i = np.where(_valid(v0), v0.values, 0.0) * ni + ni * dev * dev
                d["m2"] = red_add(m2i)
                d["mean"] = mean
        if p.isum is not None:
            s = _cat(parts, p.isum)
            vals = np.where(_valid(s), s.values, 0)
            approx = red_add(vals.astype(np.float64))
            exact = red_add(vals)
            limit = 2.0**63 if vals.dtype == np.int64 else 2.0**64
            if np.any(np.abs(approx) >= limit * (1 - 1e-12)):
                raise ProviderError(N.DATA_OVERFLOW, f"{'Int64' if vals.dtype == np.int64 else 'UInt64'} expression sum overflow")
            d["isum"] = exact
        for side in ("lo", "hi"):
            name = getattr(p, side)
            if name is None:
                continue
            s = _cat(parts, name)
            d[side] = _merge_extreme(s, rows, starts, gid, side == "lo", DataFaultError)
        if p.nulls is not None:
            d["nulls"] = red_add(_cat(parts, p.nulls).values.astype(np.int64))
        merged[c] = d
    nrows = red_add(_cat(parts, rows_name).values.astype(np.int64))

    src = plan.source
    for a in plan.aggs:
        d = merged[a.column]
        idt = src.column(a.column).dtype
        n = d["n"]
        if a.op == N.AGG_COUNT:
            out_cols.append(Series(a.name, n.astype(np.int64)))
        elif a.op == N.AGG_LEN:
            out_cols.append(Series(a.name, nrows.astype(np.int64)))
        elif a.op == N.AGG_NULL_COUNT:
            out_cols.append(Series(a.name, d["nulls"].astype(np.int64)))
        elif a.op == N.AGG_SUM:
            valid = n >= a.min_count
            if idt.kind == "f":
                vals = np.where(valid, d["fsum"], 0.0).astype(idt)
            else:
                vals = np.where(valid, d["isum"], 0)
            out_cols.append(Series(a.name, vals, valid if not valid.all() else None))
        elif a.op == N.AGG_MEAN:
            tot = d["fsum"] if idt.kind == "f" else d["isum"].astype(np.float64)
            valid = n > 0
            out_cols.append(Series(a.name, np.divide(tot, n, out=np.zeros(G), where=valid), valid))
        elif a.op in (N.AGG_VAR, N.AGG_STD):
            valid = n > a.ddof
            var = np.divide(d["m2"], n - a.ddof, out=np.zeros(G), where=valid)
            vals = np.sqrt(var) if a.op == N.AGG_STD else var
            out_cols.append(Series(a.name, vals, valid))
        elif a.op in (N.AGG_MIN, N.AGG_MAX):
            vals, valid = d["lo" if a.op == N.AGG_MIN else "hi"]
            out_cols.append(Series(a.name, vals, valid))
        else:
            raise ValueError(f"aggregation {a.op} is not supported in a sharded query")
    return DataFrame(out_cols)


def _merge_extreme(s: Series, rows, starts, gid, is_min: bool, fault):
    """Minimum (or maximum) of the ranks' extrema per group: nulls skipped,
    NaN only when every valid partial is NaN, on equal values the earliest
    rank's kept; mixed signed zeros as the extreme are a data fault."""
    G = len(starts)
    valid = _valid(s)
    v = s.values
    if G == 0:
        return v[:0], np.zeros(0, bool)
    anyvalid = np.logical_or.reduceat(valid[rows], starts)
    if v.dtype.kind == "f":
        finite = valid & ~np.isnan(v)
        fill = np.inf if is_min else -np.inf
        x = np.where(finite, v, fill).astype(np.float64)
        best = (np.minimum if is_min else np.maximum).reduceat(x[rows], starts)
        has = np.logical_or.reduceat(finite[rows], starts)
        out = np.where(has, best, np.nan).astype(v.dtype)
        # Zero extremes: the earliest partial's sign, or a fault when both occur.
        zero = has & (best == 0)
        if zero.any():
            z = finite & (v == 0)
            neg = z & np.signbit(v)
            pos = z & ~np.signbit(v)
            gneg = np.logical_or.reduceat(neg[rows], starts)
            gpos = np.logical_or.reduceat(pos[rows], starts)
            if np.any(zero & gneg & gpos):
                raise fault("Mojo GPU data fault: mixed signed-zero extrema; the CPU adjudicates")
            out = np.where(zero & gneg, np.array(-0.0, v.dtype), out)
        return out, anyvalid
    info = np.iinfo(v.dtype)
    fill = info.max if is_min else info.min
    x = np.where(valid, v, fill).astype(v.dtype)
    best = (np.minimum if is_min else np.maximum).reduceat(x[rows], starts)
    return best.astype(v.dtype), anyvalid


def split_rows(frame: DataFrame, world: int) -> list[DataFrame]:
    """Contiguous row ranges, one per rank."""
    bounds = np.linspace(0, frame.height, world + 1).astype(np.int64)
    out = []
    for r in range(world):
        a, b = int(bounds[r]), int(bounds[r + 1])
        out.append(DataFrame([Series(c, frame[c].values[a:b], None if frame[c].valid is None else frame[c].valid[a:b])
                              for c in frame.columns]))
    return out


def execute_sharded(lazy: LazyFrame | Plan, rank: int, world: int, run=None, group=None) -> DataFrame:
    """The query over all ranks' rows: this rank aggregates its contiguous
    share of `lazy`'s source frame with `run` (default: the device provider),
    the partial results are all-gathered, and every rank merges them."""
    import torch.distributed as dist

    plan = lazy.plan if isinstance(lazy, LazyFrame) else lazy
    part = split_rows(plan.source, world)[rank]
    sub, spec, rows_name = partial_plan(plan, part)
    if run is None:
        from .provider import execute

        def run(p):
            return execute(p)[0]
    mine = run(sub)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    return merge_partials(plan, gathered, spec, rows_name)
