"""Sharded group-by: the rows split across ranks (one process per GPU), each
rank aggregating its own rows on its own GPU, one exchange of the partial
groups by key, and a merge on the device that restores the result of one
query over all rows (the reference's parallel design: per-worker partial
tables merged by partition, dataframe/aggregation/hash_table.mojo:11-47).

1. Partials.  Each rank runs the query over its contiguous rows with
   aggregations a merge can combine -- counts, rows, null counts, integer
   sums (sum types are exact), means (a Float column's sum is rebuilt as
   mean x count in FP64), population variances (M2 = var0 x n) and extrema
   -- in first-appearance order (partial_plan).  On GPUs the partial result
   stays on the device (dfc_result_copy_to_device into torch tensors).
2. Exchange.  Every partial row goes to the rank that owns its key (a hash
   of the canonical key words: NaN one value, -0.0 == 0.0, nulls equal):
   one all_to_all_single of a packed int64 matrix (NCCL over NVLink on GPUs,
   gloo on CPU), after one of the row counts.  No TMA or bulk copy reads
   another GPU's memory.  A row carries its position (rank << 32 | index in
   its rank's partial result): rank r's rows all come after rank r-1's, so
   the smallest position of a group is its global first appearance.
3. Owner merge, on the owner's device (torch tensors): groups by torch.unique
   over the key words; exact integer sums from 32-bit halves (the split the
   reference's Metal kernels use, dataframe_metal/accelerator/gpu/
   filter_sum.mojo:8-14) checked against the sum type with the CPU's
   overflow message; float sums; Chan et al.'s update for M2 (the combine of
   dataframe/aggregation/function.mojo:1736-1758); extrema with the
   single-GPU null, NaN, tie and signed-zero rules; key values from the
   group's first row.
4. Order.  The owners' finished rows (one per group) are all-gathered and
   ordered by their groups' first position (maintain_order=True).
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


# ---------------------------------------------------------------------------
# Columns as int64 tensors: the raw bits of 8-byte values, narrower ones
# widened (signed types sign-extended, Float32 through its Int32 bits), so
# every column fits one int64 column of the exchanged matrix and decodes back
# exactly.
# ---------------------------------------------------------------------------
def _encode_np(values: np.ndarray) -> np.ndarray:
    dt = values.dtype
    if dt.itemsize == 8:
        return np.ascontiguousarray(values).view(np.int64)
    if dt == np.float32:
        return np.ascontiguousarray(values).view(np.int32).astype(np.int64)
    return values.astype(np.int64)


def _decode_np(bits: np.ndarray, dt: np.dtype) -> np.ndarray:
    dt = np.dtype(dt)
    bits = np.ascontiguousarray(bits, dtype=np.int64)
    if dt.itemsize == 8:
        return bits.view(dt)
    if dt == np.float32:
        return bits.astype(np.int32).view(np.float32)
    return bits.astype(dt)


class _Cols:
    """Partial columns on one device: name -> (int64 bits, valid mask, dtype)."""

    def __init__(self):
        self.bits: dict = {}
        self.valid: dict = {}
        self.dtype: dict = {}

    def add(self, name, bits, valid, dtype):
        self.bits[name], self.valid[name], self.dtype[name] = bits, valid, np.dtype(dtype)

    def rows(self) -> int:
        return int(next(iter(self.bits.values())).shape[0]) if self.bits else 0


def _frame_cols(frame: DataFrame, device) -> _Cols:
    import torch

    cols = _Cols()
    for c in frame.columns:
        s = frame[c]
        bits = torch.from_numpy(_encode_np(s.values).copy()).to(device)
        valid = torch.ones(len(s), dtype=torch.bool, device=device) if s.valid is None else \
            torch.from_numpy(np.asarray(s.valid, dtype=bool).copy()).to(device)
        cols.add(c, bits, valid, s.dtype)
    return cols


def _result_cols(result, device) -> _Cols:
    """A device result's columns as torch tensors on `device`, copied device
    to device (dfc_result_copy_to_device)."""
    import torch

    lib = N.lib()
    cols = _Cols()
    rows = result.rows
    for i, name in enumerate(result.names):
        dt, _, _ = result.column_info(i)
        raw = torch.empty(max(rows, 1), dtype=_TORCH_DTYPE[np.dtype(dt)], device=device)
        vbytes = torch.empty(max((rows + 7) // 8, 1), dtype=torch.uint8, device=device)
        # The library copies on its own stream: torch's queued work on these
        # blocks (they may be reused) completes first.
        torch.cuda.current_stream(device).synchronize()
        st = lib.dfc_result_copy_to_device(result.handle, i, raw.data_ptr(), vbytes.data_ptr())
        if st != N.OK:
            from .provider import _error

            raise _error(st, N.last_error())
        raw = raw[:rows]
        if np.dtype(dt).itemsize == 8:
            bits = raw.view(torch.int64)
        elif np.dtype(dt) == np.float32:
            bits = raw.view(torch.int32).to(torch.int64)
        else:
            bits = raw.to(torch.int64)
            if np.dtype(dt).kind == "u":  # torch reads UInt16/UInt32 through signed views
                bits &= (1 << (8 * np.dtype(dt).itemsize)) - 1
        shifts = torch.arange(8, device=device, dtype=torch.uint8)
        valid = ((vbytes.unsqueeze(1) >> shifts) & 1).reshape(-1)[:rows].bool()
        cols.add(name, bits, valid, dt)
    return cols


def _torch_dtypes():
    import torch

    return {np.dtype(np.int8): torch.int8, np.dtype(np.int16): torch.int16, np.dtype(np.int32): torch.int32,
            np.dtype(np.int64): torch.int64, np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.int16,
            np.dtype(np.uint32): torch.int32, np.dtype(np.uint64): torch.int64, np.dtype(np.float32): torch.float32,
            np.dtype(np.float64): torch.float64}


class _LazyDtypes(dict):
    def __missing__(self, key):
        self.update(_torch_dtypes())
        return dict.__getitem__(self, key)


_TORCH_DTYPE = _LazyDtypes()


# ---------------------------------------------------------------------------
# Keys: canonical words (every NaN one value, -0.0 == 0.0, a null key's word
# 0 with its null flag), their hash to an owner rank, and the exchange.
# ---------------------------------------------------------------------------
_CANON_F64 = 0x7FF8000000000000
_CANON_F32 = 0x7FC00000
_MIX1 = -0x61C8864680B583EB  # 0x9E3779B97F4A7C15 as a signed 64-bit value
_MIX2 = -0x40A7B892E31B1A47  # 0xBF58476D1CE4E5B9


def _canonical(cols: _Cols, name: str):
    import torch

    bits, valid, dt = cols.bits[name], cols.valid[name], cols.dtype[name]
    if dt == np.float64:
        f = bits.view(torch.float64)
        bits = torch.where(torch.isnan(f), torch.full_like(bits, _CANON_F64), torch.where(f == 0, torch.zeros_like(bits), bits))
    elif dt == np.float32:
        f = bits.to(torch.int32).view(torch.float32)
        bits = torch.where(torch.isnan(f), torch.full_like(bits, _CANON_F32), torch.where(f == 0, torch.zeros_like(bits), bits))
    return torch.where(valid, bits, torch.zeros_like(bits)), valid


def _key_matrix(cols: _Cols, keys: list[str]):
    """One row per partial row: the canonical key words and a null flag word."""
    import torch

    n = cols.rows()
    words, nulls = [], torch.zeros(n, dtype=torch.int64, device=_device_of(cols))
    for k, name in enumerate(keys):
        w, valid = _canonical(cols, name)
        words.append(w)
        nulls |= (~valid).to(torch.int64) << k
    return torch.stack(words + [nulls], dim=1) if words else nulls.unsqueeze(1)


def _device_of(cols: _Cols):
    return next(iter(cols.bits.values())).device


def _owner(keymat, world: int):
    """The rank owning each row's key: a multiply-xorshift hash of its words."""
    import torch

    h = torch.zeros(keymat.shape[0], dtype=torch.int64, device=keymat.device)
    for j in range(keymat.shape[1]):
        h = (h ^ keymat[:, j]) * _MIX1
        h = h ^ ((h >> 31) & ((1 << 33) - 1))
        h = h * _MIX2
    return (h & 0x7FFFFFFFFFFFFFFF) % world


def _exchange(cols: _Cols, keys: list[str], rank: int, world: int, group=None):
    """Sends every partial row to its key's owner: returns the rows this rank
    owns (in source-rank order, each rank's in its partial order) and their
    positions (rank << 32 | index in the sender's partial result)."""
    import torch
    import torch.distributed as dist

    dev = _device_of(cols)
    n = cols.rows()
    names = list(cols.bits)
    pos = (torch.arange(n, dtype=torch.int64, device=dev) | (rank << 32))
    owner = _owner(_key_matrix(cols, keys), world) if n else torch.zeros(0, dtype=torch.int64, device=dev)
    order = torch.argsort(owner, stable=True)
    counts = torch.bincount(owner, minlength=world).to(torch.int64)
    validbits = torch.zeros(n, dtype=torch.int64, device=dev)
    for i, c in enumerate(names):
        validbits |= cols.valid[c].to(torch.int64) << i
    mat = torch.stack([cols.bits[c] for c in names] + [validbits, pos], dim=1)[order].contiguous()
    recv = torch.empty_like(counts)
    dist.all_to_all_single(recv, counts, group=group)
    out = torch.empty((int(recv.sum().item()), mat.shape[1]), dtype=torch.int64, device=dev)
    dist.all_to_all_single(out, mat, recv.tolist(), counts.tolist(), group=group)
    got = _Cols()
    for i, c in enumerate(names):
        got.add(c, out[:, i].contiguous(), ((out[:, len(names)] >> i) & 1).bool(), cols.dtype[c])
    return got, out[:, len(names) + 1].contiguous()


# ---------------------------------------------------------------------------
# Owner merge (torch, on the owner's device).
# ---------------------------------------------------------------------------
def _overflow_message(input_dtype: np.dtype) -> str:
    """The CPU provider's text (dataframe/aggregation/function.mojo:2798, 2914)."""
    dt = np.dtype(input_dtype)
    if dt == np.int64:
        return "Int64 expression sum overflow"
    sum_dt = np.dtype(np.int64) if dt.itemsize <= 2 and dt.kind in "iu" else dt
    return f"{sum_dt.name} expression sum overflow"


def _exact_sum(bits, inv, G: int, signed: bool):
    """Exact per-group totals of 64-bit integers from their 32-bit halves
    (each half's sum fits int64 for fewer than 2^31 rows): (high, low) with
    total = high * 2^32 + low, low in [0, 2^32)."""
    import torch

    lo = bits & 0xFFFFFFFF
    hi = (bits >> 32) if signed else ((bits >> 32) & 0xFFFFFFFF)
    los = torch.zeros(G, dtype=torch.int64, device=bits.device).index_add_(0, inv, lo)
    his = torch.zeros(G, dtype=torch.int64, device=bits.device).index_add_(0, inv, hi)
    return his + (los >> 32), los & 0xFFFFFFFF


def _merge_extreme(bits, valid, dt: np.dtype, inv, G: int, is_min: bool):
    """Minimum (maximum) of the partial extrema per group: nulls skipped, NaN
    only when every valid partial is NaN, a zero extremum keeps the sign of
    the zeros seen (both signs: the CPU adjudicates)."""
    import torch

    from .provider import DataFaultError

    dev = bits.device
    red = "amin" if is_min else "amax"
    anyvalid = torch.zeros(G, dtype=torch.int32, device=dev).scatter_reduce_(0, inv, valid.to(torch.int32), "amax")
    if dt.kind == "f":
        v = bits.view(torch.float64) if dt == np.float64 else bits.to(torch.int32).view(torch.float32).to(torch.float64)
        finite = valid & ~torch.isnan(v)
        fill = float("inf") if is_min else float("-inf")
        x = torch.where(finite, v, torch.full_like(v, fill))
        best = torch.full((G,), fill, dtype=torch.float64, device=dev).scatter_reduce_(0, inv, x, red)
        has = torch.zeros(G, dtype=torch.int32, device=dev).scatter_reduce_(0, inv, finite.to(torch.int32), "amax") > 0
        out = torch.where(has, best, torch.full_like(best, float("nan")))
        zero = has & (best == 0)
        if bool(zero.any()):
            z = finite & (v == 0)
            neg = (z & torch.signbit(v)).to(torch.int32)
            pos = (z & ~torch.signbit(v)).to(torch.int32)
            gneg = torch.zeros(G, dtype=torch.int32, device=dev).scatter_reduce_(0, inv, neg, "amax") > 0
            gpos = torch.zeros(G, dtype=torch.int32, device=dev).scatter_reduce_(0, inv, pos, "amax") > 0
            if bool((zero & gneg & gpos).any()):
                raise DataFaultError(N.DATA_FAULT, "Mojo GPU data fault: mixed signed-zero extrema; the CPU adjudicates")
            out = torch.where(zero & gneg, torch.full_like(out, -0.0), out)
        if dt == np.float64:
            obits = out.view(torch.int64)
        else:
            obits = out.to(torch.float32).view(torch.int32).to(torch.int64)
        return obits, anyvalid > 0
    if dt == np.uint64:
        # Unsigned order through the sign-flipped bits.
        x = torch.where(valid, bits ^ (-(1 << 63)), torch.full_like(bits, (1 << 63) - 1 if is_min else -(1 << 63)))
        best = torch.full((G,), (1 << 63) - 1 if is_min else -(1 << 63), dtype=torch.int64, device=dev)
        best = best.scatter_reduce_(0, inv, x, red)
        return best ^ (-(1 << 63)), anyvalid > 0
    info = np.iinfo(dt)
    fill = int(info.max) if is_min else int(info.min)
    x = torch.where(valid, bits, torch.full_like(bits, fill))
    best = torch.full((G,), fill, dtype=torch.int64, device=dev).scatter_reduce_(0, inv, x, red)
    return best, anyvalid > 0


def _merge_owned(plan: Plan, cols: _Cols, pos, spec: dict, rows_name: str):
    """The finished rows of the groups this rank owns: per output column
    (int64 bits, valid, dtype), and each group's first position."""
    import torch

    from .provider import ProviderError

    dev = pos.device
    n = int(pos.shape[0])
    src = plan.source
    out_dtypes = _output_dtypes(plan)
    if n == 0:
        empty = torch.zeros(0, dtype=torch.int64, device=dev)
        return [(empty, empty.bool(), dt) for dt in out_dtypes], empty
    keymat = _key_matrix(cols, plan.keys)
    _, inv = torch.unique(keymat, dim=0, return_inverse=True)
    inv = inv.reshape(-1)
    G = int(inv.max().item()) + 1
    first = torch.full((G,), n, dtype=torch.int64, device=dev).scatter_reduce_(
        0, inv, torch.arange(n, dtype=torch.int64, device=dev), "amin")
    first_pos = pos[first]

    def add(x, dtype=torch.int64):
        return torch.zeros(G, dtype=dtype, device=dev).index_add_(0, inv, x)

    out = [(cols.bits[k][first], cols.valid[k][first], cols.dtype[k]) for k in plan.keys]
    merged = {}
    for c, p in spec.items():
        d = {"n": add(cols.bits[p.count])}
        ni = cols.bits[p.count].to(torch.float64)
        if p.mean is not None:
            mv = torch.where(cols.valid[p.mean], cols.bits[p.mean].view(torch.float64), torch.zeros_like(ni))
            d["fsum"] = add(mv * ni, torch.float64)
            if p.var0 is not None:
                mean = torch.where(d["n"] > 0, d["fsum"] / d["n"].clamp(min=1).to(torch.float64), torch.zeros_like(d["fsum"]))
                dev_ = mv - mean[inv]
                v0 = torch.where(cols.valid[p.var0], cols.bits[p.var0].view(torch.float64), torch.zeros_like(ni))
                d["m2"] = add(v0 * ni + ni * dev_ * dev_, torch.float64)
        if p.isum is not None:
            sdt = cols.dtype[p.isum]
            bits = torch.where(cols.valid[p.isum], cols.bits[p.isum], torch.zeros_like(cols.bits[p.isum]))
            hi, lo = _exact_sum(bits, inv, G, signed=sdt.kind == "i")
            d["isum"] = (hi, lo, sdt)
        for side in ("lo", "hi"):
            name = getattr(p, side)
            if name is not None:
                d[side] = _merge_extreme(cols.bits[name], cols.valid[name], cols.dtype[name], inv, G, side == "lo")
        if p.nulls is not None:
            d["nulls"] = add(cols.bits[p.nulls])
        merged[c] = d
    nrows = add(cols.bits[rows_name])
    true = torch.ones(G, dtype=torch.bool, device=dev)
    for a, odt in zip(plan.aggs, out_dtypes[len(plan.keys):]):
        d = merged[a.column]
        idt = src.column(a.column).dtype
        cnt = d["n"]
        if a.op == N.AGG_COUNT:
            out.append((cnt, true, odt))
        elif a.op == N.AGG_LEN:
            out.append((nrows, true, odt))
        elif a.op == N.AGG_NULL_COUNT:
            out.append((d["nulls"], true, odt))
        elif a.op == N.AGG_SUM:
            valid = cnt >= a.min_count
            if idt.kind == "f":
                s = torch.where(valid, d["fsum"], torch.zeros_like(d["fsum"]))
                bits = s.view(torch.int64) if odt == np.float64 else s.to(torch.float32).view(torch.int32).to(torch.int64)
            else:
                hi, lo, sdt = d["isum"]
                bits = _checked_total(hi, lo, sdt, valid, idt, ProviderError)
            out.append((torch.where(valid, bits, torch.zeros_like(bits)), valid, odt))
        elif a.op == N.AGG_MEAN:
            valid = cnt > 0
            if idt.kind == "f":
                tot = d["fsum"]
            else:
                hi, lo, sdt = d["isum"]
                tot = hi.to(torch.float64) * 4294967296.0 + lo.to(torch.float64)
            m = torch.where(valid, tot / cnt.clamp(min=1).to(torch.float64), torch.zeros_like(tot))
            out.append((m.view(torch.int64), valid, odt))
        elif a.op in (N.AGG_VAR, N.AGG_STD):
            valid = cnt > a.ddof
            var = torch.where(valid, d["m2"] / (cnt - a.ddof).clamp(min=1).to(torch.float64), torch.zeros_like(d["m2"]))
            v = torch.sqrt(var) if a.op == N.AGG_STD else var
            out.append((v.view(torch.int64), valid, odt))
        elif a.op in (N.AGG_MIN, N.AGG_MAX):
            bits, valid = d["lo" if a.op == N.AGG_MIN else "hi"]
            out.append((bits, valid, odt))
        else:
            raise ValueError(f"aggregation {a.op} is not supported in a sharded query")
    return out, first_pos


def _checked_total(hi, lo, sdt: np.dtype, valid, idt: np.dtype, error):
    """The exact total's bits when it fits the sum type, else the CPU's
    overflow error."""
    import torch

    if sdt.kind == "u":
        ok = (hi >= 0) & (hi < (1 << 32)) if sdt.itemsize == 8 else (hi == 0)
    else:
        ok = (hi >= -(1 << 31)) & (hi < (1 << 31)) if sdt.itemsize == 8 else (
            (hi == 0) & (lo < (1 << 31))) | ((hi == -1) & (lo >= (1 << 31)))
    if bool((valid & ~ok).any()):
        raise error(N.DATA_OVERFLOW, _overflow_message(idt))
    return (hi << 32) | lo


def _output_dtypes(plan: Plan) -> list[np.dtype]:
    src = plan.source
    out = [src.column(k).dtype for k in plan.keys]
    for a in plan.aggs:
        idt = src.column(a.column).dtype
        if a.op in (N.AGG_COUNT, N.AGG_LEN, N.AGG_NULL_COUNT):
            out.append(np.dtype(np.int64))
        elif a.op == N.AGG_SUM:
            out.append(idt if idt.kind == "f" or idt.itemsize >= 4 else np.dtype(np.int64))
        elif a.op in (N.AGG_MIN, N.AGG_MAX):
            out.append(idt)
        else:
            out.append(np.dtype(np.float64))
    return out


# ---------------------------------------------------------------------------
# Order and assembly.
# ---------------------------------------------------------------------------
def _pack(columns, first_pos):
    """One int64 matrix per owner: the output columns' bits, a word of their
    validity bits and each group's first position."""
    import torch

    validbits = torch.zeros(first_pos.shape[0], dtype=torch.int64, device=first_pos.device)
    for i, (_, valid, _) in enumerate(columns):
        validbits |= valid.to(torch.int64) << i
    return torch.stack([b for b, _, _ in columns] + [validbits, first_pos], dim=1)


def _assemble(plan: Plan, mat, dtypes) -> DataFrame:
    """The host frame of the finished rows, ordered by first position."""
    import torch

    mat = mat[torch.argsort(mat[:, -1])]
    host = mat.cpu().numpy()
    names = list(plan.keys) + [a.name for a in plan.aggs]
    width = len(names)
    cols = []
    for i, (name, dt) in enumerate(zip(names, dtypes)):
        valid = ((host[:, width] >> i) & 1).astype(bool)
        cols.append(Series(name, _decode_np(host[:, i], dt), None if valid.all() else valid))
    return DataFrame(cols)


def _gather_ordered(plan: Plan, columns, first_pos, group=None) -> DataFrame:
    """Every owner's finished rows on every rank (one all_gather of the
    packed matrices, padded to the largest), ordered by first position."""
    import torch
    import torch.distributed as dist

    mat = _pack(columns, first_pos).contiguous()
    dev = mat.device
    world = dist.get_world_size(group)
    n = torch.tensor([mat.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    pad = torch.zeros((max(max(sizes), 1), mat.shape[1]), dtype=torch.int64, device=dev)
    pad[: mat.shape[0]] = mat
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return _assemble(plan, torch.cat([b[:s] for b, s in zip(bufs, sizes)]), [dt for _, _, dt in columns])


def _take(cols: _Cols, idx) -> _Cols:
    out = _Cols()
    for c in cols.bits:
        out.add(c, cols.bits[c][idx], cols.valid[c][idx], cols.dtype[c])
    return out


def _concat(parts: list[_Cols]) -> _Cols:
    import torch

    out = _Cols()
    for c in parts[0].bits:
        out.add(c, torch.cat([p.bits[c] for p in parts]), torch.cat([p.valid[c] for p in parts]), parts[0].dtype[c])
    return out


def _check_shardable(plan: Plan) -> None:
    if plan.keys is None or not plan.keys or plan.aggs is None:
        raise ValueError("a sharded query is a group-by with at least one key")
    src = plan.source
    for name in set(plan.keys) | {a.column for a in plan.aggs}:
        s = src.column(name)
        if s.is_string or s.is_categorical:
            raise ValueError(f"column {name!r}: a sharded query reads numeric columns")
    if len(plan.keys) + len(plan.aggs) > 62:
        raise ValueError("a sharded query has at most 62 output columns")


# ---------------------------------------------------------------------------
# Entry points.
# ---------------------------------------------------------------------------
def split_rows(frame: DataFrame, world: int) -> list[DataFrame]:
    """Contiguous row ranges, one per rank."""
    bounds = np.linspace(0, frame.height, world + 1).astype(np.int64)
    out = []
    for r in range(world):
        a, b = int(bounds[r]), int(bounds[r + 1])
        out.append(DataFrame([Series(c, frame[c].values[a:b], None if frame[c].valid is None else frame[c].valid[a:b])
                              for c in frame.columns]))
    return out


def merge_partials(plan: Plan, parts: list, spec: dict, rows_name: str, owners: int | None = None,
                   device=None) -> DataFrame:
    """The query's result from the ranks' partial results in one process:
    `parts` in rank order, host DataFrames or DeviceResults (read on their
    device).  The rows are routed to `owners` owners (default one per part)
    by the exchange's key hash, each owner's rows merged as that rank would,
    and the finished rows ordered by first position."""
    import torch

    from .provider import DeviceResult

    _check_shardable(plan)
    if device is None:
        on_gpu = [p for p in parts if isinstance(p, DeviceResult)]
        device = torch.device("cuda", on_gpu[0].device) if on_gpu else torch.device("cpu")
    cols, pos = [], []
    for r, p in enumerate(parts):
        c = _result_cols(p, device) if isinstance(p, DeviceResult) else _frame_cols(p, device)
        cols.append(c)
        pos.append(torch.arange(c.rows(), dtype=torch.int64, device=device) | (r << 32))
    allc, allpos = _concat(cols), torch.cat(pos)
    owners = len(parts) if owners is None else owners
    owner = _owner(_key_matrix(allc, plan.keys), owners)
    mats, dtypes = [], _output_dtypes(plan)
    for o in range(owners):
        idx = torch.nonzero(owner == o).reshape(-1)
        columns, first_pos = _merge_owned(plan, _take(allc, idx), allpos[idx], spec, rows_name)
        mats.append(_pack(columns, first_pos))
    return _assemble(plan, torch.cat(mats), dtypes)


def execute_sharded(lazy: LazyFrame | Plan, rank: int, world: int, run=None, group=None, device=None) -> DataFrame:
    """The query over all ranks' rows, called by every rank of `group`:
    this rank aggregates its contiguous share of the source frame -- on its
    GPU (`device`, default torch's current CUDA device) with the result kept
    there, or with `run(plan) -> DataFrame` (tests: the oracle, on CPU
    tensors) -- the partial rows go to their keys' owners, each owner merges
    its groups, and every rank returns the whole result."""
    import torch

    plan = lazy.plan if isinstance(lazy, LazyFrame) else lazy
    _check_shardable(plan)
    part = split_rows(plan.source, world)[rank]
    sub, spec, rows_name = partial_plan(plan, part)
    if run is None:
        from .frame import bind
        from .provider import DeviceColumn, _regime_flags, run_bound

        index = torch.cuda.current_device() if device is None else int(device)
        bound = bind(sub)
        inputs = [DeviceColumn(s, index) for s in bound.series]
        try:
            result = run_bound(bound, inputs, flags=_regime_flags())
            try:
                cols = _result_cols(result, torch.device("cuda", index))
            finally:
                result.free()
        finally:
            for c in inputs:
                c.release()
    else:
        cols = _frame_cols(run(sub), torch.device("cpu") if device is None else device)
    got, pos = _exchange(cols, plan.keys, rank, world, group)
    columns, first_pos = _merge_owned(plan, got, pos, spec, rows_name)
    return _gather_ordered(plan, columns, first_pos, group)
