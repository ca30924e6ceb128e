"""Host-side frames, expressions and plans: the shapes the reference's core
hands a provider, restated just far enough for the filtered group-by region.

Reference shapes:
  * ``DataFrame`` of ``Series`` = typed values + validity
    (dataframe/storage/column.mojo:1-32).
  * ``LazyFrame.filter(pred).group_by(keys, maintain_order).agg(exprs)``
    (dataframe/lazy_api.mojo:418-419, 3135-3256): a SCAN -> FILTER* -> AGG
    region (dataframe/query_execution/placement.mojo:74-94).
  * ``collect(engine="accel")`` reaches the provider's ``execute``
    (dataframe/lazy_api.mojo:1763-1766).  The CPU engine is not part of this
    package: ``engine="cpu"`` raises here.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _native as N

_NP_TO_DFC = {
    np.dtype(np.int8): N.INT8,
    np.dtype(np.int16): N.INT16,
    np.dtype(np.int32): N.INT32,
    np.dtype(np.int64): N.INT64,
    np.dtype(np.uint8): N.UINT8,
    np.dtype(np.uint16): N.UINT16,
    np.dtype(np.uint32): N.UINT32,
    np.dtype(np.uint64): N.UINT64,
    np.dtype(np.float32): N.FLOAT32,
    np.dtype(np.float64): N.FLOAT64,
}
_DFC_TO_NP = {v: k for k, v in _NP_TO_DFC.items()}


def dfc_dtype(dtype: np.dtype) -> int:
    try:
        return _NP_TO_DFC[np.dtype(dtype)]
    except KeyError:
        raise TypeError(f"unsupported column type {dtype}") from None


def np_dtype(code: int) -> np.dtype:
    return _DFC_TO_NP[code]


class Series:
    """A named column: values plus an optional validity mask (True = valid).

    A column made by `from_bits` keeps its validity as the packed bitmap it
    came with (bit i of byte i // 8 set = row i valid, the layout the
    reference's columns and the provider use) and unpacks it to the bool
    mask only when `valid` is first read."""

    def __init__(self, name: str, values, valid=None, dtype=None, categories=None):
        """`values`: a numeric array, or strings (a String column, values of
        dtype object).  With `categories` the column is a Categorical: values
        are UInt32 codes into that dictionary of strings
        (dataframe/categorical.mojo:1-17)."""
        arr = np.asarray(values, dtype=dtype)
        if arr.ndim != 1:
            raise ValueError("a Series is one-dimensional")
        if arr.dtype.kind in "OUS":
            if categories is not None:
                raise TypeError("a Categorical's values are UInt32 codes")
            arr = arr.astype(object)
        else:
            dfc_dtype(arr.dtype)
        if categories is not None:
            if arr.dtype != np.uint32:
                raise TypeError("a Categorical's codes are UInt32")
            categories = np.asarray(categories, dtype=object)
        self.name = name
        self.values = np.ascontiguousarray(arr)
        self.categories = categories
        self._bits = None
        self.valid = valid

    @property
    def is_string(self) -> bool:
        return self.values.dtype == object

    @property
    def is_categorical(self) -> bool:
        return self.categories is not None

    def decoded(self) -> np.ndarray:
        """The column's strings (String or Categorical columns)."""
        if self.is_categorical:
            return self.categories[self.values]
        return self.values

    @classmethod
    def from_bits(cls, name: str, values, bits: np.ndarray | None) -> "Series":
        """A column over `values` whose validity is the packed bitmap `bits`
        (None = every row valid).  The bitmap is kept, not copied."""
        s = cls(name, values)
        n = len(s.values)
        if bits is not None:
            bits = np.asarray(bits, dtype=np.uint8)
            if len(bits) < (n + 7) // 8:
                raise ValueError("validity bitmap shorter than the values")
            if not bits_all_set(bits, n):
                s._bits = bits[: (n + 7) // 8]
        return s

    @property
    def valid(self) -> np.ndarray | None:
        if self._bits is not None:
            self._valid = unpack_validity(self._bits, len(self.values))
            self._bits = None
        return self._valid

    @valid.setter
    def valid(self, valid) -> None:
        if valid is not None:
            valid = np.asarray(valid, dtype=bool)
            if valid.shape != self.values.shape:
                raise ValueError("validity length differs from values")
            if valid.all():
                valid = None
        self._bits = None
        self._valid = valid

    @property
    def has_nulls(self) -> bool:
        return self._bits is not None or self._valid is not None

    def validity_bits(self) -> np.ndarray | None:
        """The validity as a packed little-endian bitmap (None = all valid)."""
        if self._bits is not None:
            return self._bits
        return pack_validity(self._valid)

    def __len__(self) -> int:
        return len(self.values)

    @property
    def dtype(self) -> np.dtype:
        return self.values.dtype

    def is_valid(self, i: int) -> bool:
        return self.valid is None or bool(self.valid[i])

    def item(self, i: int):
        if not self.is_valid(i):
            return None
        if self.is_categorical:
            return self.categories[self.values[i]]
        v = self.values[i]
        return v if self.is_string else v.item()

    def to_list(self) -> list:
        return [self.item(i) for i in range(len(self))]

    def slice(self, offset: int, length: int) -> "Series":
        v = None if self.valid is None else self.valid[offset : offset + length]
        return Series(self.name, self.values[offset : offset + length], v, categories=self.categories)

    def equals(self, other: "Series") -> bool:
        """Same name, dtype, length, nulls and values (NaN equals NaN)."""
        if self.name != other.name or self.dtype != other.dtype or len(self) != len(other):
            return False
        if self.is_categorical != other.is_categorical:
            return False
        if self.is_categorical and not np.array_equal(self.categories, other.categories):
            return False
        va = np.ones(len(self), bool) if self.valid is None else self.valid
        vb = np.ones(len(other), bool) if other.valid is None else other.valid
        if not np.array_equal(va, vb):
            return False
        a, b = self.values[va], other.values[vb]
        if self.dtype.kind == "f":
            return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
        return bool(np.array_equal(a, b))

    def __repr__(self) -> str:
        return f"Series({self.name!r}, {self.dtype}, {self.to_list()[:8]}{'...' if len(self) > 8 else ''})"


class DataFrame:
    def __init__(self, columns: Iterable[Series] | dict):
        if isinstance(columns, dict):
            columns = [s if isinstance(s, Series) else Series(k, s) for k, s in columns.items()]
        self._cols: list[Series] = list(columns)
        names = [c.name for c in self._cols]
        if len(set(names)) != len(names):
            raise ValueError("duplicate column names")
        lens = {len(c) for c in self._cols}
        if len(lens) > 1:
            raise ValueError("columns differ in length")

    @property
    def columns(self) -> list[str]:
        return [c.name for c in self._cols]

    @property
    def height(self) -> int:
        return len(self._cols[0]) if self._cols else 0

    def column(self, name: str) -> Series:
        for c in self._cols:
            if c.name == name:
                return c
        raise KeyError(name)

    def __getitem__(self, name: str) -> Series:
        return self.column(name)

    def item(self, row: int, name: str):
        return self.column(name).item(row)

    def lazy(self) -> "LazyFrame":
        return LazyFrame(self)

    def slice(self, offset: int, length: int) -> "DataFrame":
        return DataFrame([c.slice(offset, length) for c in self._cols])

    def group_by(self, keys, maintain_order: bool = False) -> "LazyGroupBy":
        """Eager form (dataframe/aggregation/group_by.mojo:235-356): a
        one-node lazy plan collected at once by ``agg``."""
        return _EagerGroupBy(self.lazy().group_by(keys, maintain_order=maintain_order))

    def equals(self, other: "DataFrame") -> bool:
        return self.columns == other.columns and all(a.equals(b) for a, b in zip(self._cols, other._cols))

    def __repr__(self) -> str:
        return f"DataFrame({self.height} rows: {', '.join(f'{c.name}:{c.dtype}' for c in self._cols)})"


# ---------------------------------------------------------------------------
# Expressions.
# ---------------------------------------------------------------------------
_CMP = {"<": N.LT, "<=": N.LE, ">": N.GT, ">=": N.GE, "==": N.EQ, "!=": N.NE}


@dataclass(frozen=True)
class Pred:
    """A filter predicate: a tree of comparisons and Kleene connectives."""

    kind: str  # cmp / is_null / is_not_null / and / or / not / true
    column: str | None = None
    op: str | None = None
    literal: object = None
    args: tuple = ()

    def __and__(self, other: "Pred") -> "Pred":
        return Pred("and", args=(self, other))

    def __or__(self, other: "Pred") -> "Pred":
        return Pred("or", args=(self, other))

    def __invert__(self) -> "Pred":
        return Pred("not", args=(self,))


@dataclass(frozen=True)
class AggExpr:
    op: int
    column: str
    name: str
    ddof: int = 1
    min_count: int = 0

    def alias(self, name: str) -> "AggExpr":
        return AggExpr(self.op, self.column, name, self.ddof, self.min_count)


@dataclass(frozen=True)
class Col:
    name: str

    def _cmp(self, op: str, lit) -> Pred:
        return Pred("cmp", column=self.name, op=op, literal=lit)

    def __lt__(self, lit):
        return self._cmp("<", lit)

    def __le__(self, lit):
        return self._cmp("<=", lit)

    def __gt__(self, lit):
        return self._cmp(">", lit)

    def __ge__(self, lit):
        return self._cmp(">=", lit)

    def __eq__(self, lit):  # type: ignore[override]
        return self._cmp("==", lit)

    def __ne__(self, lit):  # type: ignore[override]
        return self._cmp("!=", lit)

    __hash__ = object.__hash__

    def is_null(self) -> Pred:
        return Pred("is_null", column=self.name)

    def is_not_null(self) -> Pred:
        return Pred("is_not_null", column=self.name)

    def sum(self, min_count: int = 0) -> AggExpr:
        return AggExpr(N.AGG_SUM, self.name, self.name, min_count=min_count)

    def mean(self) -> AggExpr:
        return AggExpr(N.AGG_MEAN, self.name, self.name)

    def min(self) -> AggExpr:
        return AggExpr(N.AGG_MIN, self.name, self.name)

    def max(self) -> AggExpr:
        return AggExpr(N.AGG_MAX, self.name, self.name)

    def count(self) -> AggExpr:
        return AggExpr(N.AGG_COUNT, self.name, self.name)

    def len(self) -> AggExpr:
        return AggExpr(N.AGG_LEN, self.name, self.name)

    def null_count(self) -> AggExpr:
        return AggExpr(N.AGG_NULL_COUNT, self.name, self.name)

    def first(self) -> AggExpr:
        """The value at the group's first kept row (null when that value is)."""
        return AggExpr(N.AGG_FIRST, self.name, self.name)

    def last(self) -> AggExpr:
        """The value at the group's last kept row (null when that value is)."""
        return AggExpr(N.AGG_LAST, self.name, self.name)

    def n_unique(self) -> AggExpr:
        """Distinct values of the group: null is one value, NaN one, -0.0 == 0.0."""
        return AggExpr(N.AGG_N_UNIQUE, self.name, self.name)

    def var(self, ddof: int = 1) -> AggExpr:
        return AggExpr(N.AGG_VAR, self.name, self.name, ddof=ddof)

    def std(self, ddof: int = 1) -> AggExpr:
        return AggExpr(N.AGG_STD, self.name, self.name, ddof=ddof)


def col(name: str) -> Col:
    return Col(name)


def lit(value):
    return value


# ---------------------------------------------------------------------------
# Plans.
# ---------------------------------------------------------------------------
@dataclass
class Plan:
    """SCAN_FRAME -> FILTER* -> AGG, the region a provider receives."""

    source: DataFrame
    filters: list[Pred] = field(default_factory=list)
    keys: list[str] | None = None
    aggs: list[AggExpr] | None = None
    maintain_order: bool = False

    def describe(self) -> str:
        parts = [f"SCAN_FRAME {self.source.columns}"]
        parts += [f"FILTER {f}" for f in self.filters]
        if self.keys == []:
            parts.append(f"SELECT {[a.name for a in self.aggs]}")
        elif self.keys is not None:
            parts.append(f"AGG keys={self.keys} maintain_order={self.maintain_order} aggs={[a.name for a in self.aggs]}")
        return " -> ".join(parts)


class LazyFrame:
    def __init__(self, source: DataFrame, plan: Plan | None = None):
        self._plan = plan or Plan(source)

    @property
    def plan(self) -> Plan:
        return self._plan

    def filter(self, pred: Pred) -> "LazyFrame":
        if self._plan.keys is not None:
            raise ValueError("a filter after the aggregation is not part of this region")
        p = Plan(self._plan.source, self._plan.filters + [pred])
        return LazyFrame(p.source, p)

    def group_by(self, keys, maintain_order: bool = False) -> "LazyGroupBy":
        if isinstance(keys, str):
            keys = [keys]
        keys = list(keys)
        if not keys:
            raise ValueError("group_by needs at least one key")
        if len(set(keys)) != len(keys):
            raise ValueError("duplicate key column")
        for k in keys:
            self._plan.source.column(k)
        return LazyGroupBy(self, keys, maintain_order)

    def select(self, exprs: AggExpr | Sequence[AggExpr]) -> "LazyFrame":
        """Ungrouped reductions of the filtered rows: SCAN_FRAME -> FILTER* ->
        SELECT(col(c).sum(), ...), one output row (the reference's filtered
        reduction region, dataframe_metal/filter_plan.mojo:149-200).  An empty
        selection gives the reductions of no rows: sum 0 (null when min_count
        > 0), count, len and null_count 0, mean, min, max, var and std null."""
        if self._plan.keys is not None:
            raise ValueError("a select after the aggregation is not part of this region")
        if isinstance(exprs, AggExpr):
            exprs = [exprs]
        exprs = list(exprs)
        if not exprs:
            raise ValueError("select needs at least one reduction")
        for e in exprs:
            self._plan.source.column(e.column)
        names = [e.name for e in exprs]
        if len(set(names)) != len(names):
            raise ValueError("duplicate output column names")
        p = self._plan
        plan = Plan(p.source, list(p.filters), [], exprs, False)
        return LazyFrame(p.source, plan)

    def collect(self, engine: str = "accel") -> DataFrame:
        if engine != "accel":
            raise ValueError("this package holds only the accelerator provider: engine must be 'accel'")
        from . import provider

        return provider.execute(self)[0]


class LazyGroupBy:
    def __init__(self, frame: LazyFrame, keys: list[str], maintain_order: bool):
        self._frame = frame
        self._keys = keys
        self._maintain_order = maintain_order

    def agg(self, exprs: AggExpr | Sequence[AggExpr]) -> LazyFrame:
        if isinstance(exprs, AggExpr):
            exprs = [exprs]
        exprs = list(exprs)
        for e in exprs:
            self._frame.plan.source.column(e.column)
        names = list(self._keys) + [e.name for e in exprs]
        if len(set(names)) != len(names):
            raise ValueError("duplicate output column names")
        p = self._frame.plan
        plan = Plan(p.source, list(p.filters), list(self._keys), exprs, self._maintain_order)
        return LazyFrame(p.source, plan)

    def len(self, name: str = "len") -> LazyFrame:
        return self.agg([AggExpr(N.AGG_LEN, self._keys[0], name)])


class _EagerGroupBy:
    def __init__(self, lazy: LazyGroupBy):
        self._lazy = lazy

    def agg(self, exprs) -> DataFrame:
        return self._lazy.agg(exprs).collect()

    def len(self, name: str = "len") -> DataFrame:
        return self._lazy.len(name).collect()


# ---------------------------------------------------------------------------
# Binding: a plan as the column list, filter program and aggregation list the
# C ABI takes (binding happens before a backend is chosen in the reference,
# docs/design/accelerator-contract.md:75).
# ---------------------------------------------------------------------------
@dataclass
class Bound:
    names: list[str]                 # input column names, in `inputs` order
    series: list[Series]
    keys: list[int]
    pred: list[tuple]                # (kind, column index, cmp, literal) postfix
    aggs: list[tuple]                # (op, column index, ddof, min_count)
    out_names: list[str]
    maintain_order: bool
    # Output column index -> ("categorical" | "string", dictionary): columns
    # that come back as codes and are decoded (decode_outputs).
    decoders: dict = field(default_factory=dict)


def _bind_literal(series: Series, value):
    """A literal cast to the column's type (the core's literal coercion)."""
    kind = series.dtype.kind
    if kind == "f":
        return ("f", float(value))
    if isinstance(value, float):
        if value != value:
            raise TypeError("NaN literal against an integer column")
        if not float(value).is_integer():
            raise TypeError("fractional literal against an integer column")
        value = int(value)
    info = np.iinfo(series.dtype)
    if not info.min <= int(value) <= info.max:
        raise TypeError(f"literal {value} out of range for {series.dtype}")
    return ("u", int(value)) if series.dtype == np.uint64 else ("i", int(value))


# Aggregations that read a String or Categorical column through its codes
# (they need only equality or the row's value).
_CODED_AGGS = {N.AGG_COUNT, N.AGG_LEN, N.AGG_NULL_COUNT, N.AGG_N_UNIQUE, N.AGG_FIRST, N.AGG_LAST}


def _coded(s: Series) -> tuple[Series, str, np.ndarray]:
    """A String or Categorical column as UInt32 codes.  A Categorical keys by
    canonical codes (every code mapped to the first code with the same label,
    so repeated labels are one group) and keeps its dictionary; a String
    column is dictionary-encoded here and decoded back after the query (the
    reference groups a dictionary-coded String key by its codes and returns
    strings: dataframe/aggregation/group_by.mojo:307-317, 344-356)."""
    valid = s.valid
    if s.is_categorical:
        labels = s.categories
        first: dict = {}
        canon = np.array([first.setdefault(lab, i) for i, lab in enumerate(labels)], dtype=np.uint32)
        raw = s.values if valid is None else np.where(valid, s.values, 0).astype(np.uint32)
        codes = canon[raw] if len(labels) else np.zeros(len(s), np.uint32)
        return Series(s.name, codes, valid), "categorical", labels
    filled = s.values if valid is None else np.where(valid, s.values, "")
    uniques, inverse = np.unique(filled.astype(str).astype(object), return_inverse=True)
    return Series(s.name, inverse.astype(np.uint32), valid), "string", uniques


def _code_literal(kind: str, table: np.ndarray, value) -> int:
    """The code a string literal compares as: its (canonical) code, or one no
    row holds when the dictionary lacks it."""
    hits = np.flatnonzero(table == value) if len(table) else []
    return int(hits[0]) if len(hits) else len(table)


def bind(plan: Plan) -> Bound:
    if plan.keys is None:
        raise ValueError("the plan has no aggregation")
    src = plan.source
    names: list[str] = []
    coded: dict[str, tuple] = {}

    def idx(name: str) -> int:
        if name not in names:
            s = src.column(name)
            if s.is_string or s.is_categorical:
                coded[name] = _coded(s)
            names.append(name)
        return names.index(name)

    def series(name: str) -> Series:
        return coded[name][0] if name in coded else src.column(name)

    keys = [idx(k) for k in plan.keys]
    prog: list[tuple] = []

    def emit(p: Pred):
        if p.kind == "cmp":
            i = idx(p.column)
            if p.column in coded:
                if p.op not in ("==", "!="):
                    raise TypeError(f"only == and != compare a String or Categorical column ({p.column})")
                _, kind, table = coded[p.column]
                prog.append((N.PRED_CMP, i, _CMP[p.op], ("i", _code_literal(kind, table, p.literal))))
            else:
                prog.append((N.PRED_CMP, i, _CMP[p.op], _bind_literal(src.column(p.column), p.literal)))
        elif p.kind == "is_null":
            prog.append((N.PRED_IS_NULL, idx(p.column), 0, ("i", 0)))
        elif p.kind == "is_not_null":
            prog.append((N.PRED_IS_NOT_NULL, idx(p.column), 0, ("i", 0)))
        elif p.kind == "true":
            prog.append((N.PRED_TRUE, 0, 0, ("i", 0)))
        elif p.kind == "not":
            emit(p.args[0])
            prog.append((N.PRED_NOT, 0, 0, ("i", 0)))
        elif p.kind in ("and", "or"):
            emit(p.args[0])
            emit(p.args[1])
            prog.append((N.PRED_AND if p.kind == "and" else N.PRED_OR, 0, 0, ("i", 0)))
        else:
            raise ValueError(f"unknown predicate {p.kind}")

    for i, f in enumerate(plan.filters):
        emit(f)
        if i > 0:
            prog.append((N.PRED_AND, 0, 0, ("i", 0)))
    aggs = [(a.op, idx(a.column), a.ddof, a.min_count) for a in plan.aggs]
    decoders: dict = {}
    for k, name in enumerate(plan.keys):
        if name in coded:
            decoders[k] = coded[name][1:]
    for j, a in enumerate(plan.aggs):
        if a.column in coded:
            if a.op not in _CODED_AGGS:
                raise TypeError(f"this aggregation does not read a String or Categorical column ({a.column})")
            if a.op in (N.AGG_FIRST, N.AGG_LAST):
                decoders[len(plan.keys) + j] = coded[a.column][1:]
    return Bound(
        names=names,
        series=[series(n) for n in names],
        keys=keys,
        pred=prog,
        aggs=aggs,
        out_names=list(plan.keys) + [a.name for a in plan.aggs],
        maintain_order=plan.maintain_order,
        decoders=decoders,
    )


def decode_outputs(bound: Bound, frame: DataFrame) -> DataFrame:
    """Result columns that came back as codes: a Categorical keeps its
    dictionary, a String column gets its strings back."""
    if not bound.decoders:
        return frame
    cols = []
    for i, name in enumerate(frame.columns):
        s = frame[name]
        if i not in bound.decoders:
            cols.append(s)
            continue
        kind, table = bound.decoders[i]
        valid = s.valid
        codes = s.values.astype(np.uint32)
        if kind == "categorical":
            cols.append(Series(name, codes, valid, categories=table))
        else:
            strings = np.empty(len(s), dtype=object)
            ok = np.ones(len(s), bool) if valid is None else valid
            strings[ok] = table[codes[ok]] if len(table) else None
            cols.append(Series(name, strings, valid))
    return DataFrame(cols)


def pack_validity(valid: np.ndarray | None) -> np.ndarray | None:
    if valid is None:
        return None
    return np.packbits(valid.astype(np.uint8), bitorder="little")


def bits_all_set(bits: np.ndarray, rows: int) -> bool:
    """Whether the first `rows` bits of a little-endian bitmap are all set."""
    full = rows // 8
    head = full - full % 8
    if head and not np.all(bits[:head].view(np.uint64) == np.uint64(0xFFFFFFFFFFFFFFFF)):
        return False
    if full > head and not np.all(bits[head:full] == 0xFF):
        return False
    rem = rows % 8
    return not rem or (int(bits[full]) & ((1 << rem) - 1)) == (1 << rem) - 1


def unpack_validity(bits: np.ndarray, rows: int) -> np.ndarray:
    # unpackbits yields 0/1 bytes, which are valid booleans: a view, no copy.
    return np.unpackbits(bits, bitorder="little")[:rows].view(bool)
