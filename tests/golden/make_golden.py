"""Writes tests/golden/fixtures.json: known-answer cases transcribed from the
reference's own tests (inputs and expected outputs as those tests state them).

Run from the repository root:  python tests/golden/make_golden.py

Each case cites the reference test it comes from.  Floats are stored as
float.hex() strings so -0.0 and NaN survive; nulls as None.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

OUT = Path(__file__).resolve().parent / "fixtures.json"

I32_MIN, I32_MAX = -(2**31), 2**31 - 1
I64_MIN, I64_MAX = -(2**63), 2**63 - 1


def fl(x: float) -> str:
    return float(x).hex()


def column(dtype: str, values, valid=None):
    vals = []
    for i, v in enumerate(values):
        ok = True if valid is None else bool(valid[i])
        if dtype.startswith("float"):
            vals.append(fl(v) if ok else None)
        else:
            vals.append(int(v) if ok else None)
    return {"dtype": dtype, "values": vals}


def numbers(kind: int, values, valid):
    """_numbers of test_metal_grouped_reductions.mojo:8-21: Int32, Int64 or Float32."""
    dtype = ["int32", "int64", "float32"][kind]
    return column(dtype, values, valid)


def null_key_cases():
    """test_metal_grouped_reductions.mojo:317-466 — null keys, Int32/Int64
    extremes, filter p >= 1, sliced rows 1..6; expected order and states."""
    cases = []
    for kind in range(3):
        key_kind = 0 if kind == 0 else 1
        low = I32_MIN if key_kind == 0 else I64_MIN
        high = I32_MAX if key_kind == 0 else I64_MAX
        k = [9, low, high, low, 0, high, 0, 9]
        kv = [True, True, True, True, False, True, False, True]
        v = [99, 2, 3, 4, 5, 6, 7, 99]
        vv = [True, True, True, False, True, True, True, True]
        p = [-1, 0, 1, 2, 3, 4, 5, -1]
        sl = slice(1, 7)
        src = {
            "k": numbers(key_kind, k[sl], kv[sl]),
            "v": numbers(kind, v[sl], vv[sl]),
            "p": column("int32", p[sl]),
        }
        for filtered in (False, True):
            nonempty = [True, not filtered, True]
            keys_out = [high if filtered else low, low if filtered else high, 0]
            expected = {
                "k": numbers(key_kind, keys_out, [True, True, False]),
                "s": numbers(kind, [9 if filtered else 2, 0 if filtered else 9, 12], None),
                "n": column("int64", [2 if filtered else 1, 0 if filtered else 2, 2]),
                "avg": column("float64", [4.5 if filtered else 2.0, 0.0 if filtered else 4.5, 6.0], nonempty),
                "lo": numbers(kind, [3 if filtered else 2, 0 if filtered else 3, 5], nonempty),
                "hi": numbers(kind, [6 if filtered else 2, 0 if filtered else 6, 7], nonempty),
            }
            # Int32 sums keep Int32 (dtype.mojo:838-849); Float32 sums Float32.
            cases.append(
                {
                    "name": f"null_keys_kind{kind}_{'filtered' if filtered else 'all'}",
                    "source": "tests/execution_modes/test_metal_grouped_reductions.mojo:317-466",
                    "columns": src,
                    "filters": [["cmp", "p", ">=", 1]] if filtered else [],
                    "keys": ["k"],
                    "maintain_order": True,
                    "aggs": [
                        ["sum", "v", "s"],
                        ["count", "v", "n"],
                        ["mean", "v", "avg"],
                        ["min", "v", "lo"],
                        ["max", "v", "hi"],
                    ],
                    "expected": expected,
                }
            )
            cases.append(
                {
                    "name": f"null_keys_len_kind{kind}_{'filtered' if filtered else 'all'}",
                    "source": "tests/execution_modes/test_metal_grouped_reductions.mojo:458-465",
                    "columns": src,
                    "filters": [["cmp", "p", ">=", 1]] if filtered else [],
                    "keys": ["k"],
                    "maintain_order": True,
                    "aggs": [["len", "k", "len"]],
                    "expected": {
                        "k": numbers(key_kind, keys_out, [True, True, False]),
                        "len": column("int64", [2, 1 if filtered else 2, 2]),
                    },
                }
            )
    return cases


def cardinality_cases():
    """test_metal_grouped_reductions.mojo:494-560 — 256/257/4,096 distinct
    keys; an empty input; an all-null key of three rows."""
    cases = []
    for distinct in (256, 257, 4096):
        rows = list(range(distinct))
        cases.append(
            {
                "name": f"distinct_{distinct}",
                "source": "tests/execution_modes/test_metal_grouped_reductions.mojo:494-530",
                "columns": {"k": column("int32", rows), "v": column("int64", [r + 1 for r in rows])},
                "filters": [],
                "keys": ["k"],
                "maintain_order": True,
                "aggs": [["sum", "v", "s"], ["count", "v", "n"], ["min", "v", "lo"], ["max", "v", "hi"]],
                "expected": {
                    "k": column("int32", rows),
                    "s": column("int64", [r + 1 for r in rows]),
                    "n": column("int64", [1] * distinct),
                    "lo": column("int64", [r + 1 for r in rows]),
                    "hi": column("int64", [r + 1 for r in rows]),
                },
            }
        )
    cases.append(
        {
            "name": "empty_input",
            "source": "tests/execution_modes/test_metal_grouped_reductions.mojo:531-550",
            "columns": {"k": column("int32", []), "v": column("int64", [])},
            "filters": [],
            "keys": ["k"],
            "maintain_order": False,
            "aggs": [["sum", "v", "s", {"min_count": 1}], ["mean", "v", "avg"], ["min", "v", "lo"], ["count", "v", "n"]],
            "expected": {
                "k": column("int32", []),
                "s": column("int64", []),
                "avg": column("float64", []),
                "lo": column("int64", []),
                "n": column("int64", []),
            },
        }
    )
    cases.append(
        {
            "name": "all_null_key",
            "source": "tests/execution_modes/test_metal_grouped_reductions.mojo:551-560",
            "columns": {
                "k": column("int32", [0, 0, 0], [False, False, False]),
                "v": column("int64", [0, 0, 0], [False, False, False]),
            },
            "filters": [],
            "keys": ["k"],
            "maintain_order": False,
            "aggs": [["len", "k", "len"]],
            "expected": {"k": column("int32", [0], [False]), "len": column("int64", [3])},
        }
    )
    return cases


def float_special_case():
    """tests/public_contracts/test_grouping.mojo:71-105 — float keys -0.0 and
    0.0 are one group, every NaN one group, a null its own; the key cell is
    the group's first row; reductions of i (= row index) per group
    (integer_reductions, tests/support/reduction_contract.mojo:14-28)."""
    nan = float("nan")
    f = [-0.0, 0.0, nan, nan, 0.0]
    fv = [True, True, True, True, False]
    groups = [[0, 1], [2, 3], [4]]

    def var(xs):
        if len(xs) < 2:
            return None
        m = sum(xs) / len(xs)
        return sum((x - m) ** 2 for x in xs) / (len(xs) - 1)

    return {
        "name": "float_key_specials",
        "source": "tests/public_contracts/test_grouping.mojo:71-105",
        "columns": {"i": column("int64", list(range(5))), "f": column("float64", f, fv)},
        "filters": [],
        "keys": ["f"],
        "maintain_order": True,
        "aggs": [
            ["sum", "i", "sum"],
            ["count", "i", "count"],
            ["len", "i", "len"],
            ["min", "i", "min"],
            ["max", "i", "max"],
            ["mean", "i", "mean"],
            ["var", "i", "var"],
            ["std", "i", "std"],
        ],
        "expected": {
            "f": column("float64", [-0.0, nan, 0.0], [True, True, False]),
            "sum": column("int64", [sum(g) for g in groups]),
            "count": column("int64", [len(g) for g in groups]),
            "len": column("int64", [len(g) for g in groups]),
            "min": column("int64", [min(g) for g in groups]),
            "max": column("int64", [max(g) for g in groups]),
            "mean": column("float64", [sum(g) / len(g) for g in groups]),
            "var": column("float64", [var(g) or 0.0 for g in groups], [var(g) is not None for g in groups]),
            "std": column(
                "float64", [math.sqrt(var(g)) if var(g) is not None else 0.0 for g in groups],
                [var(g) is not None for g in groups],
            ),
        },
    }


def overflow_cases():
    """Checked sums: test_metal_grouped_reductions.mojo:755-770 (Int32 sum
    past Int32.MAX raises "int32 expression sum overflow"); the CPU's Int64
    text is "Int64 expression sum overflow" (scalar_states.mojo:35-40,
    function.mojo:2798); exact wide partials accept overflow followed by
    cancellation (docs/design/accelerator-contract.md:80-83)."""
    return [
        {
            "name": "int32_sum_overflow",
            "source": "tests/execution_modes/test_metal_grouped_reductions.mojo:764-767",
            "columns": {"k": column("int32", [0, 0, 1]), "v": column("int32", [I32_MAX, 1, 5])},
            "filters": [],
            "keys": ["k"],
            "maintain_order": True,
            "aggs": [["sum", "v", "s"]],
            "expected_error": "int32 expression sum overflow",
        },
        {
            "name": "int64_sum_overflow",
            "source": "dataframe/aggregation/scalar_states.mojo:35-40",
            "columns": {"k": column("int64", [7, 7, 8]), "v": column("int64", [I64_MIN, -1, 3])},
            "filters": [],
            "keys": ["k"],
            "maintain_order": True,
            "aggs": [["sum", "v", "s"]],
            "expected_error": "Int64 expression sum overflow",
        },
        {
            "name": "int64_overflow_then_cancel",
            "source": "docs/design/accelerator-contract.md:80-83",
            "columns": {"k": column("int64", [1, 1, 1, 2]), "v": column("int64", [I64_MAX, 1, -1, -5])},
            "filters": [],
            "keys": ["k"],
            "maintain_order": True,
            "aggs": [["sum", "v", "s"], ["mean", "v", "m"]],
            "expected": {
                "k": column("int64", [1, 2]),
                "s": column("int64", [I64_MAX, -5]),
                "m": column("float64", [float(I64_MAX) / 3.0, -5.0]),
            },
        },
        {
            "name": "filtered_overflow_row_dropped",
            "source": "tests/execution_modes/test_metal_grouped_reductions.mojo:583-598",
            "columns": {
                "k": column("int32", [0, 1]),
                "v": column("int32", [I32_MAX, 1]),
                "p": column("int32", [0, 1]),
            },
            "filters": [["cmp", "p", ">", 0]],
            "keys": ["k"],
            "maintain_order": True,
            "aggs": [["sum", "v", "s"]],
            "expected": {"k": column("int32", [1]), "s": column("int32", [1])},
        },
    ]


def welford_case():
    """docs/design/metal-moments.md:139-147: for [2^60, 2^60 + 256] the
    CPU's population variance is 32,768 (exact: 16,384).  The oracle must
    reproduce the CPU value; the provider reports a data fault so the CPU
    adjudicates, as the reference's Metal provider does."""
    return {
        "name": "welford_two_values",
        "source": "docs/design/metal-moments.md:139-147",
        "columns": {"k": column("int32", [0, 0]), "x": column("int64", [2**60, 2**60 + 256])},
        "filters": [],
        "keys": ["k"],
        "maintain_order": True,
        "aggs": [["var", "x", "var0", {"ddof": 0}]],
        "expected": {"k": column("int32", [0]), "var0": column("float64", [32768.0])},
        "device_expect": "data_fault",
    }


def bench_engine_small_case():
    """benchmarks/bench_gpu_groupby_engine.mojo:12-58 scenario 0: 4,099 rows,
    17 keys (row * 7919) % 17, values row % 1009 - 504 with every 19th row
    null; min, max, sum, count in first-appearance order (exact)."""
    rows, card = 4099, 17
    keys = [(r * 7919) % card for r in range(rows)]
    vals = [r % 1009 - 504 for r in range(rows)]
    valid = [r % 19 != 0 for r in range(rows)]
    order = []
    groups: dict[int, list[int]] = {}
    for r in range(rows):
        if keys[r] not in groups:
            groups[keys[r]] = []
            order.append(keys[r])
        if valid[r]:
            groups[keys[r]].append(vals[r])
    return {
        "name": "bench_engine_4099x17",
        "source": "benchmarks/bench_gpu_groupby_engine.mojo:12-58",
        "columns": {"key": column("int64", keys), "value": column("int64", vals, valid)},
        "filters": [],
        "keys": ["key"],
        "maintain_order": True,
        "aggs": [["min", "value", "min"], ["max", "value", "max"], ["sum", "value", "sum"], ["count", "value", "count"]],
        "expected": {
            "key": column("int64", order),
            "min": column("int64", [min(groups[k]) for k in order]),
            "max": column("int64", [max(groups[k]) for k in order]),
            "sum": column("int64", [sum(groups[k]) for k in order]),
            "count": column("int64", [len(groups[k]) for k in order]),
        },
    }


def main() -> None:
    cases = null_key_cases() + cardinality_cases() + [float_special_case()] + overflow_cases()
    cases += [welford_case(), bench_engine_small_case()]
    OUT.write_text(json.dumps({"cases": cases}, indent=None, separators=(",", ":")))
    print(f"{OUT}: {len(cases)} cases, {OUT.stat().st_size} bytes")


if __name__ == "__main__":
    main()
