"""Loads tests/golden/known_answers.json and expands its table specs into host
columns (numpy arrays, Utf8 columns, masked arrays for NULLs).  The generator
formulas are the reference fixtures' own (cited in make_known_answers.py)."""
from __future__ import annotations

import json
from pathlib import Path
from typing import Dict, List

import numpy as np

from falcondb_b200 import Utf8

GOLDEN = Path(__file__).resolve().parent / "golden" / "known_answers.json"


def cases() -> List[dict]:
    return json.loads(GOLDEN.read_text())["cases"]


def _explicit(spec: dict) -> Dict[str, object]:
    out = {}
    for c in spec["columns"]:
        vals = c["values"]
        if c["type"] == "utf8":
            out[c["name"]] = Utf8.from_strings(vals)
        else:
            dt = np.int64 if c["type"] == "int64" else np.float64
            mask = np.array([v is None for v in vals], dtype=bool)
            data = np.array([0 if v is None else v for v in vals], dtype=dt)
            out[c["name"]] = np.ma.MaskedArray(data, mask=mask) if mask.any() else data
    return out


def build_table(spec: dict) -> Dict[str, object]:
    g = spec.get("gen")
    if g is None:
        return _explicit(spec)
    n = spec.get("rows", 0)
    i = np.arange(n, dtype=np.int64)
    if g == "count_star":  # count_star_filter.rs:15-37
        return {
            "n": i,
            "maybe": np.ma.MaskedArray(i, mask=(i % 3 == 0)),
            "s": Utf8(np.asarray(i % 3, dtype=np.uint32), ["a", "b", "c"]),
        }
    if g == "split_700k":  # aggregate.rs:3519-3597
        total = 700_000
        j = np.arange(total, dtype=np.int64)
        return {"dept": Utf8(np.asarray(j % 5, dtype=np.uint32), ["eng", "sales", "hr", "ops", "legal"]), "v": j}
    if g == "join_db_left":  # join_and_parquet_paths.rs:27-33
        return {"k": i, "lv": i * 2}
    if g == "join_db_right":
        k = i + spec.get("base", 0)
        return {"k": k, "rv": k * 3}
    if g == "bench":  # query_bench.rs:103-122
        return {"id": i, "dept": Utf8(np.asarray(i % 5, dtype=np.uint32), ["eng", "hr", "finance", "ops", "legal"]),
                "score": (i % 100).astype(np.float64) + 0.5}
    if g == "lookup":  # query_bench.rs:486-500: every tenth id
        m = n // 10
        j = np.arange(m, dtype=np.int64)
        return {"lid": j * 10, "label": Utf8(np.asarray(j % 5, dtype=np.uint32), ["eng", "hr", "finance", "ops", "legal"])}
    raise ValueError(f"unknown generator {g}")


def check_result(case: dict, res) -> None:
    exp = case["expect"]
    if "scalar" in exp:
        got = res.to_rows()[0][0]
        assert got == exp["scalar"], f"{case['name']}: got {got}, want {exp['scalar']}"
    if "rows" in exp:
        rows = res.to_rows()
        want = exp["rows"]
        if exp.get("sorted"):
            rows, want = sorted(rows), sorted(want)
        assert rows == want, f"{case['name']}: got {rows}, want {want}"
    if "head_rows" in exp:
        rows = res.to_rows()[:len(exp["head_rows"])]
        assert rows == exp["head_rows"], f"{case['name']}: got {rows}, want {exp['head_rows']}"
    if "row_count" in exp:
        assert res.row_count() == exp["row_count"], f"{case['name']}: {res.row_count()} rows"
    if "first_col_sorted" in exp:
        got = sorted(r[0] for r in res.to_rows())
        assert got == exp["first_col_sorted"], f"{case['name']}: got {got}"
