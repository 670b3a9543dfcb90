"""ORACLE — test infrastructure only.

ctypes front end of ``oracle/liboracle.so``: the serial CPU restatement of
FalconDB's operators (oracle.cpp) and the reference-shaped multi-threaded CPU
engine (refengine.cpp).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg may import it; the product never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Optional, Tuple

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib: Optional[C.CDLL] = None

P = C.c_void_p
U64 = C.c_uint64
_SIGS = {
    "orc_cmp_mask": (None, [C.c_int, P, P, U64, C.c_int, C.c_int, C.c_int64, C.c_double, P]),
    "orc_code_mask": (None, [P, P, U64, P, C.c_uint32, P]),
    "orc_popcount": (U64, [P, U64]),
    "orc_mask_rows": (U64, [P, U64, P]),
    "orc_sum_lanes_f64": (C.c_double, [P, U64]),
    "orc_sum_serial_f64": (C.c_double, [P, U64]),
    "orc_checked_sum_i64": (C.c_int, [P, U64, P]),
    "orc_agg": (C.c_int, [C.c_int, C.c_int, P, P, P, U64, P, P]),
    "orc_sum_i64_masked": (C.c_int, [P, P, P, U64, P]),
    "orc_present_codes": (None, [P, P, P, U64, C.c_uint32, P]),
    "orc_group_codes": (None, [P, P, P, U64, C.c_uint32, P, P, P, P, P, P, P, P, P, P, P]),
    "orc_group_i64": (U64, [P, P, P, P, U64, P, P, P, P, P]),
    "orc_join_agg": (None, [P, P, P, P, U64, P, P, P, P, U64, C.c_int, P, P, P, P]),
    "orc_join_pairs": (U64, [P, P, U64, P, P, U64, C.c_int, P, P, U64]),
    "orc_topk": (U64, [C.c_int, P, P, U64, C.c_uint32, C.c_int, C.c_int, P]),
    "orc_sort": (None, [C.c_int, P, P, U64, C.c_int, C.c_int, P]),
    "orc_distinct": (U64, [C.c_int, P, P, U64, P]),
    "ref_hardware_threads": (C.c_int, []),
    "ref_sum_f64": (C.c_double, [P, U64, C.c_int]),
    "ref_count_cmp_f64": (U64, [P, U64, C.c_int, C.c_double]),
    "ref_present_codes": (None, [P, U64, C.c_uint32, C.c_int, P]),
    "ref_topk": (U64, [C.c_int, P, U64, C.c_uint32, C.c_int, P]),
    "ref_sort": (None, [C.c_int, P, P, U64, C.c_int, C.c_int, C.c_int, P]),
    "ref_filter_group_codes": (None, [P, P, P, U64, C.c_uint32, C.c_int, C.c_double, C.c_int, P, P, P]),
    "ref_join_agg": (None, [P, P, U64, P, P, U64, C.c_int, C.c_int, P, P, P]),
    "ref_group_i64": (U64, [P, P, U64, C.c_int]),
}


def build() -> Path:
    """Compile liboracle.so with the committed Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


# ---------------------------------------------------------------------------- serial oracle
def cmp_mask(values: np.ndarray, op: int, literal, validity: Optional[np.ndarray] = None) -> np.ndarray:
    v = np.ascontiguousarray(values)
    dtype = 2 if v.dtype.kind == "f" else 1
    v = v.astype(np.float64 if dtype == 2 else np.int64, copy=False)
    out = np.zeros(max(1, (len(v) + 63) // 64), dtype=np.uint64)
    lit_type = 2 if isinstance(literal, (float, np.floating)) else 1
    lib().orc_cmp_mask(dtype, _p(v), _p(_c(validity, np.uint64)), len(v), op, lit_type,
                       int(literal) if lit_type == 1 else 0, float(literal) if lit_type == 2 else 0.0, _p(out))
    return out


def code_mask(codes: np.ndarray, passing, validity=None) -> np.ndarray:
    c = _c(codes, np.uint32)
    pas = np.asarray(passing, dtype=np.uint8)
    out = np.zeros(max(1, (len(c) + 63) // 64), dtype=np.uint64)
    lib().orc_code_mask(_p(c), _p(_c(validity, np.uint64)), len(c), _p(pas), len(pas), _p(out))
    return out


def popcount(words: np.ndarray) -> int:
    w = _c(words, np.uint64)
    return int(lib().orc_popcount(_p(w), len(w)))


def mask_rows(words: np.ndarray, n: int) -> np.ndarray:
    w = _c(words, np.uint64)
    out = np.zeros(max(1, n), dtype=np.uint32)
    k = lib().orc_mask_rows(_p(w), n, _p(out))
    return out[:k]


def sum_lanes(v: np.ndarray) -> float:
    v = _c(v, np.float64)
    return float(lib().orc_sum_lanes_f64(_p(v), len(v)))


def sum_serial(v: np.ndarray) -> float:
    v = _c(v, np.float64)
    return float(lib().orc_sum_serial_f64(_p(v), len(v)))


def checked_sum_i64(v: np.ndarray) -> Optional[int]:
    v = _c(v, np.int64)
    out = np.zeros(1, dtype=np.int64)
    return int(out[0]) if lib().orc_checked_sum_i64(_p(v), len(v), _p(out)) else None


def agg(func: int, values: np.ndarray, mask=None, validity=None) -> Tuple[Optional[float], int]:
    """(value or None for SQL NULL, contributing count) of COUNT/SUM/AVG/MIN/MAX."""
    v = np.ascontiguousarray(values)
    dtype = 2 if v.dtype.kind == "f" else 1
    v = v.astype(np.float64 if dtype == 2 else np.int64, copy=False)
    val = np.zeros(1, dtype=np.float64)
    cnt = np.zeros(1, dtype=np.int64)
    ok = lib().orc_agg(func, dtype, _p(v), _p(_c(validity, np.uint64)), _p(_c(mask, np.uint64)), len(v),
                       _p(val), _p(cnt))
    return (float(val[0]) if ok else None), int(cnt[0])


def sum_i64_exact(values, mask=None, validity=None) -> Optional[int]:
    v = _c(values, np.int64)
    out = np.zeros(1, dtype=np.int64)
    ok = lib().orc_sum_i64_masked(_p(v), _p(_c(validity, np.uint64)), _p(_c(mask, np.uint64)), len(v), _p(out))
    return int(out[0]) if ok else None


def present_codes(codes, dict_len, mask=None, validity=None) -> np.ndarray:
    c = _c(codes, np.uint32)
    out = np.zeros(max(1, dict_len), dtype=np.uint8)
    lib().orc_present_codes(_p(c), _p(_c(validity, np.uint64)), _p(_c(mask, np.uint64)), len(c), dict_len, _p(out))
    return out[:dict_len]


def group_codes(codes, dict_len, mask=None, fvals=None, ivals=None, kvalid=None, fvalid=None, ivalid=None):
    """Per-group dict over groups 0..dict_len (dict_len = NULL key)."""
    c = _c(codes, np.uint32)
    ng = dict_len + 1
    arrs = {k: np.zeros(ng, dtype=dt) for k, dt in
            [("rows", np.int64), ("fsum", np.float64), ("fcnt", np.int64), ("isum", np.float64),
             ("icnt", np.int64), ("fmin", np.float64), ("fmax", np.float64)]}
    fv = _c(fvals, np.float64)
    iv = _c(ivals, np.int64)
    lib().orc_group_codes(_p(c), _p(_c(kvalid, np.uint64)), _p(_c(mask, np.uint64)), len(c), dict_len, _p(fv),
                          _p(_c(fvalid, np.uint64)), _p(iv), _p(_c(ivalid, np.uint64)), _p(arrs["rows"]),
                          _p(arrs["fsum"]), _p(arrs["fcnt"]), _p(arrs["isum"]), _p(arrs["icnt"]),
                          _p(arrs["fmin"]), _p(arrs["fmax"]))
    return arrs


def group_i64(keys, vals, mask=None, kvalid=None):
    k = _c(keys, np.int64)
    v = _c(vals, np.float64)
    n = len(k)
    out = {"key": np.zeros(n + 1, np.int64), "count": np.zeros(n + 1, np.int64), "sum": np.zeros(n + 1),
           "min": np.zeros(n + 1), "max": np.zeros(n + 1)}
    g = lib().orc_group_i64(_p(k), _p(_c(kvalid, np.uint64)), _p(v), _p(_c(mask, np.uint64)), n, _p(out["key"]),
                            _p(out["count"]), _p(out["sum"]), _p(out["min"]), _p(out["max"]))
    return {kk: vv[:g] for kk, vv in out.items()}


def join_agg(bkeys, bpay, pkeys, pval, join_type, bvalid=None, bpvalid=None, pvalid=None, pvvalid=None):
    bk, bp, pk, pv = _c(bkeys, np.int64), _c(bpay, np.int64), _c(pkeys, np.int64), _c(pval, np.float64)
    o = [np.zeros(1, np.int64), np.zeros(1, np.int64), np.zeros(1, np.int64), np.zeros(1, np.float64)]
    lib().orc_join_agg(_p(bk), _p(_c(bvalid, np.uint64)), _p(bp), _p(_c(bpvalid, np.uint64)), len(bk), _p(pk),
                       _p(_c(pvalid, np.uint64)), _p(pv), _p(_c(pvvalid, np.uint64)), len(pk), join_type,
                       *[_p(x) for x in o])
    return {"count": int(o[0][0]), "sum_payload": int(o[1][0]), "payload_rows": int(o[2][0]),
            "sum_value": float(o[3][0])}


def join_pairs(bkeys, pkeys, join_type, bvalid=None, pvalid=None):
    bk, pk = _c(bkeys, np.int64), _c(pkeys, np.int64)
    cap = 0
    n = lib().orc_join_pairs(_p(bk), _p(_c(bvalid, np.uint64)), len(bk), _p(pk), _p(_c(pvalid, np.uint64)), len(pk),
                             join_type, None, None, 0)
    left = np.zeros(max(1, n), np.uint32)
    right = np.zeros(max(1, n), np.uint32)
    lib().orc_join_pairs(_p(bk), _p(_c(bvalid, np.uint64)), len(bk), _p(pk), _p(_c(pvalid, np.uint64)), len(pk),
                         join_type, _p(left), _p(right), n)
    return left[:n], right[:n]


def topk(values, k, desc, nulls_last=None, validity=None) -> np.ndarray:
    v = np.ascontiguousarray(values)
    dtype = 2 if v.dtype.kind == "f" else 1
    v = v.astype(np.float64 if dtype == 2 else np.int64, copy=False)
    if nulls_last is None:
        nulls_last = desc
    out = np.zeros(max(1, k), dtype=np.uint32)
    m = lib().orc_topk(dtype, _p(v), _p(_c(validity, np.uint64)), len(v), k, int(desc), int(nulls_last), _p(out))
    return out[:m]


def sort(values, desc, nulls_last=None, validity=None) -> np.ndarray:
    """Every row number in ORDER BY order (orc_sort)."""
    v = np.ascontiguousarray(values)
    dtype = 2 if v.dtype.kind == "f" else 1
    v = v.astype(np.float64 if dtype == 2 else np.int64, copy=False)
    if nulls_last is None:
        nulls_last = desc
    out = np.zeros(max(1, len(v)), dtype=np.uint32)
    lib().orc_sort(dtype, _p(v), _p(_c(validity, np.uint64)), len(v), int(desc), int(nulls_last), _p(out))
    return out[:len(v)]


def distinct(values, validity=None) -> np.ndarray:
    """Row numbers of each value's first occurrence (orc_distinct).  A uint32
    array is taken as UTF8 codes."""
    v = np.ascontiguousarray(values)
    if v.dtype == np.uint32:
        dtype = 3
    elif v.dtype.kind == "f":
        dtype, v = 2, v.astype(np.float64, copy=False)
    else:
        dtype, v = 1, v.astype(np.int64, copy=False)
    out = np.zeros(max(1, len(v)), dtype=np.uint32)
    k = lib().orc_distinct(dtype, _p(v), _p(_c(validity, np.uint64)), len(v), _p(out))
    return out[:k]


# ---------------------------------------------------------------------------- reference-shaped engine
def hardware_threads() -> int:
    return int(lib().ref_hardware_threads())


def ref_sum_f64(v, threads):
    v = _c(v, np.float64)
    return float(lib().ref_sum_f64(_p(v), len(v), threads))


def ref_count_cmp_f64(v, op, lit):
    v = _c(v, np.float64)
    return int(lib().ref_count_cmp_f64(_p(v), len(v), op, float(lit)))


def ref_present_codes(codes, dict_len, threads):
    c = _c(codes, np.uint32)
    out = np.zeros(max(1, dict_len), np.uint8)
    lib().ref_present_codes(_p(c), len(c), dict_len, threads, _p(out))
    return out[:dict_len]


def ref_topk(values, k, desc):
    v = np.ascontiguousarray(values)
    dtype = 2 if v.dtype.kind == "f" else 1
    out = np.zeros(max(1, k), np.uint32)
    m = lib().ref_topk(dtype, _p(v), len(v), k, int(desc), _p(out))
    return out[:m]


def ref_sort(values, desc, threads, nulls_last=None, validity=None) -> np.ndarray:
    """The reference-shaped parallel full sort (ref_sort): row numbers in order."""
    v = np.ascontiguousarray(values)
    dtype = 2 if v.dtype.kind == "f" else 1
    v = v.astype(np.float64 if dtype == 2 else np.int64, copy=False)
    if nulls_last is None:
        nulls_last = desc
    out = np.zeros(max(1, len(v)), dtype=np.uint32)
    lib().ref_sort(dtype, _p(v), _p(_c(validity, np.uint64)), len(v), int(desc), int(nulls_last), int(threads),
                   _p(out))
    return out[:len(v)]


def ref_filter_group_codes(codes, score, salary, dict_len, op, lit, threads):
    c, s, sa = _c(codes, np.uint32), _c(score, np.float64), _c(salary, np.int64)
    rows, fs, is_ = np.zeros(dict_len, np.int64), np.zeros(dict_len), np.zeros(dict_len)
    lib().ref_filter_group_codes(_p(c), _p(s), _p(sa), len(c), dict_len, op, float(lit), threads, _p(rows), _p(fs),
                                 _p(is_))
    return rows, fs, is_


def ref_join_agg(bkeys, bpay, pkeys, pval, join_type, threads):
    bk, bp, pk = _c(bkeys, np.int64), _c(bpay, np.int64), _c(pkeys, np.int64)
    pv = _c(pval, np.float64)
    o = [np.zeros(1, np.int64), np.zeros(1, np.int64), np.zeros(1, np.float64)]
    lib().ref_join_agg(_p(bk), _p(bp), len(bk), _p(pk), _p(pv), len(pk), join_type, threads, *[_p(x) for x in o])
    return int(o[0][0]), int(o[1][0]), float(o[2][0])


def ref_group_i64(keys, vals, threads):
    k, v = _c(keys, np.int64), _c(vals, np.float64)
    return int(lib().ref_group_i64(_p(k), _p(v), len(k), threads))


# ---------------------------------------------------------------------------- reference MIN/MAX rules
# Python restatements (small inputs only) of how the reference's own code
# treats NaN and +-inf in MIN / MAX.  Its results depend on how the table is
# cut into batches, so they take the batch size (65,536 rows in the
# reference's tables).  The engine does not reproduce them; the tests use
# these to record, case by case, where its batch-independent rule differs.
REF_BATCH_ROWS = 65_536


def _batches(n, batch_rows):
    return [(s, min(n, s + batch_rows)) for s in range(0, n, batch_rows)] or [(0, 0)]


def ref_minmax_nokey(values, is_min, validity=None, batch_rows=REF_BATCH_ROWS):
    """No-key MIN / MAX (accumulate_typed, aggregate.rs:3286-3375).

    Per batch: a FLOAT64 column with no NULL in the batch folds f64::min /
    f64::max (NaN skipped) from +inf / -inf and contributes only when that
    fold is finite (3308-3320, 3351-3363), so a batch holding -inf (MIN) or
    +inf (MAX), or only NaN, contributes nothing.  Otherwise (NULLs present,
    or an integer column) the valid values are scanned with `<` / `>` from
    +inf / -inf (NaN never replaces the running value) and the batch
    contributes its running value whenever it had any valid value, +inf /
    -inf included (3322-3330, 3365-3373).  Batches combine with f64::min /
    f64::max.  Returns None for SQL NULL."""
    v = np.asarray(values)
    is_float = v.dtype.kind == "f"
    valid = (np.ones(len(v), bool) if validity is None else
             np.array([(int(validity[i >> 6]) >> (i & 63)) & 1 == 1 for i in range(len(v))], dtype=bool))
    fmin = lambda a, b: b if np.isnan(a) else (a if np.isnan(b) else min(a, b))
    fmax = lambda a, b: b if np.isnan(a) else (a if np.isnan(b) else max(a, b))
    comb = fmin if is_min else fmax
    value = None
    for s, e in _batches(len(v), batch_rows):
        if e <= s:
            continue
        if is_float and valid[s:e].all():
            chunk = float("inf") if is_min else float("-inf")
            for x in v[s:e]:
                chunk = comb(chunk, float(x))
            if np.isfinite(chunk):
                value = chunk if value is None else comb(value, chunk)
            continue
        cur = float("inf") if is_min else float("-inf")
        anyv = False
        for i in range(s, e):
            if not valid[i]:
                continue
            x = float(v[i])
            if (x < cur) if is_min else (x > cur):
                cur = x
            anyv = True
        if anyv:
            value = cur if value is None else comb(value, cur)
    return value


def ref_minmax_group(keys, values, is_min, batch_rows=REF_BATCH_ROWS):
    """GROUP BY MIN / MAX (accumulate_batch, aggregate.rs:1092-1169, merged
    by merge_state_entry, 1351-1390, in batch order).

    Within a batch a group's first value is taken as it is, NaN included,
    and a later value replaces it only when `<` (MIN) / `>` (MAX) holds, so a
    leading NaN stays.  Batch states merge the same way.  Returns
    {key: value}; NaN is a value here, not NULL."""
    k = np.asarray(keys)
    v = np.asarray(values, dtype=np.float64)
    better = (lambda a, b: a < b) if is_min else (lambda a, b: a > b)
    total = {}
    for s, e in _batches(len(k), batch_rows):
        state = {}
        for i in range(s, e):
            g, x = int(k[i]), float(v[i])
            if g not in state or better(x, state[g]):
                state[g] = x
        for g, x in state.items():
            if g not in total or better(x, total[g]):
                total[g] = x
    return total


# ---------------------------------------------------------------------------- several sort keys, whole-row DISTINCT
def _ord_u64(v: np.ndarray) -> np.ndarray:
    """f64_ord_key (sort.rs:451-454) of a float64 array, or the sign flip of
    an int64 array: unsigned keys whose order is the SQL order."""
    if v.dtype.kind == "f":
        b = np.ascontiguousarray(v, dtype=np.float64).view(np.uint64)
        return np.where(b >> np.uint64(63) == 0, b ^ np.uint64(1 << 63), ~b)
    return np.ascontiguousarray(v, dtype=np.int64).view(np.uint64) ^ np.uint64(1 << 63)


def sort_multi(keys, n: int) -> np.ndarray:
    """Rows 0..n-1 in ORDER BY order over several keys (sort_merged,
    sort.rs:118-165): key by key, each ascending or descending with its NULLs
    first or last; ties on every key keep row order.  `keys` is a list of
    dicts: values (int64 / float64 array, or a list of str for a text
    column), valid (bool array or None), desc, nulls_last.  Text compares as
    bytes (Rust str ordering)."""
    cols = []
    for k in keys:
        vals = k["values"]
        valid = np.ones(n, bool) if k.get("valid") is None else np.asarray(k["valid"], bool)
        if isinstance(vals, list):  # text: rank by byte-wise order
            enc = [("" if s is None else s).encode() for s in vals]
            order = sorted(range(n), key=lambda i: enc[i])
            rank = np.zeros(n, np.uint64)
            prev = None
            r = 0
            for j, i in enumerate(order):
                if prev is not None and enc[i] != prev:
                    r = j
                rank[i] = r
                prev = enc[i]
            key = rank
        else:
            key = _ord_u64(np.asarray(vals))
        if k["desc"]:
            key = ~key
        nul = ~valid
        flag = np.where(nul, 1 if k["nulls_last"] else 0, 0 if k["nulls_last"] else 1).astype(np.uint64)
        key = np.where(nul, np.uint64(0), key)
        cols.append((flag, key))
    # np.lexsort: the last key is primary; stable, so ties keep row order.
    seq = []
    for flag, key in reversed(cols):
        seq += [key, flag]
    return np.lexsort(seq).astype(np.uint32) if seq else np.arange(n, dtype=np.uint32)


def distinct_multi(cols, n: int) -> np.ndarray:
    """Rows (ascending) of the first occurrence of each distinct row over
    several columns (dedup_batches, select.rs:238-269): NULL is one value per
    column; float NaNs are one value and -0.0 equals +0.0 (norm_f64,
    select.rs:201-204); text compares by value.  `cols`: list of dicts with
    values (array, or list of str) and valid (bool array or None)."""
    def cell(c, i):
        valid = c.get("valid")
        if valid is not None and not valid[i]:
            return ("null",)
        v = c["values"][i]
        if isinstance(c["values"], list):
            return ("s", v)
        if np.asarray(c["values"]).dtype.kind == "f":
            x = float(v)
            if x != x:
                return ("nan",)
            return ("f", 0.0 if x == 0.0 else x)
        return ("i", int(v))

    seen = set()
    out = []
    for i in range(n):
        t = tuple(cell(c, i) for c in cols)
        if t not in seen:
            seen.add(t)
            out.append(i)
    return np.asarray(out, dtype=np.uint32)


# ---------------------------------------------------------------------------- zone maps
ZONE_BATCH_ROWS = 65_536
ZONE_VALUES, ZONE_NAN = 1, 2
ZONE_DTYPE = np.dtype([("min_i", "<i8"), ("max_i", "<i8"), ("min_f", "<f8"), ("max_f", "<f8"),
                       ("null_count", "<u8"), ("rows", "<u4"), ("flags", "<u4")])
NULL_CODE = 0xFFFFFFFF


def _valid_bits(validity, n):
    if validity is None:
        return np.ones(n, bool)
    w = np.asarray(validity, dtype=np.uint64)
    bits = np.unpackbits(w.view(np.uint8), bitorder="little")[:n]
    return bits.astype(bool)


def zone_map(values, kind: str, validity=None, batch_rows: int = ZONE_BATCH_ROWS) -> np.ndarray:
    """Per-batch bounds and NULL counts (column_stats, stats.rs:148-260, one
    entry per Table batch, table.rs:339, 373).  kind "int" (INT64, exact
    bounds), "float" (FLOAT64: bounds over the non-NaN values, as f64::min /
    max skip NaN, with ZONE_NAN when a NaN is present) or "code" (UTF8:
    smallest and largest dictionary code; NULL_CODE counts as NULL).
    ZONE_VALUES marks a batch holding a non-NULL (non-NaN) value."""
    v = np.asarray(values)
    n = len(v)
    valid = _valid_bits(validity, n)
    nb = (n + batch_rows - 1) // batch_rows
    out = np.zeros(nb, dtype=ZONE_DTYPE)
    for b in range(nb):
        s, e = b * batch_rows, min(n, (b + 1) * batch_rows)
        x, ok = v[s:e], valid[s:e].copy()
        if kind == "code":
            ok &= x != NULL_CODE
        out["rows"][b] = e - s
        out["null_count"][b] = int((~ok).sum())
        flags = 0
        if kind == "float":
            xf = x[ok].astype(np.float64)
            if np.isnan(xf).any():
                flags |= ZONE_NAN
            xf = xf[~np.isnan(xf)]
            if len(xf):
                flags |= ZONE_VALUES
                out["min_f"][b], out["max_f"][b] = xf.min(), xf.max()
        else:
            xi = x[ok].astype(np.int64)
            if len(xi):
                flags |= ZONE_VALUES
                out["min_i"][b], out["max_i"][b] = xi.min(), xi.max()
        out["flags"][b] = flags
    return out


# Term kinds and comparison operators of the engine's predicate programs.
T_CMP, T_IS_NULL, T_IS_NOT_NULL, T_CODE_SET, T_AND, T_OR = range(6)
EQ, NE, LT, LE, GT, GE = range(6)


def _cmp_rules_out(z, kind, op, lit_is_float, lit):
    """Can no row of batch z pass `col op lit` (can_skip_comparison,
    stats.rs:70-113), with the filter's own arithmetic: INT64 or a code
    against an INT64 literal compared exactly, INT64 against a FLOAT64
    literal as float(value), FLOAT64 as double.  NULL rows fail every
    comparison and NaN rows pass NE only."""
    values = bool(z["flags"] & ZONE_VALUES)
    nan = bool(z["flags"] & ZONE_NAN)
    if kind == "float" or (kind == "int" and lit_is_float):
        lit = float(lit)
        lo, hi = ((float(z["min_f"]), float(z["max_f"])) if kind == "float"
                  else (float(int(z["min_i"])), float(int(z["max_i"]))))
        if op == NE:
            if nan:
                return False
            if not values:
                return True
            if lit != lit:
                return False
            return lo == hi == lit
        if not values or lit != lit:
            return True
    else:
        if not values:
            return True
        lit = int(lit)
        lo, hi = int(z["min_i"]), int(z["max_i"])
        if op == NE:
            return lo == hi == lit
    return {EQ: lit < lo or lit > hi, LT: lo >= lit, LE: lo > lit, GT: hi <= lit, GE: hi < lit}[op]


def zone_rule_out(zones, kinds, terms) -> np.ndarray:
    """Per batch, True when the postfix program `terms` cannot pass any row
    of it (BatchStats::can_skip, stats.rs:57-68: AND rules out when either
    side does, OR when both do).  zones[c] / kinds[c]: the zone map and kind
    of the program's column c.  A term is a dict: kind, and col, op,
    lit (int or float), lit_float (bool), or set (a Python set of codes) and
    dict_len for CODE_SET.  IS NULL rules out a batch without NULLs, IS NOT
    NULL an all-NULL one."""
    nb = len(zones[0]) if zones else 0
    out = np.zeros(nb, bool)
    for b in range(nb):
        st = []
        for t in terms:
            k = t["kind"]
            if k in (T_AND, T_OR):
                a, c = st.pop(), st.pop()
                st.append((a or c) if k == T_AND else (a and c))
                continue
            z = zones[t["col"]][b]
            kind = kinds[t["col"]]
            if k == T_IS_NULL:
                st.append(int(z["null_count"]) == 0)
            elif k == T_IS_NOT_NULL:
                st.append(int(z["null_count"]) == int(z["rows"]))
            elif k == T_CODE_SET:
                if kind != "code":
                    st.append(False)
                elif not z["flags"] & ZONE_VALUES:
                    st.append(True)
                else:
                    lo, hi = max(int(z["min_i"]), 0), min(int(z["max_i"]), t["dict_len"] - 1)
                    st.append(not any(lo <= c <= hi for c in t["set"]))
            else:
                st.append(_cmp_rules_out(z, kind, t["op"], t.get("lit_float", False), t["lit"]))
        out[b] = st.pop()
    return out


def ref_can_skip_cmp(values, op, lit) -> bool:
    """The reference's own rule for one batch (column_stats + can_skip_comparison,
    stats.rs:70-113, 148-180): bounds folded in f64 (an INT64 value goes through
    `x as f64`, then back with `as i64`), NaN skipped by f64::min / max unless
    every value is NaN, and `!=` ruled out when min == max == literal with no
    NULL.  Small inputs only; the tests use it to record where the engine's
    exact rule differs."""
    vals = [float(x) for x in values]
    if not vals:
        return False
    mn = mx = None
    for x in vals:
        mn = x if mn is None else (x if mn != mn else (mn if x != x else min(mn, x)))
        mx = x if mx is None else (x if mx != mx else (mx if x != x else max(mx, x)))
    is_int = np.asarray(values).dtype.kind in "iu"
    if is_int:  # ScalarValue::Int64(Some(x as i64)), compared again as f64
        mn, mx = float(int(mn)), float(int(mx))
    lit = float(lit)
    if op == GT:
        return mx <= lit
    if op == GE:
        return mx < lit
    if op == LT:
        return mn >= lit
    if op == LE:
        return mn > lit
    if op == EQ:
        return lit < mn or lit > mx
    return mn == mx == lit
