"""falcondb_b200 — B200 execution engine for FalconDB's relational hot path.

Python host mirror of FalconDB's entry points over the C ABI in
``include/falcondb_b200.h`` (loaded with ctypes from the in-tree
``libfalcondb_b200.so``):

* :class:`Database` — ``Database::sql`` (src/db.rs:242) and the C FFI
  (src/api/c_ffi.rs:27-144): tables are copied into HBM once and stay resident;
  :meth:`Database.sql` returns a :class:`Result`.
* :mod:`falcondb_b200.ops` — the operator layer (device pointers, the context's
  stream), one call per CPU operator routine the reference planner calls.
* :mod:`falcondb_b200.operators` — the push-based ``Operator`` / ``Pipeline``
  interface of src/query/pipeline.rs:44-178 with GPU operators behind it.

There is no CPU fallback: importing the package fails if the library is missing,
and opening a database fails without a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Any, Dict, List, Optional, Sequence, Tuple, Union

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfalcondb_b200.so"

INT64, FLOAT64, UTF8 = 1, 2, 3
EQ, NE, LT, LE, GT, GE = range(6)
AGG_COUNT_STAR, AGG_COUNT, AGG_SUM, AGG_AVG, AGG_MIN, AGG_MAX, AGG_COUNT_DISTINCT = range(7)
JOIN_INNER, JOIN_LEFT, JOIN_SEMI, JOIN_ANTI = range(4)
TERM_CMP, TERM_IS_NULL, TERM_IS_NOT_NULL, TERM_CODE_SET, TERM_AND, TERM_OR = range(6)
NO_ROW = 0xFFFFFFFF
MAX_TERMS = 16

ERRORS = {
    -1: "FDB_E_GENERIC", -2: "FDB_E_ARG", -3: "FDB_E_CUDA", -4: "FDB_E_OOM", -5: "FDB_E_SQL",
    -6: "FDB_E_NOTFOUND", -7: "FDB_E_TYPE", -8: "FDB_E_TIMEOUT", -9: "FDB_E_CAPACITY",
}


class FalconError(RuntimeError):
    """An engine error: ``code`` is the negative FDB_E_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


# ----------------------------------------------------------------------------- ABI structs
class fdb_column(C.Structure):
    _fields_ = [("name", C.c_char_p), ("dtype", C.c_int32), ("values", C.c_void_p),
                ("validity", C.c_void_p), ("dict", C.POINTER(C.c_char_p)), ("dict_len", C.c_uint32)]


class fdb_dev_column(C.Structure):
    _fields_ = [("dtype", C.c_int32), ("_pad", C.c_int32), ("values", C.c_void_p),
                ("validity", C.c_void_p), ("validity_offset", C.c_uint64)]


class fdb_pred_term(C.Structure):
    _fields_ = [("kind", C.c_int32), ("col", C.c_int32), ("op", C.c_int32), ("lit_type", C.c_int32),
                ("lit_i", C.c_int64), ("lit_f", C.c_double), ("code_set", C.c_void_p)]


class fdb_agg_spec(C.Structure):
    _fields_ = [("func", C.c_int32), ("col", C.c_int32)]


class fdb_agg_value(C.Structure):
    _fields_ = [("f", C.c_double), ("i", C.c_int64), ("n", C.c_int64), ("is_int", C.c_int32),
                ("valid", C.c_int32)]


class fdb_join_agg(C.Structure):
    _fields_ = [("count", C.c_int64), ("sum_payload", C.c_int64), ("sum_value", C.c_double),
                ("payload_rows", C.c_int64)]


class fdb_group_i64(C.Structure):
    _fields_ = [("key", C.c_int64), ("count", C.c_int64), ("sum", C.c_double), ("min", C.c_double),
                ("max", C.c_double)]


class fdb_gb_query(C.Structure):
    _fields_ = [("key", fdb_dev_column), ("value", fdb_dev_column), ("nrows", C.c_uint64),
                ("expected_groups", C.c_uint64), ("d_groups", C.c_void_p), ("capacity", C.c_uint64),
                ("d_ngroups", C.c_void_p)]


class fdb_batch_tuning(C.Structure):
    _fields_ = [("load_factor", C.c_double), ("ctas_per_sm", C.c_int32), ("tile_rows", C.c_int32)]


class fdb_serve_query(C.Structure):
    _fields_ = [("kind", C.c_int32), ("k", C.c_int32), ("nrows", C.c_uint64), ("threshold", C.c_double),
                ("c0", C.c_void_p), ("c1", C.c_void_p), ("c2", C.c_void_p), ("dict_len", C.c_uint32),
                ("_pad", C.c_uint32), ("table", C.c_void_p), ("arrival_s", C.c_double)]


SERVE_MAX_GROUPS, SERVE_MAX_K = 16, 32
SERVE_COUNT, SERVE_GROUP, SERVE_JOIN, SERVE_TOPK = range(4)


class fdb_serve_result(C.Structure):
    _fields_ = [("count", C.c_int64), ("sum_payload", C.c_int64),
                ("group_count", C.c_int64 * SERVE_MAX_GROUPS), ("group_sum0", C.c_double * SERVE_MAX_GROUPS),
                ("group_sum2", C.c_int64 * SERVE_MAX_GROUPS), ("rows", C.c_uint32 * SERVE_MAX_K),
                ("arrival_s", C.c_double), ("start_s", C.c_double), ("done_s", C.c_double),
                ("batch_size", C.c_int32), ("status", C.c_int32)]


class fdb_serve_config(C.Structure):
    _fields_ = [("max_batch", C.c_int32), ("slots", C.c_int32), ("mem_budget", C.c_uint64)]


class fdb_mem_stats(C.Structure):
    _fields_ = [("in_use", C.c_uint64), ("budget", C.c_uint64), ("scratch", C.c_uint64),
                ("pool_reserved", C.c_uint64), ("pool_used", C.c_uint64)]


class fdb_serve_stats(C.Structure):
    _fields_ = [("wall_s", C.c_double), ("qps", C.c_double), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("max_ms", C.c_double), ("mean_batch", C.c_double), ("batches", C.c_int64),
                ("peak_reserved", C.c_uint64), ("resident_bytes", C.c_uint64)]


class fdb_zone(C.Structure):
    _fields_ = [("min_i", C.c_int64), ("max_i", C.c_int64), ("min_f", C.c_double), ("max_f", C.c_double),
                ("null_count", C.c_uint64), ("rows", C.c_uint32), ("flags", C.c_uint32)]


class fdb_op_tuning(C.Structure):
    _fields_ = [("ctas_per_sm", C.c_int32), ("_pad", C.c_int32), ("min_rows_per_cta", C.c_uint64)]


TUNE_SCAN, TUNE_GROUP, TUNE_GROUP_I64, TUNE_PROBE, TUNE_TOPK = range(5)
TUNE_KINDS = ("scan", "group", "group_i64", "probe", "topk")
ZONE_BATCH_ROWS = 65536
ZONE_VALUES, ZONE_NAN = 1, 2
ZONE_DTYPE = np.dtype([("min_i", "<i8"), ("max_i", "<i8"), ("min_f", "<f8"), ("max_f", "<f8"),
                       ("null_count", "<u8"), ("rows", "<u4"), ("flags", "<u4")])
AGG_VALUE_DTYPE = np.dtype([("f", "<f8"), ("i", "<i8"), ("n", "<i8"), ("is_int", "<i4"), ("valid", "<i4")])
JOIN_AGG_DTYPE = np.dtype([("count", "<i8"), ("sum_payload", "<i8"), ("sum_value", "<f8"),
                           ("payload_rows", "<i8")])
GROUP_I64_DTYPE = np.dtype([("key", "<i8"), ("count", "<i8"), ("sum", "<f8"), ("min", "<f8"), ("max", "<f8")])

# ----------------------------------------------------------------------------- library
_lib: Optional[C.CDLL] = None

_SIGS = {
    "fdb_version": (C.c_char_p, []),
    "fdb_last_error": (C.c_char_p, []),
    "fdb_open": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "fdb_close": (None, [C.c_void_p]),
    "fdb_table_from_columns": (C.c_int64, [C.c_void_p, C.c_char_p, C.POINTER(fdb_column), C.c_int32, C.c_uint64]),
    "fdb_table_row_count": (C.c_uint64, [C.c_void_p, C.c_char_p]),
    "fdb_table_drop": (C.c_int, [C.c_void_p, C.c_char_p]),
    "fdb_table_column": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.POINTER(fdb_dev_column),
                                   C.POINTER(C.c_uint64)]),
    "fdb_sql": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "fdb_result_row_count": (C.c_uint64, [C.c_void_p]),
    "fdb_result_num_columns": (C.c_int32, [C.c_void_p]),
    "fdb_result_column_name": (C.c_char_p, [C.c_void_p, C.c_int32]),
    "fdb_result_column_dtype": (C.c_int32, [C.c_void_p, C.c_int32]),
    "fdb_result_column_values": (C.c_void_p, [C.c_void_p, C.c_int32]),
    "fdb_result_column_nulls": (C.c_void_p, [C.c_void_p, C.c_int32]),
    "fdb_result_display": (C.c_char_p, [C.c_void_p]),
    "fdb_result_free": (None, [C.c_void_p]),
    "fdb_last_kernel_ms": (C.c_double, [C.c_void_p]),
    "fdb_last_scan_rows": (C.c_uint64, [C.c_void_p]),
    "fdb_table_zone_map": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64,
                                     C.POINTER(C.c_uint64)]),
    "fdb_zone_skip": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int32, C.POINTER(fdb_pred_term),
                                C.c_int32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "fdb_set_option": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int64]),
    "fdb_get_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(fdb_op_tuning)]),
    "fdb_set_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(fdb_op_tuning)]),
    "fdb_autotune_ops": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(fdb_op_tuning),
                                   C.POINTER(C.c_double)]),
    "fdb_tuning_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "fdb_tuning_load": (C.c_int, [C.c_void_p, C.c_char_p]),
    "fdb_memory_stats": (C.c_int, [C.c_void_p, C.POINTER(fdb_mem_stats)]),
    "fdb_stream": (C.c_void_p, [C.c_void_p]),
    "fdb_synchronize": (C.c_int, [C.c_void_p]),
    "fdb_filter_mask": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_int32, C.c_uint64,
                                  C.POINTER(fdb_pred_term), C.c_int32, C.c_void_p]),
    "fdb_filter_count": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_int32, C.c_uint64,
                                   C.POINTER(fdb_pred_term), C.c_int32, C.c_void_p]),
    "fdb_compact_mask": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p]),
    "fdb_gather": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_void_p, C.c_uint64, C.c_void_p,
                             C.c_void_p]),
    "fdb_aggregate": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_int32, C.c_uint64,
                                C.POINTER(fdb_pred_term), C.c_int32, C.POINTER(fdb_agg_spec), C.c_int32,
                                C.c_void_p]),
    "fdb_aggregate_noalloc": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_int32, C.c_uint64,
                                        C.POINTER(fdb_pred_term), C.c_int32, C.POINTER(fdb_agg_spec), C.c_int32,
                                        C.c_void_p]),
    "fdb_test_stall": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32]),
    "fdb_dict_remap": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                 C.c_uint64, C.c_void_p]),
    "fdb_distinct_codes": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_int32, C.c_uint64,
                                     C.POINTER(fdb_pred_term), C.c_int32, C.c_int32, C.c_uint32, C.c_void_p]),
    "fdb_group_by_codes": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_int32, C.c_uint64,
                                     C.POINTER(fdb_pred_term), C.c_int32, C.c_int32, C.c_uint32,
                                     C.POINTER(fdb_agg_spec), C.c_int32, C.c_void_p, C.c_void_p]),
    "fdb_group_by_i64": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.POINTER(fdb_dev_column), C.c_uint64,
                                   C.POINTER(fdb_pred_term), C.c_int32, C.POINTER(fdb_dev_column), C.c_int32,
                                   C.c_uint64, C.c_double, C.c_void_p, C.c_uint64, C.c_void_p]),
    "fdb_join_build": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.POINTER(fdb_dev_column), C.c_uint64,
                                 C.c_double, C.POINTER(C.c_void_p)]),
    "fdb_join_free": (None, [C.c_void_p]),
    "fdb_join_capacity": (C.c_uint64, [C.c_void_p]),
    "fdb_join_dense": (C.c_int, [C.c_void_p]),
    "fdb_join_probe_agg": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(fdb_dev_column), C.POINTER(fdb_dev_column),
                                     C.c_uint64, C.c_int32, C.c_void_p]),
    "fdb_join_probe_pairs": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(fdb_dev_column), C.c_uint64, C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "fdb_topk": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_uint64, C.c_uint32, C.c_int32, C.c_int32,
                           C.c_void_p, C.c_void_p]),
    "fdb_sort": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_uint64, C.c_int32, C.c_int32, C.c_void_p]),
    "fdb_distinct": (C.c_int, [C.c_void_p, C.POINTER(fdb_dev_column), C.c_uint64, C.c_void_p, C.c_void_p]),
    "fdb_gb_batch_prepare": (C.c_int, [C.c_void_p, C.POINTER(fdb_gb_query), C.c_int32, C.POINTER(fdb_batch_tuning),
                                       C.POINTER(C.c_void_p)]),
    "fdb_gb_batch_run": (C.c_int, [C.c_void_p]),
    "fdb_gb_batch_free": (None, [C.c_void_p]),
    "fdb_gb_batch_autotune": (C.c_int, [C.c_void_p, C.POINTER(fdb_gb_query), C.c_int32, C.c_int32,
                                        C.POINTER(fdb_batch_tuning), C.POINTER(C.c_double)]),
    "fdb_server_start": (C.c_int, [C.c_void_p, C.POINTER(fdb_serve_config), C.POINTER(C.c_void_p)]),
    "fdb_server_submit": (C.c_int, [C.c_void_p, C.POINTER(fdb_serve_query), C.POINTER(C.c_uint64)]),
    "fdb_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int64, C.POINTER(fdb_serve_result)]),
    "fdb_server_stop": (C.c_int, [C.c_void_p, C.POINTER(fdb_serve_stats)]),
    "fdb_serve_trace": (C.c_int, [C.c_void_p, C.POINTER(fdb_serve_query), C.c_int32, C.POINTER(fdb_serve_config),
                                  C.POINTER(fdb_serve_result), C.POINTER(fdb_serve_stats)]),
}

EXPORTED = tuple(_SIGS)


def lib() -> C.CDLL:
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m falcondb_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> int:
    if rc < 0:
        raise FalconError(rc, (lib().fdb_last_error() or b"").decode())
    return rc


def version() -> str:
    return lib().fdb_version().decode()


# ----------------------------------------------------------------------------- host columns
class Utf8:
    """A dictionary-encoded text column: uint32 codes into ``dictionary``;
    code 0xFFFFFFFF is NULL (src/storage/column.rs:1257-1277)."""

    def __init__(self, codes: np.ndarray, dictionary: Sequence[str]):
        self.codes = np.ascontiguousarray(codes, dtype=np.uint32)
        self.dictionary = [str(s) for s in dictionary]

    @staticmethod
    def from_strings(values: Sequence[Optional[str]]) -> "Utf8":
        """Encode strings with a dictionary in first-appearance order
        (column.rs:1320-1346); None becomes the NULL code."""
        d: Dict[str, int] = {}
        codes = np.empty(len(values), dtype=np.uint32)
        for i, v in enumerate(values):
            if v is None:
                codes[i] = 0xFFFFFFFF
            else:
                codes[i] = d.setdefault(v, len(d))
        return Utf8(codes, list(d))

    def __len__(self) -> int:
        return len(self.codes)


def validity_words(valid: np.ndarray) -> np.ndarray:
    """Pack a bool array (True = valid) into LSB-first uint64 words."""
    valid = np.asarray(valid, dtype=bool)
    n = len(valid)
    padded = np.zeros(((n + 63) // 64) * 64, dtype=bool)
    padded[:n] = valid
    return np.packbits(padded.reshape(-1, 8), axis=1, bitorder="little").reshape(-1).view(np.uint64).copy()


class DeviceUtf8(Utf8):
    """A text column whose codes are already on the device (a CUDA tensor of
    int32 holding uint32 codes, e.g. from fdb_dict_remap); create_table copies
    them device to device."""

    def __init__(self, codes, dictionary: Sequence[str]):
        self.codes = codes
        self.dictionary = [str(s) for s in dictionary]


ColumnLike = Union[np.ndarray, Utf8, "np.ma.MaskedArray"]


# ----------------------------------------------------------------------------- results
class Result:
    """A host-side query result (mirror of QueryResult, src/db.rs:25-27)."""

    def __init__(self, handle: int, kernel_ms: float):
        L = lib()
        self.kernel_ms = kernel_ms
        self.columns: List[str] = []
        self.dtypes: List[int] = []
        self.data: Dict[str, Any] = {}
        self.nulls: Dict[str, np.ndarray] = {}
        n = L.fdb_result_row_count(handle)
        self.rows = int(n)
        for j in range(L.fdb_result_num_columns(handle)):
            name = L.fdb_result_column_name(handle, j).decode()
            dt = L.fdb_result_column_dtype(handle, j)
            ptr = L.fdb_result_column_values(handle, j)
            nptr = L.fdb_result_column_nulls(handle, j)
            nulls = (np.ctypeslib.as_array(C.cast(nptr, C.POINTER(C.c_uint8)), (n,)).astype(bool).copy()
                     if nptr and n else np.zeros(n, dtype=bool))
            if dt == INT64:
                vals = (np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int64)), (n,)).copy() if n
                        else np.zeros(0, np.int64))
            elif dt == FLOAT64:
                vals = (np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), (n,)).copy() if n
                        else np.zeros(0, np.float64))
            else:
                arr = C.cast(ptr, C.POINTER(C.c_char_p))
                vals = [None if nulls[i] else arr[i].decode() for i in range(n)]
            key = name
            k = 1
            while key in self.data:
                key = f"{name}_{k}"
                k += 1
            self.columns.append(key)
            self.dtypes.append(dt)
            self.data[key] = vals
            self.nulls[key] = nulls
        # The display table is formatted on first use (QueryResult::display,
        # db.rs:63-64), from the copied columns.
        self._display: Optional[str] = None

    @property
    def display(self) -> str:
        if self._display is None:
            self._display = self._format()
        return self._display

    def _format(self) -> str:
        """The result as the engine's text table (fdb_result_display's layout)."""
        cells = [[("NULL" if self.nulls[k][r] else _fmt(self.value(r, k), dt)) for k, dt in
                  zip(self.columns, self.dtypes)] for r in range(self.rows)]
        w = [max([len(k)] + [len(row[j]) for row in cells]) for j, k in enumerate(self.columns)]
        line = "".join("+" + "-" * (x + 2) for x in w) + "+\n"
        out = [line, "".join(f"| {k}{' ' * (w[j] - len(k) + 1)}" for j, k in enumerate(self.columns)) + "|\n", line]
        for row in cells:
            out.append("".join(f"| {c}{' ' * (w[j] - len(c) + 1)}" for j, c in enumerate(row)) + "|\n")
        out.append(line)
        out.append(f"{self.rows} row{'' if self.rows == 1 else 's'}\n")
        return "".join(out)

    def row_count(self) -> int:
        return self.rows

    def column(self, i: Union[int, str]):
        key = self.columns[i] if isinstance(i, int) else i
        return self.data[key]

    def value(self, row: int, col: Union[int, str]):
        key = self.columns[col] if isinstance(col, int) else col
        if self.nulls[key][row]:
            return None
        v = self.data[key][row]
        return v.item() if hasattr(v, "item") else v

    def to_rows(self) -> List[List[str]]:
        """Rows as display strings, the shape the reference's tests compare."""
        out = []
        for r in range(self.rows):
            row = []
            for key, dt in zip(self.columns, self.dtypes):
                v = self.value(r, key)
                row.append("NULL" if v is None else _fmt(v, dt))
            out.append(row)
        return out

    def __repr__(self) -> str:
        return self.display


def _fmt(v, dt) -> str:
    """A cell as display text: NaN, inf and -inf as Rust prints them, whole
    floats without a fraction, others in the shortest form that reads back."""
    if dt == FLOAT64:
        f = float(v)
        if f != f:
            return "NaN"
        if f in (float("inf"), float("-inf")):
            return "inf" if f > 0 else "-inf"
        if f == int(f) and abs(f) < 1e15:
            return str(int(f))
        return repr(f)
    return str(v)


# ----------------------------------------------------------------------------- database
class DevColumn:
    """Device view of a resident column (pointers are owned by the Database)."""

    def __init__(self, raw: fdb_dev_column, nrows: int):
        self.raw = raw
        self.nrows = nrows

    @property
    def dtype(self) -> int:
        return self.raw.dtype

    @property
    def ptr(self) -> int:
        return self.raw.values

    @property
    def validity(self) -> int:
        return self.raw.validity or 0


class Database:
    """A GPU context with resident tables.

    ``mem_budget`` caps the device memory this context may hold (0 = 90 % of
    what is free when it opens).
    """

    def __init__(self, device: int = 0, mem_budget: int = 0):
        h = C.c_void_p()
        check(lib().fdb_open(device, mem_budget, C.byref(h)))
        self._h = h
        self.device = device
        self._keep: Dict[str, Any] = {}
        self._schemas: Dict[str, List[Tuple[str, int, bool]]] = {}
        self.generation = 0  # bumped by every table create / drop (catalog caches check it)

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise FalconError(-2, "database is closed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib().fdb_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "Database":
        return self

    def __exit__(self, *a) -> None:
        self.close()

    # -- tables -----------------------------------------------------------------------
    def create_table(self, name: str, columns: Dict[str, ColumnLike], nrows: Optional[int] = None) -> int:
        """Create (or replace) table ``name`` from host columns: numpy int64 /
        float64 arrays, :class:`Utf8`, or masked arrays (mask = NULL).  Arrays
        in pinned memory upload asynchronously and must stay unchanged until
        :meth:`synchronize` or a query on the table."""
        cols = (fdb_column * max(1, len(columns)))()
        keep: List[Any] = []
        n = nrows
        for j, (cname, col) in enumerate(columns.items()):
            validity = None
            if isinstance(col, Utf8):
                values = col.codes
                dtype = UTF8
                enc = [s.encode() for s in col.dictionary]
                darr = (C.c_char_p * max(1, len(enc)))(*enc)
                keep += [enc, darr]
                cols[j].dict = C.cast(darr, C.POINTER(C.c_char_p))
                cols[j].dict_len = len(enc)
            else:
                if isinstance(col, np.ma.MaskedArray):
                    validity = validity_words(~np.ma.getmaskarray(col))
                    col = np.ma.getdata(col)
                arr = np.asarray(col)
                if arr.dtype.kind == "f":
                    values, dtype = np.ascontiguousarray(arr, dtype=np.float64), FLOAT64
                elif arr.dtype.kind in "iub":
                    values, dtype = np.ascontiguousarray(arr, dtype=np.int64), INT64
                else:
                    raise FalconError(-7, f"column {cname}: unsupported dtype {arr.dtype}")
            if n is None:
                n = len(values)
            elif len(values) != n:
                raise FalconError(-2, f"column {cname} has {len(values)} rows, expected {n}")
            keep += [values, validity]
            cols[j].name = cname.encode()
            cols[j].dtype = dtype
            if hasattr(values, "data_ptr"):  # device codes (DeviceUtf8)
                cols[j].values = values.data_ptr() if len(values) else None
            else:
                cols[j].values = values.ctypes.data if len(values) else None
            cols[j].validity = validity.ctypes.data if validity is not None else None
        rc = lib().fdb_table_from_columns(self.handle, name.encode(), cols, len(columns), n or 0)
        check(rc)
        # Keep host buffers referenced until the upload is known complete.
        self._keep[name] = keep
        self.generation += 1
        self._schemas[name] = [(cname, UTF8 if isinstance(col, Utf8) else
                                (FLOAT64 if np.asarray(np.ma.getdata(col)).dtype.kind == "f" else INT64),
                                isinstance(col, np.ma.MaskedArray)) for cname, col in columns.items()]
        self._dicts = getattr(self, "_dicts", {})
        for cname, col in columns.items():
            if isinstance(col, Utf8):
                self._dicts[(name, cname)] = list(col.dictionary)
        return int(rc)

    def dictionary(self, table: str, column: str) -> List[str]:
        """The dictionary of a Utf8 column created through :meth:`create_table`."""
        try:
            return self._dicts[(table, column)]
        except (AttributeError, KeyError):
            raise FalconError(-6, f"no dictionary for {table}.{column}") from None

    def create_table_from_pointers(self, name: str, specs: List[Tuple[str, int, int]], nrows: int) -> int:
        """Create a table from raw host pointers: ``specs`` = [(name, dtype, ptr)]
        (dtype INT64 / FLOAT64; UTF8 needs :meth:`create_table`)."""
        self.generation += 1
        cols = (fdb_column * max(1, len(specs)))()
        for j, (cname, dtype, ptr) in enumerate(specs):
            cols[j].name = cname.encode()
            cols[j].dtype = dtype
            cols[j].values = ptr
            cols[j].validity = None
        return int(check(lib().fdb_table_from_columns(self.handle, name.encode(), cols, len(specs), nrows)))

    def table_row_count(self, name: str) -> int:
        return int(lib().fdb_table_row_count(self.handle, name.encode()))

    def drop_table(self, name: str) -> None:
        check(lib().fdb_table_drop(self.handle, name.encode()))
        self.generation += 1
        self._keep.pop(name, None)
        self._schemas.pop(name, None)

    def tables(self) -> List[str]:
        """Names of the tables created through :meth:`create_table`, sorted."""
        return sorted(self._schemas)

    def table_info(self, name: str) -> Optional[Dict[str, Any]]:
        """Name, row count and columns (name, type, nullable) of a table created
        through :meth:`create_table` (Database::table_info, db.rs:2727-2741);
        None if there is no such table."""
        cols = self._schemas.get(name)
        if cols is None:
            return None
        tname = {INT64: "Int64", FLOAT64: "Float64", UTF8: "Utf8"}
        return {"name": name, "row_count": self.table_row_count(name), "col_count": len(cols),
                "columns": [{"name": c, "data_type": tname[d], "nullable": nl} for c, d, nl in cols]}

    def column(self, table: str, column: str) -> DevColumn:
        raw = fdb_dev_column()
        n = C.c_uint64()
        check(lib().fdb_table_column(self.handle, table.encode(), column.encode(), C.byref(raw), C.byref(n)))
        return DevColumn(raw, int(n.value))

    # -- queries ----------------------------------------------------------------------
    def sql(self, text: str) -> Result:
        """Run one query (Database::sql, src/db.rs:242)."""
        h = C.c_void_p()
        check(lib().fdb_sql(self.handle, text.encode(), C.byref(h)))
        try:
            return Result(h.value, lib().fdb_last_kernel_ms(self.handle))
        finally:
            lib().fdb_result_free(h)

    @property
    def stream(self) -> int:
        return int(lib().fdb_stream(self.handle) or 0)

    def memory_stats(self) -> Dict[str, int]:
        """Device memory the context holds (fdb_memory_stats)."""
        st = fdb_mem_stats()
        check(lib().fdb_memory_stats(self.handle, C.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in fdb_mem_stats._fields_}

    def synchronize(self) -> None:
        check(lib().fdb_synchronize(self.handle))

    # -- zone maps ----------------------------------------------------------------------
    def zone_map(self, table: str, column: str) -> np.ndarray:
        """The column's zone map: one ZONE_DTYPE record per 65,536-row batch
        (BatchStats, src/storage/stats.rs:22-52), computed when the table was
        loaded."""
        nb = C.c_uint64()
        check(lib().fdb_table_zone_map(self.handle, table.encode(), column.encode(), None, 0, C.byref(nb)))
        out = np.zeros(int(nb.value), dtype=ZONE_DTYPE)
        if len(out):
            check(lib().fdb_table_zone_map(self.handle, table.encode(), column.encode(), out.ctypes.data,
                                           len(out), C.byref(nb)))
        return out

    def zone_skip(self, table: str, columns: Sequence[str], terms: Sequence["fdb_pred_term"]) -> np.ndarray:
        """Per batch of `table`, True when the zone maps prove that no row
        passes the WHERE program `terms` over `columns` (can_skip,
        src/storage/stats.rs:57-113)."""
        names = (C.c_char_p * max(1, len(columns)))(*[c.encode() for c in columns])
        prog = (fdb_pred_term * max(1, len(terms)))(*terms)
        nrows = self.table_row_count(table)
        nb = (nrows + ZONE_BATCH_ROWS - 1) // ZONE_BATCH_ROWS
        words = np.zeros(max(1, (nb + 63) // 64), dtype=np.uint64)
        got = C.c_uint64()
        check(lib().fdb_zone_skip(self.handle, table.encode(), names, len(columns), prog, len(terms),
                                  words.ctypes.data, len(words), C.byref(got)))
        bits = np.unpackbits(words.view(np.uint8), bitorder="little")[:int(got.value)]
        return bits.astype(bool)

    # -- launch tuning (tuning.rs:39-53's cut-offs, tuned on the device) ---------------
    def tuning(self) -> Dict[str, Dict[str, int]]:
        """Launch tuning of each kind of streamed operator: CTAs per SM
        (0 = occupancy limit) and rows per CTA (0 = no minimum)."""
        out = {}
        for k, name in enumerate(TUNE_KINDS):
            t = fdb_op_tuning()
            check(lib().fdb_get_tuning(self.handle, k, C.byref(t)))
            out[name] = {"ctas_per_sm": int(t.ctas_per_sm), "min_rows_per_cta": int(t.min_rows_per_cta)}
        return out

    def set_tuning(self, kind: Union[int, str], ctas_per_sm: int = 0, min_rows_per_cta: int = 0) -> None:
        k = TUNE_KINDS.index(kind) if isinstance(kind, str) else int(kind)
        t = fdb_op_tuning(ctas_per_sm, 0, min_rows_per_cta)
        check(lib().fdb_set_tuning(self.handle, k, C.byref(t)))

    def autotune(self, rows: int = 1 << 24, reps: int = 5) -> Tuple[Dict[str, Dict[str, int]], Dict[str, float]]:
        """Time launch-shape candidates for every kind of streamed operator on
        `rows` synthetic rows (fdb_autotune_ops) and keep the fastest.
        Returns (choices, ms per call at `rows`)."""
        best = (fdb_op_tuning * len(TUNE_KINDS))()
        ms = (C.c_double * len(TUNE_KINDS))()
        check(lib().fdb_autotune_ops(self.handle, rows, reps, best, ms))
        return ({n: {"ctas_per_sm": int(best[k].ctas_per_sm), "min_rows_per_cta": int(best[k].min_rows_per_cta)}
                 for k, n in enumerate(TUNE_KINDS)}, {n: float(ms[k]) for k, n in enumerate(TUNE_KINDS)})

    def save_tuning(self, path: str) -> None:
        """Write the tuning cache (JSON) for this device."""
        check(lib().fdb_tuning_save(self.handle, str(path).encode()))

    def load_tuning(self, path: str) -> None:
        """Apply a tuning cache written on the same kind of device."""
        check(lib().fdb_tuning_load(self.handle, str(path).encode()))

    def set_option(self, name: str, value: int) -> None:
        """Context option (fdb_set_option): "zone_maps" 1 / 0."""
        check(lib().fdb_set_option(self.handle, name.encode(), int(value)))

    @property
    def last_scan_rows(self) -> int:
        """Rows of its table that the last single-table :meth:`sql` scanned
        after zone-map pruning."""
        return int(lib().fdb_last_scan_rows(self.handle))


__all__ = [
    "Database", "Result", "Utf8", "DeviceUtf8", "DevColumn", "FalconError", "lib", "check", "version", "validity_words",
    "INT64", "FLOAT64", "UTF8", "EQ", "NE", "LT", "LE", "GT", "GE", "AGG_COUNT_STAR", "AGG_COUNT", "AGG_SUM",
    "AGG_AVG", "AGG_MIN", "AGG_MAX", "AGG_COUNT_DISTINCT", "JOIN_INNER", "JOIN_LEFT", "JOIN_SEMI", "JOIN_ANTI",
    "NO_ROW", "EXPORTED", "ZONE_DTYPE", "ZONE_BATCH_ROWS", "ZONE_VALUES", "ZONE_NAN", "TUNE_KINDS",
]
