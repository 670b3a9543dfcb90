"""Operator layer: one call per CPU physical-operator routine of the reference.

Every function takes device columns (:class:`~falcondb_b200.DevColumn` from a
resident table, or torch CUDA tensors) and returns device tensors; the work is
queued on the context's CUDA stream and nothing synchronises unless a result is
read.  Torch is used only to hold device memory.

=========================  ===================================================
function                   reference routine (FalconTechDev/falcondb, src/)
=========================  ===================================================
``filter_mask``            Expr::eval_mask_bits / fast_cmp_mask, query/expr.rs:635-1175
``filter_count``           COUNT(*)+WHERE popcount, db.rs:1439-1476
``compact``                gather_by_bitmask row walk, storage/column.rs:1077-1123
``gather``                 Column::gather_u32, storage/column.rs:1502-1520
``aggregate``              execute_agg_only, query/aggregate.rs:1394-1528
``distinct_codes``         present_codes (COUNT DISTINCT), query/aggregate.rs:3167-3200
``group_by_codes``         GroupByExec fast_utf8_gb, query/aggregate.rs:619-836
``group_by_i64``           GroupByExec fast_i64_gb, query/aggregate.rs:840-912
``join_build``             build_hash_table / IntHashTable, query/join.rs:607-645, 1054-1351
``join_probe_agg``         probe_in_place + agg; execute_hash_semi_anti_join, join.rs:49-132, 297-375
``join_probe_pairs``       probe_one / build_output, query/join.rs:657-723, 901-975
``topk``                   execute_sort_limit / top_k_ascending, query/sort.rs:59-115, 564-620
=========================  ===================================================
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import (AGG_VALUE_DTYPE, FLOAT64, GROUP_I64_DTYPE, INT64, JOIN_AGG_DTYPE, MAX_TERMS, TERM_AND,
               TERM_CMP, TERM_CODE_SET, TERM_IS_NOT_NULL, TERM_IS_NULL, TERM_OR, UTF8, Database, DevColumn,
               FalconError, check, fdb_agg_spec, fdb_dev_column, fdb_pred_term, lib)

ColArg = Union[DevColumn, torch.Tensor, Tuple[torch.Tensor, Optional[torch.Tensor]]]

_DT = {torch.int64: INT64, torch.float64: FLOAT64, torch.int32: UTF8}


def dev_column(c: ColArg, dtype: Optional[int] = None) -> fdb_dev_column:
    """fdb_dev_column for a resident column or a CUDA tensor (int64 -> INT64,
    float64 -> FLOAT64, int32 codes -> UTF8), optionally (tensor, validity)."""
    if isinstance(c, DevColumn):
        return c.raw
    validity = None
    if isinstance(c, tuple):
        c, validity = c
    if not c.is_cuda:
        raise FalconError(-2, "operator inputs must be CUDA tensors")
    if not c.is_contiguous():
        raise FalconError(-2, "operator inputs must be contiguous")
    raw = fdb_dev_column()
    raw.dtype = dtype or _DT.get(c.dtype, 0)
    if raw.dtype == 0:
        raise FalconError(-7, f"unsupported tensor dtype {c.dtype}")
    raw.values = c.data_ptr()
    raw.validity = validity.data_ptr() if validity is not None else None
    raw.validity_offset = 0
    return raw


def _cols(cols: Sequence[ColArg]):
    arr = (fdb_dev_column * max(1, len(cols)))()
    for i, c in enumerate(cols):
        arr[i] = dev_column(c)
    return arr, len(cols)


# ----------------------------------------------------------------------------- predicates
def cmp(col: int, op: int, literal: Union[int, float]) -> fdb_pred_term:
    """`cols[col] op literal` (an int literal is Int64, a float Float64)."""
    t = fdb_pred_term()
    t.kind, t.col, t.op = TERM_CMP, col, op
    if isinstance(literal, (float, np.floating)):
        t.lit_type, t.lit_f = FLOAT64, float(literal)
    else:
        t.lit_type, t.lit_i = INT64, int(literal)
    return t


def is_null(col: int) -> fdb_pred_term:
    t = fdb_pred_term()
    t.kind, t.col = TERM_IS_NULL, col
    return t


def is_not_null(col: int) -> fdb_pred_term:
    t = fdb_pred_term()
    t.kind, t.col = TERM_IS_NOT_NULL, col
    return t


def code_set(col: int, passing: Sequence[bool], device: torch.device) -> Tuple[fdb_pred_term, torch.Tensor]:
    """Utf8 test decided per dictionary entry: rows whose code's entry passes.
    Returns the term and the device bitmap (keep it alive while used)."""
    words = max(1, (len(passing) + 63) // 64)
    bits = np.zeros(words, dtype=np.uint64)
    for i, p in enumerate(passing):
        if p:
            bits[i >> 6] |= np.uint64(1) << np.uint64(i & 63)
    dev = torch.from_numpy(bits.view(np.int64)).to(device)
    t = fdb_pred_term()
    t.kind, t.col, t.lit_i, t.code_set = TERM_CODE_SET, col, len(passing), dev.data_ptr()
    return t, dev


def AND() -> fdb_pred_term:
    t = fdb_pred_term()
    t.kind = TERM_AND
    return t


def OR() -> fdb_pred_term:
    t = fdb_pred_term()
    t.kind = TERM_OR
    return t


def _prog(prog: Sequence[fdb_pred_term]):
    if len(prog) > MAX_TERMS:
        raise FalconError(-2, "predicate has too many terms")
    arr = (fdb_pred_term * max(1, len(prog)))()
    for i, t in enumerate(prog):
        arr[i] = t
    return arr, len(prog)


def _aggs(aggs: Sequence[Tuple[int, int]]):
    arr = (fdb_agg_spec * max(1, len(aggs)))()
    for i, (f, c) in enumerate(aggs):
        arr[i].func, arr[i].col = f, c
    return arr, len(aggs)


def _dev(db: Database) -> torch.device:
    return torch.device("cuda", db.device)


_streams = {}


def lib_stream(db: Database) -> torch.cuda.ExternalStream:
    """The context's CUDA stream as a torch stream (for events and ordering)."""
    key = (id(db), db.stream)
    s = _streams.get(key)
    if s is None:
        s = torch.cuda.ExternalStream(db.stream, device=_dev(db))
        _streams[key] = s
    return s


class _Fenced:
    """Order an operator call after torch's current stream, and torch's current
    stream after the call, so tensors shared with torch are never raced."""

    def __init__(self, db: Database):
        self.db = db

    def __enter__(self):
        lib_stream(self.db).wait_stream(torch.cuda.current_stream(_dev(self.db)))

    def __exit__(self, *exc):
        torch.cuda.current_stream(_dev(self.db)).wait_stream(lib_stream(self.db))
        return False


def _bytes(n: int, db: Database) -> torch.Tensor:
    return torch.empty(max(1, n), dtype=torch.uint8, device=_dev(db))


def to_records(t: torch.Tensor, dtype: np.dtype, n: Optional[int] = None) -> np.ndarray:
    """Copy a device byte buffer of packed structs to a numpy record array."""
    raw = t.detach().cpu().numpy().tobytes()
    rec = np.frombuffer(raw, dtype=dtype)
    return rec[:n] if n is not None else rec


# ----------------------------------------------------------------------------- operators
def filter_mask(db: Database, cols: Sequence[ColArg], nrows: int, prog: Sequence[fdb_pred_term]) -> torch.Tensor:
    """WHERE mask as int64 words (bit i of word i//64 = row i passes)."""
    c, nc = _cols(cols)
    p, npr = _prog(prog)
    out = torch.empty(max(1, (nrows + 63) // 64), dtype=torch.int64, device=_dev(db))
    with _Fenced(db):
        check(lib().fdb_filter_mask(db.handle, c, nc, nrows, p, npr, out.data_ptr()))
    return out


def filter_count(db: Database, cols: Sequence[ColArg], nrows: int, prog: Sequence[fdb_pred_term],
                 out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """COUNT(*) WHERE prog, as a 1-element int64 device tensor."""
    c, nc = _cols(cols)
    p, npr = _prog(prog)
    out = out if out is not None else torch.empty(1, dtype=torch.int64, device=_dev(db))
    with _Fenced(db):
        check(lib().fdb_filter_count(db.handle, c, nc, nrows, p, npr, out.data_ptr()))
    return out


def compact(db: Database, mask: torch.Tensor, nrows: int, capacity: Optional[int] = None
            ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Row numbers (int32 tensor holding uint32) of the set mask bits, and the count."""
    capacity = nrows if capacity is None else capacity
    rows = torch.empty(max(1, capacity), dtype=torch.int32, device=_dev(db))
    cnt = torch.empty(1, dtype=torch.int64, device=_dev(db))
    with _Fenced(db):
        check(lib().fdb_compact_mask(db.handle, mask.data_ptr(), nrows, rows.data_ptr(), capacity, cnt.data_ptr()))
    return rows, cnt


def gather(db: Database, col: ColArg, rows: torch.Tensor, n: int) -> Tuple[torch.Tensor, Optional[torch.Tensor]]:
    raw = dev_column(col)
    tdt = torch.int32 if raw.dtype == UTF8 else (torch.float64 if raw.dtype == FLOAT64 else torch.int64)
    out = torch.empty(max(1, n), dtype=tdt, device=_dev(db))
    valid = torch.empty(max(1, (n + 63) // 64), dtype=torch.int64, device=_dev(db)) if raw.validity else None
    with _Fenced(db):
        check(lib().fdb_gather(db.handle, C.byref(raw), rows.data_ptr(), n, out.data_ptr(),
                           valid.data_ptr() if valid is not None else None))
    return out, valid


def aggregate(db: Database, cols: Sequence[ColArg], nrows: int, prog: Sequence[fdb_pred_term],
              aggs: Sequence[Tuple[int, int]], out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """No-key aggregates; a device byte buffer of fdb_agg_value (see to_records)."""
    c, nc = _cols(cols)
    p, npr = _prog(prog)
    a, na = _aggs(aggs)
    out = out if out is not None else _bytes(AGG_VALUE_DTYPE.itemsize * na, db)
    with _Fenced(db):
        check(lib().fdb_aggregate(db.handle, c, nc, nrows, p, npr, a, na, out.data_ptr()))
    return out


def distinct_codes(db: Database, cols: Sequence[ColArg], nrows: int, prog: Sequence[fdb_pred_term],
                   code_col: int, dict_len: int, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    c, nc = _cols(cols)
    p, npr = _prog(prog)
    out = out if out is not None else torch.empty(max(1, (dict_len + 63) // 64), dtype=torch.int64,
                                                  device=_dev(db))
    with _Fenced(db):
        check(lib().fdb_distinct_codes(db.handle, c, nc, nrows, p, npr, code_col, dict_len, out.data_ptr()))
    return out


def group_by_codes(db: Database, cols: Sequence[ColArg], nrows: int, prog: Sequence[fdb_pred_term], key_col: int,
                   dict_len: int, aggs: Sequence[Tuple[int, int]]) -> Tuple[torch.Tensor, torch.Tensor]:
    """Per-group aggregates ((dict_len+1) x naggs fdb_agg_value) and row counts."""
    c, nc = _cols(cols)
    p, npr = _prog(prog)
    a, na = _aggs(aggs)
    out = _bytes(AGG_VALUE_DTYPE.itemsize * (dict_len + 1) * na, db)
    rows = torch.empty(dict_len + 1, dtype=torch.int64, device=_dev(db))
    with _Fenced(db):
        check(lib().fdb_group_by_codes(db.handle, c, nc, nrows, p, npr, key_col, dict_len, a, na, out.data_ptr(),
                                   rows.data_ptr()))
    return out, rows


def group_by_i64(db: Database, key: ColArg, value: ColArg, nrows: int, prog: Sequence[fdb_pred_term] = (),
                 pred_cols: Sequence[ColArg] = (), expected_groups: int = 0, load_factor: float = 0.0,
                 capacity: Optional[int] = None, out: Optional[torch.Tensor] = None,
                 ngroups: Optional[torch.Tensor] = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Hash GROUP BY: (device byte buffer of fdb_group_i64, group count)."""
    capacity = (nrows + 1) if capacity is None else capacity
    k, v = dev_column(key), dev_column(value)
    pc, npc = _cols(pred_cols) if pred_cols else ((fdb_dev_column * 1)(), 0)
    p, npr = _prog(prog)
    out = out if out is not None else _bytes(GROUP_I64_DTYPE.itemsize * capacity, db)
    ngroups = ngroups if ngroups is not None else torch.empty(1, dtype=torch.int64, device=_dev(db))
    with _Fenced(db):
        check(lib().fdb_group_by_i64(db.handle, C.byref(k), C.byref(v), nrows, p, npr, pc, npc, expected_groups,
                                 load_factor, out.data_ptr(), capacity, ngroups.data_ptr()))
    return out, ngroups


class HashTable:
    """A resident join build side (keeps the payload column referenced)."""

    def __init__(self, db: Database, key: ColArg, payload: Optional[ColArg], nrows: int, load_factor: float = 0.0):
        self.db = db
        self._keep = (key, payload)
        k = dev_column(key)
        pp = C.byref(dev_column(payload)) if payload is not None else None
        h = C.c_void_p()
        with _Fenced(db):
            check(lib().fdb_join_build(db.handle, C.byref(k), pp, nrows, load_factor, C.byref(h)))
        self._h = h

    @property
    def capacity(self) -> int:
        return int(lib().fdb_join_capacity(self._h))

    @property
    def dense(self) -> bool:
        """True when the table is direct-addressed (build keys span fewer
        values than it has slots); False when keys are hashed."""
        return bool(lib().fdb_join_dense(self._h))

    def free(self) -> None:
        if self._h is not None and self._h.value:
            lib().fdb_join_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def probe_agg(self, key: ColArg, nrows: int, join_type: int, value: Optional[ColArg] = None,
                  out: Optional[torch.Tensor] = None) -> torch.Tensor:
        k = dev_column(key)
        vp = C.byref(dev_column(value)) if value is not None else None
        out = out if out is not None else _bytes(JOIN_AGG_DTYPE.itemsize, self.db)
        with _Fenced(self.db):
            check(lib().fdb_join_probe_agg(self.db.handle, self._h, C.byref(k), vp, nrows, join_type,
                                           out.data_ptr()))
        return out

    def probe_pairs(self, key: ColArg, nrows: int, join_type: int, capacity: int
                    ) -> Tuple[torch.Tensor, Optional[torch.Tensor], torch.Tensor]:
        k = dev_column(key)
        dev = _dev(self.db)
        left = torch.empty(max(1, capacity), dtype=torch.int32, device=dev)
        right = torch.empty(max(1, capacity), dtype=torch.int32, device=dev) if join_type <= 1 else None
        cnt = torch.empty(1, dtype=torch.int64, device=dev)
        with _Fenced(self.db):
            check(lib().fdb_join_probe_pairs(self.db.handle, self._h, C.byref(k), nrows, join_type,
                                             left.data_ptr(), right.data_ptr() if right is not None else None,
                                             capacity, cnt.data_ptr()))
        return left, right, cnt


def topk(db: Database, col: ColArg, nrows: int, k: int, desc: bool, nulls_last: Optional[bool] = None,
         rows: Optional[torch.Tensor] = None, count: Optional[torch.Tensor] = None
         ) -> Tuple[torch.Tensor, torch.Tensor]:
    """ORDER BY col [DESC] LIMIT k: row numbers in order (int32 holding uint32)
    and their count.  NULLs default to last for DESC, first for ASC."""
    if nulls_last is None:
        nulls_last = desc
    raw = dev_column(col)
    dev = _dev(db)
    rows = rows if rows is not None else torch.empty(max(1, k), dtype=torch.int32, device=dev)
    count = count if count is not None else torch.empty(1, dtype=torch.int64, device=dev)
    with _Fenced(db):
        check(lib().fdb_topk(db.handle, C.byref(raw), nrows, k, int(desc), int(nulls_last), rows.data_ptr(),
                         count.data_ptr()))
    return rows, count


def sort(db: Database, col: ColArg, nrows: int, desc: bool, nulls_last: Optional[bool] = None,
         rows: Optional[torch.Tensor] = None) -> torch.Tensor:
    """ORDER BY col [DESC] without LIMIT: all nrows row numbers in order
    (int32 holding uint32).  NULLs default to last for DESC, first for ASC."""
    if nulls_last is None:
        nulls_last = desc
    raw = dev_column(col)
    rows = rows if rows is not None else torch.empty(max(1, nrows), dtype=torch.int32, device=_dev(db))
    with _Fenced(db):
        check(lib().fdb_sort(db.handle, C.byref(raw), nrows, int(desc), int(nulls_last), rows.data_ptr()))
    return rows


def distinct(db: Database, col: ColArg, nrows: int, rows: Optional[torch.Tensor] = None,
             count: Optional[torch.Tensor] = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """SELECT DISTINCT col: row numbers of each value's first occurrence, in row
    order (int32 holding uint32), and their count."""
    raw = dev_column(col)
    dev = _dev(db)
    rows = rows if rows is not None else torch.empty(max(1, nrows), dtype=torch.int32, device=dev)
    count = count if count is not None else torch.empty(1, dtype=torch.int64, device=dev)
    with _Fenced(db):
        check(lib().fdb_distinct(db.handle, C.byref(raw), nrows, rows.data_ptr(), count.data_ptr()))
    return rows, count


class GroupByBatch:
    """Many int64-key GROUP BY queries (COUNT(*), SUM, MIN, MAX of a value
    column) captured as one CUDA graph: fdb_gb_batch_prepare / _run / _free.
    ``queries`` = [(key, value, nrows)] with key / value column arguments (a
    slice of a table is a tensor view); outputs are allocated here, one
    (groups, count) pair per query, ``capacity`` groups each (default nrows)."""

    def __init__(self, db: Database, queries: Sequence[Tuple[ColArg, ColArg, int]],
                 tuning: Optional[Tuple[float, int, int]] = None, expected_groups: Optional[Sequence[int]] = None,
                 capacity: Optional[Sequence[int]] = None):
        from . import fdb_batch_tuning, fdb_gb_query
        self.db = db
        nq = len(queries)
        arr = (fdb_gb_query * max(1, nq))()
        dev = _dev(db)
        self.outs: List[Tuple[torch.Tensor, torch.Tensor]] = []
        self._keep = list(queries)
        for i, (k, v, n) in enumerate(queries):
            cap = int(capacity[i]) if capacity is not None else max(1, int(n) + 1)
            groups = _bytes(GROUP_I64_DTYPE.itemsize * cap, db)
            count = torch.zeros(1, dtype=torch.int64, device=dev)
            self.outs.append((groups, count))
            arr[i].key = dev_column(k)
            arr[i].value = dev_column(v)
            arr[i].nrows = int(n)
            arr[i].expected_groups = int(expected_groups[i]) if expected_groups is not None else 0
            arr[i].d_groups = groups.data_ptr()
            arr[i].capacity = cap
            arr[i].d_ngroups = count.data_ptr()
        self._arr, self._nq = arr, nq
        # No tuning: the context's (the last autotune's, or a loaded cache's).
        t = fdb_batch_tuning(*tuning) if tuning else None
        h = C.c_void_p()
        with _Fenced(db):
            check(lib().fdb_gb_batch_prepare(db.handle, arr, nq, C.byref(t) if t is not None else None, C.byref(h)))
        self._h = h

    def run(self) -> None:
        """Replay the batch on the context stream (asynchronous)."""
        with _Fenced(self.db):
            check(lib().fdb_gb_batch_run(self._h))

    def results(self, i: int) -> np.ndarray:
        """Query i's groups as a record array (GROUP_I64_DTYPE), unordered."""
        groups, count = self.outs[i]
        return to_records(groups, GROUP_I64_DTYPE, int(count.item()))

    def free(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().fdb_gb_batch_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @staticmethod
    def autotune(db: Database, queries: Sequence[Tuple[ColArg, ColArg, int]], reps: int = 3,
                 expected_groups: Optional[Sequence[int]] = None) -> Tuple[Tuple[float, int, int], float]:
        """The fastest (load_factor, ctas_per_sm, tile_rows) for these queries and its ms per run."""
        from . import fdb_batch_tuning, fdb_gb_query
        nq = len(queries)
        arr = (fdb_gb_query * max(1, nq))()
        dev = _dev(db)
        keep = []
        for i, (k, v, n) in enumerate(queries):
            groups = _bytes(GROUP_I64_DTYPE.itemsize * (int(n) + 1), db)
            count = torch.zeros(1, dtype=torch.int64, device=dev)
            keep += [groups, count]
            arr[i].key = dev_column(k)
            arr[i].value = dev_column(v)
            arr[i].nrows = int(n)
            arr[i].expected_groups = int(expected_groups[i]) if expected_groups is not None else 0
            arr[i].d_groups = groups.data_ptr()
            arr[i].capacity = int(n) + 1
            arr[i].d_ngroups = count.data_ptr()
        best = fdb_batch_tuning()
        ms = C.c_double()
        with _Fenced(db):
            check(lib().fdb_gb_batch_autotune(db.handle, arr, nq, reps, C.byref(best), C.byref(ms)))
        return (best.load_factor, best.ctas_per_sm, best.tile_rows), ms.value


def synchronize(db: Database) -> None:
    db.synchronize()
