"""Serving loop over device-resident tables (fdb_server_* / fdb_serve_trace).

Queries come from four templates over rows [0, nrows) of resident columns
(see include/falcondb_b200.h, "Serving loop"): COUNT WHERE c0 > x; GROUP BY a
dictionary column with COUNT, SUM(c0), SUM(c2) WHERE c0 > x; an INNER join
probe against a resident build table WHERE c1 < x/100 with COUNT and
SUM(payload); and ORDER BY c0 DESC LIMIT k WHERE c0 < x.  The native scheduler
admits queries under a device-memory budget, batches what has been admitted
whenever a launch slot frees up, and replays one CUDA graph per batch.
``max_batch=1, slots=1`` is one-query-at-a-time GPU execution.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import (SERVE_COUNT, SERVE_GROUP, SERVE_JOIN, SERVE_TOPK, Database, check, fdb_serve_config,
               fdb_serve_query, fdb_serve_result, fdb_serve_stats, lib)

__all__ = ["Query", "ServeStats", "Server", "serve_trace", "count_query", "group_query", "join_query",
           "topk_query", "SERVE_COUNT", "SERVE_GROUP", "SERVE_JOIN", "SERVE_TOPK"]


@dataclass
class Query:
    kind: int
    nrows: int
    threshold: float
    c0: int
    c1: int = 0
    c2: int = 0
    dict_len: int = 0
    table: int = 0
    k: int = 0
    arrival_s: float = 0.0

    def raw(self) -> fdb_serve_query:
        q = fdb_serve_query()
        q.kind, q.k, q.nrows, q.threshold = self.kind, self.k, self.nrows, self.threshold
        q.c0, q.c1, q.c2 = self.c0 or None, self.c1 or None, self.c2 or None
        q.dict_len, q.table, q.arrival_s = self.dict_len, self.table or None, self.arrival_s
        return q


def count_query(score_ptr: int, nrows: int, x: float, **kw) -> Query:
    return Query(SERVE_COUNT, nrows, x, score_ptr, **kw)


def group_query(score_ptr: int, codes_ptr: int, salary_ptr: int, dict_len: int, nrows: int, x: float, **kw) -> Query:
    return Query(SERVE_GROUP, nrows, x, score_ptr, codes_ptr, salary_ptr, dict_len=dict_len, **kw)


def join_query(key_ptr: int, value_ptr: int, table_handle: int, nrows: int, x: float, **kw) -> Query:
    return Query(SERVE_JOIN, nrows, x, key_ptr, value_ptr, table=table_handle, **kw)


def topk_query(score_ptr: int, nrows: int, x: float, k: int = 10, **kw) -> Query:
    return Query(SERVE_TOPK, nrows, x, score_ptr, k=k, **kw)


@dataclass
class ServeStats:
    wall_s: float
    qps: float
    p50_ms: float
    p99_ms: float
    max_ms: float
    mean_batch: float
    batches: int
    peak_reserved: int
    resident_bytes: int


def _stats(s: fdb_serve_stats) -> ServeStats:
    return ServeStats(s.wall_s, s.qps, s.p50_ms, s.p99_ms, s.max_ms, s.mean_batch, s.batches, s.peak_reserved,
                      s.resident_bytes)


def _config(max_batch: int, slots: int, mem_budget: int) -> fdb_serve_config:
    c = fdb_serve_config()
    c.max_batch, c.slots, c.mem_budget = max_batch, slots, mem_budget
    return c


class Server:
    """An online serving loop: submit() returns a ticket, wait() its result."""

    def __init__(self, db: Database, max_batch: int = 128, slots: int = 4, mem_budget: int = 0):
        self.db = db
        h = C.c_void_p()
        cfg = _config(max_batch, slots, mem_budget)
        check(lib().fdb_server_start(db.handle, C.byref(cfg), C.byref(h)))
        self._h = h

    def submit(self, q: Query) -> int:
        t = C.c_uint64()
        raw = q.raw()
        check(lib().fdb_server_submit(self._h, C.byref(raw), C.byref(t)))
        return int(t.value)

    def wait(self, ticket: int, timeout_s: Optional[float] = None) -> fdb_serve_result:
        r = fdb_serve_result()
        ns = -1 if timeout_s is None else int(timeout_s * 1e9)
        check(lib().fdb_server_wait(self._h, ticket, ns, C.byref(r)))
        return r

    def stop(self) -> ServeStats:
        st = fdb_serve_stats()
        h, self._h = self._h, None
        check(lib().fdb_server_stop(h, C.byref(st)))
        return _stats(st)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().fdb_server_stop(self._h, None)
            except Exception:
                pass


def serve_trace(db: Database, queries: Sequence[Query], max_batch: int = 128, slots: int = 4,
                mem_budget: int = 0) -> Tuple[List[fdb_serve_result], ServeStats]:
    """Submit each query at its arrival_s (seconds from the start) and collect
    every result; returns (results in query order, stats)."""
    n = len(queries)
    arr = (fdb_serve_query * max(1, n))()
    for i, q in enumerate(queries):
        arr[i] = q.raw()
    out = (fdb_serve_result * max(1, n))()
    st = fdb_serve_stats()
    cfg = _config(max_batch, slots, mem_budget)
    check(lib().fdb_serve_trace(db.handle, arr, n, C.byref(cfg), out, C.byref(st)))
    return [out[i] for i in range(n)], _stats(st)
