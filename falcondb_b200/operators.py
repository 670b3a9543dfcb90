"""Push-based physical operators over device-resident columns.

Mirror of FalconDB's operator contract (src/query/pipeline.rs:44-178 and
src/query/operators.rs:28-224): an :class:`Operator` takes one chunk at a time
and answers :class:`OpResult` ``Emit(batch)`` / ``Empty`` / ``Done``; blocking
operators answer in :meth:`Operator.flush`; a :class:`Pipeline` pushes chunks
through a chain, stops reading once a stage says ``Done`` (LIMIT), and flushes
the stages in order so a blocking stage's output still travels the rest of the
chain.  A GPU operator is therefore a drop-in for the matching CPU plan node.

What differs is the chunk: the reference cuts batches into 2048-row chunks that
fit a CPU core's L1.  Here a chunk is a *view* of device columns (no copy) of
up to :data:`CHUNK_ROWS` rows, enough to give every SM of a B200 many tiles;
each stage is one or a few kernel launches on the context's stream.

Every compute step calls the engine's kernels through the C ABI
(:mod:`falcondb_b200.ops`); there is no host fallback.  Host synchronisation
happens only where a row count must reach the host to size an output (a
filtered chunk, a group count).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Dict, Iterable, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import (AGG_AVG, AGG_COUNT, AGG_COUNT_STAR, AGG_MAX, AGG_MIN, AGG_SUM, AGG_VALUE_DTYPE, EQ, FLOAT64, GE, GT,
               GROUP_I64_DTYPE, INT64, JOIN_AGG_DTYPE, JOIN_ANTI, JOIN_SEMI, LE, LT, NE, TERM_AND, TERM_OR, UTF8,
               Database, DevColumn, FalconError, fdb_dev_column, fdb_pred_term)
from . import ops

#: Rows per chunk: 8M rows of an 8-byte column is 64 MB, several tiles for
#: each of the 148 SMs and well past the point where launch cost matters.
CHUNK_ROWS = 1 << 23

_ESIZE = {INT64: 8, FLOAT64: 8, UTF8: 4}
_TORCH = {INT64: torch.int64, FLOAT64: torch.float64, UTF8: torch.int32}


# ----------------------------------------------------------------------------- data
@dataclass
class Column:
    """A device column view: element address, type, validity words (LSB-first
    bit per row, or 0) and the bit offset of row 0 in them.  ``keep`` holds the
    tensors or table the memory belongs to; ``dictionary`` the strings of a
    Utf8 column's codes."""

    dtype: int
    values: int
    nrows: int
    validity: int = 0
    voff: int = 0
    dictionary: Optional[List[str]] = None
    keep: Any = None

    def raw(self) -> fdb_dev_column:
        r = fdb_dev_column()
        r.dtype = self.dtype
        r.values = self.values if self.nrows else None
        r.validity = self.validity or None
        r.validity_offset = self.voff
        return r

    def slice(self, start: int, n: int) -> "Column":
        """Rows [start, start+n) as a view (shifts the address and the validity bit offset)."""
        if start < 0 or n < 0 or start + n > self.nrows:
            raise FalconError(-2, f"slice [{start}, {start + n}) outside {self.nrows} rows")
        return Column(self.dtype, self.values + start * _ESIZE[self.dtype], n, self.validity,
                      self.voff + start if self.validity else 0, self.dictionary, self.keep)

    def to_numpy(self) -> np.ndarray:
        """Values as a host array (NULLs left as stored: see :meth:`valid_numpy`)."""
        if self.nrows == 0:
            return np.zeros(0, dtype={INT64: np.int64, FLOAT64: np.float64, UTF8: np.uint32}[self.dtype])
        t = _view(self.values, self.nrows, self.dtype)
        a = t.cpu().numpy()
        return a.view(np.uint32) if self.dtype == UTF8 else a

    def valid_numpy(self) -> np.ndarray:
        if not self.validity:
            return np.ones(self.nrows, dtype=bool)
        w0 = self.voff // 64
        nw = (self.voff + self.nrows + 63) // 64 - w0
        words = _view(self.validity + 8 * w0, nw, INT64).cpu().numpy().view(np.uint64)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little").astype(bool)
        s = self.voff - 64 * w0
        return bits[s:s + self.nrows]


def _view(addr: int, n: int, dtype: int) -> torch.Tensor:
    """A torch tensor over existing device memory (no copy, no ownership)."""
    cls = {INT64: C.c_int64, FLOAT64: C.c_double, UTF8: C.c_int32}[dtype]

    class _Iface:
        __cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(cls).str, "data": (addr, False),
                                    "version": 2}

    return torch.as_tensor(_Iface(), device="cuda")


def tensor_column(t: torch.Tensor, validity: Optional[torch.Tensor] = None,
                  dictionary: Optional[List[str]] = None) -> Column:
    """A column over a contiguous CUDA tensor (int64, float64, or int32 Utf8 codes)."""
    if not t.is_cuda or not t.is_contiguous():
        raise FalconError(-2, "columns must be contiguous CUDA tensors")
    dt = {torch.int64: INT64, torch.float64: FLOAT64, torch.int32: UTF8}.get(t.dtype)
    if dt is None:
        raise FalconError(-7, f"unsupported tensor dtype {t.dtype}")
    return Column(dt, t.data_ptr(), t.numel(), validity.data_ptr() if validity is not None else 0, 0,
                  dictionary, (t, validity))


@dataclass
class Batch:
    """A RecordBatch of device columns sharing a row count (table.rs:46-49)."""

    columns: Dict[str, Column]
    nrows: int

    def row_count(self) -> int:
        return self.nrows

    def column(self, name: str) -> Column:
        try:
            return self.columns[name]
        except KeyError:
            raise FalconError(-6, f"unknown column {name}") from None

    @property
    def names(self) -> List[str]:
        return list(self.columns)

    def slice(self, start: int, n: int) -> "Batch":
        return Batch({k: c.slice(start, n) for k, c in self.columns.items()}, n)

    @staticmethod
    def from_table(db: Database, table: str, names: Sequence[str]) -> "Batch":
        """Views of a resident table's columns."""
        cols: Dict[str, Column] = {}
        n = db.table_row_count(table)
        for name in names:
            dc = db.column(table, name)
            r = dc.raw
            d = db.dictionary(table, name) if r.dtype == UTF8 else None
            cols[name] = Column(r.dtype, r.values or 0, dc.nrows, r.validity or 0, r.validity_offset, d,
                                (db, table))
        return Batch(cols, n)

    def to_numpy(self) -> Dict[str, np.ndarray]:
        """Host copy: numeric columns as arrays (masked where NULL), Utf8 as object arrays of strings."""
        out: Dict[str, np.ndarray] = {}
        for k, c in self.columns.items():
            v = c.to_numpy()
            ok = c.valid_numpy()
            if c.dtype == UTF8:
                d = c.dictionary or []
                s = np.array([d[x] if (x < len(d) and o) else None for x, o in zip(v.tolist(), ok.tolist())],
                             dtype=object)
                out[k] = s
            else:
                out[k] = np.ma.MaskedArray(v, mask=~ok) if c.validity else v
        return out


# ----------------------------------------------------------------------------- contract
class OpResult:
    """What an operator did with a chunk (pipeline.rs:46-58)."""

    __slots__ = ("kind", "batch")
    EMIT, EMPTY, DONE = "Emit", "Empty", "Done"

    def __init__(self, kind: str, batch: Optional[Batch] = None):
        self.kind = kind
        self.batch = batch

    @staticmethod
    def Emit(batch) -> "OpResult":
        return OpResult(OpResult.EMIT, batch)

    def __repr__(self) -> str:
        return f"OpResult.{self.kind}" + (f"({self.batch.row_count()} rows)" if self.batch is not None else "")


OpResult.Empty = OpResult(OpResult.EMPTY)
OpResult.Done = OpResult(OpResult.DONE)


class Operator:
    """One pipeline stage (pipeline.rs:60-72)."""

    def process(self, chunk) -> OpResult:
        raise NotImplementedError

    def flush(self) -> List[Any]:
        """Called once after the last chunk; blocking operators answer here."""
        return []

    def name(self) -> str:
        raise NotImplementedError


def into_chunks(batch, chunk_rows: int = CHUNK_ROWS) -> List[Any]:
    """Views of at most ``chunk_rows`` rows each (pipeline.rs:77-92)."""
    n = batch.row_count()
    if n <= chunk_rows:
        return [batch]
    return [batch.slice(s, min(chunk_rows, n - s)) for s in range(0, n, chunk_rows)]


class Pipeline:
    """A chain of operators driven by pushing chunks (pipeline.rs:95-178)."""

    def __init__(self, ops_: Sequence[Operator], chunk_rows: int = CHUNK_ROWS):
        self.ops = list(ops_)
        self.chunk_rows = chunk_rows

    def is_empty(self) -> bool:
        return not self.ops

    def stage_names(self) -> List[str]:
        return [o.name() for o in self.ops]

    def run(self, inputs: Iterable[Any]) -> List[Any]:
        out: List[Any] = []
        stop = False
        for batch in inputs:
            for chunk in into_chunks(batch, self.chunk_rows):
                if not self._push_from(0, chunk, out):
                    stop = True  # a downstream stage is satisfied (LIMIT): stop reading
                    break
            if stop:
                break
        self._flush_from(0, out)
        return out

    def _push_from(self, idx: int, chunk, out: List[Any]) -> bool:
        """Push into stage idx onward; False when a stage answered Done."""
        while True:
            if idx >= len(self.ops):
                if chunk.row_count() > 0:
                    out.append(chunk)
                return True
            r = self.ops[idx].process(chunk)
            if r.kind == OpResult.EMIT:
                chunk = r.batch
                idx += 1
                continue
            return r.kind != OpResult.DONE

    def _flush_from(self, idx: int, out: List[Any]) -> None:
        for i in range(idx, len(self.ops)):
            for batch in self.ops[i].flush():
                stopped = False
                for chunk in into_chunks(batch, self.chunk_rows):
                    if not self._push_from(i + 1, chunk, out):
                        stopped = True  # the rest of the flushed rows are not needed
                        break
                if stopped:
                    break


# ----------------------------------------------------------------------------- predicates
class Expr:
    """A WHERE expression over column names, compiled per batch to the engine's
    postfix predicate program (fdb_pred_term, at most 16 terms)."""

    def __and__(self, other: "Expr") -> "Expr":
        return _Bool(TERM_AND, self, other)

    def __or__(self, other: "Expr") -> "Expr":
        return _Bool(TERM_OR, self, other)

    def columns(self) -> List[str]:
        raise NotImplementedError

    def emit(self, batch: Batch, index: Dict[str, int], terms: List[fdb_pred_term], keep: List[Any]) -> None:
        raise NotImplementedError


class col(Expr):
    """Column reference; comparisons with a literal build leaves."""

    def __init__(self, name: str):
        self.name_ = name

    def _cmp(self, op: int, lit) -> Expr:
        return _Leaf(self.name_, "cmp", op, lit)

    def __lt__(self, v): return self._cmp(LT, v)
    def __le__(self, v): return self._cmp(LE, v)
    def __gt__(self, v): return self._cmp(GT, v)
    def __ge__(self, v): return self._cmp(GE, v)
    def __eq__(self, v): return self._cmp(EQ, v)  # noqa: E704
    def __ne__(self, v): return self._cmp(NE, v)  # noqa: E704
    __hash__ = object.__hash__

    def is_null(self) -> Expr:
        return _Leaf(self.name_, "null", 0, None)

    def is_not_null(self) -> Expr:
        return _Leaf(self.name_, "notnull", 0, None)

    def isin(self, values: Sequence[Any]) -> Expr:
        return _Leaf(self.name_, "in", 0, list(values))


class _Leaf(Expr):
    def __init__(self, name: str, kind: str, op: int, lit):
        self.name_, self.kind, self.op, self.lit = name, kind, op, lit

    def columns(self) -> List[str]:
        return [self.name_]

    def emit(self, batch, index, terms, keep):
        c = batch.column(self.name_)
        j = index[self.name_]
        if self.kind == "null":
            terms.append(ops.is_null(j))
        elif self.kind == "notnull":
            terms.append(ops.is_not_null(j))
        elif c.dtype == UTF8:
            # String predicates become a set of dictionary codes (expr.rs:1143-1171).
            d = c.dictionary or []
            if self.kind == "in":
                passing = [s in set(self.lit) for s in d]
            else:
                import operator as _o
                f = {EQ: _o.eq, NE: _o.ne, LT: _o.lt, LE: _o.le, GT: _o.gt, GE: _o.ge}[self.op]
                passing = [f(s, self.lit) for s in d]
            t, bits = ops.code_set(j, passing, torch.device("cuda", torch.cuda.current_device()))
            keep.append(bits)
            terms.append(t)
        elif self.kind == "in":
            for i, v in enumerate(self.lit):
                terms.append(ops.cmp(j, EQ, v))
                if i:
                    terms.append(ops.OR())
            if not self.lit:
                terms.append(ops.cmp(j, NE, 0))
                terms.append(ops.cmp(j, EQ, 0))
                terms.append(ops.AND())  # always false
        else:
            terms.append(ops.cmp(j, self.op, self.lit))


class _Bool(Expr):
    def __init__(self, kind: int, a: Expr, b: Expr):
        self.kind, self.a, self.b = kind, a, b

    def columns(self) -> List[str]:
        return self.a.columns() + self.b.columns()

    def emit(self, batch, index, terms, keep):
        self.a.emit(batch, index, terms, keep)
        self.b.emit(batch, index, terms, keep)
        t = fdb_pred_term()
        t.kind = self.kind
        terms.append(t)


def compile_expr(expr: Optional[Expr], batch: Batch) -> Tuple[List[Column], List[fdb_pred_term], List[Any]]:
    """(input columns, postfix program over their positions, buffers to keep alive)."""
    if expr is None:
        return [], [], []
    names: List[str] = []
    for n in expr.columns():
        if n not in names:
            names.append(n)
    if len(names) > 4:
        raise FalconError(-2, "a WHERE over more than 4 columns per scan")
    index = {n: i for i, n in enumerate(names)}
    terms: List[fdb_pred_term] = []
    keep: List[Any] = []
    expr.emit(batch, index, terms, keep)
    return [batch.column(n) for n in names], terms, keep


def _raws(cols: Sequence[Column]):
    arr = (fdb_dev_column * max(1, len(cols)))()
    for i, c in enumerate(cols):
        arr[i] = c.raw()
    return arr


# ----------------------------------------------------------------------------- operators
def _concat(db: Database, chunks: List[Batch], names: Sequence[str]) -> Batch:
    """One batch over held chunks: the chunks' own range when they are adjacent
    views of the same columns (the common case, a scan of a resident table),
    else a device copy."""
    if len(chunks) == 1:
        return chunks[0]
    n = sum(c.row_count() for c in chunks)
    out: Dict[str, Column] = {}
    for name in names:
        parts = [c.column(name) for c in chunks]
        p0 = parts[0]
        es = _ESIZE[p0.dtype]
        adjacent = all(q.values == p0.values + es * sum(x.nrows for x in parts[:i]) and q.validity == p0.validity
                       and (not q.validity or q.voff == p0.voff + sum(x.nrows for x in parts[:i]))
                       for i, q in enumerate(parts))
        if adjacent:
            out[name] = Column(p0.dtype, p0.values, n, p0.validity, p0.voff, p0.dictionary, [q.keep for q in parts])
            continue
        if any(q.validity for q in parts):
            raise FalconError(-2, f"column {name}: held chunks with NULLs must be adjacent views")
        vals = torch.cat([_view(q.values, q.nrows, q.dtype) for q in parts if q.nrows])
        out[name] = tensor_column(vals, None, p0.dictionary)
    return Batch(out, n)


class FilterOp(Operator):
    """WHERE: drops the rows that fail the predicate (operators.rs:28-46)."""

    def __init__(self, db: Database, predicate: Expr):
        self.db = db
        self.predicate = predicate

    def process(self, chunk: Batch) -> OpResult:
        n = chunk.row_count()
        cols, prog, keep = compile_expr(self.predicate, chunk)
        mask = ops.filter_mask(self.db, _as_args(cols), n, prog)
        rows, cnt = ops.compact(self.db, mask, n)
        k = int(cnt.item())
        if k == 0:
            return OpResult.Empty
        return OpResult.Emit(_gather(self.db, chunk, rows, k))

    def name(self) -> str:
        return "Filter"


def _arg(c: Column) -> DevColumn:
    """The ops-layer argument for a column view."""
    return DevColumn(c.raw(), c.nrows)


def _as_args(cols: Sequence[Column]) -> List[DevColumn]:
    return [_arg(c) for c in cols]


def _gather(db: Database, b: Batch, rows: torch.Tensor, k: int) -> Batch:
    """Rows `rows[:k]` of every column of b, as new device columns."""
    out: Dict[str, Column] = {}
    for name, c in b.columns.items():
        v, val = ops.gather(db, _arg(c), rows, k)
        out[name] = tensor_column(v[:k], val, c.dictionary)
    return Batch(out, k)


class ProjectOp(Operator):
    """SELECT list of column references, optionally renamed (operators.rs:48-66).
    Expressions other than column references are not on the GPU path."""

    def __init__(self, columns: Sequence[Union[str, Tuple[str, str]]]):
        self.columns = [(c, c) if isinstance(c, str) else (c[0], c[1]) for c in columns]

    def process(self, chunk: Batch) -> OpResult:
        return OpResult.Emit(Batch({alias: chunk.column(src) for src, alias in self.columns}, chunk.row_count()))

    def name(self) -> str:
        return "Project"


class LimitOp(Operator):
    """LIMIT / OFFSET; answers Done once the limit is met, so the source stops
    reading (operators.rs:68-120)."""

    def __init__(self, offset: int = 0, limit: Optional[int] = None):
        self.skip = offset
        self.take = limit

    def process(self, chunk) -> OpResult:
        if self.take == 0:
            return OpResult.Done
        n = chunk.row_count()
        if self.skip >= n:
            self.skip -= n
            return OpResult.Empty
        start, self.skip = self.skip, 0
        available = n - start
        take = available if self.take is None else min(self.take, available)
        if self.take is not None:
            self.take -= take
        if take == 0:
            return OpResult.Done
        return OpResult.Emit(chunk.slice(start, take))

    def name(self) -> str:
        return "Limit"


class SortOp(Operator):
    """ORDER BY one column [DESC] [LIMIT k], blocking (operators.rs:122-148):
    with LIMIT k <= 4096 the GPU top-k (execute_sort_limit's top_k path,
    sort.rs:59-115), otherwise the GPU radix sort of the FLOAT64 / INT64 key
    (sort_merged -> try_typed_sort, sort.rs:118-133, 209-350) and then the
    LIMIT.  Ties follow arrival order; several keys raise."""

    def __init__(self, db: Database, keys: Sequence[Tuple[str, bool]], limit: Optional[int],
                 nulls_last: Optional[bool] = None):
        if len(keys) != 1:
            raise FalconError(-5, "SortOp orders by one column on the GPU")
        self.db = db
        self.key, self.desc = keys[0]
        self.limit = limit
        self.nulls_last = nulls_last
        self.held: List[Batch] = []

    def process(self, chunk: Batch) -> OpResult:
        self.held.append(chunk)
        return OpResult.Empty

    def flush(self) -> List[Batch]:
        if not self.held:
            return []
        held, self.held = self.held, []
        b = _concat(self.db, held, held[0].names)
        n = b.row_count()
        if n == 0 or self.limit == 0:
            return []
        if self.limit is not None and self.limit <= 4096:
            rows, cnt = ops.topk(self.db, _arg(b.column(self.key)), n, self.limit, self.desc, self.nulls_last)
            k = int(cnt.item())
        else:
            rows = ops.sort(self.db, _arg(b.column(self.key)), n, self.desc, self.nulls_last)
            k = n if self.limit is None else min(n, self.limit)
        return [_gather(self.db, b, rows, k)] if k else []

    def name(self) -> str:
        return "Sort"


@dataclass
class AggSpec:
    """One aggregate: func (AGG_*), input column (None for COUNT(*)), output name."""

    func: int
    column: Optional[str]
    alias: str


class AggregateOp(Operator):
    """GROUP BY with aggregates, or no-key aggregates; blocking
    (operators.rs:150-180, GroupByExec::execute aggregate.rs:535).  Chunks are
    held and aggregated together at flush, as the reference does.

    * no key: fdb_aggregate (COUNT(*), COUNT, SUM, AVG, MIN, MAX);
    * a Utf8 key: the dictionary-code GROUP BY (up to 4 aggregates);
    * an Int64 key: the hash GROUP BY with one value column, whose output
      carries COUNT(*), SUM, MIN, MAX (and AVG = SUM / COUNT(value)) of it.
    Output columns: the key (if any) then one column per aggregate; COUNT is
    Int64, the rest Float64 (aggregate.rs:3390-3420)."""

    def __init__(self, db: Database, aggs: Sequence[AggSpec], group_by: Optional[str] = None,
                 where: Optional[Expr] = None, expected_groups: int = 0):
        self.db = db
        self.aggs = list(aggs)
        self.group_by = group_by
        self.where = where
        self.expected_groups = expected_groups
        self.held: List[Batch] = []
        if not 1 <= len(self.aggs) <= 4:
            raise FalconError(-2, "between 1 and 4 aggregates")

    def process(self, chunk: Batch) -> OpResult:
        self.held.append(chunk)
        return OpResult.Empty

    def _inputs(self, b: Batch) -> Tuple[List[Column], List[fdb_pred_term], List[Any], Dict[str, int]]:
        """Scan columns (the WHERE's first, in the order its program refers to
        them, then the key and aggregate inputs), the program, and the index of
        each column name in the scan."""
        pcols, prog, keep = compile_expr(self.where, b)
        index: Dict[str, int] = {}
        for n in (self.where.columns() if self.where else []):
            index.setdefault(n, len(index))
        for n in ([self.group_by] if self.group_by else []) + [a.column for a in self.aggs if a.column]:
            index.setdefault(n, len(index))
        if len(index) > 4:
            raise FalconError(-2, "at most 4 distinct columns per aggregate scan")
        return [b.column(n) for n in index], prog, keep, index

    def flush(self) -> List[Batch]:
        held, self.held = self.held, []
        if not held:
            held = []
        names = sorted({n for h in held for n in h.names})
        b = _concat(self.db, held, names) if held else None
        n = b.row_count() if b is not None else 0
        if self.group_by is None:
            return [self._no_key(b, n)]
        if b is None or n == 0:
            return []
        key = b.column(self.group_by)
        if key.dtype == UTF8:
            return [self._by_codes(b, n)]
        return [self._by_i64(b, n)]

    def _no_key(self, b: Optional[Batch], n: int) -> Batch:
        dev = torch.device("cuda", self.db.device)
        if b is None or n == 0:
            recs = np.zeros(len(self.aggs), dtype=AGG_VALUE_DTYPE)
        else:
            cols, prog, keep, index = self._inputs(b)
            specs = [(a.func, index[a.column] if a.column else 0) for a in self.aggs]
            out = ops.aggregate(self.db, _as_args(cols), n, prog, specs)
            recs = ops.to_records(out, AGG_VALUE_DTYPE, len(self.aggs))
        cols_out: Dict[str, Column] = {}
        for a, r in zip(self.aggs, recs):
            if a.func in (AGG_COUNT_STAR, AGG_COUNT):
                t = torch.tensor([int(r["i"]) if n else 0], dtype=torch.int64, device=dev)
                cols_out[a.alias] = tensor_column(t)
            else:
                valid = bool(r["valid"])
                t = torch.tensor([float(r["f"]) if valid else 0.0], dtype=torch.float64, device=dev)
                vw = torch.tensor([1 if valid else 0], dtype=torch.int64, device=dev)
                cols_out[a.alias] = tensor_column(t, vw)
        return Batch(cols_out, 1)

    def _by_codes(self, b: Batch, n: int) -> Batch:
        cols, prog, keep, index = self._inputs(b)
        key = b.column(self.group_by)
        d = key.dictionary or []
        specs = [(a.func, index[a.column] if a.column else 0) for a in self.aggs]
        out, grows = ops.group_by_codes(self.db, _as_args(cols), n, prog, index[self.group_by], len(d), specs)
        recs = ops.to_records(out, AGG_VALUE_DTYPE, (len(d) + 1) * len(self.aggs)).reshape(len(d) + 1,
                                                                                           len(self.aggs))
        rows = grows.cpu().numpy()
        present = [g for g in range(len(d) + 1) if rows[g] > 0]
        return self._emit_groups(np.array(present, dtype=np.int64), recs[present], d, codes=True)

    def _by_i64(self, b: Batch, n: int) -> Batch:
        values = {a.column for a in self.aggs if a.column}
        if len(values) > 1:
            raise FalconError(-2, "the Int64-key GROUP BY aggregates one value column")
        key = b.column(self.group_by)
        vcol = b.column(values.pop()) if values else key
        pcols, prog, keep = compile_expr(self.where, b)
        if len(pcols) > 2:
            raise FalconError(-2, "the Int64-key GROUP BY takes a WHERE over at most 2 columns")
        out, ng = ops.group_by_i64(self.db, _arg(key), _arg(vcol), n, prog=prog, pred_cols=_as_args(pcols),
                                   expected_groups=self.expected_groups)
        g = int(ng.item())
        recs = ops.to_records(out, GROUP_I64_DTYPE, g)
        recs = recs[np.argsort(recs["key"], kind="stable")]
        dev = torch.device("cuda", self.db.device)
        cols_out: Dict[str, Column] = {self.group_by: tensor_column(
            torch.from_numpy(np.ascontiguousarray(recs["key"])).to(dev))}
        for a in self.aggs:
            if a.func in (AGG_COUNT_STAR, AGG_COUNT):
                if a.func == AGG_COUNT and vcol.validity:
                    raise FalconError(-2, "COUNT(value) over a nullable value column is not in the GPU hash GROUP BY")
                v = recs["count"].astype(np.int64)
            elif a.func == AGG_SUM:
                v = recs["sum"]
            elif a.func == AGG_AVG:
                v = recs["sum"] / np.maximum(recs["count"], 1)
            elif a.func == AGG_MIN:
                v = recs["min"]
            elif a.func == AGG_MAX:
                v = recs["max"]
            else:
                raise FalconError(-2, "aggregate not supported by the Int64-key GROUP BY")
            cols_out[a.alias] = tensor_column(torch.from_numpy(np.ascontiguousarray(v)).to(dev))
        return Batch(cols_out, g)

    def _emit_groups(self, gids: np.ndarray, recs: np.ndarray, d: List[str], codes: bool) -> Batch:
        dev = torch.device("cuda", self.db.device)
        g = len(gids)
        kc = np.where(gids < len(d), gids, 0xFFFFFFFF).astype(np.uint32).view(np.int32)
        key_valid = (gids < len(d))
        words = np.zeros(max(1, (g + 63) // 64), dtype=np.uint64)
        for i in np.nonzero(key_valid)[0]:
            words[i >> 6] |= np.uint64(1) << np.uint64(i & 63)
        cols_out: Dict[str, Column] = {self.group_by: tensor_column(
            torch.from_numpy(np.ascontiguousarray(kc)).to(dev),
            torch.from_numpy(words.view(np.int64)).to(dev), d)}
        for j, a in enumerate(self.aggs):
            r = recs[:, j] if g else np.zeros(0, dtype=AGG_VALUE_DTYPE)
            if a.func in (AGG_COUNT_STAR, AGG_COUNT):
                cols_out[a.alias] = tensor_column(torch.from_numpy(r["i"].astype(np.int64)).to(dev))
            else:
                ok = r["valid"].astype(bool)
                w = np.zeros(max(1, (g + 63) // 64), dtype=np.uint64)
                for i in np.nonzero(ok)[0]:
                    w[i >> 6] |= np.uint64(1) << np.uint64(i & 63)
                cols_out[a.alias] = tensor_column(torch.from_numpy(np.ascontiguousarray(r["f"])).to(dev),
                                                  torch.from_numpy(w.view(np.int64)).to(dev))
        return Batch(cols_out, g)

    def name(self) -> str:
        return "Aggregate"


class DistinctOp(Operator):
    """SELECT DISTINCT of one column, blocking (operators.rs:182-205 ->
    dedup_batches, select.rs:238-457): each value's first row in arrival order,
    on the GPU (fdb_distinct).  FLOAT64 NaNs are one value and -0.0 == +0.0;
    all NULLs are one value."""

    def __init__(self, db: Database, column: str):
        self.db = db
        self.column = column
        self.held: List[Batch] = []

    def process(self, chunk: Batch) -> OpResult:
        self.held.append(chunk)
        return OpResult.Empty

    def flush(self) -> List[Batch]:
        held, self.held = self.held, []
        if not held:
            return []
        b = _concat(self.db, held, [self.column])
        n = b.row_count()
        if n == 0:
            return []
        rows, cnt = ops.distinct(self.db, _arg(b.column(self.column)), n)
        k = int(cnt.item())
        return [_gather(self.db, b, rows, k)] if k else []

    def name(self) -> str:
        return "Distinct"


class HashJoinProbeOp(Operator):
    """Probe side of an equi-join on one Int64 key against a resident build
    table (ops.HashTable), the join type fixed per operator.

    * ``mode="agg"`` (blocking): COUNT(*) and SUM(build payload) of the join
      (for SEMI / ANTI, SUM of the probe column ``value`` instead, as their
      output keeps probe columns only, join.rs:45-48); one row at flush;
    * ``mode="rows"`` (SEMI / ANTI, streaming): emits the kept probe rows of
      each chunk (execute_hash_semi_anti_join's keep mask, join.rs:49-132)."""

    def __init__(self, db: Database, table: "ops.HashTable", key: str, join_type: int, mode: str = "agg",
                 value: Optional[str] = None):
        if mode not in ("agg", "rows"):
            raise FalconError(-2, "mode is 'agg' or 'rows'")
        if mode == "rows" and join_type not in (JOIN_SEMI, JOIN_ANTI):
            raise FalconError(-2, "row output is for SEMI / ANTI joins")
        self.db, self.table, self.key, self.join_type, self.mode, self.value = db, table, key, join_type, mode, value
        self.acc = {"count": 0, "sum_payload": 0, "payload_rows": 0, "sum_value": 0.0}
        self.partials: List[torch.Tensor] = []

    def process(self, chunk: Batch) -> OpResult:
        n = chunk.row_count()
        k = chunk.column(self.key)
        if self.mode == "agg":
            v = _arg(chunk.column(self.value)) if self.value else None
            self.partials.append(self.table.probe_agg(_arg(k), n, self.join_type, v))
            return OpResult.Empty
        left, _, cnt = self.table.probe_pairs(_arg(k), n, self.join_type, n)
        m = int(cnt.item())
        if m == 0:
            return OpResult.Empty
        # Kept rows come back in arbitrary order; the reference keeps probe order.
        rows = torch.sort(left[:m].to(torch.int64))[0].to(torch.int32)
        return OpResult.Emit(_gather(self.db, chunk, rows, m))

    def flush(self) -> List[Batch]:
        if self.mode != "agg":
            return []
        tot = {"count": 0, "sum_payload": 0, "payload_rows": 0, "sum_value": 0.0}
        for t in self.partials:
            r = ops.to_records(t, JOIN_AGG_DTYPE, 1)[0]
            tot["count"] += int(r["count"])
            tot["sum_payload"] += int(r["sum_payload"])
            tot["payload_rows"] += int(r["payload_rows"])
            tot["sum_value"] += float(r["sum_value"])
        self.partials = []
        dev = torch.device("cuda", self.db.device)
        semi_anti = self.join_type in (JOIN_SEMI, JOIN_ANTI)
        if semi_anti:
            s = torch.tensor([tot["sum_value"]], dtype=torch.float64, device=dev)
            ok = tot["payload_rows"] > 0
        else:
            s = torch.tensor([float(tot["sum_payload"])], dtype=torch.float64, device=dev)
            ok = tot["payload_rows"] > 0
        vw = torch.tensor([1 if ok else 0], dtype=torch.int64, device=dev)
        return [Batch({"count": tensor_column(torch.tensor([tot["count"]], dtype=torch.int64, device=dev)),
                       "sum": tensor_column(s, vw)}, 1)]

    def name(self) -> str:
        return "HashJoinProbe"
