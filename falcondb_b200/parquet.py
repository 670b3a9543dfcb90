"""Parquet -> HBM loader (read_parquet / read_parquet_projected,
src/storage/parquet_io.rs:290-500, with the type mapping of
arrow_array_to_falcon, 118-231).

The file is decoded on the host by pyarrow's multi-threaded reader, every
column is converted to the engine's layout, and the table is uploaded once
with ``Database.create_table``.  Text columns get ONE dictionary for the whole
file, in first-appearance order.  The reference builds a dictionary per
65,536-row batch (column.rs:1320-1346) and its Utf8 GROUP BY reads batch 0's
dictionary for every batch (aggregate.rs:655-658), which mislabels groups when
batches disagree.  A global dictionary cannot.

Type mapping (the engine holds INT64, FLOAT64 and UTF8 columns):

* Int8/16/32/64, UInt8/16/64 -> INT64.  UInt32 wraps to i32 first, as the
  reference's ``a.value(i) as i32`` does (parquet_io.rs:166-167).
* Float64 -> FLOAT64.  Float32 -> FLOAT64, widened exactly (the reference keeps
  an f32 column).
* Utf8 / LargeUtf8 -> UTF8 codes over the global dictionary.
* Date32 -> INT64 days.  Timestamp[us] -> INT64 microseconds; other units are
  rejected, as the reference's TimestampMicrosecondArray downcast does.
* Boolean -> INT64 0 / 1 (the engine has no boolean column).
* Null -> INT64, every row NULL.
* Decimal128 and anything else -> FDB_E_TYPE.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple, Union

import numpy as np

from . import Database, FalconError, Utf8

__all__ = ["read_parquet_columns", "load_parquet"]

ColumnLike = Union[np.ndarray, np.ma.MaskedArray, Utf8]


def _pa():
    try:
        import pyarrow as pa
        import pyarrow.compute as pc
        import pyarrow.parquet as pq
    except ImportError as e:  # pragma: no cover - pyarrow ships with the image
        raise FalconError(-1, f"pyarrow is needed to read Parquet: {e}") from None
    return pa, pc, pq


def _with_nulls(values: np.ndarray, valid: Optional[np.ndarray]) -> ColumnLike:
    if valid is None or valid.all():
        return values
    return np.ma.masked_array(values, mask=~valid)


def _valid(arr) -> Optional[np.ndarray]:
    if arr.null_count == 0:
        return None
    return np.asarray(arr.is_valid().to_numpy(zero_copy_only=False), dtype=bool)


def _convert(name: str, arr) -> ColumnLike:
    """One column (a pyarrow ChunkedArray) in the engine's layout."""
    pa, pc, _ = _pa()
    t = arr.type
    n = len(arr)
    valid = _valid(arr)
    if pa.types.is_null(t):
        return np.ma.masked_array(np.zeros(n, dtype=np.int64), mask=np.ones(n, dtype=bool))
    if pa.types.is_boolean(t):
        v = np.asarray(arr.fill_null(False).to_numpy(zero_copy_only=False), dtype=np.int64)
        return _with_nulls(v, valid)
    if pa.types.is_integer(t):
        v = np.asarray(arr.fill_null(0).to_numpy(zero_copy_only=False))
        if t == pa.uint32():
            v = v.astype(np.uint32).view(np.int32)
        return _with_nulls(v.astype(np.int64), valid)
    if pa.types.is_floating(t):
        if pa.types.is_float16(t):
            raise FalconError(-7, f"column {name}: float16 is not supported")
        v = np.asarray(arr.fill_null(0).to_numpy(zero_copy_only=False)).astype(np.float64)
        return _with_nulls(v, valid)
    if pa.types.is_date32(t):
        v = np.asarray(arr.cast(pa.int32()).fill_null(0).to_numpy(zero_copy_only=False)).astype(np.int64)
        return _with_nulls(v, valid)
    if pa.types.is_timestamp(t):
        if t.unit != "us":
            raise FalconError(-7, f"column {name}: timestamp[{t.unit}] (only microseconds are read)")
        v = np.asarray(arr.cast(pa.int64()).fill_null(0).to_numpy(zero_copy_only=False))
        return _with_nulls(v, valid)
    if pa.types.is_dictionary(t) and (pa.types.is_string(t.value_type) or pa.types.is_large_string(t.value_type)):
        # Text read as per-row-group dictionaries: merge them into one, then
        # renumber it in order of first appearance in the file (so the codes
        # do not depend on how a writer ordered its dictionary pages).  NULL
        # rows take the engine's NULL code.
        if n == 0:
            return Utf8(np.zeros(0, dtype=np.uint32), [])
        arr = arr.unify_dictionaries()
        dictionary = arr.chunk(0).dictionary
        idx = np.concatenate([np.asarray(ch.indices.fill_null(-1).to_numpy(zero_copy_only=False), dtype=np.int64)
                              for ch in arr.chunks])
        present = idx >= 0
        if not present.any():
            return Utf8(np.full(n, 0xFFFFFFFF, dtype=np.uint32), [])
        order = np.asarray(pc.unique(pa.array(idx[present])).to_numpy(zero_copy_only=False), dtype=np.int64)
        lut = np.zeros(len(dictionary), dtype=np.int64)
        lut[order] = np.arange(len(order))
        codes = np.where(present, lut[np.where(present, idx, 0)], 0xFFFFFFFF).astype(np.uint32)
        words = dictionary.to_pylist()
        return Utf8(codes, [str(words[o]) for o in order])
    if pa.types.is_string(t) or pa.types.is_large_string(t):
        return _convert(name, arr.dictionary_encode())
    raise FalconError(-7, f"column {name}: Parquet type {t} is not supported")


def read_parquet_columns(path: str, columns: Optional[Sequence[str]] = None
                         ) -> Tuple[Dict[str, ColumnLike], int]:
    """The columns of a Parquet file (all, or `columns` in that order) in the
    engine's layout, and the row count."""
    pa, _, pq = _pa()
    try:
        schema = pq.read_schema(path)
        want = list(columns) if columns is not None else list(schema.names)
        text = [f.name for f in schema if f.name in want and (pa.types.is_string(f.type) or
                                                               pa.types.is_large_string(f.type))]
        # Text columns come back dictionary-encoded: no string per row is built.
        table = pq.read_table(path, columns=want, use_threads=True, read_dictionary=text)
    except (OSError, ValueError, KeyError) as e:
        raise FalconError(-1, f"cannot read {path}: {e}") from None
    out: Dict[str, ColumnLike] = {}
    for name in table.column_names:
        out[name] = _convert(name, table.column(name))
    return out, table.num_rows


def load_parquet(db: Database, path: str, table: str, columns: Optional[Sequence[str]] = None) -> int:
    """Read a Parquet file into device table `table` (created or replaced);
    returns the row count."""
    cols, n = read_parquet_columns(path, columns)
    if not cols:
        raise FalconError(-2, f"{path}: no columns to load")
    db.create_table(table, cols, nrows=n)
    return n
