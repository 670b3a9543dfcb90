"""Parquet -> HBM loader (read_parquet / read_parquet_projected,
src/storage/parquet_io.rs:290-500, with the type mapping of
arrow_array_to_falcon, 118-231).

The file is decoded on the host by pyarrow's multi-threaded reader, every
column is converted to the engine's layout, and the table is uploaded once
with ``Database.create_table``.  Text columns get ONE dictionary for the whole
file.  The reference builds a dictionary per 65,536-row batch
(column.rs:1320-1346) and its Utf8 GROUP BY reads batch 0's dictionary for
every batch (aggregate.rs:655-658), which mislabels groups when batches
disagree.  A global dictionary cannot.

``load_parquet`` builds that dictionary on the GPU side: text columns are
read dictionary-encoded, the host merges only the row groups' dictionaries
(distinct strings; merged order: chunk by chunk, each chunk's dictionary in
its own order, which for dictionaries written in order of first appearance
is the file's first-appearance order), each row group's indices are copied
to the device unchanged, and fdb_dict_remap turns them into merged codes
there.  ``read_parquet_columns`` returns host columns instead, with the
dictionary renumbered by first appearance in the rows.

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


def _merge_chunk_dictionaries(arr):
    """The merged dictionary of a dictionary-encoded text column (strings in
    order of first appearance in the chunks' dictionaries, chunk by chunk)
    and, per chunk, the merged code of each of its dictionary entries.  Only
    the dictionaries are read here: they hold distinct strings, not rows."""
    merged: Dict[str, int] = {}
    words: List[str] = []
    remaps = []
    for ch in arr.chunks:
        d = ch.dictionary.to_pylist()
        r = np.empty(len(d), dtype=np.uint32)
        for j, w in enumerate(d):
            w = str(w)
            g = merged.get(w)
            if g is None:
                g = merged[w] = len(words)
                words.append(w)
            r[j] = g
        remaps.append(r)
    return words, remaps


def _text_on_device(db: Database, arr):
    """A dictionary-encoded text column as device codes over one merged
    dictionary: each chunk's indices are copied to the device as they are,
    and fdb_dict_remap turns them into merged codes there."""
    import torch

    from . import DeviceUtf8, check, lib
    from .ops import _Fenced, _dev

    pa, _, _ = _pa()
    dev = _dev(db)
    n = len(arr)
    words, remaps = _merge_chunk_dictionaries(arr)
    starts = np.zeros(len(arr.chunks) + 1, dtype=np.uint64)
    idx = torch.empty(max(1, n), dtype=torch.int32, device=dev)
    at = 0
    for c, ch in enumerate(arr.chunks):
        m = len(ch)
        if m:
            local = np.array(ch.indices.cast(pa.int32()).fill_null(-1).to_numpy(zero_copy_only=False),
                             dtype=np.int32)  # a writable copy for torch
            idx[at:at + m].copy_(torch.from_numpy(local))
        at += m
        starts[c + 1] = at
    offs = np.zeros(len(remaps), dtype=np.uint64)
    if len(remaps) > 1:
        offs[1:] = np.cumsum([len(r) for r in remaps[:-1]])
    remap = np.concatenate(remaps) if remaps else np.zeros(0, np.uint32)
    d_starts = torch.from_numpy(starts.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(offs.view(np.int64)).to(dev)
    d_remap = torch.from_numpy(np.ascontiguousarray(remap).view(np.int32) if len(remap) else
                               np.zeros(1, np.int32)).to(dev)
    codes = torch.empty(max(1, n), dtype=torch.int32, device=dev)
    with _Fenced(db):
        check(lib().fdb_dict_remap(db.handle, idx.data_ptr(), n, d_starts.data_ptr(), len(arr.chunks),
                                   d_remap.data_ptr(), d_offs.data_ptr(), len(remap), codes.data_ptr()))
    return DeviceUtf8(codes[:n], words), (idx, d_starts, d_offs, d_remap)


def load_parquet(db: Database, path: str, table: str, columns: Optional[Sequence[str]] = None) -> int:
    """Read a Parquet file into device table `table` (created or replaced);
    returns the row count.  Numeric columns are decoded on the host; text
    columns keep their per-row-group dictionaries until the GPU merges them
    (fdb_dict_remap), so no string and no per-row code is built on the host."""
    pa, _, pq = _pa()
    try:
        schema = pq.read_schema(path)
        want = list(columns) if columns is not None else list(schema.names)
        text = [f.name for f in schema if f.name in want and (pa.types.is_string(f.type) or
                                                               pa.types.is_large_string(f.type))]
        tbl = pq.read_table(path, columns=want, use_threads=True, read_dictionary=text)
    except (OSError, ValueError, KeyError) as e:
        raise FalconError(-1, f"cannot read {path}: {e}") from None
    if not tbl.column_names:
        raise FalconError(-2, f"{path}: no columns to load")
    n = tbl.num_rows
    cols: Dict[str, ColumnLike] = {}
    keep = []
    for name in tbl.column_names:
        arr = tbl.column(name)
        t = arr.type
        if (pa.types.is_dictionary(t) and (pa.types.is_string(t.value_type) or pa.types.is_large_string(t.value_type))
                and n > 0):
            cols[name], bufs = _text_on_device(db, arr)
            keep.append(bufs)
        else:
            cols[name] = _convert(name, arr)
    db.create_table(table, cols, nrows=n)
    db.synchronize()  # the device codes were copied into the table before the buffers go
    return n
