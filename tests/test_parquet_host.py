"""The Parquet loader's host side on the CPU: the reference's Arrow type
mapping (parquet_io.rs:118-231), NULLs, and one dictionary per text column
across row groups that see their strings in different orders."""
import numpy as np
import pytest

pa = pytest.importorskip("pyarrow")
pq = pytest.importorskip("pyarrow.parquet")

from falcondb_b200 import FalconError, Utf8  # noqa: E402
from falcondb_b200 import parquet as P  # noqa: E402


def _write(tmp_path, table, **kw):
    path = str(tmp_path / "t.parquet")
    pq.write_table(table, path, **kw)
    return path


def test_types_and_nulls(tmp_path):
    t = pa.table({
        "i8": pa.array([1, -2, None], type=pa.int8()),
        "u32": pa.array([1, 4_000_000_000, 7], type=pa.uint32()),
        "u64": pa.array([1, 2**63 + 5, 3], type=pa.uint64()),
        "f32": pa.array([0.1, None, -2.5], type=pa.float32()),
        "f64": pa.array([1.5, 2.5, None], type=pa.float64()),
        "b": pa.array([True, False, None]),
        "d": pa.array([0, 19000, None], type=pa.date32()),
        "ts": pa.array([1, 2, 3], type=pa.timestamp("us")),
        "n": pa.array([None, None, None], type=pa.null()),
        "s": pa.array(["x", None, "y"]),
    })
    cols, n = P.read_parquet_columns(_write(tmp_path, t))
    assert n == 3
    assert list(np.ma.getdata(cols["i8"])) == [1, -2, 0] and list(np.ma.getmaskarray(cols["i8"])) == [0, 0, 1]
    assert cols["u32"].tolist() == [1, 4_000_000_000 - 2**32, 7]  # wraps to i32 (parquet_io.rs:166-167)
    assert cols["u64"].tolist()[1] == 2**63 + 5 - 2**64
    f32 = cols["f32"]
    assert f32.dtype == np.float64 and np.ma.getdata(f32)[0] == np.float64(np.float32(0.1))
    assert list(np.ma.getmaskarray(f32)) == [0, 1, 0]
    assert list(np.ma.getdata(cols["b"])) == [1, 0, 0] and list(np.ma.getmaskarray(cols["b"])) == [0, 0, 1]
    assert list(np.ma.getdata(cols["d"]))[:2] == [0, 19000]
    assert cols["ts"].tolist() == [1, 2, 3]
    assert np.ma.getmaskarray(cols["n"]).all()
    s = cols["s"]
    assert isinstance(s, Utf8) and s.dictionary == ["x", "y"] and list(s.codes) == [0, 0xFFFFFFFF, 1]


def test_one_dictionary_across_row_groups(tmp_path):
    """Row groups that meet the strings in different orders (the reference's
    per-batch dictionary hazard, aggregate.rs:655-658): one first-appearance
    dictionary, codes that name the right strings in every group."""
    vals = ["eng", "hr", "ops"] * 400 + ["ops", "hr", "eng", "fin"] * 300
    t = pa.table({"dept": pa.array(vals), "v": pa.array(np.arange(len(vals), dtype=np.int64))})
    path = _write(tmp_path, t, row_group_size=1000)
    assert pq.ParquetFile(path).num_row_groups > 1
    cols, n = P.read_parquet_columns(path)
    d = cols["dept"]
    assert d.dictionary == ["eng", "hr", "ops", "fin"]
    assert [d.dictionary[c] for c in d.codes] == vals
    assert cols["v"].tolist() == list(range(n))


def test_text_edge_cases(tmp_path):
    t = pa.table({"none": pa.array([None, None], type=pa.string()), "one": pa.array(["a", "a"]),
                  "big": pa.array(["x", "y"], type=pa.large_string())})
    cols, n = P.read_parquet_columns(_write(tmp_path, t))
    assert cols["none"].dictionary == [] and list(cols["none"].codes) == [0xFFFFFFFF] * 2
    assert cols["one"].dictionary == ["a"] and list(cols["one"].codes) == [0, 0]
    assert cols["big"].dictionary == ["x", "y"]
    empty = pa.table({"s": pa.array([], type=pa.string()), "v": pa.array([], type=pa.int64())})
    cols, n = P.read_parquet_columns(_write(tmp_path, empty))
    assert n == 0 and len(cols["s"].codes) == 0


def test_projection_and_errors(tmp_path):
    t = pa.table({"a": pa.array([1, 2]), "b": pa.array([3.0, 4.0]),
                  "dec": pa.array([1, 2], type=pa.decimal128(10, 2)),
                  "ns": pa.array([1, 2], type=pa.timestamp("ns"))})
    path = _write(tmp_path, t)
    cols, n = P.read_parquet_columns(path, ["b", "a"])
    assert list(cols) == ["b", "a"] and n == 2
    with pytest.raises(FalconError):
        P.read_parquet_columns(path, ["dec"])
    with pytest.raises(FalconError):
        P.read_parquet_columns(path, ["ns"])
    with pytest.raises(FalconError):
        P.read_parquet_columns(str(tmp_path / "missing.parquet"))


def test_chunk_dictionaries_merge_without_touching_rows():
    """The GPU loader's host half: the row groups' dictionaries (distinct
    strings) merge chunk by chunk into one dictionary, each chunk's entries
    mapped to merged codes; remapping each chunk's indices through its table
    gives every row's string (checked here on the host)."""
    import pyarrow as pa

    from falcondb_b200 import parquet as P

    chunks = [pa.DictionaryArray.from_arrays(pa.array([0, 1, 1, None, 0], pa.int32()), pa.array(["b", "a"])),
              pa.DictionaryArray.from_arrays(pa.array([2, 0, 1], pa.int32()), pa.array(["a", "c", "b"])),
              pa.DictionaryArray.from_arrays(pa.array([0, 0], pa.int32()), pa.array(["d"]))]
    arr = pa.chunked_array(chunks)
    words, remaps = P._merge_chunk_dictionaries(arr)
    assert words == ["b", "a", "c", "d"]
    assert [list(r) for r in remaps] == [[0, 1], [1, 2, 0], [3]]
    rows = []
    for ch, r in zip(arr.chunks, remaps):
        for k in ch.indices.to_pylist():
            rows.append(None if k is None else words[r[k]])
    assert rows == ["b", "a", "a", None, "b", "b", "a", "c", "d", "d"]
