"""GPU parity of ORDER BY without LIMIT against the oracle's restatement of
sort_merged -> try_typed_sort -> assemble (sort.rs:118-133, 209-350, 773-791):
bit-exact row lists, (order key, row) order, NULL rows first or last in row
order.  Full-size cases check size-independent properties instead: the output
is a permutation and the keys it reads are non-decreasing."""
import ctypes as C

import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run(db, col, n, desc, nulls_last=None):
    rows = ops.sort(db, col, n, desc, nulls_last)
    return rows[:n].cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 65_537, 1_000_003])
@pytest.mark.parametrize("desc", [False, True])
def test_sort_f64_random(db, n, desc):
    v = np.random.default_rng(n).standard_normal(n) * 1e3
    assert np.array_equal(run(db, dev(v), n, desc), O.sort(v, desc))


@pytest.mark.parametrize("n", [7, 5000, 300_001])
@pytest.mark.parametrize("desc", [False, True])
def test_sort_i64_full_range(db, n, desc):
    """Keys varying in every byte, the int64 extremes included."""
    rng = np.random.default_rng(n + 1)
    v = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64, endpoint=True)
    v[0] = np.iinfo(np.int64).min
    v[-1] = np.iinfo(np.int64).max
    assert np.array_equal(run(db, dev(v), n, desc), O.sort(v, desc))


def test_sort_float_specials(db):
    """NaN (both signs), +-inf, +-0.0, subnormals, repeated values."""
    base = np.array([3.0, -0.0, 0.0, np.nan, -1.0, np.inf, 3.0, -np.inf, 5e-324, -5e-324,
                     np.float64(np.nan) * -1, 1e308, -1e308, 0.0, -0.0])
    v = np.tile(base, 701)
    n = len(v)
    for desc in (False, True):
        assert np.array_equal(run(db, dev(v), n, desc), O.sort(v, desc)), desc


@pytest.mark.parametrize("n", [9, 10_000, 2_000_003])
def test_sort_ties_keep_row_order(db, n):
    for v in (np.full(n, 42.5), np.zeros(n, dtype=np.int64), (np.arange(n) % 3).astype(np.int64),
              (np.arange(n) // 1000).astype(np.float64)):
        for desc in (False, True):
            assert np.array_equal(run(db, dev(v), n, desc), O.sort(v, desc)), (v.dtype, desc)


@pytest.mark.parametrize("n", [1, 63, 64, 65, 4097, 100_003])
@pytest.mark.parametrize("nulls_last", [False, True])
def test_sort_nulls(db, n, nulls_last):
    rng = np.random.default_rng(n)
    v = rng.random(n) * 10
    valid = rng.random(n) > 0.3
    words = F.validity_words(valid)
    for desc in (False, True):
        got = run(db, (dev(v), dev(words.view(np.int64))), n, desc, nulls_last)
        assert np.array_equal(got, O.sort(v, desc, nulls_last=nulls_last, validity=words)), desc


def test_sort_all_null_and_no_null_bitmap(db):
    n = 5000
    v = np.arange(n, dtype=np.float64)
    none = F.validity_words(np.zeros(n, dtype=bool))
    allv = F.validity_words(np.ones(n, dtype=bool))
    for nl in (False, True):
        assert list(run(db, (dev(v), dev(none.view(np.int64))), n, True, nl)) == list(range(n))
        assert np.array_equal(run(db, (dev(v), dev(allv.view(np.int64))), n, True, nl), O.sort(v, True))


@pytest.mark.parametrize("voff", [1, 37, 64, 100])
def test_sort_validity_offset(db, voff):
    """A column whose validity bits start at bit `voff` of its bitmap."""
    n = 10_007
    rng = np.random.default_rng(voff)
    v = rng.integers(-50, 50, n).astype(np.int64)
    valid = rng.random(n) > 0.25
    shifted = np.concatenate([np.zeros(voff, dtype=bool), valid])
    words = F.validity_words(shifted)
    dv, dw = dev(v), dev(words.view(np.int64))
    raw = F.fdb_dev_column()
    raw.dtype = F.INT64
    raw.values = dv.data_ptr()
    raw.validity = dw.data_ptr()
    raw.validity_offset = voff
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    F.check(F.lib().fdb_sort(db.handle, C.byref(raw), n, 0, 1, out.data_ptr()))
    torch.cuda.synchronize()
    exp = O.sort(v, False, nulls_last=True, validity=F.validity_words(valid))
    assert np.array_equal(out.cpu().numpy().view(np.uint32), exp)


def test_sort_empty_and_errors(db):
    v = dev(np.zeros(4, dtype=np.float64))
    assert ops.sort(db, v, 0, False).numel() >= 1
    with pytest.raises(F.FalconError):
        ops.sort(db, dev(np.zeros(4, dtype=np.int32)), 4, False)


@pytest.mark.parametrize("dtype", [np.float64, np.int64])
def test_sort_full_size_properties(db, dtype):
    """100M rows: a permutation whose order keys never decrease (ties in row
    order), checked on the device."""
    n = 100_000_000
    g = torch.Generator(device="cuda").manual_seed(7)
    if dtype == np.float64:
        t = torch.rand(n, device="cuda", dtype=torch.float64, generator=g) * 100
    else:
        t = torch.randint(-(1 << 40), 1 << 40, (n,), device="cuda", dtype=torch.int64, generator=g)
    for desc in (False, True):
        rows = ops.sort(db, t, n, desc)[:n].long()
        seen = torch.zeros(n, dtype=torch.bool, device="cuda")
        seen[rows] = True
        assert bool(seen.all())
        s = t[rows]
        d = s[1:] - s[:-1]
        assert bool((d <= 0).all() if desc else (d >= 0).all())
        ties = d == 0
        assert bool((rows[1:][ties] > rows[:-1][ties]).all())
        del rows, seen, s, d, ties
        torch.cuda.empty_cache()


# ----------------------------------------------------------------------------- DISTINCT
def run_distinct(db, col, n):
    rows, cnt = ops.distinct(db, col, n)
    return rows[:int(cnt.item())].cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 2, 100, 4097, 65_537, 1_000_003])
def test_distinct_int_and_float(db, n):
    rng = np.random.default_rng(n)
    for card in (1, 7, 1000, n):
        v = rng.integers(-card, card + 1, n).astype(np.int64)
        assert np.array_equal(run_distinct(db, dev(v), n), O.distinct(v)), ("i64", card)
        f = v.astype(np.float64) * 0.25
        assert np.array_equal(run_distinct(db, dev(f), n), O.distinct(f)), ("f64", card)


def test_distinct_float_specials(db):
    base = np.array([np.nan, -0.0, 0.0, -np.nan, 2.0, np.inf, -np.inf, 5e-324, -5e-324, 1e308])
    v = np.tile(base, 997)[np.random.default_rng(3).permutation(9970)]
    assert np.array_equal(run_distinct(db, dev(v), len(v)), O.distinct(v))


@pytest.mark.parametrize("n", [5, 4096, 300_007])
def test_distinct_utf8_codes(db, n):
    codes = np.random.default_rng(n).integers(0, 12, n).astype(np.uint32)
    codes[::5] = 0xFFFFFFFF  # the NULL code is one value
    got = run_distinct(db, dev(codes.view(np.int32)), n)
    assert np.array_equal(got, O.distinct(codes))


@pytest.mark.parametrize("n", [1, 64, 65, 10_007])
def test_distinct_nulls(db, n):
    rng = np.random.default_rng(n)
    v = rng.integers(0, 20, n).astype(np.int64)
    valid = rng.random(n) > 0.4
    words = F.validity_words(valid)
    got = run_distinct(db, (dev(v), dev(words.view(np.int64))), n)
    assert np.array_equal(got, O.distinct(v, validity=words))
    none = F.validity_words(np.zeros(n, dtype=bool))
    assert list(run_distinct(db, (dev(v), dev(none.view(np.int64))), n)) == [0]


def test_distinct_empty_and_errors(db):
    rows, cnt = ops.distinct(db, dev(np.zeros(4, dtype=np.int64)), 0)
    assert int(cnt.item()) == 0
    with pytest.raises(F.FalconError):
        ops.distinct(db, dev(np.zeros(4, dtype=np.int16)), 4)


def test_distinct_full_size_properties(db):
    """100M rows, 10M-value domain: the kept rows ascend, hold every value once,
    and each is its value's first row (checked against a scatter-min on the
    device)."""
    n = 100_000_000
    g = torch.Generator(device="cuda").manual_seed(11)
    t = torch.randint(0, 10_000_000, (n,), device="cuda", dtype=torch.int64, generator=g)
    rows, cnt = ops.distinct(db, t, n)
    k = int(cnt.item())
    r = rows[:k].long()
    assert bool((r[1:] > r[:-1]).all())
    vals = t[r]
    assert k == int(torch.unique(t).numel()) == int(torch.unique(vals).numel())
    first = torch.full((10_000_000,), n, dtype=torch.int64, device="cuda")
    first.scatter_reduce_(0, t, torch.arange(n, device="cuda"), reduce="amin")
    assert bool((first[vals] == r).all())


def _sort_table(n, seed):
    """id, a text column over an unsorted dictionary with NULLs, a nullable
    INT64 column with many ties, and a FLOAT64 column with -0.0 / NaN."""
    r = np.random.default_rng(seed)
    labels = ["pear", "apple", "fig", "kiwi", "Zebra", "apple2", "é", "", "b", "ba"]
    codes = r.integers(0, len(labels), n).astype(np.uint32)
    codes[r.random(n) < 0.05] = 0xFFFFFFFF
    sal = r.integers(0, 50, n)
    sal_valid = r.random(n) > 0.1
    score = np.round(r.random(n) * 20, 1)
    score[::97] = -0.0
    score[::131] = np.nan
    return {"id": np.arange(n, dtype=np.int64), "dept": F.Utf8(codes, labels),
            "salary": np.ma.MaskedArray(sal, mask=~sal_valid), "score": score}


def _okey(t, name, desc, nulls_last=None):
    col = t[name]
    nl = desc if nulls_last is None else nulls_last
    if isinstance(col, F.Utf8):
        vals = [None if c == 0xFFFFFFFF else col.dictionary[c] for c in col.codes]
        return {"values": vals, "valid": np.array([v is not None for v in vals]), "desc": desc, "nulls_last": nl}
    if isinstance(col, np.ma.MaskedArray):
        return {"values": np.ma.getdata(col), "valid": ~np.ma.getmaskarray(col), "desc": desc, "nulls_last": nl}
    return {"values": col, "valid": None, "desc": desc, "nulls_last": nl}


@pytest.mark.parametrize("order_by,keys", [
    ("dept, salary DESC", [("dept", False, None), ("salary", True, None)]),
    ("dept DESC NULLS FIRST, score", [("dept", True, False), ("score", False, None)]),
    ("salary, score DESC, dept", [("salary", False, None), ("score", True, None), ("dept", False, None)]),
    ("dept", [("dept", False, None)]),
    ("score NULLS LAST, dept DESC", [("score", False, True), ("dept", True, None)]),
])
def test_order_by_several_keys_and_text_keys(db, order_by, keys):
    """ORDER BY several keys and text keys on the GPU (stable radix passes,
    last key first; text by dictionary rank) against the oracle's several-key
    sort, with and without WHERE and LIMIT."""
    n = 200_003
    t = _sort_table(n, seed=len(order_by))
    db.create_table("t", t)
    order = O.sort_multi([_okey(t, k, d, nl) for k, d, nl in keys], n)
    got = db.sql(f"SELECT id FROM t ORDER BY {order_by}").column(0)
    assert np.array_equal(np.asarray(got), order)
    got = db.sql(f"SELECT id FROM t ORDER BY {order_by} LIMIT 5000").column(0)
    assert np.array_equal(np.asarray(got), order[:5000])
    # With a WHERE: the selected rows' positions are sorted, then mapped back.
    sel = np.flatnonzero(t["score"] > 5.0)
    sub = {k: (F.Utf8(v.codes[sel], v.dictionary) if isinstance(v, F.Utf8) else v[sel]) for k, v in t.items()}
    want = sel[O.sort_multi([_okey(sub, k, d, nl) for k, d, nl in keys], len(sel))]
    got = db.sql(f"SELECT id FROM t WHERE score > 5 ORDER BY {order_by}").column(0)
    assert np.array_equal(np.asarray(got), want)


def test_distinct_over_several_columns(db):
    """SELECT DISTINCT over several columns on the GPU: the first occurrence of
    each distinct row, in row order, against the oracle's whole-row DISTINCT
    (NULL one value per column; NaN one value; -0.0 equal to +0.0; text by
    value, with one string under two codes)."""
    n = 300_001
    r = np.random.default_rng(5)
    labels = ["x", "y", "x", "z"]  # "x" under two codes
    codes = r.integers(0, 4, n).astype(np.uint32)
    codes[::50] = 0xFFFFFFFF
    a = r.integers(0, 30, n)
    av = r.random(n) > 0.05
    f = np.round(r.random(n) * 4) - 2.0
    f[::7] = -0.0
    f[::11] = np.nan
    t = {"d": F.Utf8(codes, labels), "a": np.ma.MaskedArray(a, mask=~av), "f": f}
    db.create_table("t", t)
    dv = [None if c == 0xFFFFFFFF else labels[c] for c in codes]
    cols = [{"values": dv, "valid": np.array([v is not None for v in dv])}, {"values": a, "valid": av},
            {"values": f}]
    want = O.distinct_multi(cols, n)
    res = db.sql("SELECT DISTINCT d, a, f FROM t")
    assert res.row_count() == len(want)
    assert res.column(0) == [dv[i] for i in want]
    got_a = [res.value(i, 1) for i in range(res.row_count())]
    assert got_a == [int(a[i]) if av[i] else None for i in want]
    # Two columns, after a WHERE.
    sel = np.flatnonzero((a < 10) & av)  # WHERE a < 10 drops the NULL rows
    want2 = sel[O.distinct_multi([{"values": a[sel], "valid": av[sel]}, {"values": f[sel]}], len(sel))]
    res2 = db.sql("SELECT DISTINCT a, f FROM t WHERE a < 10")
    assert res2.row_count() == len(want2)
    got_f = np.asarray([res2.value(i, 1) for i in range(res2.row_count())], dtype=np.float64)
    assert np.array_equal(got_f, f[want2], equal_nan=True)
