"""Pins the oracle (oracle/oracle.cpp) to the reference's own known answers.

Every case of tests/golden/known_answers.json (transcribed from FalconDB's test
suites, file:line in each case) is recomputed here through the oracle's
functions, plus the reference's property tests for lane sums
(aggregate.rs:3655-3701) and top-k (tests/top_k_scan.rs).  CPU only.
"""
import numpy as np
import pytest

import falcondb_b200 as F
from oracle import oracle as O
from tests.known_answers import build_table, cases

EQ, NE, LT, LE, GT, GE = range(6)


def _valid(col):
    if isinstance(col, np.ma.MaskedArray):
        return F.validity_words(~np.ma.getmaskarray(col)), np.ma.getdata(col)
    return None, col


def _mask_and(a, b):
    return a & b


def _is_null_words(col, n):
    v, _ = _valid(col)
    if v is None:
        return np.zeros(max(1, (n + 63) // 64), np.uint64)
    words = ~v
    if n % 64:
        words[-1] &= np.uint64((1 << (n % 64)) - 1)
    return words


def _count_star_mask(t, pred):
    n = len(t["n"])
    nn = t["n"]
    mv, md = _valid(t["maybe"])
    s = t["s"]
    like_b = [d.startswith("b") for d in s.dictionary]
    leaf = {
        "n >= 0": lambda: O.cmp_mask(nn, GE, 0),
        "n < 0": lambda: O.cmp_mask(nn, LT, 0),
        "n >= 0 AND n < 100000": lambda: O.cmp_mask(nn, GE, 0) & O.cmp_mask(nn, LT, 100000),
        "n > 10": lambda: O.cmp_mask(nn, GT, 10),
        "maybe IS NULL": lambda: _is_null_words(t["maybe"], n),
        "maybe IS NOT NULL": lambda: (mv if mv is not None else O.cmp_mask(nn, GE, -(2**62))),
        "s = 'a'": lambda: O.code_mask(s.codes, [d == "a" for d in s.dictionary]),
        "s <> 'a'": lambda: O.code_mask(s.codes, [d != "a" for d in s.dictionary]),
        "s LIKE 'b%'": lambda: O.code_mask(s.codes, like_b),
        "n IN (1, 2, 3)": lambda: O.cmp_mask(nn, EQ, 1) | O.cmp_mask(nn, EQ, 2) | O.cmp_mask(nn, EQ, 3),
        "n NOT IN (1, 2, 3)": lambda: O.cmp_mask(nn, NE, 1) & O.cmp_mask(nn, NE, 2) & O.cmp_mask(nn, NE, 3),
        "n > 5 AND n < 20": lambda: O.cmp_mask(nn, GT, 5) & O.cmp_mask(nn, LT, 20),
        "n < 2 OR n > 9995": lambda: O.cmp_mask(nn, LT, 2) | O.cmp_mask(nn, GT, 9995),
    }
    return leaf[pred]()


ALL = cases()


@pytest.mark.parametrize("case", [c for c in ALL if c["name"].startswith("count_star_filter")],
                         ids=lambda c: c["name"])
def test_count_star_filter(case):
    t = build_table(case["tables"]["t"])
    pred = case["sql"].split(" WHERE ", 1)[1]
    assert O.popcount(_count_star_mask(t, pred)) == int(case["expect"]["scalar"])


def _case(name):
    return next(c for c in ALL if c["name"] == name)


def test_count_col_counts_non_null():
    c = _case("count_col_counts_non_null")
    t = build_table(c["tables"]["t"])
    v, d = _valid(t["maybe"])
    mask = O.cmp_mask(t["n"], GE, 0)
    val, cnt = O.agg(1, d, mask=mask, validity=v)
    assert cnt == 200 == int(c["expect"]["scalar"])


def _group_rows(t, key, fcol=None, icol=None):
    k = t[key]
    g = O.group_codes(k.codes, len(k.dictionary),
                      fvals=None if fcol is None else t[fcol], ivals=None if icol is None else t[icol])
    return g, k.dictionary


def test_sql_integration_group_by():
    t = build_table(_case("group_by_count")["tables"]["t"])
    g, d = _group_rows(t, "dept")
    assert {d[i]: int(g["rows"][i]) for i in range(len(d))} == {"eng": 3, "hr": 2}
    t = build_table(_case("group_by_sum")["tables"]["t"])
    g, d = _group_rows(t, "dept", icol="salary")
    assert {d[i]: g["isum"][i] for i in range(len(d))} == {"eng": 220.0, "hr": 170.0}
    t = build_table(_case("group_by_avg")["tables"]["t"])
    g, d = _group_rows(t, "dept", icol="score")
    avg = {d[i]: g["isum"][i] / g["icnt"][i] for i in range(len(d))}
    assert avg["eng"] == 15.0
    t = build_table(_case("group_by_min_max")["tables"]["t"])
    _, mn = O.agg(4, t["score"]), None
    assert O.agg(4, t["score"])[0] == 5.0 and O.agg(5, t["score"])[0] == 10.0
    t = build_table(_case("group_by_single_group")["tables"]["t"])
    g, d = _group_rows(t, "dept", icol="n")
    assert g["isum"][0] == 6.0
    t = build_table(_case("group_by_all_unique")["tables"]["t"])
    g, d = _group_rows(t, "dept")
    assert int((g["rows"] > 0).sum()) == 3


def test_sql_integration_counts_and_distinct():
    t = build_table(_case("aggregate_without_group_by")["tables"]["t"])
    assert O.agg(1, t["n"])[1] == 5
    t = build_table(_case("count_on_empty_table")["tables"]["t"])
    assert O.agg(1, t["n"])[1] == 0
    t = build_table(_case("count_distinct_basic")["tables"]["t"])
    pres = O.present_codes(t["dept"].codes, len(t["dept"].dictionary))
    assert len({t["dept"].dictionary[i] for i in np.flatnonzero(pres)}) == 2


def test_parallel_group_by_matches_a_single_batch():
    c = _case("parallel_group_by_matches_a_single_batch")
    t = build_table(c["tables"]["t"])
    g, d = _group_rows(t, "dept", icol="v")
    got = sorted([d[i], str(int(g["icnt"][i])), str(int(g["isum"][i]))] for i in range(len(d)))
    assert got == c["expect"]["rows"]


def test_agg_only_count_sum_min_max():
    t = build_table(_case("agg_only_count_sum")["tables"]["t"])
    assert O.agg(1, t["score"])[1] == 5
    assert O.agg(2, t["score"])[0] == 40.0
    assert O.agg(4, t["score"])[0] == 6.0 and O.agg(5, t["score"])[0] == 10.0


def test_null_join_keys_match_nothing():
    tabs = _case("null_key_inner")["tables"]
    l, r = build_table(tabs["l"]), build_table(tabs["r"])
    lv, ld = _valid(l["k"])
    rv, rd = _valid(r["rk"])
    want = {0: 1, 1: 4, 2: 1, 3: 3}
    for jt, n in want.items():
        assert O.join_agg(rd, None, ld, None, jt, bvalid=rv, pvalid=lv)["count"] == n
        left, right = O.join_pairs(rd, ld, jt, bvalid=rv, pvalid=lv)
        assert len(left) == n


def test_join_and_parquet_paths():
    for name, jt in [("inner_join_keeps_every_match", 0), ("inner_join_below_threshold", 0),
                     ("left_join_keeps_unmatched_rows", 1), ("join_with_no_overlap", 0)]:
        c = _case(name)
        l, r = build_table(c["tables"]["l"]), build_table(c["tables"]["r"])
        assert O.join_agg(r["k"], r["rv"], l["k"], None, jt)["count"] == c["expect"]["row_count"], name
    c = _case("join_result_matches_a_small_reference")
    l, r = build_table(c["tables"]["l"]), build_table(c["tables"]["r"])
    left, right = O.join_pairs(r["k"], l["k"], 0)
    ks = sorted(int(l["k"][i]) for i in left if l["k"][i] < 3)
    assert [str(k) for k in ks] == c["expect"]["first_col_sorted"]


@pytest.mark.parametrize("rows", [100_000, 1_000_000])
def test_query_bench_assertions(rows):
    b = build_table({"gen": "bench", "rows": rows})
    lk = build_table({"gen": "lookup", "rows": rows})
    assert O.sum_lanes(b["score"]) == rows // 100 * 5000
    assert O.popcount(O.cmp_mask(b["score"], GT, 50)) == rows // 2
    assert O.join_agg(lk["lid"], None, b["id"], None, 0)["count"] == rows // 10
    assert O.join_agg(lk["lid"], None, b["id"], None, 1)["count"] == rows
    assert O.join_agg(lk["lid"], None, b["id"], None, 2)["count"] == rows // 10
    assert O.join_agg(lk["lid"], None, b["id"], None, 3)["count"] == rows - rows // 10


@pytest.mark.parametrize("n", [0, 1, 7, 8, 9, 15, 16, 17, 1000, 65_537])
def test_lane_sum_matches_a_plain_sum(n):
    """aggregate.rs:3655-3670: |lanes - plain| <= max(|plain| 1e-12, 1e-9)."""
    vals = (np.arange(n) % 100).astype(np.float64) + 0.5
    plain = O.sum_serial(vals)
    assert abs(O.sum_lanes(vals) - plain) <= max(abs(plain) * 1e-12, 1e-9)


def test_lane_sum_integers_and_overflow():
    """aggregate.rs:3672-3692 and the checked i64 sum (3087-3104)."""
    for n in [0, 1, 7, 8, 9, 17, 1000, 65_537]:
        v = np.arange(n, dtype=np.int64) - 500
        assert O.checked_sum_i64(v) == int(v.sum())
    big = np.array([1 << 62, 1 << 62, 1 << 62], dtype=np.int64)
    assert O.checked_sum_i64(big) is None


ROWS = 1000


def _topk_fixture():
    """tests/top_k_scan.rs:58-80: scattered distinct scores, NULL every 97th row."""
    i = np.arange(ROWS)
    scores = ((i * 7919) % ROWS).astype(np.float64) + 0.5
    null = i % 97 == 0
    return scores, F.validity_words(~null), null


def _full_sort_head(scores, null, k, desc, nulls_last):
    keyed = [r for r in range(len(scores)) if not null[r]]
    keyed.sort(key=lambda r: (-scores[r] if desc else scores[r], r))
    nulls = [r for r in range(len(scores)) if null[r]]
    order = keyed + nulls if nulls_last else nulls + keyed
    return order[:k]


@pytest.mark.parametrize("k", [1, 5, 10, 15, 100])
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("nulls_last", [False, True])
def test_topk_is_the_head_of_the_full_sort(k, desc, nulls_last):
    scores, valid, null = _topk_fixture()
    got = O.topk(scores, k, desc, nulls_last=nulls_last, validity=valid)
    assert list(got) == _full_sort_head(scores, null, k, desc, nulls_last)


def test_topk_ties_break_on_row_ascending():
    """An all-equal column (top_k_scan.rs ties case): the first k rows."""
    v = np.full(5000, 3.25)
    assert list(O.topk(v, 10, True)) == list(range(10))
    assert list(O.topk(v, 10, False)) == list(range(10))


def test_topk_ascending_column_desc():
    v = np.arange(100_000, dtype=np.int64)
    assert list(O.topk(v, 10, True)) == list(range(99_999, 99_989, -1))


def _xorshift_keys(n):
    """sort.rs:1677-1690: xorshift64 keys from 0x2545F4914F6CDD1D."""
    state, out = 0x2545F4914F6CDD1D, []
    m = (1 << 64) - 1
    for _ in range(n):
        state ^= (state << 13) & m
        state ^= state >> 7
        state ^= (state << 17) & m
        out.append(state)
    return out


def test_full_sort_known_answers():
    """sort.rs:1642-1672 (make_batch, sort_asc, sort_desc) and 1729-1740
    (sort_nulls_last)."""
    score = np.array([7.0, 9.5, 8.0, 6.0])
    asc = O.sort(score, False)
    assert score[asc[0]] == 6.0 and score[asc[3]] == 9.5
    assert score[O.sort(score, True)[0]] == 9.5
    x = np.array([1.0, 0.0, 3.0])
    valid = F.validity_words(np.array([True, False, True]))
    assert list(O.sort(x, False, nulls_last=True, validity=valid)) == [0, 2, 1]
    assert list(O.sort(x, False, nulls_last=False, validity=valid)) == [1, 0, 2]


def test_full_sort_matches_the_tuple_sort_of_order_keys():
    """sort.rs:1675-1690 (radix_sort_matches_comparison_sort): 2 * 8192 + 37
    xorshift keys sort as (key, row) tuples.  An INT64 column whose values are
    key XOR 2^63 has exactly these order keys."""
    keys = _xorshift_keys(2 * 8192 + 37)
    vals = np.array([k ^ (1 << 63) for k in keys], dtype=np.uint64).view(np.int64)
    expect = [r for _, r in sorted((k, r) for r, k in enumerate(keys))]
    assert list(O.sort(vals, False)) == expect


def test_full_sort_constant_and_duplicate_keys():
    """sort.rs:1693-1705: constant keys keep row order; i % 3 keys sort as
    (key, row) tuples."""
    n = 8192 + 5
    assert list(O.sort(np.full(n, 42, dtype=np.int64), False)) == list(range(n))
    dup = np.arange(n, dtype=np.int64) % 3
    assert list(O.sort(dup, False)) == [r for _, r in sorted((int(dup[r]), r) for r in range(n))]


def test_full_sort_large_float_column_is_ordered():
    """sort.rs:1707-1723: 16,384 scattered floats come out non-decreasing."""
    n = 2 * 8192
    i = np.arange(n)
    v = ((i * 7919) % n).astype(np.float64) - n // 2
    got = v[O.sort(v, False)]
    assert np.all(np.diff(got) >= 0)
    assert sorted(O.sort(v, False)) == list(range(n))


def test_full_sort_float_order_keys():
    """f64_ord_key (sort.rs:451-454): -0.0 before +0.0, NaN after +inf, DESC
    flips the keys, ties stay in row order in both directions."""
    v = np.array([3.0, -0.0, 0.0, np.nan, -1.0, np.inf, 3.0, -np.inf])
    assert list(O.sort(v, False)) == [7, 4, 1, 2, 0, 6, 5, 3]
    assert list(O.sort(v, True)) == [3, 5, 0, 6, 2, 1, 4, 7]


def test_full_sort_head_is_the_topk():
    scores, valid, null = _topk_fixture()
    for desc in (False, True):
        for nulls_last in (False, True):
            full = O.sort(scores, desc, nulls_last=nulls_last, validity=valid)
            assert list(full) == _full_sort_head(scores, null, ROWS, desc, nulls_last)
            assert list(full[:15]) == list(O.topk(scores, 15, desc, nulls_last=nulls_last, validity=valid))


def test_distinct_known_answers():
    """tests/sort_and_dedup_paths.rs:143-206 and sql_integration.rs:1326-1338,
    restated on the oracle: first occurrence kept, in row order."""
    assert list(O.distinct(np.array([1, 2, 1, 3, 2], dtype=np.int64))) == [0, 1, 3]
    assert list(O.distinct(np.array([7, 7, 7], dtype=np.int64))) == [0]
    v = np.array([0, 0, 1], dtype=np.int64)  # two NULLs then 1: NULLs are one value
    assert list(O.distinct(v, validity=F.validity_words(np.array([False, False, True])))) == [0, 2]
    assert list(O.distinct(np.array([0, 1, 0], dtype=np.uint32))) == [0, 1]  # alpha, beta, alpha
    assert len(O.distinct(np.array([1.5, 2.5, 1.5]))) == 2
    assert len(O.distinct(np.concatenate([[1], np.arange(40) % 5]).astype(np.int64))) == 5
    assert len(O.distinct(np.arange(3000, dtype=np.int64) % 137)) == 137
    assert len(O.distinct(np.array([0, 1, 0, 1, 0], dtype=np.uint32))) == 2  # eng, hr
    n = np.array([3, 1, 2, 1, 3], dtype=np.int64)  # DISTINCT n ORDER BY n: ORDER BY first, then dedup
    order = O.sort(n, False)
    assert list(n[order][O.distinct(n[order])]) == [1, 2, 3]


def test_distinct_float_equality():
    """row_eq / norm_f64 (select.rs:201-236): NaNs are one value, -0.0 == +0.0."""
    v = np.array([np.nan, -0.0, 0.0, -np.nan, 2.0, np.inf, -np.inf, 2.0, np.inf])
    assert list(O.distinct(v)) == [0, 1, 4, 5, 6]


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_reference_engine_sort_agrees_with_the_oracle(threads):
    """ref_sort (pair loop + parallel tuple sort, sort.rs:270-345, 692-698) is
    the serial oracle's full sort, NULLs included."""
    rng = np.random.default_rng(threads)
    for n in [0, 1, 4097, 100_003]:
        v = rng.standard_normal(n)
        v[::5] = 0.25
        for desc in (False, True):
            assert np.array_equal(O.ref_sort(v, desc, threads), O.sort(v, desc))
    i = rng.integers(-20, 20, 50_001)
    w = F.validity_words(rng.random(50_001) > 0.3)
    for nl in (False, True):
        assert np.array_equal(O.ref_sort(i, False, threads, nulls_last=nl, validity=w),
                              O.sort(i, False, nulls_last=nl, validity=w))


def test_reference_engine_agrees_with_the_serial_oracle():
    """The timed CPU baseline computes the same answers as the serial oracle."""
    from falcondb_b200 import workloads as W

    t = W.table_t(300_000, seed=3)
    sc = t["score"]
    assert abs(O.ref_sum_f64(sc, 4) - O.sum_serial(sc)) <= abs(O.sum_serial(sc)) * 1e-12
    assert O.ref_count_cmp_f64(sc, GT, 50.0) == O.popcount(O.cmp_mask(sc, GT, 50))
    assert list(O.ref_topk(sc, 10, True)) == list(O.topk(sc, 10, True))
    assert list(O.ref_topk(t["id"], 10, True)) == list(O.topk(t["id"], 10, True))
    pres = O.ref_present_codes(t["dept"].codes, 12, 4)
    assert list(pres) == list(O.present_codes(t["dept"].codes, 12))
    rows, fs, is_ = O.ref_filter_group_codes(t["dept"].codes, sc, t["salary"], 12, GT, 50.0, 4)
    g = O.group_codes(t["dept"].codes, 12, mask=O.cmp_mask(sc, GT, 50), fvals=sc, ivals=t["salary"])
    assert list(rows) == list(g["rows"][:12])
    assert np.allclose(fs, g["fsum"][:12], rtol=1e-12, atol=0)
    assert list(is_) == list(g["isum"][:12])
    b, p = W.join_tables(10_000, 200_000)
    for jt in range(4):
        c, ps, vs = O.ref_join_agg(b["key"], b["payload"], p["key"], p["value"], jt, 4)
        o = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
        assert c == o["count"]
        if jt <= 1:
            assert ps == o["sum_payload"]
        else:
            assert abs(vs - o["sum_value"]) <= abs(o["sum_value"]) * 1e-12


def _key(t, name, desc=False, nulls_last=None):
    """A sort_multi key over column `name` of a known-answer table."""
    col = t[name]
    if isinstance(col, F.Utf8):
        vals = [None if c == 0xFFFFFFFF else col.dictionary[c] for c in col.codes]
        valid = np.array([v is not None for v in vals])
        return {"values": vals, "valid": valid, "desc": desc, "nulls_last": desc if nulls_last is None else nulls_last}
    vd, data = _valid(col)
    valid = None if vd is None else ~np.ma.getmaskarray(col)
    return {"values": np.asarray(data), "valid": valid, "desc": desc,
            "nulls_last": desc if nulls_last is None else nulls_last}


def _cells(t, name, order):
    col = t[name]
    if isinstance(col, F.Utf8):
        return ["NULL" if col.codes[r] == 0xFFFFFFFF else col.dictionary[col.codes[r]] for r in order]
    return [str(int(col[r])) if np.asarray(col).dtype.kind == "i" else ("%g" % col[r]) for r in order]


@pytest.mark.parametrize("name,keys,outcols", [
    ("order_by_string", [("name", False, None)], ["name"]),
    ("order_by_multi_key", [("dept", False, None), ("score", True, None)], ["dept", "score"]),
    ("sort_text_by_string_not_dictionary_position[ASC]", [("s", False, None)], ["s"]),
    ("sort_text_by_string_not_dictionary_position[DESC]", [("s", True, None)], ["s"]),
    ("sort_text_places_nulls[s ASC]", [("s", False, None)], ["s"]),
    ("sort_text_places_nulls[s ASC NULLS LAST]", [("s", False, True)], ["s"]),
    ("sort_text_places_nulls[s DESC]", [("s", True, None)], ["s"]),
    ("sort_equal_strings_keep_row_order[ASC]", [("s", False, None)], ["id"]),
    ("sort_equal_strings_keep_row_order[DESC]", [("s", True, None)], ["id"]),
    ("sort_all_distinct_text_column", [("s", False, None)], ["s"]),
    ("sort_multi_key", [("dept", False, None), ("score", True, None)], ["dept", "score"]),
])
def test_multi_key_and_text_sort_known_answers(name, keys, outcols):
    """sql_integration.rs:210-226 and sort.rs:979-1060, 1747-1766 restated
    on the oracle's several-key sort (sort_merged, sort.rs:118-165; text by
    string, sort.rs:352-382; NULLs first ascending unless NULLS LAST)."""
    c = _case(name)
    t = build_table(c["tables"]["t"])
    n = len(next(iter(t.values())).codes if isinstance(next(iter(t.values())), F.Utf8) else next(iter(t.values())))
    order = O.sort_multi([_key(t, k, d, nl) for k, d, nl in keys], n)
    got = [list(r) for r in zip(*[_cells(t, oc, order) for oc in outcols])]
    exp = c["expect"]
    want = exp.get("rows") or exp.get("head_rows")
    assert got[:len(want)] == want


def test_distinct_whole_rows_known_answer():
    """tests/sort_and_dedup_paths.rs:162-165 on the oracle's whole-row DISTINCT,
    plus NULLs as one value and float equality across columns."""
    c = _case("distinct_compares_whole_rows")
    t = build_table(c["tables"]["t"])
    a, b = t["a"], t["b"]
    cols = [{"values": np.asarray(a)}, {"values": [b.dictionary[x] for x in b.codes]}]
    assert len(O.distinct_multi(cols, 3)) == c["expect"]["row_count"]
    x = np.array([1.0, np.nan, -0.0, 0.0, 1.0, np.nan])
    y = np.array([5, 6, 7, 7, 5, 6])
    yv = np.array([True, False, True, True, True, False])
    assert list(O.distinct_multi([{"values": x}, {"values": y, "valid": yv}], 6)) == [0, 1, 2]
