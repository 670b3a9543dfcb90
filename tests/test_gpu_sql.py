"""Database.sql on the GPU: every known answer of the reference's own tests
(tests/golden/known_answers.json) and the headline query shapes against the
oracle."""
import numpy as np
import pytest

import falcondb_b200 as F
from falcondb_b200 import workloads as W
from oracle import oracle as O
from tests.known_answers import build_table, cases, check_result

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def load(db, tables):
    for name, spec in tables.items():
        db.create_table(name, build_table(spec))


@pytest.mark.parametrize("case", cases(), ids=lambda c: c["name"])
def test_known_answer(db, case):
    load(db, case["tables"])
    res = db.sql(case["sql"])
    check_result(case, res)


def test_config0_query(db):
    n = 1_000_000
    t = W.table_t(n, seed=1)
    db.create_table("t", t)
    res = db.sql("SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM t WHERE score > 50 GROUP BY dept ORDER BY dept")
    mask = O.cmp_mask(t["score"], F.GT, 50)
    g = O.group_codes(t["dept"].codes, 12, mask=mask, fvals=t["score"], ivals=t["salary"])
    assert res.row_count() == 12
    assert res.column(0) == W.DEPTS  # ORDER BY dept
    for i in range(12):
        assert res.column(1)[i] == g["rows"][i]
        assert abs(res.column(2)[i] - g["fsum"][i]) <= RTOL * g["fsum"][i]
        assert res.column(3)[i] == g["isum"][i] / g["icnt"][i]


def test_config1_queries(db):
    n = 2_000_003
    t = W.table_t(n, seed=2)
    db.create_table("t", t)
    s = db.sql("SELECT SUM(score) FROM t").column(0)[0]
    want = O.sum_serial(t["score"])
    assert abs(s - want) <= RTOL * want
    assert db.sql("SELECT COUNT(*) FROM t WHERE score > 50").column(0)[0] == O.popcount(
        O.cmp_mask(t["score"], F.GT, 50))
    assert db.sql("SELECT COUNT(DISTINCT dept) FROM t").column(0)[0] == 12
    top = db.sql("SELECT id, score FROM t ORDER BY score DESC LIMIT 10")
    rows = O.topk(t["score"], 10, True)
    assert list(top.column(0)) == list(t["id"][rows])
    assert list(top.column(1)) == list(t["score"][rows])
    top2 = db.sql("SELECT id FROM t ORDER BY id DESC LIMIT 10")
    assert list(top2.column(0)) == list(range(n - 1, n - 11, -1))


def test_config2_join_queries(db):
    b, p = W.join_tables(100_000, 1_000_003, seed=5)
    db.create_table("b", b)
    db.create_table("p", p)
    for sql, jt in [("SELECT COUNT(*), SUM(b.payload) FROM p JOIN b ON p.key = b.key", F.JOIN_INNER),
                    ("SELECT COUNT(*), SUM(b.payload) FROM p LEFT JOIN b ON p.key = b.key", F.JOIN_LEFT)]:
        r = db.sql(sql)
        want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
        assert r.column(0)[0] == want["count"] and r.column(1)[0] == float(want["sum_payload"])
    for sql, jt in [("SELECT COUNT(*), SUM(value) FROM p WHERE EXISTS (SELECT 1 FROM b WHERE b.key = p.key)",
                     F.JOIN_SEMI),
                    ("SELECT COUNT(*), SUM(value) FROM p WHERE NOT EXISTS (SELECT 1 FROM b WHERE b.key = p.key)",
                     F.JOIN_ANTI)]:
        r = db.sql(sql)
        want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
        assert r.column(0)[0] == want["count"]
        assert abs(r.column(1)[0] - want["sum_value"]) <= RTOL * want["sum_value"]


def test_config3_group_by(db):
    n = 1_000_000
    g = W.groupby_table(n, distinct=200_000, seed=4)
    db.create_table("g", g)
    r = db.sql("SELECT key, COUNT(*), SUM(v), MIN(v), MAX(v) FROM g GROUP BY key ORDER BY key")
    want = O.group_i64(g["key"], g["v"])
    assert np.array_equal(np.asarray(r.column(0)), want["key"])
    assert np.array_equal(np.asarray(r.column(1)), want["count"])
    rel = np.abs(np.asarray(r.column(2)) - want["sum"]) / np.abs(want["sum"])
    assert rel.max() <= RTOL
    assert np.array_equal(np.asarray(r.column(3)), want["min"])


def test_where_with_projection_and_limit(db):
    t = W.table_t(100_000, seed=9)
    db.create_table("t", t)
    r = db.sql("SELECT id, score FROM t WHERE score > 99.9 AND dept = 'd03' ORDER BY score DESC LIMIT 5")
    sel = np.flatnonzero((t["score"] > 99.9) & (t["dept"].codes == 3))
    order = sel[np.lexsort((sel, -t["score"][sel]))][:5]
    assert list(r.column(0)) == list(order)
    r2 = db.sql("SELECT COUNT(*) FROM t WHERE dept IN ('d01', 'd02') OR salary < 31000")
    want = int(((t["dept"].codes == 1) | (t["dept"].codes == 2) | (t["salary"] < 31000)).sum())
    assert r2.column(0)[0] == want


def test_errors_are_reported(db):
    db.create_table("t", {"x": np.arange(10, dtype=np.int64)})
    with pytest.raises(F.FalconError) as e:
        db.sql("SELECT y FROM t")
    assert e.value.code == -6
    with pytest.raises(F.FalconError) as e:
        db.sql("SELEKT x FROM t")
    assert e.value.code == -5
    with pytest.raises(F.FalconError):
        db.sql("SELECT x FROM nope")


def test_order_by_without_small_limit_sorts_on_the_gpu(db):
    """ORDER BY one numeric column with no LIMIT, or one above the top-k bound,
    with and without WHERE, by name, alias and position: the oracle's full sort
    (try_typed_sort, sort.rs:209-350) of the selected rows."""
    t = W.table_t(300_000, seed=5)
    db.create_table("t", t)
    r = db.sql("SELECT id, score FROM t ORDER BY score")
    assert list(r.column(0)) == list(O.sort(t["score"], False))
    r = db.sql("SELECT score AS s, id FROM t ORDER BY s DESC LIMIT 10000")
    assert list(r.column(1)) == list(O.sort(t["score"], True)[:10000])
    r = db.sql("SELECT id FROM t ORDER BY 1 DESC")
    assert list(r.column(0)) == list(range(299_999, -1, -1))
    sel = np.flatnonzero(t["score"] > 60)
    r = db.sql("SELECT id, salary FROM t WHERE score > 60 ORDER BY salary DESC")
    assert list(r.column(0)) == list(sel[O.sort(t["salary"][sel], True)])
    r = db.sql("SELECT id FROM t WHERE score > 60 ORDER BY score LIMIT 5000")
    assert list(r.column(0)) == list(sel[O.sort(t["score"][sel], False)][:5000])


@pytest.mark.parametrize("nulls", ["", " NULLS FIRST", " NULLS LAST"])
def test_order_by_nullable_column(db, nulls):
    n = 50_000
    rng = np.random.default_rng(3)
    x = np.ma.masked_array(rng.standard_normal(n), mask=rng.random(n) < 0.2)
    x[5] = -0.0
    x[6] = 0.0
    db.create_table("u", {"id": np.arange(n, dtype=np.int64), "x": x})
    valid = F.validity_words(~np.ma.getmaskarray(x))
    for desc in (False, True):
        nl = desc if not nulls else nulls == " NULLS LAST"
        r = db.sql(f"SELECT id FROM u ORDER BY x{' DESC' if desc else ''}{nulls}")
        want = O.sort(np.ma.getdata(x), desc, nulls_last=nl, validity=valid)
        assert list(r.column(0)) == list(want), (desc, nulls)


def test_select_distinct(db):
    """SELECT DISTINCT: each value's first row in output order (dedup_batches,
    select.rs:238-457), after ORDER BY and LIMIT (db.rs:1699-1729); the
    reference's own cases (sort_and_dedup_paths.rs:143-206,
    sql_integration.rs:1326-1338) restated."""
    db.create_table("t", {"v": np.array([1, 2, 1, 3, 2], dtype=np.int64)})
    assert list(db.sql("SELECT DISTINCT v FROM t").column(0)) == [1, 2, 3]
    db.create_table("t", {"v": np.array([7, 7, 7], dtype=np.int64)})
    assert list(db.sql("SELECT DISTINCT v FROM t").column(0)) == [7]
    db.create_table("t", {"v": np.ma.masked_array(np.array([0, 0, 1], dtype=np.int64), mask=[True, True, False])})
    assert db.sql("SELECT DISTINCT v FROM t").rows == 2
    db.create_table("t", {"s": F.Utf8(np.array([0, 1, 0], dtype=np.uint32), ["alpha", "beta"])})
    assert list(db.sql("SELECT DISTINCT s FROM t").column(0)) == ["alpha", "beta"]
    db.create_table("t", {"v": np.array([1.5, 2.5, 1.5])})
    assert db.sql("SELECT DISTINCT v FROM t").rows == 2
    db.create_table("t", {"v": np.arange(3000, dtype=np.int64) % 137})
    assert db.sql("SELECT DISTINCT v FROM t").rows == 137
    db.create_table("t", {"n": np.array([3, 1, 2, 1, 3], dtype=np.int64)})
    assert list(db.sql("SELECT DISTINCT n FROM t ORDER BY n ASC").column(0)) == [1, 2, 3]
    assert list(db.sql("SELECT DISTINCT n FROM t ORDER BY n DESC LIMIT 3").column(0)) == [3, 2]
    assert list(db.sql("SELECT DISTINCT n FROM t LIMIT 3").column(0)) == [3, 1, 2]
    # Whole rows (dedup_batches): the same column twice is one distinct value per row.
    assert list(db.sql("SELECT DISTINCT n, n FROM t").column(0)) == [3, 1, 2]


@pytest.mark.parametrize("n", [1000, 1_000_003])
def test_select_distinct_against_the_oracle(db, n):
    rng = np.random.default_rng(n)
    t = W.table_t(n, seed=4)
    sal = t["salary"] % 5000
    f = np.round(rng.standard_normal(n), 2)
    f[::997] = np.nan
    f[1::991] = -0.0
    f[2::983] = 0.0
    xv = rng.integers(0, 300, n).astype(np.int64)
    null = rng.random(n) < 0.05
    db.create_table("u", {"id": t["id"], "dept": t["dept"], "salary": sal, "f": f,
                          "x": np.ma.masked_array(xv, mask=null)})
    r = db.sql("SELECT DISTINCT salary FROM u")
    assert list(r.column(0)) == list(sal[O.distinct(sal)])
    got = np.array(db.sql("SELECT DISTINCT f FROM u").column(0), dtype=np.float64)
    exp = f[O.distinct(f)]
    assert np.array_equal(got, exp, equal_nan=True)
    assert np.array_equal(np.signbit(got), np.signbit(exp))  # the first zero's sign is kept
    sel = np.flatnonzero(sal > 1000)
    keep = sel[O.distinct(xv[sel], validity=F.validity_words(~null[sel]))]
    r = db.sql("SELECT DISTINCT x FROM u WHERE salary > 1000")
    assert r.rows == len(keep)
    assert [None if null[k] else int(xv[k]) for k in keep] == [r.value(i, 0) for i in range(r.rows)]
    r = db.sql("SELECT DISTINCT dept FROM u")
    assert list(r.column(0)) == [W.DEPTS[c] for c in t["dept"].codes[O.distinct(t["dept"].codes)]]


def _row_numbers(vals, desc):
    """ROW_NUMBER() OVER (ORDER BY vals): try_dense_partition_sort
    (window.rs:308-331) -- f64 order keys, ties by position -- via the oracle's
    sort of the values as f64."""
    rn = np.empty(len(vals), dtype=np.int64)
    rn[O.sort(np.asarray(vals, dtype=np.float64), desc)] = np.arange(1, len(vals) + 1)
    return rn


@pytest.mark.parametrize("n", [20, 1_000_003])
def test_row_number_over_order_by(db, n):
    t = W.table_t(n, seed=6)
    db.create_table("t", t)
    r = db.sql("SELECT id, ROW_NUMBER() OVER (ORDER BY score DESC) AS rn FROM t")
    assert r.rows == n
    assert list(r.column(0)) == list(range(n))
    assert np.array_equal(np.asarray(r.column(1)), _row_numbers(t["score"], True))
    r = db.sql("SELECT ROW_NUMBER() OVER (ORDER BY salary) AS rn, id FROM t WHERE score > 30")
    sel = np.flatnonzero(t["score"] > 30)
    assert list(r.column(1)) == list(sel)
    assert np.array_equal(np.asarray(r.column(0)), _row_numbers(t["salary"][sel], False))
    r = db.sql("SELECT id, ROW_NUMBER() OVER (ORDER BY score DESC) AS rn FROM t ORDER BY rn LIMIT 5")
    assert list(r.column(0)) == list(O.sort(t["score"], True)[:5])
    r = db.sql("SELECT id, ROW_NUMBER() OVER () AS rn FROM t WHERE score < 10")
    assert list(r.column(1)) == list(range(1, int((t["score"] < 10).sum()) + 1))


def test_row_number_semantics(db):
    # window.rs:978-995 restated without PARTITION BY: salaries 100, 120, 90,
    # 80, 110 DESC -> 3, 1, 4, 5, 2.
    db.create_table("t", {"salary": np.array([100, 120, 90, 80, 110], dtype=np.int64)})
    r = db.sql("SELECT salary, ROW_NUMBER() OVER (ORDER BY salary DESC) AS rn FROM t")
    assert list(r.column(1)) == [3, 1, 4, 5, 2]
    # An INT64 key is read as f64 (expr.rs:232): 2^60 + 1, 2^60, 2^60 + 2 are one
    # value there, so they number in row order.
    big = np.array([2**60 + 1, 2**60, 2**60 + 2, 5], dtype=np.int64)
    db.create_table("b", {"k": big})
    assert list(db.sql("SELECT ROW_NUMBER() OVER (ORDER BY k) AS rn FROM b").column(0)) == [2, 3, 4, 1]
    with pytest.raises(F.FalconError) as e:
        db.sql("SELECT ROW_NUMBER() OVER (PARTITION BY k ORDER BY k) FROM b")
    assert e.value.code == -5
