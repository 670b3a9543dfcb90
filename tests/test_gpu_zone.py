"""Zone maps on the GPU (stats.rs:22-113; execute_select's batch skip,
select.rs:115-137): the maps computed at load against the oracle, batch
pruning through fdb_zone_skip against the oracle, SQL answers identical with
pruning on and off (and to the oracle), and the int64-key GROUP BY taking its
key range from the zone map with the same answer as the sizing pass."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops
from oracle import oracle as O

pytestmark = pytest.mark.gpu
BR = F.ZONE_BATCH_ROWS


def masked(values, valid):
    return np.ma.masked_array(values, mask=~valid)


def words_of(valid):
    w = np.packbits(valid, bitorder="little")
    return np.concatenate([w, np.zeros((-len(w)) % 8, np.uint8)]).view(np.uint64)


def same_zone(got, want, kind):
    assert len(got) == len(want)
    for f in ("null_count", "rows", "flags"):
        assert np.array_equal(got[f], want[f]), f
    has = (want["flags"] & O.ZONE_VALUES) != 0
    if kind == "float":
        assert np.array_equal(got["min_f"][has], want["min_f"][has])
        assert np.array_equal(got["max_f"][has], want["max_f"][has])
    else:
        assert np.array_equal(got["min_i"][has], want["min_i"][has])
        assert np.array_equal(got["max_i"][has], want["max_i"][has])


@pytest.fixture
def zt(db):
    """3 batches and a ragged tail: a sorted id, a float with NULLs, NaN and
    +-inf, a text column with NULL codes and a batch that is all NULL."""
    rng = np.random.default_rng(3)
    n = 3 * BR + 1234
    ident = np.arange(n, dtype=np.int64) * 3 - 1000
    f = rng.normal(0, 10, n)
    f[rng.random(n) < 0.001] = np.nan
    f[7] = np.inf
    f[BR + 5] = -np.inf
    fvalid = rng.random(n) >= 0.01
    fvalid[2 * BR:3 * BR] = False                       # batch 2: all NULL
    codes = rng.integers(0, 5, n).astype(np.uint32)
    codes[:BR] = rng.integers(0, 2, BR)                 # batch 0: codes 0..1 only
    codes[rng.random(n) < 0.01] = 0xFFFFFFFF
    dictionary = ["a", "b", "c", "d", "e"]
    db.create_table("z", {"id": ident, "f": masked(f, fvalid), "s": F.Utf8(codes, dictionary)})
    return dict(n=n, id=ident, f=f, fvalid=fvalid, codes=codes, dict=dictionary)


def test_zone_maps_match_the_oracle(db, zt):
    same_zone(db.zone_map("z", "id"), O.zone_map(zt["id"], "int"), "int")
    same_zone(db.zone_map("z", "f"), O.zone_map(zt["f"], "float", words_of(zt["fvalid"])), "float")
    same_zone(db.zone_map("z", "s"), O.zone_map(zt["codes"], "code"), "code")
    zf = db.zone_map("z", "f")
    assert zf["flags"][2] == 0 and zf["null_count"][2] == BR   # the all-NULL batch
    assert zf["max_f"][0] == np.inf and zf["min_f"][1] == -np.inf


def test_empty_and_replaced_tables(db):
    db.create_table("e", {"x": np.zeros(0, dtype=np.int64)})
    assert len(db.zone_map("e", "x")) == 0
    assert col(db.sql("SELECT COUNT(*) FROM e WHERE x > 3"), 0) == [0]
    a = np.arange(BR + 10, dtype=np.int64)
    db.create_table("r", {"x": a})
    assert db.zone_map("r", "x")["max_i"][1] == BR + 9
    db.create_table("r", {"x": a + 100})                    # same layout: overwritten in place
    z = db.zone_map("r", "x")
    assert (z["min_i"][0], z["max_i"][1]) == (100, BR + 109)
    assert col(db.sql("SELECT COUNT(*) FROM r WHERE x < 100"), 0) == [0]


def test_zone_skip_matches_the_oracle(db, zt):
    dev = torch.device("cuda", 0)
    t_set, keep = ops.code_set(2, [False, True, False, False, False], dev)   # s = 'b'
    programs = [
        ([ops.cmp(0, F.GE, int(zt["id"][2 * BR]))], [dict(kind=O.T_CMP, col=0, op=O.GE, lit=int(zt["id"][2 * BR]))]),
        ([ops.cmp(0, F.LT, 5.5)], [dict(kind=O.T_CMP, col=0, op=O.LT, lit=5.5, lit_float=True)]),
        ([ops.cmp(1, F.GT, 1e9)], [dict(kind=O.T_CMP, col=1, op=O.GT, lit=1e9, lit_float=True)]),
        ([ops.cmp(1, F.NE, 0.0)], [dict(kind=O.T_CMP, col=1, op=O.NE, lit=0.0, lit_float=True)]),
        ([ops.is_not_null(1)], [dict(kind=O.T_IS_NOT_NULL, col=1)]),
        ([ops.is_null(0)], [dict(kind=O.T_IS_NULL, col=0)]),
        ([t_set], [dict(kind=O.T_CODE_SET, col=2, set={1}, dict_len=5)]),
        ([ops.cmp(0, F.GE, int(zt["id"][BR])), ops.cmp(1, F.GT, 1e9), ops.OR()],
         [dict(kind=O.T_CMP, col=0, op=O.GE, lit=int(zt["id"][BR])),
          dict(kind=O.T_CMP, col=1, op=O.GT, lit=1e9, lit_float=True), dict(kind=O.T_OR)]),
        ([ops.cmp(0, F.LT, int(zt["id"][BR])), ops.is_null(1), ops.AND()],
         [dict(kind=O.T_CMP, col=0, op=O.LT, lit=int(zt["id"][BR])), dict(kind=O.T_IS_NULL, col=1),
          dict(kind=O.T_AND)]),
    ]
    zones = [O.zone_map(zt["id"], "int"), O.zone_map(zt["f"], "float", words_of(zt["fvalid"])),
             O.zone_map(zt["codes"], "code")]
    kinds = ["int", "float", "code"]
    fired = 0
    for prog, oterms in programs:
        got = db.zone_skip("z", ["id", "f", "s"], prog)
        want = O.zone_rule_out(zones, kinds, oterms)
        assert np.array_equal(got, want), oterms
        fired += int(got.sum())
    assert fired >= 6
    del keep


def sql_both(db, q):
    """The query with zone maps on, then off: (result on, scanned rows on)."""
    db.set_option("zone_maps", 1)
    on = db.sql(q)
    scanned = db.last_scan_rows
    db.set_option("zone_maps", 0)
    off = db.sql(q)
    db.set_option("zone_maps", 1)
    assert on.row_count() == off.row_count() and on.columns == off.columns, q
    for c in range(len(on.columns)):
        for r in range(on.row_count()):
            x, y = on.value(r, c), off.value(r, c)
            if isinstance(x, float) and isinstance(y, float):
                # FP64 sums: the scanned range changes how rows split over
                # CTAs, so the summation order (1e-12 relative).
                assert abs(x - y) <= 1e-12 * max(abs(x), abs(y)) or (x != x and y != y), (q, x, y)
            else:
                assert x == y, (q, x, y)
    return on, scanned


def col(res, c):
    return [res.value(r, c) for r in range(res.row_count())]


def test_sql_answers_with_pruning(db):
    n = 20 * BR + 77
    rng = np.random.default_rng(9)
    ident = np.arange(n, dtype=np.int64)
    score = rng.random(n) * 100
    codes = rng.integers(0, 12, n).astype(np.uint32)
    depts = [f"d{i:02d}" for i in range(12)]
    db.create_table("t", {"id": ident, "score": score, "dept": F.Utf8(codes, depts)})

    lo = 18 * BR + 5
    res, scanned = sql_both(db, f"SELECT COUNT(*) FROM t WHERE id >= {lo}")
    assert col(res, 0) == [n - lo] and scanned == n - 18 * BR

    res, scanned = sql_both(db, f"SELECT SUM(score), MIN(score), COUNT(*) FROM t WHERE id < {BR + 3} AND score > 50")
    sel = (ident < BR + 3) & (score > 50)
    assert col(res, 2) == [int(sel.sum())] and scanned == 2 * BR
    assert abs(col(res, 0)[0] - O.sum_serial(score[sel])) <= 1e-12 * col(res, 0)[0]
    assert col(res, 1)[0] == score[sel].min()

    q = f"SELECT dept, COUNT(*), SUM(score) FROM t WHERE id >= {5 * BR} AND id < {7 * BR - 1} GROUP BY dept ORDER BY dept"
    res, scanned = sql_both(db, q)
    sel = (ident >= 5 * BR) & (ident < 7 * BR - 1)
    assert scanned == 2 * BR
    assert col(res, 1) == [int(((codes == i) & sel).sum()) for i in range(12)]

    q = f"SELECT id, score FROM t WHERE id > {n - 100} ORDER BY score DESC LIMIT 5"
    res, scanned = sql_both(db, q)
    tail = np.arange(n - 99, n)
    want = tail[np.argsort(-score[tail], kind="stable")][:5]
    assert col(res, 0) == want.tolist() and scanned == BR + 77   # batches 19 and 20

    res, scanned = sql_both(db, "SELECT DISTINCT dept FROM t WHERE id < 10 ORDER BY dept")
    assert col(res, 0) == sorted({depts[c] for c in codes[:10]}) and scanned == BR

    # Nothing can pass: every batch is ruled out.
    res, scanned = sql_both(db, "SELECT COUNT(*), SUM(score) FROM t WHERE id > 1000000000")
    assert col(res, 0) == [0] and col(res, 1) == [None] and scanned == 0
    res, _ = sql_both(db, "SELECT id FROM t WHERE id < -5")
    assert res.row_count() == 0
    res, _ = sql_both(db, "SELECT dept, COUNT(*) FROM t WHERE id < -5 GROUP BY dept")
    assert res.row_count() == 0

    # Text predicates rule batches out through their code range.
    one = np.zeros(n, dtype=np.uint32)
    one[3 * BR:3 * BR + 10] = 1
    db.create_table("u", {"id": ident, "s": F.Utf8(one, ["x", "y"])})
    res, scanned = sql_both(db, "SELECT COUNT(*) FROM u WHERE s = 'y'")
    assert col(res, 0) == [10] and scanned == BR
    res, scanned = sql_both(db, "SELECT COUNT(*) FROM u WHERE s IN ('y') OR id < 3")
    assert col(res, 0) == [13] and scanned == 4 * BR

    # No WHERE, or a WHERE that rules nothing out: the whole table.
    _, scanned = sql_both(db, "SELECT COUNT(*) FROM t WHERE score > 50")
    assert scanned == n


def test_group_by_key_range_from_zone_maps(db):
    rng = np.random.default_rng(5)
    n = 4 * BR + 999
    keys = rng.integers(-2000, 3000, n).astype(np.int64)
    vals = rng.normal(0, 1, n)
    db.create_table("g", {"k": keys, "v": vals})
    k, v = db.column("g", "k"), db.column("g", "v")
    got = {}
    for on in (1, 0):
        db.set_option("zone_maps", on)
        out, ng = ops.group_by_i64(db, k, v, n)
        got[on] = ops.to_records(out, F.GROUP_I64_DTYPE, int(ng.item()))
    db.set_option("zone_maps", 1)
    assert np.array_equal(got[1]["key"], got[0]["key"]) and np.array_equal(got[1]["count"], got[0]["count"])
    assert np.array_equal(got[1]["min"], got[0]["min"]) and np.array_equal(got[1]["max"], got[0]["max"])
    assert np.allclose(got[1]["sum"], got[0]["sum"], rtol=1e-12, atol=1e-12)
    gk, cnt = np.unique(keys, return_counts=True)
    assert np.array_equal(got[1]["key"], gk) and np.array_equal(got[1]["count"], cnt)
    # A view of the rows from batch 2 on (a pointer into the column).
    view = F.DevColumn(ops.dev_column(k), n - 2 * BR)
    view.raw.values = k.raw.values + 2 * BR * 8
    vv = F.DevColumn(ops.dev_column(v), n - 2 * BR)
    vv.raw.values = v.raw.values + 2 * BR * 8
    out, ng = ops.group_by_i64(db, view, vv, n - 2 * BR)
    rec = ops.to_records(out, F.GROUP_I64_DTYPE, int(ng.item()))
    gk, cnt = np.unique(keys[2 * BR:], return_counts=True)
    assert np.array_equal(rec["key"], gk) and np.array_equal(rec["count"], cnt)
    # Through SQL.
    res = db.sql("SELECT k, COUNT(*), MAX(v) FROM g GROUP BY k ORDER BY k")
    gk, cnt = np.unique(keys, return_counts=True)
    assert col(res, 0) == gk.tolist() and col(res, 1) == cnt.tolist()
