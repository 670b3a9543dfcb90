"""Parity at the benchmark configurations' full sizes.

The other GPU tests hold the kernels to the oracle on inputs the oracle
finishes in seconds.  These run the same comparisons at the sizes the
benchmark measures, so that every path the full sizes reach is pinned: the
100M-row streamed scans and top-k sample bounds, the join probe over 100M
rows against both table kinds, the HyperLogLog-sized global table of the
100M-row Zipf GROUP BY (about 4.85M groups), and the serving loop over
100M-row tables with batches of mixed sizes.

Bars, as everywhere: counts, COUNT(DISTINCT), integer sums, MIN/MAX, join
counts and integer payload sums, and top-k row lists (ties by row ascending)
bit-exact; FP64 SUM/AVG within 1e-12 relative of the serial FP64 oracle.
Each test takes tens of seconds (data generation and the oracle on the
host dominate)."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops, serving as S, workloads as W
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
RTOL = 1e-12
N = 100_000_000


def close(got, want):
    return abs(got - want) <= RTOL * abs(want)


def test_config1_scan_and_topk_100M(db):
    """SUM(score); COUNT(*) WHERE score > 50; COUNT(DISTINCT dept);
    ORDER BY score DESC LIMIT 10; ORDER BY id DESC LIMIT 10 over 100M rows,
    through Database::sql."""
    t = W.table_t(N, seed=1)
    db.create_table("t", t)
    try:
        s = db.sql("SELECT SUM(score) FROM t").column(0)[0]
        assert close(s, O.sum_serial(t["score"]))
        c = db.sql("SELECT COUNT(*) FROM t WHERE score > 50").column(0)[0]
        assert c == O.popcount(O.cmp_mask(t["score"], F.GT, 50))
        d = db.sql("SELECT COUNT(DISTINCT dept) FROM t").column(0)[0]
        assert d == int(O.present_codes(t["dept"].codes, 12).sum())
        top = db.sql("SELECT id, score FROM t ORDER BY score DESC LIMIT 10")
        rows = O.topk(t["score"], 10, True)
        assert list(top.column(0)) == list(t["id"][rows])
        assert list(top.column(1)) == list(t["score"][rows])
        top_id = db.sql("SELECT id FROM t ORDER BY id DESC LIMIT 10")
        assert list(top_id.column(0)) == list(t["id"][O.topk(t["id"], 10, True)])
        # The ascending sides and a larger k reach the other top-k kernels.
        lo = db.sql("SELECT id FROM t ORDER BY score ASC LIMIT 100")
        assert list(lo.column(0)) == list(O.topk(t["score"], 100, False))
    finally:
        db.drop_table("t")


@pytest.mark.parametrize("hashed", [False, True], ids=["dense_table", "hashed_table"])
def test_config2_joins_1M_x_100M(db, hashed):
    """INNER / LEFT with COUNT(*), SUM(b.payload); SEMI / ANTI (EXISTS / NOT
    EXISTS) with COUNT(*), SUM(value) over a 1M-row build side and a 100M-row
    probe side.  The configuration's keys make a direct-addressed table; the
    same keys scattered (x 7919 + 3) make a hashed one."""
    b, p = W.join_tables(1_000_000, N, seed=7)
    if hashed:
        b["key"] = b["key"] * 7919 + 3
        p["key"] = p["key"] * 7919 + 3
    db.create_table("b", b)
    db.create_table("p", p)
    try:
        for sql, jt in [("SELECT COUNT(*), SUM(b.payload) FROM p JOIN b ON p.key = b.key", F.JOIN_INNER),
                        ("SELECT COUNT(*), SUM(b.payload) FROM p LEFT JOIN b ON p.key = b.key", F.JOIN_LEFT)]:
            r = db.sql(sql)
            want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
            assert r.column(0)[0] == want["count"]
            assert r.column(1)[0] == float(want["sum_payload"])
        for sql, jt in [("SELECT COUNT(*), SUM(value) FROM p WHERE EXISTS (SELECT 1 FROM b WHERE b.key = p.key)",
                         F.JOIN_SEMI),
                        ("SELECT COUNT(*), SUM(value) FROM p WHERE NOT EXISTS "
                         "(SELECT 1 FROM b WHERE b.key = p.key)", F.JOIN_ANTI)]:
            r = db.sql(sql)
            want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
            assert r.column(0)[0] == want["count"]
            assert close(r.column(1)[0], want["sum_value"])
    finally:
        db.drop_table("b")
        db.drop_table("p")


def test_config3_zipf_group_by_100M(db):
    """GROUP BY key with COUNT(*), SUM(v), MIN(v), MAX(v) over 100M rows of
    Zipf(1.1) keys on a 10M-value domain, through Database::sql (the global
    table sized from a HyperLogLog estimate): every group's key, count, MIN
    and MAX exactly, every SUM within 1e-12."""
    g = W.groupby_table(N, distinct=10_000_000, seed=11)
    db.create_table("g", g)
    try:
        r = db.sql("SELECT key, COUNT(*), SUM(v), MIN(v), MAX(v) FROM g GROUP BY key ORDER BY key")
        want = O.group_i64(g["key"], g["v"])
        assert r.row_count() == len(want["key"])
        assert len(want["key"]) > 4_000_000
        assert np.array_equal(np.asarray(r.column(0)), want["key"])
        assert np.array_equal(np.asarray(r.column(1)), want["count"])
        rel = np.abs(np.asarray(r.column(2)) - want["sum"]) / np.abs(want["sum"])
        assert rel.max() <= RTOL
        assert np.array_equal(np.asarray(r.column(3)), want["min"])
        assert np.array_equal(np.asarray(r.column(4)), want["max"])
    finally:
        db.drop_table("g")


def test_config0_filter_group_by_100M(db):
    """The filter -> GROUP BY dept query of the CPU configuration at 100M
    rows (the fused lane kernel's large launch shape)."""
    t = W.table_t(N, seed=3)
    db.create_table("t", t)
    try:
        res = db.sql("SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM t WHERE score > 50 "
                     "GROUP BY dept ORDER BY dept")
        mask = O.cmp_mask(t["score"], F.GT, 50)
        g = O.group_codes(t["dept"].codes, 12, mask=mask, fvals=t["score"], ivals=t["salary"])
        assert res.column(0) == W.DEPTS
        for i in range(12):
            assert res.column(1)[i] == g["rows"][i]
            assert close(res.column(2)[i], g["fsum"][i])
            assert res.column(3)[i] == g["isum"][i] / g["icnt"][i]
    finally:
        db.drop_table("t")


def test_config4_serving_mix_100M_alone_and_batched(db):
    """The serving mix over 100M-row resident tables (the four templates,
    table prefixes log-uniform in 10k..100M rows, thresholds uniform in
    [0, 100)): each answer equals the oracle's, run one query at a time and
    in continuous batches."""
    t = W.table_t(N, seed=31)
    codes = t["dept"].codes
    cols = {"score": torch.from_numpy(t["score"]).cuda(), "dept": torch.from_numpy(codes.view(np.int32)).cuda(),
            "salary": torch.from_numpy(t["salary"]).cuda()}
    bt, pt = W.join_tables(1_000_000, N, seed=32)
    cols["pkey"] = torch.from_numpy(pt["key"]).cuda()
    cols["pval"] = torch.from_numpy(pt["value"]).cuda()
    ht = ops.HashTable(db, torch.from_numpy(bt["key"]).cuda(), torch.from_numpy(bt["payload"]).cuda(),
                       len(bt["key"]))
    torch.cuda.synchronize()
    try:
        r = np.random.default_rng(2000)
        qs = []
        for i in range(96):
            kind = i % 4
            n = int(min(N, np.floor(10 ** (4 + 4 * r.random()))))
            x = float(r.random() * 100)
            if kind == S.SERVE_COUNT:
                q = S.count_query(cols["score"].data_ptr(), n, x)
            elif kind == S.SERVE_GROUP:
                q = S.group_query(cols["score"].data_ptr(), cols["dept"].data_ptr(), cols["salary"].data_ptr(),
                                  12, n, x)
            elif kind == S.SERVE_JOIN:
                q = S.join_query(cols["pkey"].data_ptr(), cols["pval"].data_ptr(), ht._h.value, n, x)
            else:
                q = S.topk_query(cols["score"].data_ptr(), n, x, k=10)
            qs.append(q)
        alone, st1 = S.serve_trace(db, qs, max_batch=1, slots=1)
        batched, st2 = S.serve_trace(db, qs, max_batch=128, slots=2)
        assert st1.mean_batch == 1 and st2.mean_batch > 1
        score, sal, pk, pv = t["score"], t["salary"], pt["key"], pt["value"]
        for q, a, bres in zip(qs, alone, batched):
            assert a.status == 0 and bres.status == 0
            n, x = q.nrows, q.threshold
            if q.kind == S.SERVE_COUNT:
                want = int((score[:n] > x).sum())
                assert a.count == want and bres.count == want
            elif q.kind == S.SERVE_GROUP:
                sel = score[:n] > x
                c = codes[:n][sel]
                cnt = np.bincount(c, minlength=12)
                s2 = np.bincount(c, weights=sal[:n][sel].astype(np.float64), minlength=12)
                # bincount adds each group's weights one by one in row order:
                # the serial FP64 sum per group.
                s0 = np.bincount(c, weights=score[:n][sel], minlength=12)
                for rr in (a, bres):
                    assert list(rr.group_count[:12]) == list(cnt)
                    assert list(rr.group_sum2[:12]) == [int(v) for v in s2]
                    for gi in range(12):
                        assert abs(rr.group_sum0[gi] - s0[gi]) <= RTOL * max(abs(s0[gi]), 1e-300)
            elif q.kind == S.SERVE_JOIN:
                keys = pk[:n][pv[:n] < x / 100]
                o = O.join_agg(bt["key"], bt["payload"], keys, np.zeros(len(keys)), F.JOIN_INNER)
                assert (a.count, a.sum_payload) == (o["count"], o["sum_payload"])
                assert (bres.count, bres.sum_payload) == (o["count"], o["sum_payload"])
            else:
                idx = np.nonzero(score[:n] < x)[0]
                want = list(idx[O.topk(score[:n][idx], q.k, True)])
                for rr in (a, bres):
                    assert rr.count == len(want) and list(rr.rows[:rr.count]) == want
    finally:
        ht.free()
        del cols
        torch.cuda.empty_cache()
