"""Serving loop (fdb_serve_trace / fdb_server_*): every answer equals the
oracle's for the query alone, whether the query ran by itself (one query at a
time), in a large batch, or in batches that formed as queries arrived; COUNT,
GROUP BY counts and integer sums and join results exactly, FP64 sums within
1e-12 relative, top-k rows exactly (ties by row ascending)."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops, serving as S, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-12
N = 2_000_003


@pytest.fixture(scope="module")
def env(db):
    t = W.table_t(N, seed=31)
    codes = t["dept"].codes
    cols = {"score": torch.from_numpy(t["score"]).cuda(), "dept": torch.from_numpy(codes.view(np.int32)).cuda(),
            "salary": torch.from_numpy(t["salary"]).cuda()}
    bt, pt = W.join_tables(100_000, N, seed=32)
    cols["pkey"] = torch.from_numpy(pt["key"]).cuda()
    cols["pval"] = torch.from_numpy(pt["value"]).cuda()
    ht = ops.HashTable(db, torch.from_numpy(bt["key"]).cuda(), torch.from_numpy(bt["payload"]).cuda(),
                       len(bt["key"]))
    torch.cuda.synchronize()
    host = {"score": t["score"], "codes": codes, "salary": t["salary"], "pkey": pt["key"], "pval": pt["value"],
            "bkey": bt["key"], "bpay": bt["payload"]}
    yield cols, ht, host
    ht.free()


def make_queries(cols, ht, nq, seed, rate=None):
    r = np.random.default_rng(seed)
    qs = []
    t = 0.0
    for i in range(nq):
        kind = int(r.integers(0, 4))
        n = int(min(N, max(1, np.floor(10 ** (1 + 5.3 * r.random())))))
        x = float(r.random() * 100)
        if rate:
            t += float(r.exponential(1.0 / rate))
        if kind == S.SERVE_COUNT:
            q = S.count_query(cols["score"].data_ptr(), n, x)
        elif kind == S.SERVE_GROUP:
            q = S.group_query(cols["score"].data_ptr(), cols["dept"].data_ptr(), cols["salary"].data_ptr(), 12, n, x)
        elif kind == S.SERVE_JOIN:
            q = S.join_query(cols["pkey"].data_ptr(), cols["pval"].data_ptr(), ht._h.value, n, x)
        else:
            q = S.topk_query(cols["score"].data_ptr(), n, x, k=int(r.choice([1, 10, 32])))
        q.arrival_s = t
        qs.append(q)
    return qs


def expect(q, host):
    n, x = q.nrows, q.threshold
    if q.kind == S.SERVE_COUNT:
        return int((host["score"][:n] > x).sum())
    if q.kind == S.SERVE_GROUP:
        sel = host["score"][:n] > x
        c = host["codes"][:n][sel]
        return (np.bincount(c, minlength=12), np.bincount(c, weights=host["score"][:n][sel], minlength=12),
                np.bincount(c, weights=host["salary"][:n][sel].astype(np.float64), minlength=12))
    if q.kind == S.SERVE_JOIN:
        pk = host["pkey"][:n][host["pval"][:n] < x / 100]
        o = O.join_agg(host["bkey"], host["bpay"], pk, np.zeros(len(pk)), F.JOIN_INNER)
        return o["count"], o["sum_payload"]
    v = host["score"][:n]
    idx = np.nonzero(v < x)[0]
    order = O.topk(v[idx], q.k, True)
    return list(idx[order])


def check(q, r, host):
    assert r.status == 0
    want = expect(q, host)
    if q.kind == S.SERVE_COUNT:
        assert r.count == want
    elif q.kind == S.SERVE_GROUP:
        cnt, s0, s2 = want
        assert list(r.group_count[:12]) == list(cnt)
        assert list(r.group_sum2[:12]) == [int(v) for v in s2]  # integer sums, exact
        for g in range(12):
            assert abs(r.group_sum0[g] - s0[g]) <= RTOL * max(abs(s0[g]), 1e-300)
    elif q.kind == S.SERVE_JOIN:
        assert (r.count, r.sum_payload) == want
    else:
        assert r.count == len(want) and list(r.rows[:r.count]) == want


def test_serve_alone_in_a_batch_and_as_they_arrive(db, env):
    cols, ht, host = env
    qs = make_queries(cols, ht, 160, seed=1)
    serial, st1 = S.serve_trace(db, qs, max_batch=1, slots=1)
    batched, st2 = S.serve_trace(db, qs, max_batch=128, slots=4)
    assert st1.mean_batch == 1 and st2.mean_batch > 1
    for q, a, b in zip(qs, serial, batched):
        check(q, a, host)
        check(q, b, host)
    arriving = make_queries(cols, ht, 160, seed=1, rate=4000.0)  # same queries, Poisson arrivals
    res, st3 = S.serve_trace(db, arriving, max_batch=64, slots=3)
    for q, r in zip(arriving, res):
        check(q, r, host)
        assert r.done_s >= r.start_s >= r.arrival_s - 1e-6
    assert st3.p99_ms >= st3.p50_ms > 0


def test_serve_memory_budget_limits_batches(db, env):
    cols, ht, host = env
    qs = make_queries(cols, ht, 40, seed=2)
    _, st = S.serve_trace(db, qs, max_batch=128, slots=1)
    res, st_small = S.serve_trace(db, qs, max_batch=128, slots=1, mem_budget=st.resident_bytes + 4096)
    assert st_small.mean_batch < st.mean_batch
    for q, r in zip(qs, res):
        check(q, r, host)


def test_online_server_submit_wait(db, env):
    cols, ht, host = env
    qs = make_queries(cols, ht, 30, seed=3)
    srv = S.Server(db, max_batch=16, slots=2)
    tickets = [srv.submit(q) for q in qs]
    for q, t in zip(qs, tickets):
        check(q, srv.wait(t, timeout_s=30.0), host)
    with pytest.raises(F.FalconError):
        srv.wait(tickets[0], timeout_s=0.0)  # a ticket is handed out once
    st = srv.stop()
    assert st.batches >= 1 and st.qps > 0


def test_serve_join_on_a_hashed_table(db, env):
    """JOIN queries served over a table whose keys hash (they span far more
    values than it has slots); the fixture's table is direct-addressed."""
    cols, ht, host = env
    bkey = host["bkey"] * 7919 + 3
    pkey = host["pkey"] * 7919 + 3
    hh = ops.HashTable(db, torch.from_numpy(bkey).cuda(), torch.from_numpy(host["bpay"]).cuda(), len(bkey))
    assert ht.dense and not hh.dense
    dpk = torch.from_numpy(pkey).cuda()
    r = np.random.default_rng(77)
    qs = []
    for i in range(24):
        n = int(min(N, max(1, np.floor(10 ** (1 + 5.3 * r.random())))))
        qs.append(S.join_query(dpk.data_ptr(), cols["pval"].data_ptr(), hh._h.value, n, float(r.random() * 100)))
    # Batches of up to 16 (groups of several queries probe once and share the
    # result), then one query at a time (a one-query group filters, probes and
    # counts in one pass).
    for mb in (16, 1):
        res, _ = S.serve_trace(db, qs, max_batch=mb, slots=1)
        for q, rr in zip(qs, res):
            assert rr.status == 0
            sel = pkey[:q.nrows][host["pval"][:q.nrows] < q.threshold / 100]
            o = O.join_agg(bkey, host["bpay"], sel, np.zeros(len(sel)), F.JOIN_INNER)
            assert (rr.count, rr.sum_payload) == (o["count"], o["sum_payload"])
    hh.free()


def test_serve_many_group_queries_in_one_batch(db, env):
    """40 GROUP queries in one batch: up to 32 that cover a whole unit are
    answered together by threshold rank, the rest one by one.  Thresholds
    repeat and reach both ends of the score range, prefixes differ (so queries
    cover units partly) and two dictionary sizes are mixed; every answer must
    match the query run alone."""
    cols, ht, host = env
    r = np.random.default_rng(40)
    thr = [50.0, 50.0, 50.0, -1.0, 100.0, 0.0, 99.9] + [float(x) for x in r.random(33) * 100]
    qs = []
    for i, x in enumerate(thr):
        n = N if i % 3 else int(r.integers(1, N))
        dict_len = 12 if i % 5 else 7
        qs.append(S.group_query(cols["score"].data_ptr(), cols["dept"].data_ptr(), cols["salary"].data_ptr(),
                                dict_len, n, x))
    res, st = S.serve_trace(db, qs, max_batch=64, slots=1)
    assert st.batches >= 1
    for q, rr in zip(qs, res):
        assert rr.status == 0
        n, x, d = q.nrows, q.threshold, q.dict_len
        sel = host["score"][:n] > x
        c = host["codes"][:n][sel]
        keep = c < d
        c = c[keep]
        cnt = np.bincount(c, minlength=16)
        s0 = np.bincount(c, weights=host["score"][:n][sel][keep], minlength=16)
        s2 = np.bincount(c, weights=host["salary"][:n][sel][keep].astype(np.float64), minlength=16)
        assert list(rr.group_count[:16]) == list(cnt)
        assert list(rr.group_sum2[:16]) == [int(v) for v in s2]
        for gi in range(16):
            assert abs(rr.group_sum0[gi] - s0[gi]) <= RTOL * max(abs(s0[gi]), 1e-300)


def test_serve_many_count_and_join_queries_in_one_batch(db, env):
    """40 COUNT and 40 JOIN queries in one batch: those covering a whole unit
    are answered together by threshold rank (a suffix sum of binned rows for
    COUNT, a prefix sum for JOIN's value < limit), the rest one by one.
    Thresholds repeat and reach both ends; prefixes differ."""
    cols, ht, host = env
    r = np.random.default_rng(41)
    thr = [50.0, 50.0, 50.0, -1.0, 100.0, 0.0, 99.9, 100.5] + [float(x) for x in r.random(32) * 100]
    qs = []
    for i, x in enumerate(thr):
        n = N if i % 3 else int(r.integers(1, N))
        qs.append(S.count_query(cols["score"].data_ptr(), n, x))
        qs.append(S.join_query(cols["pkey"].data_ptr(), cols["pval"].data_ptr(), ht._h.value, n, x))
    res, _ = S.serve_trace(db, qs, max_batch=128, slots=1)
    for q, rr in zip(qs, res):
        check(q, rr, host)
