"""GPU parity of the push-based operators (falcondb_b200.operators) against
the oracle and plain numpy, through the same C ABI kernels as the operator
layer.  The cases restate the reference's operator tests (operators.rs:250-404)
and add the config-0 query shape as a Filter -> Aggregate pipeline.  A small
chunk size (2048 rows, the reference's) exercises every chunk boundary."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops, workloads as W
from falcondb_b200.operators import (AggSpec, AggregateOp, Batch, DistinctOp, FilterOp, HashJoinProbeOp, LimitOp,
                                     Pipeline, ProjectOp, SortOp, col, tensor_column)
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CH = 2048
RTOL = 1e-12


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def vbatch(vals):
    return Batch({"v": tensor_column(dev(np.asarray(vals, dtype=np.int64)))}, len(vals))


def values(batches, name="v"):
    out = []
    for b in batches:
        out += [int(x) for x in b.column(name).to_numpy()]
    return out


def fbatch(vals):
    return Batch({"f": tensor_column(dev(np.asarray(vals, dtype=np.float64)))}, len(vals))


def fvalues(batches):
    return np.concatenate([b.column("f").to_numpy() for b in batches]) if batches else np.zeros(0)


def run(ops_, *batches):
    return Pipeline(ops_, chunk_rows=CH).run(list(batches))


def test_filter_keeps_matching_rows_and_can_match_nothing(db):
    assert values(run([FilterOp(db, col("v") > 4990)], vbatch(range(5000)))) == list(range(4991, 5000))
    assert run([FilterOp(db, col("v") > 999_999)], vbatch(range(5000))) == []


def test_filter_then_limit_and_offset(db):
    assert values(run([FilterOp(db, col("v") > 100), LimitOp(0, 3)], vbatch(range(5000)))) == [101, 102, 103]
    assert values(run([LimitOp(3000, 5)], vbatch(range(5000)))) == list(range(3000, 3005))


def test_sort_with_a_top_n_bound_across_chunks(db):
    got = run([SortOp(db, [("v", False)], 4)], vbatch(list(reversed(range(5000)))))
    assert values(got) == [0, 1, 2, 3]
    got = run([FilterOp(db, col("v") > 4995), SortOp(db, [("v", False)], 10)], vbatch(list(reversed(range(5000)))))
    assert values(got) == [4996, 4997, 4998, 4999]
    got = run([SortOp(db, [("v", True)], 10), LimitOp(0, 3)], vbatch(range(5000)))
    assert values(got) == [4999, 4998, 4997]


def test_sort_ties_follow_arrival_order(db):
    v = np.random.default_rng(3).integers(0, 5, 20_000)
    got = run([ProjectOp([("v", "k")]), SortOp(db, [("k", True)], 50)], vbatch(v))
    assert values(got, "k") == list(v[O.topk(v, 50, True)])


def test_distinct_removes_duplicates_across_chunks(db):
    got = run([DistinctOp(db, "v")], vbatch([i % 100 for i in range(5000)]))
    assert values(got) == list(range(100))


def test_sort_without_a_limit_and_above_the_top_k_bound(db):
    """SortOp with no LIMIT, or one above 4096, runs the GPU radix sort
    (try_typed_sort, sort.rs:209-350): the oracle's full sort, ties in
    arrival order."""
    v = np.random.default_rng(8).integers(0, 50, 20_000)
    got = run([SortOp(db, [("v", True)], None)], vbatch(v))
    assert values(got) == list(v[O.sort(v, True)])
    got = run([SortOp(db, [("v", False)], 10_000), LimitOp(9_990, 100)], vbatch(v))
    assert values(got) == list(v[O.sort(v, False)][9_990:10_000])
    f = np.random.default_rng(9).standard_normal(9_000)
    got = fvalues(run([SortOp(db, [("f", False)], None)], fbatch(f)))
    assert np.array_equal(got, f[O.sort(f, False)])


def test_distinct_keeps_first_occurrences_in_arrival_order(db):
    """dedup_batches (select.rs:238-457): first occurrence wins, in the order
    rows arrive across chunks; float NaNs are one value, -0.0 == +0.0."""
    v = np.random.default_rng(4).integers(0, 3000, 20_000)
    assert values(run([DistinctOp(db, "v")], vbatch(v))) == list(v[O.distinct(v)])
    f = np.array([2.5, np.nan, -0.0, 2.5, 0.0, np.nan, 1.0] * 700)
    got = fvalues(run([DistinctOp(db, "f")], fbatch(f)))
    exp = f[O.distinct(f)]
    assert len(got) == len(exp) == 4
    assert np.array_equal(got, exp, equal_nan=True)


def test_config0_filter_group_by_pipeline(db):
    """SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM t WHERE score > 50 GROUP BY dept."""
    n = 1_000_000
    t = W.table_t(n, seed=5)
    db.create_table("op_t", {"dept": t["dept"], "score": t["score"], "salary": t["salary"]})
    b = Batch.from_table(db, "op_t", ["dept", "score", "salary"])
    aggs = [AggSpec(F.AGG_COUNT_STAR, None, "count"), AggSpec(F.AGG_SUM, "score", "sum_score"),
            AggSpec(F.AGG_AVG, "salary", "avg_salary")]
    # The WHERE fused into the aggregate scan, and as a separate FilterOp stage.
    for stages in ([AggregateOp(db, aggs, group_by="dept", where=col("score") > 50)],
                   [FilterOp(db, col("score") > 50), AggregateOp(db, aggs, group_by="dept")]):
        got = Pipeline(stages, chunk_rows=1 << 18).run([b])
        assert len(got) == 1
        h = got[0].to_numpy()
        mask = O.cmp_mask(t["score"], F.GT, 50)
        g = O.group_codes(t["dept"].codes, 12, mask=mask, fvals=t["score"], ivals=t["salary"])
        present = [d for d in range(12) if g["rows"][d]]
        assert list(h["dept"]) == [W.DEPTS[d] for d in present]
        assert list(h["count"]) == [int(g["rows"][d]) for d in present]
        for j, d in enumerate(present):
            assert abs(h["sum_score"][j] - g["fsum"][d]) <= RTOL * abs(g["fsum"][d])
            assert h["avg_salary"][j] == g["isum"][d] / g["icnt"][d]
    db.drop_table("op_t")


def test_no_key_and_int64_key_aggregates(db):
    n = 300_000
    r = np.random.default_rng(9)
    k = r.integers(0, 1000, n)
    v = r.random(n)
    b = Batch({"k": tensor_column(dev(k)), "v": tensor_column(dev(v))}, n)
    got = run([AggregateOp(db, [AggSpec(F.AGG_COUNT_STAR, None, "c"), AggSpec(F.AGG_MAX, "v", "mx"),
                                AggSpec(F.AGG_SUM, "k", "sk")], where=col("v") < 0.5)], b)
    h = got[0].to_numpy()
    sel = v < 0.5
    assert int(h["c"][0]) == int(sel.sum()) and float(h["mx"][0]) == float(v[sel].max())
    assert float(h["sk"][0]) == float(k[sel].sum())
    got = run([AggregateOp(db, [AggSpec(F.AGG_COUNT_STAR, None, "c"), AggSpec(F.AGG_SUM, "v", "s"),
                                AggSpec(F.AGG_MIN, "v", "mn")], group_by="k")], b)
    h = got[0].to_numpy()
    want = O.group_i64(k, v)
    assert np.array_equal(h["k"], want["key"]) and np.array_equal(h["c"], want["count"])
    assert np.array_equal(h["mn"], want["min"])
    assert np.max(np.abs(h["s"] - want["sum"]) / np.abs(want["sum"])) <= RTOL


def test_hash_join_probe_operator(db):
    bt, pt = W.join_tables(50_000, 400_000, seed=4)
    ht = ops.HashTable(db, dev(bt["key"]), dev(bt["payload"]), len(bt["key"]))
    probe = Batch({"key": tensor_column(dev(pt["key"])), "value": tensor_column(dev(pt["value"]))}, len(pt["key"]))
    for jt in (F.JOIN_INNER, F.JOIN_LEFT, F.JOIN_SEMI, F.JOIN_ANTI):
        value = "value" if jt in (F.JOIN_SEMI, F.JOIN_ANTI) else None
        got = Pipeline([HashJoinProbeOp(db, ht, "key", jt, value=value)], chunk_rows=1 << 16).run([probe])
        h = got[0].to_numpy()
        want = O.join_agg(bt["key"], bt["payload"], pt["key"], pt["value"], jt)
        assert int(h["count"][0]) == want["count"]
        if value:
            assert abs(float(h["sum"][0]) - want["sum_value"]) <= RTOL * abs(want["sum_value"])
        else:
            assert float(h["sum"][0]) == float(want["sum_payload"])
    got = Pipeline([HashJoinProbeOp(db, ht, "key", F.JOIN_SEMI, mode="rows"), LimitOp(0, 1000)],
                   chunk_rows=1 << 16).run([probe])
    kept = np.isin(pt["key"], bt["key"])
    assert values(got, "key") == [int(x) for x in pt["key"][kept][:1000]]
    ht.free()
