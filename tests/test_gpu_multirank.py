"""Multi-rank queries through the API (falcondb_b200.distributed): two ranks,
each a process with its own context on the one GPU of this machine, each
holding a contiguous row shard; the engine's kernels produce every partial
record and the ranks combine them over gloo.  Rank 0 checks each answer
against the oracle over the whole table.  The two processes' kernels never
wait on each other: the only exchange is the host-side collectives."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    import torch.distributed as dist

    import falcondb_b200 as F
    from falcondb_b200 import distributed as D, workloads as W
    from oracle import oracle as O

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    db = F.Database(0)
    try:
        sdb = D.ShardedDatabase(db)
        n = 1_000_003
        t = W.table_t(n, seed=17)
        sdb.load("t", t)
        aggs = [(F.AGG_SUM, "score"), (F.AGG_AVG, "score"), (F.AGG_MIN, "score"), (F.AGG_MAX, "salary"),
                (F.AGG_SUM, "salary"), (F.AGG_COUNT_STAR, "score")]
        rec = sdb.aggregate("t", aggs)
        cnt = sdb.count_where("t", "score", F.GT, 50)
        nd = sdb.count_distinct("t", "dept")
        tops = {d: sdb.topk("t", "score", 10, d) for d in (True, False)}
        top_id = sdb.topk("t", "id", 10, True)
        # Join: the build side lives on rank 0 only.
        bt, pt = W.join_tables(50_000, n, seed=18)
        sdb.load("p", pt)
        jr = {jt: sdb.join_agg("p", "key", jt, probe_value="value" if jt >= F.JOIN_SEMI else None,
                               build_key=bt["key"] if rank == 0 else None,
                               build_payload=bt["payload"] if rank == 0 else None, build_rows=len(bt["key"]))
              for jt in (F.JOIN_INNER, F.JOIN_LEFT, F.JOIN_SEMI, F.JOIN_ANTI)}
        # High-cardinality GROUP BY: partials routed to their owner, gathered on rank 0.
        g = W.groupby_table(n, distinct=300_000, seed=19)
        sdb.load("g", g)
        groups = sdb.group_by_i64("g", "key", "v")
        if rank == 0:
            s = O.sum_serial(t["score"])
            assert abs(rec[0]["f"] - s) <= RTOL * s
            assert abs(rec[1]["f"] - s / n) <= 1e-11 * (s / n)
            assert rec[2]["f"] == t["score"].min() and rec[3]["f"] == t["salary"].max()
            # SUM over INT64 is a Float64 record (exact below 2^53), COUNT(*) an Int64 one.
            assert rec[4]["is_int"] == 0 and rec[4]["f"] == float(int(t["salary"].sum()))
            assert rec[5]["is_int"] == 1 and rec[5]["i"] == n
            assert cnt == O.popcount(O.cmp_mask(t["score"], F.GT, 50))
            assert nd == 12
            for d in (True, False):
                assert list(tops[d]) == list(O.topk(t["score"], 10, d))
            assert list(top_id) == list(range(n - 1, n - 11, -1))
            for jt, got in jr.items():
                want = O.join_agg(bt["key"], bt["payload"], pt["key"], pt["value"], jt)
                assert int(got[0]["count"]) == want["count"]
                if jt <= F.JOIN_LEFT:
                    assert int(got[0]["sum_payload"]) == want["sum_payload"]
                else:
                    assert abs(float(got[0]["sum_value"]) - want["sum_value"]) <= RTOL * want["sum_value"]
            want = O.group_i64(g["key"], g["v"])
            assert np.array_equal(groups["key"], want["key"]) and np.array_equal(groups["count"], want["count"])
            assert np.array_equal(groups["min"], want["min"]) and np.array_equal(groups["max"], want["max"])
            assert np.max(np.abs(groups["sum"] - want["sum"]) / np.abs(want["sum"])) <= RTOL
        else:
            assert groups is None
    finally:
        db.close()
        dist.destroy_process_group()


def test_two_ranks_through_the_api_match_the_whole_table():
    mp.start_processes(_worker, args=(2, _free_port()), nprocs=2, join=True, start_method="spawn")
