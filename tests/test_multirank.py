"""Multi-rank combine logic (falcondb_b200.shard) with two gloo ranks on CPU.

Each rank takes its contiguous shard of seeded data, computes the partial a
GPU would produce for it (here with the oracle, on the host), and the ranks
combine through torch.distributed.  Rank 0 checks the combined answer against
the oracle over the whole input: counts, integer sums, top-k rows, join
results and GROUP BY keys/counts/MIN/MAX exactly, FP64 sums within 1e-12."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

RTOL = 1e-12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ord_keys(v, desc):
    b = v.view(np.uint64)
    k = np.where(b >> np.uint64(63), ~b, b ^ np.uint64(1 << 63))
    return ~k if desc else k


def _agg_record(func, values, is_int):
    """A partial in the layout fdb_aggregate writes (k_scan.cu): COUNT /
    COUNT(*) as Int64 records (`i`, is_int 1); SUM, AVG, MIN and MAX as
    Float64 records (`f`, is_int 0), an INT64 SUM being its exact total
    converted to f64 (the reference types SUM as Float64)."""
    from oracle import oracle as O

    import falcondb_b200 as F
    rec = np.zeros(1, dtype=F.AGG_VALUE_DTYPE)[0]
    val, cnt = O.agg(func, values)
    rec["n"] = cnt
    if func in (F.AGG_COUNT_STAR, F.AGG_COUNT):
        rec["is_int"] = 1
        rec["i"] = cnt
        rec["valid"] = 1
    elif val is not None:
        rec["valid"] = 1
        if func == F.AGG_SUM and is_int:
            rec["f"] = float(int(O.sum_i64_exact(values)))
        else:
            rec["f"] = val
    return rec


def _worker(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import falcondb_b200 as F
    from falcondb_b200 import shard, workloads as W
    from oracle import oracle as O

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 200_003
        t = W.table_t(n, seed=7)
        s0, cnt = shard.shard_range(n, rank, world)
        sl = slice(s0, s0 + cnt)

        # No-key aggregates.
        funcs = [F.AGG_COUNT_STAR, F.AGG_SUM, F.AGG_AVG, F.AGG_MIN, F.AGG_MAX]
        local = np.array([_agg_record(f, t["score"][sl], False) for f in funcs], dtype=F.AGG_VALUE_DTYPE)
        got = shard.combine_aggregates(local, funcs)
        isum = shard.combine_aggregates(np.array([_agg_record(F.AGG_SUM, t["salary"][sl], True)],
                                                 dtype=F.AGG_VALUE_DTYPE), [F.AGG_SUM])
        # Top-k over global rows.
        for desc in (True, False):
            rows = O.topk(t["score"][sl], 10, desc) + s0
            keys = _ord_keys(t["score"][rows], desc)
            gk, gr = shard.combine_topk(keys, rows, 10)
            if rank == 0:
                assert list(gr) == list(O.topk(t["score"], 10, desc))
        # Join: build side replicated from rank 0, probe sharded.
        bt, pt = W.join_tables(20_000, n, seed=3)
        import torch
        bk, bp = shard.broadcast_columns([torch.from_numpy(bt["key"]) if rank == 0 else None,
                                          torch.from_numpy(bt["payload"]) if rank == 0 else None],
                                         [len(bt["key"])] * 2, [torch.int64] * 2)
        assert np.array_equal(bk.numpy(), bt["key"])
        jl = O.join_agg(bk.numpy(), bp.numpy(), pt["key"][sl], pt["value"][sl], F.JOIN_INNER)
        jrec = np.zeros(1, dtype=F.JOIN_AGG_DTYPE)
        for f in ("count", "sum_payload", "payload_rows", "sum_value"):
            jrec[0][f] = jl[f]
        jg = shard.combine_join(jrec)
        # High-cardinality GROUP BY: exchange by key owner, then gather.
        g = W.groupby_table(n, distinct=50_000, seed=5)
        part = O.group_i64(g["key"][sl], g["v"][sl])
        recs = np.zeros(len(part["key"]), dtype=F.GROUP_I64_DTYPE)
        for f in ("key", "count", "sum", "min", "max"):
            recs[f] = part[f]
        mine = shard.exchange_groups(recs)
        owners = shard._owner(mine["key"], world)
        assert np.all(owners == rank)  # each rank holds only the keys it owns
        allg = shard.gather_groups(mine)

        if rank == 0:
            for j, f in enumerate(funcs):
                want, c = O.agg(f, t["score"])
                if f == F.AGG_COUNT_STAR:
                    assert got[j]["i"] == n
                elif f in (F.AGG_MIN, F.AGG_MAX):
                    assert got[j]["f"] == want
                else:
                    assert abs(got[j]["f"] - want) <= RTOL * abs(want)
            assert isum[0]["f"] == float(int(O.sum_i64_exact(t["salary"])))
            jw = O.join_agg(bt["key"], bt["payload"], pt["key"], pt["value"], F.JOIN_INNER)
            assert (int(jg[0]["count"]), int(jg[0]["sum_payload"])) == (jw["count"], jw["sum_payload"])
            want = O.group_i64(g["key"], g["v"])
            assert np.array_equal(allg["key"], want["key"]) and np.array_equal(allg["count"], want["count"])
            assert np.array_equal(allg["min"], want["min"]) and np.array_equal(allg["max"], want["max"])
            assert np.max(np.abs(allg["sum"] - want["sum"]) / np.abs(want["sum"])) <= RTOL
    finally:
        dist.destroy_process_group()


def test_shard_ranges_cover_every_row():
    from falcondb_b200 import shard

    for n in (0, 1, 7, 100_003):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_range(n, r, world) for r in range(world)]
            assert sum(c for _, c in parts) == n
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(world - 1))


def test_two_rank_combines_match_the_whole_input():
    mp.start_processes(_worker, args=(2, _free_port()), nprocs=2, join=True, start_method="spawn")
