"""Multi-GPU queries through the operator API: one process per GPU, every
table split into contiguous row shards (one per rank), the single-GPU kernels
run on the local shard, and the engine's own partial records combined with
the exchange steps of :mod:`falcondb_b200.shard`.

The reference runs in one process (rayon threads over 65,536-row batches); a
query here gives the same answer as the same query on one GPU over the whole
table: counts, integer sums, top-k rows, join results and GROUP BY groups
exactly, FP64 sums within 1e-12 relative (partials are folded in rank order,
so they are repeatable too).  No kernel reads another GPU's memory: the
exchanges are NCCL (or, in host tests, gloo) collectives of a few KB per
query, plus the join build side broadcast once and the GROUP BY partials
routed to their owner rank.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from . import AGG_COUNT_STAR, AGG_VALUE_DTYPE, FLOAT64, GROUP_I64_DTYPE, JOIN_AGG_DTYPE, Database, Utf8, fdb_pred_term
from . import ops, shard

__all__ = ["ShardedDatabase", "order_keys"]


def order_keys(values: np.ndarray, desc: bool) -> np.ndarray:
    """The top-k's order keys of FLOAT64 / INT64 values (f64_ord_key,
    src/query/sort.rs:451-454; the sign flip for int64; NOT for DESC)."""
    v = np.ascontiguousarray(values)
    b = v.view(np.uint64)
    if v.dtype.kind == "f":
        k = np.where(b >> np.uint64(63), ~b, b ^ np.uint64(1 << 63))
    else:
        k = b ^ np.uint64(1 << 63)
    return ~k if desc else k


class ShardedDatabase:
    """A GPU context per rank over this rank's row shard of every table.

    ``load(name, columns)`` takes the whole table's host columns on every rank
    (or only this rank's rows, with ``total_rows``) and keeps rows
    ``shard_range(n, rank, world)`` resident on this rank's GPU.  Query
    methods return the global answer on every rank (GROUP BY: on rank ``dst``).
    """

    def __init__(self, db: Database, group=None):
        self.db = db
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self._rows: Dict[str, Tuple[int, int]] = {}  # table -> (first global row, local rows)
        self._dicts: Dict[Tuple[str, str], List[str]] = {}

    # ------------------------------------------------------------------ tables
    def load(self, name: str, columns: Dict[str, object], total_rows: Optional[int] = None) -> Tuple[int, int]:
        """Make this rank's shard of table `name` resident; returns (first
        global row, rows here)."""
        first = next(iter(columns.values()))
        n = len(first.codes) if isinstance(first, Utf8) else len(first)
        if total_rows is None:
            start, cnt = shard.shard_range(n, self.rank, self.world)
            local = {}
            for k, c in columns.items():
                if isinstance(c, Utf8):
                    local[k] = Utf8(np.ascontiguousarray(c.codes[start:start + cnt]), c.dictionary)
                else:
                    local[k] = c[start:start + cnt]
        else:
            start, cnt = shard.shard_range(total_rows, self.rank, self.world)
            if n != cnt:
                raise ValueError(f"rank {self.rank} holds rows [{start}, {start + cnt}) of {name}, got {n} rows")
            local = columns
        for k, c in local.items():
            if isinstance(c, Utf8):
                self._dicts[(name, k)] = list(c.dictionary)
        self.db.create_table(name, local, nrows=cnt)
        self.db.synchronize()
        self._rows[name] = (start, cnt)
        return start, cnt

    def _col(self, table: str, col: str):
        return self.db.column(table, col)

    # ------------------------------------------------------------------ queries
    def aggregate(self, table: str, aggs: Sequence[Tuple[int, str]], where: Sequence[fdb_pred_term] = (),
                  where_cols: Sequence[str] = ()) -> np.ndarray:
        """No-key aggregates (execute_agg_only): AGG_VALUE_DTYPE records, one
        per (func, column); `where` terms index `where_cols` first, then the
        aggregate columns."""
        names = list(where_cols)
        for _, c in aggs:
            if c not in names:
                names.append(c)
        cols = [self._col(table, c) for c in names]
        spec = [(f, names.index(c) if f != AGG_COUNT_STAR else 0) for f, c in aggs]
        n = self._rows[table][1]
        # fdb_aggregate takes up to 4 aggregates per scan.
        local = np.concatenate([ops.to_records(ops.aggregate(self.db, cols, n, list(where), spec[i:i + 4]),
                                               AGG_VALUE_DTYPE, len(spec[i:i + 4]))
                                for i in range(0, len(spec), 4)])
        return shard.combine_aggregates(local, [f for f, _ in aggs], self.group)

    def count_where(self, table: str, col: str, op: int, literal) -> int:
        """COUNT(*) WHERE col op literal (the popcount path)."""
        n = self._rows[table][1]
        cnt = ops.filter_count(self.db, [self._col(table, col)], n, [ops.cmp(0, op, literal)])
        local = np.array([int(cnt.item())], dtype=np.int64)
        parts = shard._all_gather_bytes(local.view(np.uint8), self.group)
        return int(sum(int(p.view(np.int64)[0]) for p in parts))

    def count_distinct(self, table: str, col: str) -> int:
        """COUNT(DISTINCT text column): the OR of every rank's code presence
        bitmap, counted as distinct strings."""
        d = self._dicts[(table, col)]
        n = self._rows[table][1]
        words = ops.distinct_codes(self.db, [self._col(table, col)], n, [], 0, len(d))
        bits = shard.combine_presence(words.cpu().numpy().view(np.uint64), self.group)
        return len({d[i] for i in range(len(d)) if (int(bits[i >> 6]) >> (i & 63)) & 1})

    def topk(self, table: str, col: str, k: int, desc: bool) -> np.ndarray:
        """ORDER BY col [DESC] LIMIT k over the whole table: global row
        numbers, ties by row ascending (top_k_ascending, sort.rs:564-620)."""
        start, n = self._rows[table]
        c = self._col(table, col)
        rows, cnt = ops.topk(self.db, c, n, k, desc)
        m = int(cnt.item())
        local_rows = rows[:m]
        if m:
            vals, _ = ops.gather(self.db, c, local_rows, m)
            v = vals.cpu().numpy()[:m]
        else:
            v = np.zeros(0, dtype=np.float64 if c.raw.dtype == FLOAT64 else np.int64)
        grow = local_rows.cpu().numpy().view(np.uint32).astype(np.uint64) + np.uint64(start)
        _, g = shard.combine_topk(order_keys(v, desc), grow, k, self.group)
        return g

    def join_agg(self, probe_table: str, probe_key: str, join_type: int, probe_value: Optional[str] = None,
                 build_key: Optional[np.ndarray] = None, build_payload: Optional[np.ndarray] = None,
                 build_rows: int = 0, src: int = 0) -> np.ndarray:
        """Hash join with COUNT(*) / SUM aggregates: the build side, held by
        rank `src`, is broadcast and built on every GPU; each rank probes its
        shard; the partials are summed (JOIN_AGG_DTYPE record)."""
        dev = torch.device("cuda", torch.cuda.current_device())
        bk, bp = shard.broadcast_columns(
            [torch.from_numpy(np.ascontiguousarray(build_key)) if self.rank == src else None,
             torch.from_numpy(np.ascontiguousarray(build_payload)) if self.rank == src else None],
            [build_rows, build_rows], [torch.int64, torch.int64], src=src, group=self.group)
        bk, bp = bk.to(dev), bp.to(dev)
        h = ops.HashTable(self.db, bk, bp, build_rows)
        try:
            n = self._rows[probe_table][1]
            val = self._col(probe_table, probe_value) if probe_value else None
            out = h.probe_agg(self._col(probe_table, probe_key), n, join_type, value=val)
            local = ops.to_records(out, JOIN_AGG_DTYPE, 1)
        finally:
            h.free()
        return shard.combine_join(local, self.group)

    def group_by_i64(self, table: str, key: str, value: str, dst: int = 0) -> Optional[np.ndarray]:
        """GROUP BY key with COUNT(*), SUM, MIN, MAX of value: each rank's
        groups go to the rank owning the key and are merged there; rank `dst`
        receives every group (sorted by key), the others None."""
        n = self._rows[table][1]
        out, ng = ops.group_by_i64(self.db, self._col(table, key), self._col(table, value), n)
        local = ops.to_records(out, GROUP_I64_DTYPE, int(ng.item()))
        mine = shard.exchange_groups(local, self.group)
        return shard.gather_groups(mine, dst=dst, group=self.group)
