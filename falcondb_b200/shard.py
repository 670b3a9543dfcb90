"""Row-range sharding across GPUs and the exchange steps that combine per-GPU
partial results (one process per GPU, torch.distributed: NCCL between GPUs,
gloo for host tests).

Every operator on the path is data-parallel over rows; each rank runs the
single-GPU kernels on its contiguous shard and the ranks then exchange small
partials:

* no-key aggregates: every rank's fdb_agg_value records are gathered and
  combined in rank order, so FP64 sums are the same on every rank and from run
  to run (``combine_aggregates``);
* top-k: each rank's k best (order key, global row) pairs are gathered and
  merged with the same (key, row) order the kernels use (``combine_topk``);
* hash join: the build side is replicated (``broadcast_columns``); each rank
  probes its shard and the COUNT / SUM partials are summed (``combine_join``);
* high-cardinality GROUP BY: each rank's groups are routed to the rank that
  owns hash(key) % world (an all-to-all of variable-size records) and merged
  there (``exchange_groups``); ``gather_groups`` collects them on one rank.

The reference is single-process (rayon threads over 65,536-row batches); the
combine rules restate its merge steps: merge_state_entry
(src/query/aggregate.rs:1351-1390) for aggregates and groups, and the
(key, row) order of top_k_ascending (src/query/sort.rs:564-620) for top-k.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from . import (AGG_AVG, AGG_COUNT, AGG_COUNT_STAR, AGG_MAX, AGG_MIN, AGG_SUM, AGG_VALUE_DTYPE, GROUP_I64_DTYPE,
               JOIN_AGG_DTYPE)


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """(first row, row count) of this rank's contiguous shard of n rows."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def _device(group=None) -> torch.device:
    backend = dist.get_backend(group)
    return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


def _all_gather_bytes(buf: np.ndarray, group=None) -> List[np.ndarray]:
    """All-gather a fixed-size byte array from every rank (rank order)."""
    dev = _device(group)
    t = torch.from_numpy(np.ascontiguousarray(buf).view(np.uint8).copy()).to(dev)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return [o.cpu().numpy() for o in out]


def fold_aggregates(parts: Sequence[np.ndarray], funcs: Sequence[int]) -> np.ndarray:
    """Fold per-rank no-key aggregate records (AGG_VALUE_DTYPE, one per func,
    as fdb_aggregate returns them; parts in rank order) into the global ones.
    FP64 partials are folded in rank order, so results are repeatable."""
    out = np.zeros(len(funcs), dtype=AGG_VALUE_DTYPE)
    for j, f in enumerate(funcs):
        recs = [p[j] for p in parts]
        n = sum(int(r["n"]) for r in recs)
        out[j]["n"] = n
        out[j]["is_int"] = recs[0]["is_int"]
        valid = [r for r in recs if r["valid"]]
        if f in (AGG_COUNT_STAR, AGG_COUNT):
            out[j]["i"] = sum(int(r["i"]) for r in recs)
            out[j]["f"] = float(out[j]["i"])
            out[j]["valid"] = 1
        elif f == AGG_SUM:
            if recs[0]["is_int"]:
                out[j]["i"] = sum(int(r["i"]) for r in valid)
                out[j]["f"] = float(out[j]["i"])
            else:
                acc = 0.0
                for r in valid:
                    acc += float(r["f"])
                out[j]["f"] = acc
            out[j]["valid"] = 1 if valid else 0
        elif f == AGG_AVG:
            # Each rank's AVG times its count is its sum (exact for integer data
            # below 2^53; within one rounding per rank otherwise).
            s = 0.0
            for r in valid:
                s += float(r["f"]) * float(r["n"])
            out[j]["f"] = s / n if n else 0.0
            out[j]["valid"] = 1 if valid else 0
        elif f in (AGG_MIN, AGG_MAX):
            vals = [float(r["f"]) for r in valid]
            out[j]["f"] = (min(vals) if f == AGG_MIN else max(vals)) if vals else 0.0
            out[j]["valid"] = 1 if vals else 0
        else:
            raise ValueError(f"aggregate {f} has no shard combine (COUNT DISTINCT: OR the presence bitmaps)")
    return out


def combine_aggregates(local: np.ndarray, funcs: Sequence[int], group=None) -> np.ndarray:
    """fold_aggregates over every rank's records, on every rank."""
    parts = [p.view(AGG_VALUE_DTYPE) for p in _all_gather_bytes(local.view(np.uint8), group)]
    return fold_aggregates(parts, funcs)


def combine_presence(local_words: np.ndarray, group=None) -> np.ndarray:
    """COUNT(DISTINCT code): OR of every rank's dictionary-code presence bitmap."""
    parts = _all_gather_bytes(local_words.view(np.uint8), group)
    out = np.zeros_like(local_words.view(np.uint64))
    for p in parts:
        out |= p.view(np.uint64)
    return out


def _pad_topk(keys: np.ndarray, rows: np.ndarray, k: int) -> np.ndarray:
    pk = np.full(k, np.iinfo(np.uint64).max, dtype=np.uint64)
    pr = np.full(k, np.iinfo(np.uint64).max, dtype=np.uint64)
    m = min(k, len(keys))
    pk[:m] = np.asarray(keys, dtype=np.uint64)[:m]
    pr[:m] = np.asarray(rows, dtype=np.uint64)[:m]
    return np.concatenate([pk, pr])


def fold_topk(parts: Sequence[np.ndarray], k: int) -> Tuple[np.ndarray, np.ndarray]:
    """Merge per-rank padded (key[k], row[k]) lists into the global k best
    (ascending (order key, global row))."""
    ak = np.concatenate([p[:k] for p in parts])
    ar = np.concatenate([p[k:] for p in parts])
    live = ~((ak == np.iinfo(np.uint64).max) & (ar == np.iinfo(np.uint64).max))
    ak, ar = ak[live], ar[live]
    order = np.lexsort((ar, ak))[:k]
    return ak[order], ar[order]


def combine_topk(keys: np.ndarray, rows: np.ndarray, k: int, group=None) -> Tuple[np.ndarray, np.ndarray]:
    """Merge every rank's k best (order key, global row) pairs, each rank's
    list padded to k, into the global k best (ascending (key, row)), on every rank."""
    parts = [p.view(np.uint64) for p in _all_gather_bytes(_pad_topk(keys, rows, k).view(np.uint8), group)]
    return fold_topk(parts, k)


def fold_join(parts: Sequence[np.ndarray]) -> np.ndarray:
    """Sum per-rank join partials (JOIN_AGG_DTYPE records: count, sum_payload,
    payload_rows exact; sum_value folded in rank order)."""
    out = np.zeros(1, dtype=JOIN_AGG_DTYPE)
    for f in ("count", "sum_payload", "payload_rows"):
        out[0][f] = sum(int(p[f]) for p in parts)
    acc = 0.0
    for p in parts:
        acc += float(p["sum_value"])
    out[0]["sum_value"] = acc
    return out


def combine_join(local: np.ndarray, group=None) -> np.ndarray:
    """fold_join over every rank's join partial, on every rank."""
    return fold_join([p.view(JOIN_AGG_DTYPE)[0] for p in _all_gather_bytes(local.view(np.uint8), group)])


def all_gather_parts(parts: Sequence[np.ndarray], group=None) -> List[List[np.ndarray]]:
    """Several fixed-size byte arrays from every rank in one collective:
    result[r][j] is rank r's array j (same sizes on every rank)."""
    sizes = [int(np.ascontiguousarray(p).view(np.uint8).size) for p in parts]
    flat = (np.concatenate([np.ascontiguousarray(p).view(np.uint8).ravel() for p in parts]) if parts
            else np.zeros(0, np.uint8))
    out = []
    for blob in _all_gather_bytes(flat, group):
        o, off = [], 0
        for sz in sizes:
            o.append(blob[off:off + sz])
            off += sz
        out.append(o)
    return out


def broadcast_columns(cols: Sequence[Optional[torch.Tensor]], lengths: Sequence[int], dtypes: Sequence[torch.dtype],
                      src: int = 0, group=None) -> List[torch.Tensor]:
    """Replicate columns held by rank `src` (the join build side) on every rank."""
    dev = _device(group)
    out = []
    for c, n, dt in zip(cols, lengths, dtypes):
        t = c.to(dev) if (dist.get_rank(group) == src and c is not None) else torch.empty(n, dtype=dt, device=dev)
        dist.broadcast(t, src=src, group=group)
        out.append(t)
    return out


def _owner(keys: np.ndarray, world: int) -> np.ndarray:
    h = (keys.astype(np.uint64) ^ np.uint64(1 << 63)) * np.uint64(0x9E3779B97F4A7C15)
    return (h >> np.uint64(32)) % np.uint64(world)


def _merge_groups(recs: np.ndarray) -> np.ndarray:
    """Fold group partials that share a key (merge_state_entry,
    aggregate.rs:1351-1390): counts and sums add, MIN / MAX take the extreme of
    the non-NaN partials."""
    if len(recs) == 0:
        return recs
    recs = recs[np.argsort(recs["key"], kind="stable")]
    starts = np.nonzero(np.r_[True, recs["key"][1:] != recs["key"][:-1]])[0]
    out = np.zeros(len(starts), dtype=GROUP_I64_DTYPE)
    out["key"] = recs["key"][starts]
    out["count"] = np.add.reduceat(recs["count"], starts)
    out["sum"] = np.add.reduceat(recs["sum"], starts)
    mn = np.where(np.isnan(recs["min"]), np.inf, recs["min"])
    mx = np.where(np.isnan(recs["max"]), -np.inf, recs["max"])
    out["min"] = np.minimum.reduceat(mn, starts)
    out["max"] = np.maximum.reduceat(mx, starts)
    out["min"][np.isinf(out["min"]) & (out["min"] > 0)] = np.nan
    out["max"][np.isinf(out["max"]) & (out["max"] < 0)] = np.nan
    return out


def exchange_groups(local: np.ndarray, group=None) -> np.ndarray:
    """Route every rank's GROUP BY partials (GROUP_I64_DTYPE) to the rank that
    owns each key (hash % world) and merge them there; returns this rank's
    final groups (disjoint across ranks)."""
    world = dist.get_world_size(group)
    dev = _device(group)
    local = np.ascontiguousarray(local)
    dest = _owner(local["key"], world)
    order = np.argsort(dest, kind="stable")
    send = local[order]
    counts = np.bincount(dest.astype(np.int64), minlength=world).astype(np.int64)
    cnt_t = torch.from_numpy(counts).to(dev)
    recv_counts = torch.empty_like(cnt_t)
    dist.all_to_all_single(recv_counts, cnt_t, group=group)
    rc = recv_counts.cpu().numpy()
    isz = GROUP_I64_DTYPE.itemsize
    send_t = torch.from_numpy(send.view(np.uint8).copy()).to(dev)
    recv_t = torch.empty(int(rc.sum()) * isz, dtype=torch.uint8, device=dev)
    dist.all_to_all_single(recv_t, send_t, output_split_sizes=[int(c) * isz for c in rc],
                           input_split_sizes=[int(c) * isz for c in counts], group=group)
    return _merge_groups(recv_t.cpu().numpy().view(GROUP_I64_DTYPE))


def gather_groups(mine: np.ndarray, dst: int = 0, group=None) -> Optional[np.ndarray]:
    """All ranks' final groups on rank dst (sorted by key); None elsewhere."""
    objs = [None] * dist.get_world_size(group) if dist.get_rank(group) == dst else None
    dist.gather_object(mine, objs, dst=dst, group=group)
    if objs is None:
        return None
    allg = np.concatenate(objs) if objs else np.zeros(0, dtype=GROUP_I64_DTYPE)
    return allg[np.argsort(allg["key"], kind="stable")]
