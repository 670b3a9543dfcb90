"""Benchmark: scanned GB/s of the scan / filter / top-k hot path on B200.

Workload (the reference's scan + top-k configuration, 100M rows): table t with
id int64 0..N-1, dept Utf8 uniform over 12 labels, score f64 uniform [0,100),
salary int64 uniform [30000,200000] (seeded synthetic data); one step runs the
five queries
    SUM(score); COUNT(*) WHERE score > 50; COUNT(DISTINCT dept);
    ORDER BY score DESC LIMIT 10; ORDER BY id DESC LIMIT 10 (ties: id asc)
over the whole table.  Algorithmic bytes per row at the reference's storage
widths: 8 + 8 + 4 + 8 + 8 = 36 B/row.

* value   : device-resident columns, the operator layer on the context stream,
            CUDA events around K steps (inputs are 0.4-0.8 GB per column, far
            larger than the 126 MB L2, so no flush is needed between steps).
* e2e     : the public API with host buffers: each step uploads the columns
            from pinned host memory (fdb_table_from_columns) and runs the five
            queries through fdb_sql, results read back to the host.
* roofline: the dominant query's kernels, algorithmic bytes / CUDA-event time,
            against the measured HBM copy bandwidth (MEASURED_PEAKS.json).
* cpu_baseline: the reference-shaped CPU engine (oracle/refengine.cpp, a C++
            restatement of FalconDB's rayon operators) on this host's cores.

`python bench.py --impl reference` times that CPU engine alone (the reference
arm).  Under torchrun each rank holds its own 100M-row shard (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_ROWS = 100_000_000
BYTES_PER_ROW = {"sum_score": 8, "count_where": 8, "count_distinct": 4, "topk_score": 8, "topk_id": 8}
QUERIES = {
    "sum_score": "SELECT SUM(score) FROM {t}",
    "count_where": "SELECT COUNT(*) FROM {t} WHERE score > 50",
    "count_distinct": "SELECT COUNT(DISTINCT dept) FROM {t}",
    "topk_score": "SELECT id, score FROM {t} ORDER BY score DESC LIMIT 10",
    "topk_id": "SELECT id FROM {t} ORDER BY id DESC LIMIT 10",
}
LAUNCHES_PER_STEP = 7  # sum 1, count 1, distinct 1, top-k (sample + main) x 2
METRIC = "scanned GB/s vs 8 TB/s HBM"
# How the int64-key GROUP BY sizes its table in these runs.
ZONE_SIZING = ("key range from the key column's zone maps (computed on the GPU when the table is loaded, per "
               "65,536-row batch, as Table::append_batch computes BatchStats); no pass over the keys inside the "
               "timed call. ms_with_sizing_pass: the same call with zone maps off, which first reads the keys once "
               "(HyperLogLog estimate and key range)")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel: str):
    """Per-launch DRAM bytes of `kernel` from a committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        v = d.get(kernel)
        if isinstance(v, dict):
            return v.get("dram_bytes_per_launch_full_size")
    return None


class Clocks:
    """SM clock and clock-event (throttle) reasons sampled through NVML every
    millisecond while the timed region runs (the region is tens of ms, too short
    for nvidia-smi's sampling period).  Reads only; changes no GPU setting."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self._nvml = None

    def _handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            from cuda import cudart

            err, bus = cudart.cudaDeviceGetPCIBusId(64, self.device)
            bus = bus.decode() if isinstance(bus, bytes) else bus
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.strip("\x00"))
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading

        try:
            nv, h = self._handle()
        except Exception:
            return self
        self._nvml = nv
        self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    r = get_reasons(h)
                    for bit, name in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(name)
                except Exception:
                    pass
                time.sleep(0.001)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        time.sleep(0.003)
        return self

    def __exit__(self, *a):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "NVML, 1 ms polling"}


def make_table(n: int, seed: int):
    from falcondb_b200 import workloads as W

    return W.table_t(n, seed=seed)


# ----------------------------------------------------------------------------- GPU arm
def run_gpu(args):
    import torch
    import torch.distributed as dist

    import falcondb_b200 as F
    from falcondb_b200 import ops

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    n = args.rows
    t = make_table(n, seed=1 + rank)

    db = F.Database(local)
    if args.tuning:
        db.load_tuning(args.tuning)
    db.create_table("t", t)
    db.synchronize()
    cs = {c: db.column("t", c) for c in ("id", "dept", "score")}
    lib_stream = ops.lib_stream(db)

    # Device result buffers reused every step (no allocation in the timed region).
    r_sum = ops._bytes(F.AGG_VALUE_DTYPE.itemsize, db)
    r_cnt = torch.empty(1, dtype=torch.int64, device=dev)
    r_dist = torch.empty(1, dtype=torch.int64, device=dev)
    r_top1 = torch.empty(10, dtype=torch.int32, device=dev)
    r_top1c = torch.empty(1, dtype=torch.int64, device=dev)
    r_top2 = torch.empty(10, dtype=torch.int32, device=dev)
    r_top2c = torch.empty(1, dtype=torch.int64, device=dev)
    pred = [ops.cmp(0, F.GT, 50)]
    L = F.lib()
    from falcondb_b200 import fdb_agg_spec, fdb_dev_column, fdb_pred_term
    import ctypes as C

    def col_arr(*cols):
        a = (fdb_dev_column * len(cols))()
        for i, c in enumerate(cols):
            a[i] = c.raw
        return a

    c_score, c_dept, c_id = col_arr(cs["score"]), col_arr(cs["dept"]), col_arr(cs["id"])
    p_arr = (fdb_pred_term * 1)(pred[0])
    a_sum = (fdb_agg_spec * 1)()
    a_sum[0].func, a_sum[0].col = F.AGG_SUM, 0
    h = db.handle

    def q_sum():
        F.check(L.fdb_aggregate(h, c_score, 1, n, None, 0, a_sum, 1, r_sum.data_ptr()))

    def q_count():
        F.check(L.fdb_filter_count(h, c_score, 1, n, p_arr, 1, r_cnt.data_ptr()))

    def q_distinct():
        F.check(L.fdb_distinct_codes(h, c_dept, 1, n, None, 0, 0, 12, r_dist.data_ptr()))

    def q_top_score():
        F.check(L.fdb_topk(h, C.byref(cs["score"].raw), n, 10, 1, 1, r_top1.data_ptr(), r_top1c.data_ptr()))

    def q_top_id():
        F.check(L.fdb_topk(h, C.byref(cs["id"].raw), n, 10, 1, 1, r_top2.data_ptr(), r_top2c.data_ptr()))

    steps = [("sum_score", q_sum), ("count_where", q_count), ("count_distinct", q_distinct),
             ("topk_score", q_top_score), ("topk_id", q_top_id)]
    combined = {}

    def combine():
        # Every rank's partials of the five queries in one all-gather (the
        # shard's SUM record, COUNT, code presence bitmap, and each top-k as
        # order keys plus global row numbers), folded in rank order.
        from falcondb_b200 import distributed as D, shard
        vs, _ = ops.gather(db, cs["score"], r_top1, 10)
        vi, _ = ops.gather(db, cs["id"], r_top2, 10)
        base = np.uint64(rank * n)
        rows1 = r_top1.cpu().numpy().view(np.uint32).astype(np.uint64) + base
        rows2 = r_top2.cpu().numpy().view(np.uint32).astype(np.uint64) + base
        parts = [ops.to_records(r_sum, F.AGG_VALUE_DTYPE, 1), r_cnt.cpu().numpy(), r_dist.cpu().numpy(),
                 shard._pad_topk(D.order_keys(vs.cpu().numpy()[:10], True), rows1, 10),
                 shard._pad_topk(D.order_keys(vi.cpu().numpy()[:10], True), rows2, 10)]
        got = shard.all_gather_parts(parts)
        combined["sum"] = shard.fold_aggregates([g[0].view(F.AGG_VALUE_DTYPE) for g in got], [F.AGG_SUM])
        combined["count"] = sum(int(g[1].view(np.int64)[0]) for g in got)
        combined["distinct"] = int(np.bitwise_or.reduce([g[2].view(np.uint64)[0] for g in got]))
        combined["top_score"] = shard.fold_topk([g[3].view(np.uint64) for g in got], 10)[1]
        combined["top_id"] = shard.fold_topk([g[4].view(np.uint64) for g in got], 10)[1]

    def one_step(evs=None):
        for j, (name, fn) in enumerate(steps):
            if evs is not None:
                evs[j][0].record(lib_stream)
            fn()
            if evs is not None:
                evs[j][1].record(lib_stream)
        if world > 1:
            combine()

    torch.cuda.synchronize()
    for _ in range(args.warmup):
        one_step()
    db.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    K = args.steps
    evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in steps]
           for _ in range(K)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        start.record(lib_stream)
        for k in range(K):
            one_step(evs[k])
        stop.record(lib_stream)
        db.synchronize()
        torch.cuda.synchronize()
    clocks = clk.summary()
    ms = start.elapsed_time(stop)
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    per_q = {name: sum(evs[k][j][0].elapsed_time(evs[k][j][1]) for k in range(K)) / K
             for j, (name, _) in enumerate(steps)}

    # After timing, every answer of the last step against the oracle: the
    # FP64 SUM within 1e-12 of the serial sum, the count, the distinct set and
    # both top-k row lists (ties by row ascending) exactly.
    from oracle import oracle as O
    got_sum = float(ops.to_records(r_sum, F.AGG_VALUE_DTYPE, 1)[0]["f"])
    want_sum = O.sum_serial(t["score"])
    assert abs(got_sum - want_sum) <= 1e-12 * abs(want_sum), (got_sum, want_sum)
    assert int(r_cnt.item()) == O.popcount(O.cmp_mask(t["score"], F.GT, 50))
    present = O.present_codes(t["dept"].codes, 12)
    assert int(r_dist.cpu().numpy().view(np.uint64)[0]) == sum(1 << i for i in range(12) if present[i])
    assert int(r_top1c.item()) == 10 and int(r_top2c.item()) == 10
    assert list(r_top1.cpu().numpy()) == list(O.topk(t["score"], 10, True))
    assert list(r_top2.cpu().numpy()) == list(O.topk(t["id"], 10, True))

    bytes_per_step = sum(BYTES_PER_ROW.values()) * n
    value = world * bytes_per_step * K / (ms / 1e3) / 1e9

    # ---------------- e2e through the public API (host buffers) ----------------
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, F, t, n, db, torch, world, dist, local)

    result = None
    if rank == 0:
        peak, peak_kind = peaks()
        dom = max(per_q, key=per_q.get)
        achieved = BYTES_PER_ROW[dom] * n / (per_q[dom] / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "frac_vs_8TBs": round(achieved / 8000.0, 4),
                "traffic": traffic_from_profiles(dom),
                "algorithmic_bytes_per_launch": BYTES_PER_ROW[dom] * n}
        per_query = {q: {"ms": round(per_q[q], 4),
                         "GB/s": round(BYTES_PER_ROW[q] * n / (per_q[q] / 1e3) / 1e9, 1),
                         "frac_of_measured_hbm": round(BYTES_PER_ROW[q] * n / (per_q[q] / 1e3) / 1e9 / peak, 4)}
                     for q in per_q}
        result = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(ms / K, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64/int64", "data": "synthetic (seeded)",
            "config": {"workload": "scan+top-k 100M rows: SUM(score); COUNT(*) WHERE score>50; "
                                   "COUNT(DISTINCT dept); ORDER BY score DESC LIMIT 10; ORDER BY id DESC LIMIT 10",
                       "rows_per_gpu": n, "bytes_per_row": sum(BYTES_PER_ROW.values()),
                       "l2_flush": "not needed: every input column (400-800 MB) exceeds the 126 MB L2",
                       "parallelism": f"row shards x{world}"},
            "roofline": roof, "per_query": per_query, "e2e": e2e, "gpu_launches": LAUNCHES_PER_STEP * K,
            "clocks": clocks, "extra_keys": ["per_query"],
        }
        if not args.no_cpu:
            result["cpu_baseline"] = cpu_baseline(t, n, args.cpu_threads)
    if world == 1 and not args.no_configs:
        extra = run_configs(args, db, t, n, peaks()[0])
        result.update(extra)
        result["extra_keys"] = ["per_query"] + list(extra)
    db.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_e2e(args, F, t, n, db, torch, world, dist, local):
    """Each step: pinned host columns -> fdb_table_from_columns (async upload,
    score first) -> the five queries through fdb_sql -> results on the host."""
    pinned = {}
    for name, arr in (("score", t["score"]), ("dept", t["dept"].codes), ("id", t["id"])):
        tt = torch.empty(arr.nbytes, dtype=torch.uint8, pin_memory=True)
        tt.numpy()[:] = np.frombuffer(arr.tobytes(), dtype=np.uint8)
        pinned[name] = tt
    from falcondb_b200 import fdb_column
    import ctypes as C

    cols = (fdb_column * 3)()
    dict_enc = [s.encode() for s in t["dept"].dictionary]
    darr = (C.c_char_p * len(dict_enc))(*dict_enc)
    for j, (name, dt) in enumerate((("score", F.FLOAT64), ("dept", F.UTF8), ("id", F.INT64))):
        cols[j].name = name.encode()
        cols[j].dtype = dt
        cols[j].values = pinned[name].data_ptr()
        cols[j].validity = None
        if dt == F.UTF8:
            cols[j].dict = C.cast(darr, C.POINTER(C.c_char_p))
            cols[j].dict_len = len(dict_enc)
    L = F.lib()
    h2d = n * (8 + 4 + 8)
    d2h = 0

    def step():
        nonlocal d2h
        F.check(L.fdb_table_from_columns(db.handle, b"e2e", cols, 3, n))
        out = 0
        for sql in QUERIES.values():
            r = db.sql(sql.format(t="e2e"))
            out += 8 * r.rows * len(r.columns)  # result values read back (8 B each)
        d2h = out

    for _ in range(max(1, args.warmup)):
        step()
    db.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        step()
    db.synchronize()
    el = time.perf_counter() - t0
    if world > 1:
        tt = torch.tensor([el], device=torch.device("cuda", local))
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        el = float(tt.item())
    value = world * sum(BYTES_PER_ROW.values()) * n * args.e2e_steps / el / 1e9
    return {"value": round(value, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": round(el / args.e2e_steps * 1e3, 3), "steps": args.e2e_steps,
            "path": "fdb_table_from_columns (pinned host) + 5 x fdb_sql"}


# ----------------------------------------------------------------------------- the other configurations
def run_configs(args, db, t, n, peak):
    """One line's extra keys: the other BASELINE configurations at full size,
    each timed with CUDA events on the library stream (K steps after 3
    warm-ups; every input column exceeds the 126 MB L2) and checked against
    the oracle after timing.

    * filter_groupby_100M: SELECT dept, COUNT(*), SUM(score), AVG(salary)
      WHERE score > 50 GROUP BY dept over the headline's 100M-row table
      (20 B/row).
    * join_{inner,left,semi,anti}: 1M-row build (key a permutation of
      0..1M-1, payload uniform [0, 1e6)), 100M-row probe (key uniform
      [0, 2M), value uniform [0, 1)); COUNT(*) with SUM(payload), or with
      SUM(value) for SEMI / ANTI (8 B/probe row of key, +8 B of value).
    * aggregate_where_100M: SELECT COUNT(*), SUM(score), AVG(salary),
      MAX(score) WHERE score > 50 over the headline table (16 B/row).
    * zone_prune: SELECT COUNT(*), SUM(score) WHERE id >= 99M through
      fdb_sql over the headline table (id ascending), zone maps on and off:
      host wall time per query.
    * groupby_zipf: 100M rows, key Zipf(1.1) over 10M values, COUNT / SUM /
      MIN / MAX of v, the key range from the zone maps; the same call with
      the sizing pass beside it (16 B/row + 40 B/group).
    * groupby_batched: 64 GROUP BY queries over slices of that table, sizes
      log-uniform in [10k, 10M] rows, one captured graph against the same
      queries one by one.
    * serving: 10,000 queries of the four templates, Poisson at 2000 qps,
      batched against one at a time, plus an offered-load sweep."""
    import torch

    import falcondb_b200 as F
    from falcondb_b200 import ops, serving as S, workloads as W
    from oracle import oracle as O

    dev = torch.device("cuda", 0)
    stream = ops.lib_stream(db)
    K, Wm = max(3, min(args.steps, 10)), 3
    L = F.lib()
    extra = {}

    def rate(name, ms, nbytes, **kw):
        gbs = nbytes / (ms / 1e3) / 1e9
        d = {"ms": round(ms, 4), "algorithmic_bytes": int(nbytes), "GB/s": round(gbs, 1),
             "frac_of_measured_hbm": round(gbs / peak, 4), "oracle_checked": True, "steps": K, "warmup": Wm}
        d.update(kw)
        extra[name] = d

    # --- configuration 0's query at 100M rows (the headline table) ---------
    cols = [db.column("t", c) for c in ("dept", "score", "salary")]
    prog = [ops.cmp(1, F.GT, 50)]
    aggs = [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_AVG, 2)]
    res = ops._bytes(F.AGG_VALUE_DTYPE.itemsize * 13 * 3, db)
    grows = torch.empty(13, dtype=torch.int64, device=dev)
    ca, nc = ops._cols(cols)
    pa, npr = ops._prog(prog)
    aa, na = ops._aggs(aggs)
    ms = _time_steps(lambda: F.check(L.fdb_group_by_codes(db.handle, ca, nc, n, pa, npr, 0, 12, aa, na,
                                                          res.data_ptr(), grows.data_ptr())), K, Wm, stream, torch)
    g0 = O.group_codes(t["dept"].codes, 12, mask=O.cmp_mask(t["score"], F.GT, 50), fvals=t["score"],
                       ivals=t["salary"])
    rec = ops.to_records(res, F.AGG_VALUE_DTYPE).reshape(13, 3)
    assert list(grows.cpu().numpy()[:12]) == list(g0["rows"][:12])
    for d in range(12):
        assert abs(rec[d, 1]["f"] - g0["fsum"][d]) <= 1e-12 * g0["fsum"][d]
        assert rec[d, 2]["f"] == g0["isum"][d] / g0["icnt"][d]
    rate("filter_groupby_100M", ms, 20 * n, rows=n,
         query="SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM t WHERE score > 50 GROUP BY dept")

    # --- aggregates under one WHERE compare (execute_agg_only) ----------------
    cols2 = [db.column("t", c) for c in ("score", "salary")]
    aggs2 = [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 0), (F.AGG_AVG, 1), (F.AGG_MAX, 0)]
    res2 = ops._bytes(F.AGG_VALUE_DTYPE.itemsize * 4, db)
    ca2, nc2 = ops._cols(cols2)
    pa2, npr2 = ops._prog([ops.cmp(0, F.GT, 50)])
    aa2, na2 = ops._aggs(aggs2)
    ms = _time_steps(lambda: F.check(L.fdb_aggregate(db.handle, ca2, nc2, n, pa2, npr2, aa2, na2, res2.data_ptr())),
                     K, Wm, stream, torch)
    rec = ops.to_records(res2, F.AGG_VALUE_DTYPE, 4)
    sel = t["score"] > 50
    assert rec[0]["i"] == int(sel.sum())
    assert abs(rec[1]["f"] - O.sum_serial(t["score"][sel])) <= 1e-12 * rec[1]["f"]
    assert rec[2]["f"] == float(O.sum_i64_exact(t["salary"][sel])) / int(sel.sum())
    assert rec[3]["f"] == float(t["score"][sel].max())
    rate("aggregate_where_100M", ms, 16 * n, rows=n,
         query="SELECT COUNT(*), SUM(score), AVG(salary), MAX(score) FROM t WHERE score > 50")

    # --- zone-map pruning (execute_select's batch skip, select.rs:115-137) ---
    lo = n - n // 100
    qz = f"SELECT COUNT(*), SUM(score) FROM t WHERE id >= {lo}"
    walls = {}
    for on in (0, 1):
        db.set_option("zone_maps", on)
        for _ in range(Wm):
            db.sql(qz)
        t0 = time.perf_counter()
        for _ in range(K):
            r = db.sql(qz)
        walls[on] = (time.perf_counter() - t0) / K * 1e3
        scanned = db.last_scan_rows
        assert r.value(0, 0) == n - lo
        assert abs(r.value(0, 1) - O.sum_serial(t["score"][lo:])) <= 1e-12 * r.value(0, 1)
    extra["zone_prune"] = {"query": qz.replace("FROM t", "FROM t (id ascending)"), "rows": n,
                           "ms_pruned": round(walls[1], 4), "ms_full_scan": round(walls[0], 4),
                           "rows_scanned_pruned": scanned, "oracle_checked": True, "steps": K, "warmup": Wm,
                           "timing": "host wall time of fdb_sql, result fetched"}

    # --- configuration 2: 1M x 100M joins ------------------------------------
    b, p = W.join_tables(1_000_000, n, seed=7)
    db.create_table("b", b)
    db.create_table("p", p)
    bk, bp = db.column("b", "key"), db.column("b", "payload")
    pk, pv = db.column("p", "key"), db.column("p", "value")
    out = ops._bytes(F.JOIN_AGG_DTYPE.itemsize, db)
    ms_build = _time_steps(lambda: ops.HashTable(db, bk, bp, len(b["key"])).free(), 3, 2, stream, torch)
    ht = ops.HashTable(db, bk, bp, len(b["key"]))
    for jt, name in [(F.JOIN_INNER, "inner"), (F.JOIN_LEFT, "left"), (F.JOIN_SEMI, "semi"), (F.JOIN_ANTI, "anti")]:
        val = pv if jt >= F.JOIN_SEMI else None
        ms = _time_steps(lambda: ht.probe_agg(pk, n, jt, value=val, out=out), K, Wm, stream, torch)
        got = ops.to_records(out, F.JOIN_AGG_DTYPE, 1)[0]
        want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
        assert int(got["count"]) == want["count"]
        if jt <= F.JOIN_LEFT:
            assert int(got["sum_payload"]) == want["sum_payload"]
        else:
            assert abs(float(got["sum_value"]) - want["sum_value"]) <= 1e-12 * abs(want["sum_value"])
        rate(f"join_{name}", ms, (16 if jt >= F.JOIN_SEMI else 8) * n, build_rows=len(b["key"]), probe_rows=n,
             count=int(got["count"]), table="direct-addressed" if ht.dense else "hashed",
             build_ms=round(ms_build, 4))

    # --- configuration 3: Zipf GROUP BY, single and batched ------------------
    g = W.groupby_table(n, distinct=10_000_000, seed=11)
    db.create_table("g", g)
    gk, gv = db.column("g", "key"), db.column("g", "v")
    cap = 12_000_000
    outb = ops._bytes(F.GROUP_I64_DTYPE.itemsize * cap, db)
    ng = torch.empty(1, dtype=torch.int64, device=dev)
    # With the key column's zone maps off, the same call first reads the keys
    # once (HyperLogLog estimate and key range); timed too, for comparison.
    db.set_option("zone_maps", 0)
    ms_pass = _time_steps(lambda: ops.group_by_i64(db, gk, gv, n, capacity=cap, out=outb, ngroups=ng), K, Wm,
                          stream, torch)
    db.set_option("zone_maps", 1)
    ms = _time_steps(lambda: ops.group_by_i64(db, gk, gv, n, capacity=cap, out=outb, ngroups=ng), K, Wm, stream,
                     torch)
    groups = int(ng.item())
    rec = ops.to_records(outb, F.GROUP_I64_DTYPE, groups)
    rec = rec[np.argsort(rec["key"], kind="stable")]
    want = O.group_i64(g["key"], g["v"])
    assert np.array_equal(rec["key"], want["key"]) and np.array_equal(rec["count"], want["count"])
    assert np.array_equal(rec["min"], want["min"]) and np.array_equal(rec["max"], want["max"])
    assert float((np.abs(rec["sum"] - want["sum"]) / np.abs(want["sum"])).max()) <= 1e-12
    del rec, want
    rate("groupby_zipf", ms, 16 * n + 40 * groups, rows=n, groups=groups, distinct_domain=10_000_000, zipf_s=1.1,
         table_sizing=ZONE_SIZING, ms_with_sizing_pass=round(ms_pass, 4))

    kt = torch.from_numpy(g["key"]).to(dev)
    vt = torch.from_numpy(g["v"]).to(dev)
    rng = np.random.default_rng(64)
    sizes = np.minimum(np.floor(10 ** (4 + 3 * rng.random(64))).astype(np.int64), n)
    offs = [int(rng.integers(0, n - s + 1)) for s in sizes]
    qs = [(kt[o:o + int(s)], vt[o:o + int(s)], int(s)) for o, s in zip(offs, sizes)]
    tuning, _ = ops.GroupByBatch.autotune(db, qs, reps=2)
    batch = ops.GroupByBatch(db, qs, tuning=tuning)
    ms_batch = _time_steps(batch.run, K, Wm, stream, torch)
    bgroups = [int(batch.outs[i][1].item()) for i in range(len(qs))]
    souts = [(ops._bytes(F.GROUP_I64_DTYPE.itemsize * (gq + 1), db), torch.empty(1, dtype=torch.int64, device=dev))
             for gq in bgroups]

    def serial():
        for (kk, vv, sz), gq, (ob, nb2) in zip(qs, bgroups, souts):
            ops.group_by_i64(db, kk, vv, sz, expected_groups=max(gq, 1), capacity=gq + 1, out=ob, ngroups=nb2)
    ms_serial = _time_steps(serial, K, Wm, stream, torch)
    assert [int(nb2.item()) for _, nb2 in souts] == bgroups
    for i in np.argsort(sizes)[::16]:  # four queries of spread sizes against the oracle
        o, sz = offs[i], int(sizes[i])
        r = ops.to_records(batch.outs[i][0], F.GROUP_I64_DTYPE, bgroups[i])
        r = r[np.argsort(r["key"], kind="stable")]
        w = O.group_i64(g["key"][o:o + sz], g["v"][o:o + sz])
        assert np.array_equal(r["key"], w["key"]) and np.array_equal(r["count"], w["count"])
        assert float((np.abs(r["sum"] - w["sum"]) / np.abs(w["sum"])).max()) <= 1e-12
    batch.free()
    rows_total = int(sizes.sum())
    rate("groupby_batched", ms_batch, 16 * rows_total + 40 * sum(bgroups), queries=len(qs), rows_total=rows_total,
         groups_total=sum(bgroups), ms_serial=round(ms_serial, 4), speedup_vs_serial=round(ms_serial / ms_batch, 2),
         qps_batched=round(len(qs) / (ms_batch / 1e3), 1), qps_serial=round(len(qs) / (ms_serial / 1e3), 1),
         tuning={"load_factor": tuning[0], "ctas_per_sm": tuning[1], "tile_rows": tuning[2]},
         oracle_checked_queries=4, serial="the same queries one by one, tables sized to the exact group counts")
    del kt, vt, qs, souts
    db.drop_table("g")
    del g
    torch.cuda.empty_cache()

    # --- configuration 4: serving --------------------------------------------
    extra["serving"] = serve_configuration(args, db, t, n, p, b, ht, S, O, F, torch)
    ht.free()
    db.drop_table("b")
    db.drop_table("p")
    return extra


def serve_configuration(args, db, t, n, p, b, ht, S, O, F, torch):
    """10,000 queries (filter-count, filter-group-by, inner join, top-k drawn
    uniformly) over prefixes of the resident tables, prefix sizes log-uniform
    in [10k, 100M] rows, thresholds uniform in [0, 100), Poisson arrivals at
    2000 qps, under a 40 GB device budget: continuous batching against one
    query at a time, then an offered-load sweep up to 3x the serial mode's
    saturated throughput.  Every batched answer equals the one-at-a-time
    answer; 32 of them (8 per template) are checked against the oracle."""
    score = db.column("t", "score").raw.values
    dept = db.column("t", "dept").raw.values
    sal = db.column("t", "salary").raw.values
    pkey = db.column("p", "key").raw.values
    pval = db.column("p", "value").raw.values
    rng = np.random.default_rng(2000)
    nq, rate0 = args.serve_queries, 2000.0
    kinds, rows, xs = [], [], []
    for _ in range(nq):
        kinds.append(int(rng.integers(0, 4)))
        rows.append(int(min(n, np.floor(10 ** (4 + (np.log10(n) - 4) * rng.random())))))
        xs.append(float(rng.random() * 100))
    gaps = rng.exponential(1.0, nq)  # unit-rate Poisson gaps, scaled per offered load

    def queries(qps):
        qs, at = [], 0.0
        for i in range(nq):
            at += gaps[i] / qps if qps else 0.0
            k, r, x = kinds[i], rows[i], xs[i]
            if k == S.SERVE_COUNT:
                q = S.count_query(score, r, x)
            elif k == S.SERVE_GROUP:
                q = S.group_query(score, dept, sal, 12, r, x)
            elif k == S.SERVE_JOIN:
                q = S.join_query(pkey, pval, ht._h.value, r, x)
            else:
                q = S.topk_query(score, r, x, k=10)
            q.arrival_s = at
            qs.append(q)
        return qs

    budget = 40 << 30
    slots = args.serve_slots
    S.serve_trace(db, queries(0)[:200], max_batch=128, slots=slots, mem_budget=budget)  # warm-up
    live = queries(rate0)
    res_b, live_b = S.serve_trace(db, live, max_batch=128, slots=slots, mem_budget=budget)
    res_s, live_s = S.serve_trace(db, live, max_batch=1, slots=1, mem_budget=budget)
    burst = queries(0)
    _, sat_b = S.serve_trace(db, burst, max_batch=128, slots=slots, mem_budget=budget)
    _, sat_s = S.serve_trace(db, burst, max_batch=1, slots=1, mem_budget=budget)

    def same(a, c):
        return (a.status == 0 and c.status == 0 and a.count == c.count and a.sum_payload == c.sum_payload
                and list(a.group_count) == list(c.group_count) and list(a.group_sum2) == list(c.group_sum2)
                and all(abs(x - y) <= 1e-12 * max(abs(y), 1e-300) for x, y in zip(a.group_sum0, c.group_sum0))
                and list(a.rows[:a.count]) == list(c.rows[:c.count]))
    assert all(same(a, c) for a, c in zip(res_b, res_s))
    # Oracle: 8 queries per template.
    score_h, codes_h, sal_h = t["score"], t["dept"].codes, t["salary"]
    checked = {k: 0 for k in range(4)}
    for q, r in zip(live, res_b):
        if checked[q.kind] >= 8:
            continue
        checked[q.kind] += 1
        m, x = q.nrows, q.threshold
        if q.kind == S.SERVE_COUNT:
            assert r.count == int((score_h[:m] > x).sum())
        elif q.kind == S.SERVE_GROUP:
            sel = score_h[:m] > x
            c = codes_h[:m][sel]
            assert list(r.group_count[:12]) == list(np.bincount(c, minlength=12))
            assert list(r.group_sum2[:12]) == [int(v) for v in np.bincount(c, weights=sal_h[:m][sel].astype(float),
                                                                          minlength=12)]
            s0 = np.bincount(c, weights=score_h[:m][sel], minlength=12)
            assert all(abs(r.group_sum0[j] - s0[j]) <= 1e-12 * max(abs(s0[j]), 1e-300) for j in range(12))
        elif q.kind == S.SERVE_JOIN:
            keys = p["key"][:m][p["value"][:m] < x / 100]
            o = O.join_agg(b["key"], b["payload"], keys, np.zeros(len(keys)), F.JOIN_INNER)
            assert (r.count, r.sum_payload) == (o["count"], o["sum_payload"])
        else:
            idx = np.nonzero(score_h[:m] < x)[0]
            assert list(r.rows[:r.count]) == list(idx[O.topk(score_h[:m][idx], q.k, True)])

    def d(st):
        return {"qps": round(st.qps, 1), "p50_ms": round(st.p50_ms, 4), "p99_ms": round(st.p99_ms, 4),
                "max_ms": round(st.max_ms, 4), "mean_batch": round(st.mean_batch, 2)}

    # Offered-load sweep: serial at 90 % of its saturated rate, batched at 1x,
    # 2x and 3x that saturated rate.
    sweep = {"serial_saturated_qps": round(sat_s.qps, 1), "serial": {}, "batched": {}}
    s90 = 0.9 * sat_s.qps
    _, st = S.serve_trace(db, queries(s90), max_batch=1, slots=1, mem_budget=budget)
    sweep["serial"][f"{s90:.0f}"] = d(st)
    for mult in (1, 2, 3):
        off = mult * sat_s.qps
        _, st = S.serve_trace(db, queries(off), max_batch=128, slots=slots, mem_budget=budget)
        sweep["batched"][f"{off:.0f}"] = d(st)
    return {"unit": "queries/s", "queries": nq, "arrival_qps": rate0, "slots": slots, "max_batch": 128,
            "mem_budget_bytes": budget, "table_rows": n, "prefix_rows": "log-uniform [10k, 100M]",
            "at_2000qps": {"batched": d(live_b), "serial": d(live_s)},
            "saturated": {"batched": d(sat_b), "serial": d(sat_s)},
            "throughput_speedup": round(sat_b.qps / sat_s.qps, 2) if sat_s.qps else None,
            "offered_load_sweep": sweep, "results_identical_batched_vs_serial": True,
            "oracle_checked": True, "oracle_checked_queries": 32}


# ----------------------------------------------------------------------------- CPU baseline
def cpu_queries(t, n, threads):
    from oracle import oracle as O

    t0 = time.perf_counter()
    O.ref_sum_f64(t["score"][:n], threads)
    O.ref_count_cmp_f64(t["score"][:n], 4, 50.0)
    O.ref_present_codes(t["dept"].codes[:n], 12, threads)
    O.ref_topk(t["score"][:n], 10, True)
    O.ref_topk(t["id"][:n], 10, True)
    return time.perf_counter() - t0


def cpu_baseline(t, n, threads):
    from oracle import oracle as O

    threads = threads or O.hardware_threads()
    cpu_queries(t, min(n, 2_000_000), threads)  # warm
    el = cpu_queries(t, n, threads)
    value = sum(BYTES_PER_ROW.values()) * n / el / 1e9
    return {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"one pass of the 5 queries over all {n} rows (reference-shaped C++ engine: "
                      "SUM/COUNT DISTINCT parallel over 65,536-row batches, COUNT WHERE and top-k serial "
                      "over batches as in the reference)",
            "seconds": round(el, 3)}


# ----------------------------------------------------------------------------- secondary workloads
def radix_bytes_per_row(passes: int, keys_last: bool) -> int:
    """Algorithmic bytes per row of the radix sort: the key build (read 8,
    write 12); per digit pass the digit count (the 8-byte keys in the first
    pass, then the 1-byte digits that the previous scatter wrote), the scatter
    (read 12; write 12, or only the 4-byte row in a last pass that stores no
    keys) and, before every pass but the last, the next pass's digit (1)."""
    b = 20
    for p in range(passes):
        last = p == passes - 1
        b += (8 if p == 0 else 1) + 12 + (12 if keys_last or not last else 4) + (0 if last else 1)
    return b


def _time_steps(fn, K, W, stream, torch):
    """CUDA-event time of K calls of fn() on `stream` after W warm-ups."""
    for _ in range(W):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(K):
        fn()
    e.record(stream)
    torch.cuda.synchronize()
    return s.elapsed_time(e) / K


def run_secondary(args):
    """Per-operator lines for the other hot-path rows (not the headline):
    filter_groupby (fused WHERE -> GROUP BY dept, 20 B/row), aggregate
    (aggregates under one WHERE compare, 16 B/row), join (1M build x
    100M probe, INNER/LEFT/SEMI/ANTI), groupby (100M Zipf keys, 16 B/row + 40 B
    per group)."""
    import torch

    import falcondb_b200 as F
    from falcondb_b200 import ops, workloads as W
    from oracle import oracle as O

    dev = torch.device("cuda", 0)
    db = F.Database(0)
    if args.tuning:
        db.load_tuning(args.tuning)
    stream = ops.lib_stream(db)
    peak, peak_kind = peaks()
    out = []
    n = args.rows
    K, Wm = args.steps, args.warmup

    def line(name, ms, nbytes, extra):
        gbs = nbytes / (ms / 1e3) / 1e9
        d = {"metric": METRIC, "workload": name, "value": round(gbs, 1), "unit": "GB/s", "ms": round(ms, 4),
             "frac_of_measured_hbm": round(gbs / peak, 4), "frac_vs_8TBs": round(gbs / 8000, 4),
             "algorithmic_bytes": nbytes, "steps": K, "warmup": Wm}
        d.update(extra)
        out.append(d)

    if args.workload in ("filter_groupby", "all"):
        for rows in sorted({1_000_000, n}):
            t = W.table_t(rows, seed=1)
            db.create_table("t", t)
            cols = [db.column("t", c) for c in ("dept", "score", "salary")]
            prog = [ops.cmp(1, F.GT, 50)]
            aggs = [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_AVG, 2)]
            res = ops._bytes(F.AGG_VALUE_DTYPE.itemsize * 13 * 3, db)
            grows = torch.empty(13, dtype=torch.int64, device=dev)
            L = F.lib()
            ca, nc = ops._cols(cols)
            pa, npr = ops._prog(prog)
            aa, na = ops._aggs(aggs)

            def q():
                F.check(L.fdb_group_by_codes(db.handle, ca, nc, rows, pa, npr, 0, 12, aa, na, res.data_ptr(),
                                             grows.data_ptr()))
            ms = _time_steps(q, K, Wm, stream, torch)
            g = O.group_codes(t["dept"].codes, 12, mask=O.cmp_mask(t["score"], F.GT, 50), fvals=t["score"],
                              ivals=t["salary"])
            assert list(grows.cpu().numpy()[:12]) == list(g["rows"][:12])
            line("filter_groupby", ms, 20 * rows, {"rows": rows, "query": "SELECT dept, COUNT(*), SUM(score), "
                                                   "AVG(salary) FROM t WHERE score > 50 GROUP BY dept"})
            db.drop_table("t")

    if args.workload in ("aggregate", "all"):
        # Aggregates under one WHERE compare (FilterAggOp): 16 B/row of score
        # and salary; then SUM(salary) alone under the same WHERE for scale.
        t = W.table_t(n, seed=1)
        db.create_table("t", t)
        cols = [db.column("t", c) for c in ("score", "salary")]
        L = F.lib()
        sel = t["score"] > 50
        ca, nc = ops._cols(cols)
        pa, npr = ops._prog([ops.cmp(0, F.GT, 50)])
        for name, aggs in (("aggregate_where", [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 0), (F.AGG_AVG, 1),
                                                (F.AGG_MAX, 0)]),
                           ("sum_where", [(F.AGG_SUM, 1)])):
            res = ops._bytes(F.AGG_VALUE_DTYPE.itemsize * len(aggs), db)
            aa, na = ops._aggs(aggs)
            ms = _time_steps(lambda: F.check(L.fdb_aggregate(db.handle, ca, nc, n, pa, npr, aa, na, res.data_ptr())),
                             K, Wm, stream, torch)
            rec = ops.to_records(res, F.AGG_VALUE_DTYPE, len(aggs))
            if name == "aggregate_where":
                assert rec[0]["i"] == int(sel.sum())
                assert abs(rec[1]["f"] - O.sum_serial(t["score"][sel])) <= 1e-12 * rec[1]["f"]
                assert rec[2]["f"] == float(O.sum_i64_exact(t["salary"][sel])) / int(sel.sum())
                assert rec[3]["f"] == float(t["score"][sel].max())
                q = "SELECT COUNT(*), SUM(score), AVG(salary), MAX(score) FROM t WHERE score > 50"
            else:
                assert rec[0]["f"] == float(O.sum_i64_exact(t["salary"][sel]))
                q = "SELECT SUM(salary) FROM t WHERE score > 50"
            line(name, ms, 16 * n, {"rows": n, "query": q})
        db.drop_table("t")

    if args.workload in ("join", "all"):
        nb, npb = 1_000_000, n
        b0, p0 = W.join_tables(nb, npb, seed=7)
        # The build keys are a permutation of 0..nb-1, so the table is direct-
        # addressed; "_hashed" scatters every key (x 7919 + 3) so that the same
        # join runs on a hashed table.
        for tag, scale in (("", None), ("_hashed", 7919)):
            b, p = dict(b0), dict(p0)
            if scale:
                b["key"] = b0["key"] * scale + 3
                p["key"] = p0["key"] * scale + 3
            db.create_table("b", b)
            db.create_table("p", p)
            bk, bp = db.column("b", "key"), db.column("b", "payload")
            pk, pv = db.column("p", "key"), db.column("p", "value")
            res = ops._bytes(F.JOIN_AGG_DTYPE.itemsize, db)
            ms_build = _time_steps(lambda: ops.HashTable(db, bk, bp, nb).free(), max(3, K // 5), 2, stream, torch)
            h = ops.HashTable(db, bk, bp, nb)
            for jt, name in [(F.JOIN_INNER, "inner"), (F.JOIN_LEFT, "left"), (F.JOIN_SEMI, "semi"),
                             (F.JOIN_ANTI, "anti")]:
                val = pv if jt >= F.JOIN_SEMI else None
                ms = _time_steps(lambda: h.probe_agg(pk, npb, jt, value=val, out=res), K, Wm, stream, torch)
                got = ops.to_records(res, F.JOIN_AGG_DTYPE, 1)[0]
                nbytes = 8 * npb + (8 * npb if jt >= F.JOIN_SEMI else 0)
                line(f"join_probe_{name}{tag}", ms, nbytes, {
                    "build_rows": nb, "probe_rows": npb, "count": int(got["count"]),
                    "table": "direct-addressed" if h.dense else "hashed", "build_ms": round(ms_build, 4),
                    "query_ms_build_plus_probe": round(ms + ms_build, 4),
                    "query_GBps": round((nbytes + 16 * nb) / ((ms + ms_build) / 1e3) / 1e9, 1)})
            want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], F.JOIN_INNER)
            got = ops.to_records(h.probe_agg(pk, npb, F.JOIN_INNER, out=res), F.JOIN_AGG_DTYPE, 1)[0]
            assert int(got["count"]) == want["count"] and int(got["sum_payload"]) == want["sum_payload"]
            h.free()
            db.drop_table("b")
            db.drop_table("p")

    if args.workload in ("groupby", "all"):
        g = W.groupby_table(n, distinct=10_000_000, seed=11)
        db.create_table("g", g)
        gk, gv = db.column("g", "key"), db.column("g", "v")
        cap = 12_000_000
        outb = ops._bytes(F.GROUP_I64_DTYPE.itemsize * cap, db)
        ng = torch.empty(1, dtype=torch.int64, device=dev)
        lf = args.load_factor

        def q():
            ops.group_by_i64(db, gk, gv, n, expected_groups=0, load_factor=lf, capacity=cap, out=outb,
                             ngroups=ng)
        db.set_option("zone_maps", 0)
        ms_pass = _time_steps(q, K, Wm, stream, torch)
        db.set_option("zone_maps", 1)
        ms = _time_steps(q, K, Wm, stream, torch)
        groups = int(ng.item())
        # After timing: every group against the oracle (keys, counts, MIN/MAX
        # exactly; SUM within 1e-12 relative).
        rec = ops.to_records(outb, F.GROUP_I64_DTYPE, groups)
        rec = rec[np.argsort(rec["key"], kind="stable")]
        want = O.group_i64(g["key"], g["v"])
        assert np.array_equal(rec["key"], want["key"]) and np.array_equal(rec["count"], want["count"])
        assert np.array_equal(rec["min"], want["min"]) and np.array_equal(rec["max"], want["max"])
        assert float((np.abs(rec["sum"] - want["sum"]) / np.abs(want["sum"])).max()) <= 1e-12
        del rec, want
        line("groupby_zipf", ms, 16 * n + 40 * groups, {"rows": n, "groups": groups, "distinct_domain": 10_000_000,
                                                        "zipf_s": 1.1, "load_factor": lf, "oracle_checked": True,
                                                        "table_sizing": ZONE_SIZING,
                                                        "ms_with_sizing_pass": round(ms_pass, 4)})
        db.drop_table("g")

    if args.workload in ("batch", "all"):
        # 64 GROUP BY key queries over slices of the 100M-row Zipf table, sizes
        # log-uniform in [10k, 10M] rows, offsets uniform: one captured graph
        # (the autotuner's tuning) against the same queries run one by one.
        g = W.groupby_table(n, distinct=10_000_000, seed=11)
        db.create_table("g", g)
        kt = torch.from_numpy(g["key"]).to(dev)
        vt = torch.from_numpy(g["v"]).to(dev)
        rng = np.random.default_rng(64)
        sizes = np.minimum(np.floor(10 ** (4 + 3 * rng.random(64))).astype(np.int64), n)
        offs = [int(rng.integers(0, n - s + 1)) for s in sizes]
        qs = [(kt[o:o + int(s)], vt[o:o + int(s)], int(s)) for o, s in zip(offs, sizes)]
        rows_total = int(sizes.sum())
        tuning, tuned_ms = ops.GroupByBatch.autotune(db, qs, reps=2)
        b = ops.GroupByBatch(db, qs, tuning=tuning)
        ms_batch = _time_steps(b.run, K, Wm, stream, torch)
        groups = [int(b.outs[i][1].item()) for i in range(len(qs))]
        outs = [(ops._bytes(F.GROUP_I64_DTYPE.itemsize * (gq + 1), db), torch.empty(1, dtype=torch.int64, device=dev))
                for gq in groups]

        def serial():
            for (kk, vv, s), gq, (ob, nb) in zip(qs, groups, outs):
                ops.group_by_i64(db, kk, vv, s, expected_groups=max(gq, 1), capacity=gq + 1, out=ob, ngroups=nb)
        ms_serial = _time_steps(serial, K, Wm, stream, torch)
        assert [int(nb.item()) for _, nb in outs] == groups
        b.free()
        nbytes = 16 * rows_total + 40 * sum(groups)
        line("groupby_batched", ms_batch, nbytes, {
            "queries": len(qs), "rows_total": rows_total, "groups_total": sum(groups),
            "qps_batched": round(len(qs) / (ms_batch / 1e3), 1), "ms_serial": round(ms_serial, 4),
            "qps_serial": round(len(qs) / (ms_serial / 1e3), 1), "speedup_vs_serial": round(ms_serial / ms_batch, 2),
            "tuning": {"load_factor": tuning[0], "ctas_per_sm": tuning[1], "tile_rows": tuning[2]},
            "serial": "the same 64 queries as fdb_group_by_i64 calls in sequence, tables sized to the exact "
                      "group counts"})
        db.drop_table("g")
    if args.workload in ("sort", "all"):
        # ORDER BY score DESC over 100M FLOAT64 rows, no LIMIT: an LSD radix
        # sort of (order key, row) pairs (bytes per row: radix_bytes_per_row).
        host_sc = W.table_t(n, seed=1)["score"]
        sc = torch.from_numpy(host_sc).to(dev)
        rows_out = torch.empty(n, dtype=torch.int32, device=dev)
        ms = _time_steps(lambda: ops.sort(db, sc, n, True, rows=rows_out), K, Wm, stream, torch)
        bits = host_sc.view(np.uint64)
        ordk = np.where(bits >> np.uint64(63) == 0, bits ^ np.uint64(1 << 63), ~bits)  # f64_ord_key
        vary = int(np.bitwise_or.reduce(ordk)) ^ int(np.bitwise_and.reduce(ordk))
        passes = sum(1 for byte in range(8) if (vary >> (8 * byte)) & 255)
        del bits, ordk
        r = rows_out[:n].long()
        s_sorted = sc[r]
        assert bool((s_sorted[1:] <= s_sorted[:-1]).all())
        seen = torch.zeros(n, dtype=torch.bool, device=dev)
        seen[r] = True
        assert bool(seen.all())
        del r, s_sorted, seen
        nbytes = n * radix_bytes_per_row(passes, keys_last=False)
        sample = 10_000_000 if n >= 10_000_000 else n
        hs = sc[:sample].cpu().numpy()
        threads = args.cpu_threads or O.hardware_threads()
        t0 = time.perf_counter()
        O.ref_sort(hs, True, threads)
        cpu_s = time.perf_counter() - t0
        line("sort", ms, nbytes, {"rows": n, "query": "SELECT score FROM t ORDER BY score DESC",
                                  "digit_passes": passes, "mrows_per_s": round(n / (ms / 1e3) / 1e6, 1),
                                  "cpu_sample": {"rows": sample, "mrows_per_s": round(sample / cpu_s / 1e6, 2),
                                                 "cores": threads, "kind": "port",
                                                 "what": "reference-shaped sort: (order key, row) pair loop, "
                                                         "parallel tuple sort (oracle/refengine.cpp ref_sort)"}})
        # SELECT DISTINCT score (first occurrence per value, row order): the same
        # radix sort on value keys (every pass writes keys), a run-head pass
        # (read 12 per row, a bit per row of mask) and the mask's compaction
        # (4 bytes per kept row).
        dcount = torch.empty(1, dtype=torch.int64, device=dev)
        ms_d = _time_steps(lambda: ops.distinct(db, sc, n, rows=rows_out, count=dcount), K, Wm, stream, torch)
        kept = int(dcount.item())
        assert kept == int(torch.unique(sc).numel())
        hs_d = hs[:2_000_000]
        t0 = time.perf_counter()
        O.distinct(hs_d)
        cpu_d = time.perf_counter() - t0
        line("distinct", ms_d, n * (radix_bytes_per_row(passes, keys_last=True) + 12) + n // 4 + kept * 4,
             {"rows": n, "query": "SELECT DISTINCT score FROM t", "distinct_values": kept,
              "mrows_per_s": round(n / (ms_d / 1e3) / 1e6, 1),
              "cpu_sample": {"rows": len(hs_d), "mrows_per_s": round(len(hs_d) / cpu_d / 1e6, 2), "cores": 1,
                             "kind": "port", "what": "oracle hash-set first-occurrence scan"}})
        del rows_out
        torch.cuda.empty_cache()
        # The same operators end to end through Database::sql at the sizes the
        # reference publishes them (100K and 1M rows): host wall time per query,
        # result rows fetched to host memory included.
        for rows in (100_000, 1_000_000):
            db.create_table("s", W.table_t(rows, seed=2))
            for name, sql in (("order_by_full", "SELECT id FROM s ORDER BY score DESC"),
                              ("distinct", "SELECT DISTINCT score FROM s"),
                              ("row_number", "SELECT ROW_NUMBER() OVER (ORDER BY score DESC) AS rn FROM s")):
                for _ in range(Wm):
                    db.sql(sql)
                times = []
                for _ in range(K):
                    t0 = time.perf_counter()
                    r = db.sql(sql)
                    times.append((time.perf_counter() - t0) * 1e3)
                out.append({"metric": "SQL wall time", "workload": f"sql_{name}", "rows": rows, "query": sql,
                            "value": round(statistics.median(times), 4), "unit": "ms", "result_rows": r.rows,
                            "steps": K, "warmup": Wm, "higher_is_better": False})
            db.drop_table("s")
    if args.workload in ("parquet", "all"):
        # The configuration's table t (id, dept, score, salary) as a Parquet
        # file of 65,536-row row groups, loaded into HBM: host decode by
        # pyarrow, text dictionaries merged and remapped on the GPU.
        import tempfile

        import pyarrow as pa
        import pyarrow.parquet as pq

        from falcondb_b200 import parquet as P
        tp = W.table_t(n, seed=3)
        with tempfile.TemporaryDirectory() as tmp:
            path = f"{tmp}/t.parquet"
            dept = pa.DictionaryArray.from_arrays(pa.array(tp["dept"].codes.view(np.int32)),
                                                  pa.array(tp["dept"].dictionary))
            pq.write_table(pa.table({"id": tp["id"], "dept": dept, "score": tp["score"], "salary": tp["salary"]}),
                           path, row_group_size=65_536)
            size = Path(path).stat().st_size
            times = []
            for _ in range(3):
                t0 = time.perf_counter()
                P.load_parquet(db, path, "pq")
                times.append(time.perf_counter() - t0)
            cnt = db.sql("SELECT COUNT(*) FROM pq WHERE score > 50").column(0)[0]
            assert cnt == O.popcount(O.cmp_mask(tp["score"], F.GT, 50))
            g = db.sql("SELECT dept, COUNT(*) FROM pq GROUP BY dept ORDER BY dept")
            want = np.bincount(tp["dept"].codes, minlength=12)
            assert list(g.column(0)) == W.DEPTS and list(g.column(1)) == list(want)
            db.drop_table("pq")
        out.append({"metric": "Parquet load time", "workload": "parquet_load", "rows": n, "file_bytes": size,
                    "value": round(min(times), 3), "unit": "s", "higher_is_better": False,
                    "runs_s": [round(x, 3) for x in times], "row_group_rows": 65_536,
                    "what": "load_parquet: pyarrow host decode (all host threads) + GPU dictionary merge + upload",
                    "oracle_checked": True})
    if args.workload in ("rest", "all"):
        run_rest(args, db, out)
    if args.workload in ("serve", "all"):
        run_serving(args, db, out, peak)
    if args.workload == "serve_single":
        run_serving_single(args, db, out)
    db.close()
    return out


def run_rest(args, db, out):
    """POST /sql through the REST front end: 32 closed-loop HTTP clients send
    2000 requests (500 on the fdb_sql-only leg) drawn from the four serving
    templates (random thresholds)
    over a 10M-row table and a 1M x 10M join.  Once with the serving loop
    batching template requests, once with every request through fdb_sql (the
    reference server's one-request-at-a-time shape).  Client-side latency and
    throughput; every answer is checked against a fdb_sql run of the same text."""
    import json
    import urllib.request
    from concurrent.futures import ThreadPoolExecutor

    from falcondb_b200 import rest as R, workloads as W

    db.create_table("t", W.table_t(10_000_000, seed=21))
    b, p = W.join_tables(1_000_000, 10_000_000, seed=22)
    db.create_table("b", b)
    db.create_table("p", p)
    rng = np.random.default_rng(23)
    shapes = ["SELECT COUNT(*) FROM t WHERE score > {x}",
              "SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM t WHERE score > {x} GROUP BY dept",
              "SELECT id, score FROM t WHERE score < {x} ORDER BY score DESC LIMIT 10",
              "SELECT COUNT(*), SUM(b.payload) FROM p JOIN b ON p.key = b.key WHERE p.value < {y}"]
    texts = []
    for _ in range(2000):
        x = round(float(rng.uniform(0, 100)), 2)
        texts.append(shapes[int(rng.integers(0, 4))].format(x=x, y=f"{x / 100:.4f}"))
    check = {t: db.sql(t).rows for t in set(texts[:50])}

    def post(port, sql):
        req = urllib.request.Request(f"http://127.0.0.1:{port}/sql", data=json.dumps({"sql": sql}).encode(),
                                     method="POST", headers={"Content-Type": "application/json"})
        t0 = time.perf_counter()
        with urllib.request.urlopen(req, timeout=120) as r:
            body = json.loads(r.read())
        return sql, body, (time.perf_counter() - t0) * 1e3

    res = {}
    for batching in (True, False):
        # The fdb_sql-only leg runs a quarter of the requests: it is the slow one.
        run_texts = texts if batching else texts[:500]
        srv = R.RestServer(db, port=0, batching=batching, max_batch=64, slots=2).start()
        try:
            with ThreadPoolExecutor(32) as ex:
                list(ex.map(lambda s_: post(srv.port, s_), texts[:64]))  # warm-up
                t0 = time.perf_counter()
                got = list(ex.map(lambda s_: post(srv.port, s_), run_texts))
                wall = time.perf_counter() - t0
        finally:
            srv.stop()
        for sql, body, _ in got:
            if sql in check:
                assert body["row_count"] == check[sql], sql
        lat = np.array([g[2] for g in got])
        served = sum(1 for g in got if g[1]["path"] == "serving")
        res[batching] = {"requests": len(run_texts), "qps": round(len(run_texts) / wall, 1),
                         "p50_ms": round(float(np.percentile(lat, 50)), 3),
                         "p99_ms": round(float(np.percentile(lat, 99)), 3), "served": served,
                         "mean_batch": round(float(np.mean([g[1].get("batch_size", 1) for g in got])), 2)}
    out.append({"metric": "REST /sql throughput", "workload": "rest_sql", "value": res[True]["qps"],
                "unit": "requests/s", "higher_is_better": True, "requests": len(texts), "clients": 32,
                "batched": res[True], "sql_only": res[False],
                "speedup_vs_sql_only": round(res[True]["qps"] / res[False]["qps"], 2),
                "tables": "t: 10M rows; join: 1M build x 10M probe"})
    for name in ("t", "b", "p"):
        db.drop_table(name)


def run_serving(args, db, out, peak):
    """10,000 queries from the 4 serving templates (filter-count, filter-group-by,
    inner join, top-k) over prefixes of 100M-row resident tables, prefix sizes
    log-uniform in [10k, 100M] rows, thresholds uniform in [0, 100), arriving as
    a Poisson process at 2000 qps; served with continuous batching and one query
    at a time, in real time (latency) and all at once (throughput)."""
    import torch

    from falcondb_b200 import ops, serving as S, workloads as W

    n = args.rows
    t = W.table_t(n, seed=1)
    dev = torch.device("cuda", 0)
    cols = {"score": torch.from_numpy(t["score"]).to(dev), "dept": torch.from_numpy(t["dept"].codes.view(np.int32)).to(dev),
            "salary": torch.from_numpy(t["salary"]).to(dev)}
    del t
    bt, pt = W.join_tables(1_000_000, n, seed=7)
    cols["pkey"] = torch.from_numpy(pt["key"]).to(dev)
    cols["pval"] = torch.from_numpy(pt["value"]).to(dev)
    del pt
    ht = ops.HashTable(db, torch.from_numpy(bt["key"]).to(dev), torch.from_numpy(bt["payload"]).to(dev),
                       len(bt["key"]))
    torch.cuda.synchronize()
    rng = np.random.default_rng(2000)
    nq, rate = args.serve_queries, 2000.0
    qs = []
    at = 0.0
    for _ in range(nq):
        kind = int(rng.integers(0, 4))
        rows = int(min(n, np.floor(10 ** (4 + (np.log10(n) - 4) * rng.random()))))
        x = float(rng.random() * 100)
        at += float(rng.exponential(1.0 / rate))
        if kind == S.SERVE_COUNT:
            q = S.count_query(cols["score"].data_ptr(), rows, x)
        elif kind == S.SERVE_GROUP:
            q = S.group_query(cols["score"].data_ptr(), cols["dept"].data_ptr(), cols["salary"].data_ptr(), 12, rows, x)
        elif kind == S.SERVE_JOIN:
            q = S.join_query(cols["pkey"].data_ptr(), cols["pval"].data_ptr(), ht._h.value, rows, x)
        else:
            q = S.topk_query(cols["score"].data_ptr(), rows, x, k=10)
        q.arrival_s = at
        qs.append(q)
    budget = 40 << 30
    burst = [S.Query(**{**q.__dict__, "arrival_s": 0.0}) for q in qs]
    S.serve_trace(db, burst[:200], max_batch=128, slots=4, mem_budget=budget)  # warm-up
    res_b, live_b = S.serve_trace(db, qs, max_batch=128, slots=args.serve_slots, mem_budget=budget)
    res_s, live_s = S.serve_trace(db, qs, max_batch=1, slots=1, mem_budget=budget)
    _, sat_b = S.serve_trace(db, burst, max_batch=128, slots=args.serve_slots, mem_budget=budget)
    _, sat_s = S.serve_trace(db, burst, max_batch=1, slots=1, mem_budget=budget)
    same = all(a.status == 0 and b.status == 0 and a.count == b.count and a.sum_payload == b.sum_payload
               and list(a.group_count) == list(b.group_count) and list(a.rows[:a.count]) == list(b.rows[:b.count])
               for a, b in zip(res_b, res_s))
    ht.free()

    def d(st):
        return {"qps": round(st.qps, 1), "p50_ms": round(st.p50_ms, 4), "p99_ms": round(st.p99_ms, 4),
                "max_ms": round(st.max_ms, 4), "mean_batch": round(st.mean_batch, 2), "batches": st.batches}

    def by_kind(res):
        names = {S.SERVE_COUNT: "count", S.SERVE_GROUP: "group", S.SERVE_JOIN: "join", S.SERVE_TOPK: "topk"}
        outk = {}
        for kind, name in names.items():
            lat = sorted((r.done_s - r.arrival_s) * 1e3 for q, r in zip(qs, res) if q.kind == kind)
            big = sorted((r.done_s - r.arrival_s) * 1e3 for q, r in zip(qs, res) if q.kind == kind and q.nrows >= n // 2)
            if lat:
                outk[name] = {"p50_ms": round(lat[len(lat) // 2], 4), "p99_ms": round(lat[int(0.99 * (len(lat) - 1))], 4),
                              "p50_ms_rows_ge_half": round(big[len(big) // 2], 4) if big else None}
        return outk
    out.append({"metric": METRIC, "workload": "serving", "value": round(sat_b.qps, 1), "unit": "queries/s",
                "higher_is_better": True, "queries": nq, "arrival_qps": rate,
                "templates": "filter-count, filter-group-by, inner join, top-k (uniform)",
                "table_rows": n, "prefix_rows": "log-uniform [10k, 100M]", "thresholds": "uniform [0, 100)",
                "mem_budget_bytes": budget, "slots": args.serve_slots, "max_batch": 128, "resident_bytes": live_b.resident_bytes,
                "peak_reserved_bytes": live_b.peak_reserved,
                "at_2000qps": {"batched": d(live_b), "serial": d(live_s)},
                "at_2000qps_by_template": {"batched": by_kind(res_b), "serial": by_kind(res_s)},
                "saturated": {"batched": d(sat_b), "serial": d(sat_s)},
                "throughput_speedup": round(sat_b.qps / sat_s.qps, 2) if sat_s.qps else None,
                "results_identical_batched_vs_serial": same})


def run_serving_single(args, db, out):
    """Each serving template on its own: 20 queries over all n rows of the
    serving tables, 20 ms apart, so that every query runs alone on the GPU;
    the line reports each template's median latency (submit to result on the
    host) over the last 17.  Launch order: 20 COUNT, 20 GROUP, 20 JOIN, 20
    TOPK batches."""
    import torch

    from falcondb_b200 import ops, serving as S, workloads as W

    n = args.rows
    dev = torch.device("cuda", 0)
    t = W.table_t(n, seed=1)
    score = torch.from_numpy(t["score"]).to(dev)
    dept = torch.from_numpy(t["dept"].codes.view(np.int32)).to(dev)
    sal = torch.from_numpy(t["salary"]).to(dev)
    del t
    bt, pt = W.join_tables(1_000_000, n, seed=7)
    pkey = torch.from_numpy(pt["key"]).to(dev)
    pval = torch.from_numpy(pt["value"]).to(dev)
    del pt
    ht = ops.HashTable(db, torch.from_numpy(bt["key"]).to(dev), torch.from_numpy(bt["payload"]).to(dev),
                       len(bt["key"]))
    torch.cuda.synchronize()
    make = {
        "count": lambda: S.count_query(score.data_ptr(), n, 50.0),
        "group": lambda: S.group_query(score.data_ptr(), dept.data_ptr(), sal.data_ptr(), 12, n, 50.0),
        "join": lambda: S.join_query(pkey.data_ptr(), pval.data_ptr(), ht._h.value, n, 50.0),
        "topk": lambda: S.topk_query(score.data_ptr(), n, 50.0, k=10),
    }
    lat = {}
    for name, f in make.items():
        qs = []
        for i in range(20):
            q = f()
            q.arrival_s = 0.02 * i
            qs.append(q)
        res, _ = S.serve_trace(db, qs, max_batch=128, slots=1, mem_budget=40 << 30)
        ms = sorted((r.done_s - r.arrival_s) * 1e3 for r in res[3:])
        lat[name] = round(ms[len(ms) // 2], 4)
    ht.free()
    out.append({"metric": METRIC, "workload": "serving_single", "unit": "ms", "higher_is_better": False,
                "rows": n, "median_latency_ms": lat,
                "queries": "20 per template over all rows, 20 ms apart (threshold 50; join value < 0.5; k = 10)"})


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from oracle import oracle as O

    threads = args.cpu_threads or O.hardware_threads()
    n = args.rows
    t = make_table(n, seed=1)
    for _ in range(args.warmup):
        cpu_queries(t, n, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_queries(t, n, threads)
    el = time.perf_counter() - t0
    value = sum(BYTES_PER_ROW.values()) * n * args.steps / el / 1e9
    base = {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"{args.steps} passes of the 5 queries over {n} rows"}
    return {"metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(el / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64/int64", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": {"workload": "scan+top-k 100M rows (the 5 queries), reference-shaped C++ CPU engine",
                       "rows": n},
            "cpu_baseline": base,
            "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--rows", type=int, default=N_ROWS)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations' extra keys (1 GPU only)")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--workload", default="scan",
                    choices=["scan", "filter_groupby", "aggregate", "join", "groupby", "batch", "sort", "parquet", "rest", "serve", "serve_single",
                             "all"],
                    help="scan = the headline line; the others print per-operator lines")
    ap.add_argument("--load-factor", type=float, default=0.5)
    ap.add_argument("--tuning", default="", help="a launch-tuning cache (fdb_tuning_save) to load first")
    ap.add_argument("--serve-queries", type=int, default=10_000)
    ap.add_argument("--serve-slots", type=int, default=2)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload != "scan" and args.impl != "reference":
        for line in run_secondary(args):
            print(json.dumps(line), flush=True)
        return
    res = run_reference(args) if args.impl == "reference" else run_gpu(args)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
