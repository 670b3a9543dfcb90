"""Batched int64-key GROUP BY (fdb_gb_batch_*): many queries over slices of
one table in one captured CUDA graph.  Each query's groups must equal the
oracle's GROUP BY of its slice (counts, keys, MIN/MAX exact; SUM within
1e-12 relative), on the first replay and on later ones."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def check_query(rec, keys, vals):
    rec = rec[np.argsort(rec["key"], kind="stable")]
    want = O.group_i64(keys, vals)
    assert np.array_equal(rec["key"], want["key"])
    assert np.array_equal(rec["count"], want["count"])
    assert np.array_equal(rec["min"], want["min"]) and np.array_equal(rec["max"], want["max"])
    if len(want["sum"]):
        rel = np.abs(rec["sum"] - want["sum"]) / np.maximum(np.abs(want["sum"]), 1e-300)
        assert rel.max() <= RTOL


def slices(n_total, sizes, seed):
    r = np.random.default_rng(seed)
    return [(int(r.integers(0, n_total - s + 1)), int(s)) for s in sizes]


@pytest.mark.parametrize("tuning", [None, (0.35, 1, 4096), (0.7, 3, 16384)])
def test_batch_matches_each_query(db, tuning):
    n = 3_000_000
    t = W.groupby_table(n, distinct=1_000_000, seed=3)
    k, v = dev(t["key"]), dev(t["v"])
    sizes = [0, 1, 17, 1000, 10_000, 65_536, 65_537, 200_000, 1_000_000, 2_500_000]
    sl = slices(n, sizes, 1)
    b = ops.GroupByBatch(db, [(k[o:o + s], v[o:o + s], s) for o, s in sl], tuning=tuning)
    for rep in range(2):
        b.run()
        db.synchronize()
        for i, (o, s) in enumerate(sl):
            check_query(b.results(i), t["key"][o:o + s], t["v"][o:o + s])
    b.free()


def test_batch_null_keys_int_values_and_validity(db):
    n = 400_000
    r = np.random.default_rng(5)
    keys = r.integers(-1000, 1000, n)
    keys[::11] = np.iinfo(np.int64).min  # the NULL group
    vals = r.integers(0, 100, n)
    b = ops.GroupByBatch(db, [(dev(keys[:150_000]), dev(vals[:150_000]), 150_000),
                              (dev(keys[150_000:]), dev(vals[150_000:]), n - 150_000)])
    b.run()
    db.synchronize()
    check_query(b.results(0), keys[:150_000], vals[:150_000].astype(np.float64))
    check_query(b.results(1), keys[150_000:], vals[150_000:].astype(np.float64))
    b.free()
    # NULL values (validity on the value column): SUM/MIN/MAX skip them.
    valid = r.random(n) > 0.2
    vw = F.validity_words(valid)
    fv = r.random(n)
    b = ops.GroupByBatch(db, [(dev(keys), (dev(fv), dev(vw.view(np.int64))), n)])
    b.run()
    db.synchronize()
    rec = b.results(0)
    rec = rec[np.argsort(rec["key"], kind="stable")]
    import pandas as pd
    g = pd.DataFrame({"k": keys, "v": np.where(valid, fv, np.nan)}).groupby("k", sort=True)["v"]
    assert np.array_equal(rec["key"], g.size().index.to_numpy())
    assert np.array_equal(rec["count"], g.size().to_numpy())
    assert np.array_equal(rec["min"], g.min().to_numpy(), equal_nan=True)
    b.free()


def test_batch_too_small_a_table_reports_capacity(db):
    """A caller's expected_groups far below the truth fails loudly, never silently."""
    n = 300_000
    keys = np.random.default_rng(6).permutation(n).astype(np.int64)
    vals = np.ones(n)
    b = ops.GroupByBatch(db, [(dev(keys), dev(vals), n)], expected_groups=[1])
    b.run()
    with pytest.raises(F.FalconError):
        db.synchronize()
    b.free()
    db.synchronize()  # the error was reported once; the context is usable again


def test_batch_autotune_picks_a_working_tuning(db):
    n = 1_000_000
    t = W.groupby_table(n, distinct=100_000, seed=9)
    k, v = dev(t["key"]), dev(t["v"])
    qs = [(k[o:o + s], v[o:o + s], s) for o, s in slices(n, [5000, 50_000, 500_000], 2)]
    tuning, ms = ops.GroupByBatch.autotune(db, qs, reps=2)
    assert 0 < tuning[0] < 1 and tuning[1] >= 1 and tuning[2] >= 256 and ms > 0
    b = ops.GroupByBatch(db, qs, tuning=tuning)
    b.run()
    db.synchronize()
    for i, (kk, vv, s) in enumerate(qs):
        check_query(b.results(i), kk.cpu().numpy(), vv.cpu().numpy())
    b.free()
