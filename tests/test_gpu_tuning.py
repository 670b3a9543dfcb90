"""Launch tuning on the GPU (the counterpart of tuning.rs:39-53's cut-offs):
every kind of streamed operator gives the oracle's answer under extreme
tunings (one CTA in all; a few CTAs per SM with a row minimum), the autotuner
returns valid choices and keeps them, and the JSON cache round-trips and
refuses a file written for another device."""
import json

import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-12
EXTREMES = [(1, 1 << 40), (2, 1 << 16), (0, 0)]   # (CTAs per SM, rows per CTA); the last is the default


@pytest.fixture
def tuned_db(db, tmp_path):
    yield db
    # Back to the defaults (the batched GROUP BY's too) for the tests after.
    path = tmp_path / "defaults.json"
    db.save_tuning(path)
    doc = json.loads(path.read_text())
    doc["ops"] = {k: {"ctas_per_sm": 0, "min_rows_per_cta": 0} for k in F.TUNE_KINDS}
    doc["gb_batch"] = {"load_factor": 0, "ctas_per_sm": 0, "tile_rows": 0}
    path.write_text(json.dumps(doc))
    db.load_tuning(path)


def test_answers_do_not_depend_on_the_tuning(tuned_db):
    db = tuned_db
    n = 3_000_017
    t = W.table_t(n, seed=21)
    db.create_table("t", t)
    score, dept, salary = db.column("t", "score"), db.column("t", "dept"), db.column("t", "salary")
    mask = O.cmp_mask(t["score"], F.GT, 50)
    want_count = O.popcount(mask)
    want_sum = O.sum_serial(t["score"][O.mask_rows(mask, n)])
    g0 = O.group_codes(t["dept"].codes, 12, mask=mask, fvals=t["score"], ivals=t["salary"])
    keys = (np.arange(n, dtype=np.int64) * 7919) % 50_000
    db.create_table("g", {"k": keys, "v": t["score"]})
    gk, gv = db.column("g", "k"), db.column("g", "v")
    want_g = O.group_i64(keys, t["score"])
    b = {"key": np.random.default_rng(2).permutation(100_000).astype(np.int64),
         "payload": np.arange(100_000, dtype=np.int64)}
    db.create_table("b", b)
    ht = ops.HashTable(db, db.column("b", "key"), db.column("b", "payload"), 100_000)
    pk = (np.arange(n, dtype=np.int64) * 31) % 200_000
    db.create_table("p", {"key": pk})
    want_j = O.join_agg(b["key"], b["payload"], pk, np.zeros(n), F.JOIN_INNER)
    want_top = O.topk(t["score"], 10, True)
    try:
        for cps, rows in EXTREMES:
            for k in range(len(F.TUNE_KINDS)):
                db.set_tuning(k, cps, rows)
            cnt = ops.filter_count(db, [score], n, [ops.cmp(0, F.GT, 50)])
            assert int(cnt.item()) == want_count
            agg = ops.to_records(ops.aggregate(db, [score], n, [ops.cmp(0, F.GT, 50)], [(F.AGG_SUM, 0)]),
                                 F.AGG_VALUE_DTYPE, 1)[0]
            assert abs(agg["f"] - want_sum) <= RTOL * want_sum
            out, grows = ops.group_by_codes(db, [dept, score, salary], n, [ops.cmp(1, F.GT, 50)], 0, 12,
                                            [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_AVG, 2)])
            assert list(grows.cpu().numpy()[:12]) == list(g0["rows"][:12])
            go, ng = ops.group_by_i64(db, gk, gv, n)
            rec = ops.to_records(go, F.GROUP_I64_DTYPE, int(ng.item()))
            rec = rec[np.argsort(rec["key"], kind="stable")]
            assert np.array_equal(rec["key"], want_g["key"]) and np.array_equal(rec["count"], want_g["count"])
            assert np.array_equal(rec["min"], want_g["min"]) and np.array_equal(rec["max"], want_g["max"])
            j = ops.to_records(ht.probe_agg(db.column("p", "key"), n, F.JOIN_INNER), F.JOIN_AGG_DTYPE, 1)[0]
            assert (int(j["count"]), int(j["sum_payload"])) == (want_j["count"], want_j["sum_payload"])
            rows_out, c = ops.topk(db, score, n, 10, True)
            assert rows_out.cpu().numpy().view(np.uint32)[:int(c.item())].tolist() == want_top.tolist()
    finally:
        ht.free()


def test_autotune_keeps_valid_choices(tuned_db, tmp_path):
    db = tuned_db
    best, ms = db.autotune(rows=1 << 22, reps=3)
    assert set(best) == set(F.TUNE_KINDS) and set(ms) == set(F.TUNE_KINDS)
    for name, t in best.items():
        assert t["ctas_per_sm"] in (0, 1, 2, 3, 4), (name, t)
        assert t["min_rows_per_cta"] in (0, 1 << 15, 1 << 17, 1 << 19), (name, t)
        assert 0.0 < ms[name] < 1000.0
    assert db.tuning() == best
    # The operators still answer right under the chosen tuning.
    n = 1_000_003
    v = np.random.default_rng(1).random(n)
    db.create_table("s", {"v": v})
    cnt = ops.filter_count(db, [db.column("s", "v")], n, [ops.cmp(0, F.LT, 0.25)])
    assert int(cnt.item()) == int((v < 0.25).sum())

    # The cache file round-trips.
    path = tmp_path / "tuning.json"
    db.set_tuning("probe", 3, 1 << 17)
    db.save_tuning(path)
    doc = json.loads(path.read_text())
    assert doc["ops"]["probe"] == {"ctas_per_sm": 3, "min_rows_per_cta": 1 << 17}
    assert doc["sm_count"] == torch.cuda.get_device_properties(0).multi_processor_count
    before = db.tuning()
    for k in range(len(F.TUNE_KINDS)):
        db.set_tuning(k, 0, 0)
    db.load_tuning(path)
    assert db.tuning() == before
    # A file for another device is refused and changes nothing.
    doc["device"] = "some other GPU"
    doc["ops"]["scan"] = {"ctas_per_sm": 1, "min_rows_per_cta": 0}
    other = tmp_path / "other.json"
    other.write_text(json.dumps(doc))
    with pytest.raises(F.FalconError) as e:
        db.load_tuning(other)
    assert e.value.code == -2
    assert db.tuning() == before
    with pytest.raises(F.FalconError):
        db.load_tuning(tmp_path / "missing.json")


def test_batch_tuning_is_kept_by_the_context(tuned_db, tmp_path):
    db = tuned_db
    rng = np.random.default_rng(4)
    n = 400_000
    keys = rng.integers(0, 20_000, n).astype(np.int64)
    vals = rng.random(n)
    db.create_table("q", {"k": keys, "v": vals})
    k, v = db.column("q", "k"), db.column("q", "v")
    kt = torch.from_numpy(keys).cuda()
    vt = torch.from_numpy(vals).cuda()
    qs = [(kt[i * 50_000:(i + 1) * 50_000], vt[i * 50_000:(i + 1) * 50_000], 50_000) for i in range(4)]
    best, _ = ops.GroupByBatch.autotune(db, qs, reps=2)
    path = tmp_path / "t.json"
    db.save_tuning(path)
    gb = json.loads(path.read_text())["gb_batch"]
    assert (gb["load_factor"], gb["ctas_per_sm"], gb["tile_rows"]) == best
    b = ops.GroupByBatch(db, qs)   # no tuning given: the context's
    b.run()
    for i in range(4):
        r = b.results(i)
        r = r[np.argsort(r["key"], kind="stable")]
        want = O.group_i64(keys[i * 50_000:(i + 1) * 50_000], vals[i * 50_000:(i + 1) * 50_000])
        assert np.array_equal(r["key"], want["key"]) and np.array_equal(r["count"], want["count"])
    b.free()
    del k, v
