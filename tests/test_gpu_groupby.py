"""GPU parity of GROUP BY: dictionary-code groups (fast_utf8_gb) and int64 hash
groups (fast_i64_gb) against the oracle.  Counts and integer sums bit-exact;
FP64 sums within 1e-12 relative; MIN/MAX exact."""
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


def close(a, b):
    return abs(a - b) <= RTOL * max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("n", [1, 65, 4096, 1_000_000, 3_000_017])
def test_filter_group_by_dept(db, n):
    """The config-0 query shape: WHERE score > 50 GROUP BY dept with COUNT(*),
    SUM(score), AVG(salary)."""
    t = W.table_t(n, seed=n)
    codes, score, salary = t["dept"].codes, t["score"], t["salary"]
    cols = [dev(codes.view(np.int32)), dev(score), dev(salary)]
    out, rows = ops.group_by_codes(db, cols, n, [ops.cmp(1, F.GT, 50)], 0, 12,
                                   [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_AVG, 2), (F.AGG_MIN, 1)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE).reshape(13, 4)[:13]
    grows = rows.cpu().numpy()
    mask = O.cmp_mask(score, F.GT, 50)
    g = O.group_codes(codes, 12, mask=mask, fvals=score, ivals=salary)
    assert list(grows) == list(g["rows"])
    for d in range(12):
        if g["rows"][d] == 0:
            continue
        assert rec[d, 0]["i"] == g["rows"][d]
        assert close(rec[d, 1]["f"], g["fsum"][d])
        assert rec[d, 2]["f"] == g["isum"][d] / g["icnt"][d]  # bit-exact: integer partial sums
        assert rec[d, 3]["f"] == g["fmin"][d]


def _same_f(a, b):
    return (np.isnan(a) and np.isnan(b)) or close(a, b)


OPS = [F.EQ, F.NE, F.LT, F.LE, F.GT, F.GE]


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("n,off,lit", [(1, 0, 50), (4099, 0, 50.0), (1_000_003, 0, 50), (100_001, 1, 49.5),
                                       (16_777_219, 0, 50.0)])
def test_lane_fast_path_every_operator(db, op, n, off, lit):
    """WHERE score <op> literal GROUP BY code with COUNT(*), SUM(score),
    AVG(salary) — the specialised lane kernel's shape — over NaN scores (only
    != accepts them), scores equal to the literal, NULL and out-of-dictionary
    codes, int and float literals, (off=1) views that are not 16-byte aligned,
    which take the plain-load path, and both launch shapes (2^24 rows and
    more run the large-input shape)."""
    r = np.random.default_rng(n * 7 + op)
    tot = n + off
    codes = r.integers(0, 14, tot).astype(np.uint32)  # 12 and 13 are outside the 12-entry dictionary
    codes[::17] = 0xFFFFFFFF
    score = np.floor(r.random(tot) * 100.0)
    score[::23] = np.nan
    salary = r.integers(-(1 << 30), 1 << 30, tot)
    cols = [dev(codes.view(np.int32))[off:], dev(score)[off:], dev(salary)[off:]]
    codes, score, salary = codes[off:], score[off:], salary[off:]
    out, rows = ops.group_by_codes(db, cols, n, [ops.cmp(1, op, lit)], 0, 12,
                                   [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_AVG, 2)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE).reshape(13, 3)
    g = O.group_codes(codes, 12, mask=O.cmp_mask(score, op, lit), fvals=score, ivals=salary)
    assert list(rows.cpu().numpy()) == list(g["rows"])
    for d in range(13):
        assert rec[d, 0]["i"] == g["rows"][d]
        if g["rows"][d] == 0:
            continue
        assert _same_f(rec[d, 1]["f"], g["fsum"][d])
        assert rec[d, 2]["f"] == g["isum"][d] / g["icnt"][d]


@pytest.mark.parametrize("n", [5, 777_777])
def test_lane_fast_path_shapes(db, n):
    """The specialised lane kernel with 0, 2 and 3 summed slots over 1, 2 and
    4 staged columns (a column summed twice, int64 and FP64 slots mixed)."""
    t = W.table_t(n, seed=n)
    codes, score, salary, ids = t["dept"].codes, t["score"], t["salary"], t["id"]
    dc, ds, dsal, did = dev(codes.view(np.int32)), dev(score), dev(salary), dev(ids)
    # 1 column, COUNT(*) only.
    out, rows = ops.group_by_codes(db, [dc], n, [], 0, 12, [(F.AGG_COUNT_STAR, 0)])
    g = O.group_codes(codes, 12)
    assert list(rows.cpu().numpy()) == list(g["rows"])
    assert list(ops.to_records(out, F.AGG_VALUE_DTYPE)["i"]) == list(g["rows"])
    # 2 columns: the WHERE column summed twice.
    out, rows = ops.group_by_codes(db, [dc, ds], n, [ops.cmp(1, F.LT, 30.0)], 0, 12,
                                   [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_AVG, 1)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE).reshape(13, 3)
    g = O.group_codes(codes, 12, mask=O.cmp_mask(score, F.LT, 30.0), fvals=score)
    assert list(rows.cpu().numpy()) == list(g["rows"])
    for d in range(12):
        if g["rows"][d]:
            assert close(rec[d, 1]["f"], g["fsum"][d])
            assert close(rec[d, 2]["f"], g["fsum"][d] / g["fcnt"][d])
    # 4 columns, 3 summed slots.
    out, rows = ops.group_by_codes(db, [dc, ds, dsal, did], n, [ops.cmp(1, F.GE, 10.5)], 0, 12,
                                   [(F.AGG_SUM, 2), (F.AGG_SUM, 1), (F.AGG_AVG, 3), (F.AGG_COUNT_STAR, 0)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE).reshape(13, 4)
    mask = O.cmp_mask(score, F.GE, 10.5)
    g1 = O.group_codes(codes, 12, mask=mask, fvals=score, ivals=salary)
    g2 = O.group_codes(codes, 12, mask=mask, ivals=ids)
    assert list(rows.cpu().numpy()) == list(g1["rows"])
    for d in range(12):
        if g1["rows"][d]:
            assert rec[d, 0]["f"] == g1["isum"][d]
            assert close(rec[d, 1]["f"], g1["fsum"][d])
            assert rec[d, 2]["f"] == g2["isum"][d] / g2["icnt"][d]
            assert rec[d, 3]["i"] == g1["rows"][d]


def test_group_by_codes_nulls_and_empty_groups(db):
    n = 50_000
    r = np.random.default_rng(3)
    codes = r.integers(0, 7, n).astype(np.uint32)
    codes[::13] = 0xFFFFFFFF
    vals = r.integers(-100, 100, n)
    valid = r.random(n) > 0.3
    vw = F.validity_words(valid)
    cols = [dev(codes.view(np.int32)), (dev(vals), dev(vw.view(np.int64)))]
    out, rows = ops.group_by_codes(db, cols, n, [], 0, 10, [(F.AGG_COUNT, 1), (F.AGG_SUM, 1), (F.AGG_MAX, 1)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE).reshape(11, 3)
    grows = rows.cpu().numpy()
    g = O.group_codes(codes, 10, ivals=vals, ivalid=vw)
    assert list(grows) == list(g["rows"])
    for d in range(11):
        if g["rows"][d] == 0:
            continue
        assert rec[d, 0]["i"] == g["icnt"][d]
        assert rec[d, 1]["f"] == g["isum"][d]
        sel = (np.where(codes == 0xFFFFFFFF, 10, codes) == d) & valid
        if sel.any():
            assert rec[d, 2]["f"] == float(vals[sel].max())
        else:
            assert rec[d, 2]["valid"] == 0


def test_group_by_codes_is_repeatable(db):
    n = 2_000_000
    t = W.table_t(n, seed=5)
    cols = [dev(t["dept"].codes.view(np.int32)), dev(t["score"])]
    outs = [ops.to_records(ops.group_by_codes(db, cols, n, [], 0, 12, [(F.AGG_SUM, 1)])[0], F.AGG_VALUE_DTYPE)
            for _ in range(3)]
    assert np.array_equal(outs[0]["f"], outs[1]["f"]) and np.array_equal(outs[1]["f"], outs[2]["f"])


def _hash_groups(db, keys, vals, **kw):
    n = len(keys)
    out, ng = ops.group_by_i64(db, dev(keys), dev(vals), n, **kw)
    g = int(ng.item())
    rec = ops.to_records(out, F.GROUP_I64_DTYPE, g)
    return rec[np.argsort(rec["key"], kind="stable")]


@pytest.mark.parametrize("n,distinct", [(1, 10), (1000, 50), (200_000, 100_000), (2_000_000, 1_000_000)])
def test_hash_group_by_zipf(db, n, distinct):
    t = W.groupby_table(n, distinct=distinct, seed=n)
    rec = _hash_groups(db, t["key"], t["v"])
    want = O.group_i64(t["key"], t["v"])
    assert np.array_equal(rec["key"], want["key"])
    assert np.array_equal(rec["count"], want["count"])
    assert np.array_equal(rec["min"], want["min"]) and np.array_equal(rec["max"], want["max"])
    rel = np.abs(rec["sum"] - want["sum"]) / np.maximum(np.abs(want["sum"]), 1e-300)
    assert rel.max() <= RTOL


def test_hash_group_by_null_keys_and_int_values(db):
    n = 100_000
    r = np.random.default_rng(8)
    keys = r.integers(-50, 50, n)
    keys[::17] = np.iinfo(np.int64).min  # reads as NULL (aggregate.rs:867)
    vals = r.integers(0, 1000, n)
    rec = _hash_groups(db, keys, vals)
    want = O.group_i64(keys, vals.astype(np.float64))
    assert np.array_equal(rec["key"], want["key"])
    assert np.array_equal(rec["count"], want["count"])
    assert np.array_equal(rec["sum"], want["sum"])  # integer-valued f64 sums are exact


def test_hash_group_by_all_distinct_and_load_factor(db):
    n = 500_000
    keys = np.random.default_rng(9).permutation(n).astype(np.int64) * 7 - 3
    vals = np.random.default_rng(10).random(n)
    for lf in (0.25, 0.5, 0.7):
        rec = _hash_groups(db, keys, vals, load_factor=lf, expected_groups=n)
        assert len(rec) == n
        order = np.argsort(keys)
        assert np.array_equal(rec["key"], keys[order]) and np.array_equal(rec["sum"], vals[order])


def test_hash_group_by_with_filter(db):
    n = 300_000
    t = W.groupby_table(n, distinct=20_000, seed=12)
    sel = np.random.default_rng(13).random(n) * 100
    rec = _hash_groups(db, t["key"], t["v"], prog=[ops.cmp(0, F.LT, 25.0)], pred_cols=[dev(sel)])
    mask = O.cmp_mask(sel, F.LT, 25.0)
    want = O.group_i64(t["key"], t["v"], mask=mask)
    assert np.array_equal(rec["key"], want["key"]) and np.array_equal(rec["count"], want["count"])


def _pandas_groups(keys, vals, vvalid=None):
    """COUNT(*), SUM/MIN/MAX over the non-NULL values, per key (NULL values as NaN)."""
    import pandas as pd

    v = vals.astype(np.float64) if vvalid is None else np.where(vvalid, vals.astype(np.float64), np.nan)
    g = pd.DataFrame({"k": keys, "v": v}).groupby("k", sort=True)["v"]
    return {"key": g.size().index.to_numpy(), "count": g.size().to_numpy(), "sum": g.sum().to_numpy(),
            "min": g.min().to_numpy(), "max": g.max().to_numpy()}


def _same_groups(rec, want):
    assert np.array_equal(rec["key"], want["key"]) and np.array_equal(rec["count"], want["count"])
    assert np.array_equal(rec["min"], want["min"], equal_nan=True)
    assert np.array_equal(rec["max"], want["max"], equal_nan=True)
    rel = np.abs(rec["sum"] - want["sum"]) / np.maximum(np.abs(want["sum"]), 1e-300)
    assert rel.max() <= RTOL


def test_hash_group_by_large_with_null_values_and_keys(db):
    """850k groups (a table far larger than the CTA tables) with NULL values
    (SUM/MIN/MAX skip them, COUNT(*) counts the row) and a NULL key group."""
    n = 1_500_000
    r = np.random.default_rng(21)
    keys = r.integers(0, 1_200_000, n)
    keys[::100] = np.iinfo(np.int64).min  # the NULL group
    vals = r.random(n)
    vvalid = r.random(n) > 0.1
    vw = F.validity_words(vvalid)
    out, ng = ops.group_by_i64(db, dev(keys), (dev(vals), dev(vw.view(np.int64))), n)
    g = int(ng.item())
    rec = ops.to_records(out, F.GROUP_I64_DTYPE, g)
    rec = rec[np.argsort(rec["key"], kind="stable")]
    _same_groups(rec, _pandas_groups(keys, vals, vvalid))


def _raw_groups(db, keys, vals, **kw):
    """Groups in the order the kernel wrote them."""
    out, ng = ops.group_by_i64(db, dev(keys), dev(vals) if not isinstance(vals, tuple) else vals, len(keys), **kw)
    return ops.to_records(out, F.GROUP_I64_DTYPE, int(ng.item()))


@pytest.mark.parametrize("kind", ["dense", "hashed"])
def test_group_by_both_table_kinds(db, kind):
    """The same Zipf groups through a direct-addressed table (keys spanning
    0..D-1) and a hashed one (the keys scattered x 7919 + 3, so that their
    range is far wider than the groups): equal answers; the direct-addressed
    table writes its groups in key order."""
    n, d = 3_000_000, 400_000
    t = W.groupby_table(n, distinct=d, seed=77)
    keys = t["key"] if kind == "dense" else t["key"] * 7919 + 3
    raw = _raw_groups(db, keys, t["v"])
    if kind == "dense":
        assert np.all(np.diff(raw["key"]) > 0)
    rec = raw[np.argsort(raw["key"], kind="stable")]
    want = O.group_i64(keys, t["v"])
    assert np.array_equal(rec["key"], want["key"]) and np.array_equal(rec["count"], want["count"])
    assert np.array_equal(rec["min"], want["min"]) and np.array_equal(rec["max"], want["max"])
    rel = np.abs(rec["sum"] - want["sum"]) / np.maximum(np.abs(want["sum"]), 1e-300)
    assert rel.max() <= RTOL


@pytest.mark.parametrize("lo", [np.iinfo(np.int64).min + 1, -5_000, np.iinfo(np.int64).max - 4_999])
def test_dense_group_by_key_range_edges(db, lo):
    """Direct-addressed tables over ranges at both ends of int64 (the slot
    index is key - min in 64-bit two's complement), with INT64_MIN keys (the
    NULL group, written after every key) and NULL values."""
    n = 400_000
    r = np.random.default_rng(abs(lo) % 1000)
    keys = lo + r.integers(0, 5_000, n)
    keys[::23] = np.iinfo(np.int64).min
    vals = r.random(n) * 10  # positive: sums that cancel have no relative-error bound under reordering
    vvalid = r.random(n) > 0.2
    vw = F.validity_words(vvalid)
    raw = _raw_groups(db, keys, (dev(vals), dev(vw.view(np.int64))))
    assert raw["key"][-1] == np.iinfo(np.int64).min  # the NULL group comes last
    assert np.all(np.diff(raw["key"][:-1]) > 0)
    rec = raw[np.argsort(raw["key"], kind="stable")]
    _same_groups(rec, _pandas_groups(keys, vals, vvalid))


def test_dense_group_by_with_filter_and_int_values(db):
    n = 1_000_000
    r = np.random.default_rng(31)
    keys = r.integers(1_000, 60_000, n)
    vals = r.integers(-10**12, 10**12, n)
    sel = r.random(n) * 100
    raw = _raw_groups(db, keys, vals, prog=[ops.cmp(0, F.GE, 40.0)], pred_cols=[dev(sel)])
    assert np.all(np.diff(raw["key"]) > 0)
    want = O.group_i64(keys, vals.astype(np.float64), mask=O.cmp_mask(sel, F.GE, 40.0))
    assert np.array_equal(raw["key"], want["key"]) and np.array_equal(raw["count"], want["count"])
    assert np.array_equal(raw["min"], want["min"]) and np.array_equal(raw["max"], want["max"])
    rel = np.abs(raw["sum"] - want["sum"]) / np.maximum(np.abs(want["sum"]), 1e-300)
    assert rel.max() <= RTOL


def test_dense_group_by_capacity_error(db):
    """An output buffer smaller than the groups: FDB_E_CAPACITY at the next
    synchronisation, and the context stays usable."""
    keys = np.arange(10_000, dtype=np.int64) % 5_000
    vals = np.ones(10_000)
    with pytest.raises(F.FalconError) as e:
        ops.group_by_i64(db, dev(keys), dev(vals), len(keys), capacity=100)
        db.synchronize()
    assert e.value.code == -9
    rec = _raw_groups(db, keys, vals)
    assert len(rec) == 5_000 and np.all(rec["count"] == 2)


def _same_or_close_sums(got, want):
    """SUMs: non-finite ones (inf, -inf, NaN) exactly, the rest within RTOL."""
    fin = np.isfinite(want)
    assert np.array_equal(got[~fin], want[~fin], equal_nan=True)
    rel = np.abs(got[fin] - want[fin]) / np.maximum(np.abs(want[fin]), 1e-300)
    assert rel.max(initial=0.0) <= RTOL


@pytest.mark.parametrize("special", [False, True], ids=["plain", "nan_inf_negzero"])
def test_dense_group_by_heavy_keys(db, special):
    """A few keys carry most rows (every consumer warp's most frequent keys,
    the rows whose COUNT / SUM a warp may keep in registers), the rest spread
    over a dense 200K-key range; with NaN, +-inf and -0.0 among the heavy
    keys' values and a NULL key group.  Every group against the oracle."""
    n, d = 4_000_000, 200_000
    r = np.random.default_rng(91)
    keys = r.integers(0, d, n)
    heavy = np.array([17, 99_999, 150_001])
    pick = r.random(n)
    keys[pick < 0.3] = heavy[0]
    keys[(pick >= 0.3) & (pick < 0.45)] = heavy[1]
    keys[(pick >= 0.45) & (pick < 0.55)] = heavy[2]
    vals = r.random(n) * 100 + 1.0  # positive: a heavy key's SUM does not cancel to near zero
    if special:
        hot_rows = np.flatnonzero(np.isin(keys, heavy))
        for value, every in ((np.nan, 100_003), (np.inf, 200_003), (-np.inf, 300_007), (-0.0, 7)):
            vals[hot_rows[::every]] = value
        vals[np.flatnonzero(keys == heavy[2])[::50_000]] = np.nan  # a heavy key whose SUM is NaN
    keys[::1000] = np.iinfo(np.int64).min  # the NULL group
    raw = _raw_groups(db, keys, vals)
    assert raw["key"][-1] == np.iinfo(np.int64).min and np.all(np.diff(raw["key"][:-1]) > 0)
    rec = raw[np.argsort(raw["key"], kind="stable")]
    want = O.group_i64(keys, vals)
    assert np.array_equal(rec["key"], want["key"]) and np.array_equal(rec["count"], want["count"])
    assert np.array_equal(rec["min"], want["min"], equal_nan=True)
    assert np.array_equal(rec["max"], want["max"], equal_nan=True)
    fin = np.isfinite(want["min"])
    assert np.array_equal(np.signbit(rec["min"][fin]), np.signbit(want["min"][fin]))
    _same_or_close_sums(rec["sum"], want["sum"])


def test_dense_group_by_heavy_keys_null_values(db):
    """Heavy keys whose values are partly NULL: COUNT(*) counts every row,
    SUM / MIN / MAX skip the NULL values."""
    n, d = 3_000_000, 100_000
    r = np.random.default_rng(92)
    keys = r.integers(0, d, n)
    keys[r.random(n) < 0.5] = 4_242
    vals = r.random(n)
    vvalid = r.random(n) > 0.2
    vw = F.validity_words(vvalid)
    raw = _raw_groups(db, keys, (dev(vals), dev(vw.view(np.int64))))
    _same_groups(raw, _pandas_groups(keys, vals, vvalid))
