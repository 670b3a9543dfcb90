"""GPU parity of the hash join (build + probe) against the oracle's restatement
of IntHashTable + probe_one + execute_hash_semi_anti_join: counts and integer
payload sums bit-exact, SUM(value) within 1e-12, row-pair multisets equal."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TYPES = [F.JOIN_INNER, F.JOIN_LEFT, F.JOIN_SEMI, F.JOIN_ANTI]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def agg(db, b, p, jt, bvalid=None, pvalid=None, lf=0.0, dense=None):
    """Build, probe with aggregation, free; `dense` (when given) is the table
    mode the build must have chosen."""
    bk = (dev(b["key"]), dev(bvalid.view(np.int64))) if bvalid is not None else dev(b["key"])
    pk = (dev(p["key"]), dev(pvalid.view(np.int64))) if pvalid is not None else dev(p["key"])
    h = ops.HashTable(db, bk, dev(b["payload"]), len(b["key"]), lf)
    if dense is not None:
        assert h.dense == dense
    out = h.probe_agg(pk, len(p["key"]), jt, value=dev(p["value"]))
    rec = ops.to_records(out, F.JOIN_AGG_DTYPE, 1)[0]
    h.free()
    return rec


def check_agg(got, want, jt):
    assert got["count"] == want["count"]
    if jt <= 1:
        assert got["sum_payload"] == want["sum_payload"]
        assert got["payload_rows"] == want["payload_rows"]
    else:
        assert abs(got["sum_value"] - want["sum_value"]) <= 1e-12 * max(abs(want["sum_value"]), 1e-300)


I64 = np.iinfo(np.int64)


def _edge_probes(r, keys, n):
    """n probe keys: build keys, keys just outside the build range on both
    sides, int64 extremes and INT64_MIN."""
    lo, hi = int(keys.min()), int(keys.max())
    pk = r.choice(keys, n)
    m = n // 8
    pk[:m] = r.integers(max(I64.min + 1, lo - 5000), lo, m) if lo > I64.min + 1 else pk[:m]
    pk[m:2 * m] = r.integers(hi + 1, min(I64.max, hi + 5000), m) if hi < I64.max - 1 else pk[m:2 * m]
    pk[2 * m:2 * m + 4] = [I64.max, I64.min + 1, I64.min, lo]
    return pk


@pytest.mark.parametrize("nb,np_", [(1, 1), (10, 1000), (1000, 100_003), (100_000, 3_000_017)])
@pytest.mark.parametrize("jt", TYPES)
def test_join_agg(db, nb, np_, jt):
    b, p = W.join_tables(nb, np_, seed=nb + np_)
    got = agg(db, b, p, jt)
    want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
    assert got["count"] == want["count"]
    if jt <= 1:
        assert got["sum_payload"] == want["sum_payload"]
        assert got["payload_rows"] == want["payload_rows"]
    else:
        assert abs(got["sum_value"] - want["sum_value"]) <= 1e-12 * abs(want["sum_value"])


@pytest.mark.parametrize("jt", TYPES)
def test_join_duplicates_and_nulls(db, jt):
    r = np.random.default_rng(4)
    b = {"key": r.integers(0, 500, 3000), "payload": r.integers(0, 100, 3000)}
    p = {"key": r.integers(-10, 600, 50_000), "value": r.random(50_000)}
    bvalid = F.validity_words(r.random(3000) > 0.1)
    pvalid = F.validity_words(r.random(50_000) > 0.1)
    got = agg(db, b, p, jt, bvalid, pvalid)
    want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt, bvalid=bvalid, pvalid=pvalid)
    assert got["count"] == want["count"]
    if jt <= 1:
        assert got["sum_payload"] == want["sum_payload"]


def test_join_int64_min_key(db):
    """A build key equal to INT64_MIN (the slot sentinel's pattern) still joins."""
    mn = np.iinfo(np.int64).min
    b = {"key": np.array([mn, 5, mn, 7], dtype=np.int64), "payload": np.array([1, 2, 3, 4], dtype=np.int64)}
    p = {"key": np.array([mn, 5, 6, mn], dtype=np.int64), "value": np.array([0.5, 1.5, 2.5, 3.5])}
    for jt in TYPES:
        got = agg(db, b, p, jt)
        want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt)
        assert got["count"] == want["count"], jt
        if jt <= 1:
            assert got["sum_payload"] == want["sum_payload"], jt


@pytest.mark.parametrize("jt", TYPES)
def test_join_pairs_multiset(db, jt):
    r = np.random.default_rng(6)
    bk = r.integers(0, 2000, 5000)
    pk = r.integers(0, 4000, 100_000)
    h = ops.HashTable(db, dev(bk), None, len(bk))
    want_l, want_r = O.join_pairs(bk, pk, jt)
    left, right, cnt = h.probe_pairs(dev(pk), len(pk), jt, capacity=len(want_l) + 16)
    c = int(cnt.item())
    assert c == len(want_l)
    gl = left[:c].cpu().numpy().view(np.uint32)
    if jt <= 1:
        gr = right[:c].cpu().numpy().view(np.uint32)
        got = sorted(zip(gl.tolist(), gr.tolist()))
        assert got == sorted(zip(want_l.tolist(), want_r.tolist()))
    else:
        assert sorted(gl.tolist()) == sorted(want_l.tolist())
    h.free()


def test_join_load_factors(db):
    b, p = W.join_tables(200_000, 1_000_000, seed=3)
    want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], F.JOIN_INNER)
    for lf in (0.25, 0.5, 0.75):
        assert agg(db, b, p, F.JOIN_INNER, lf=lf)["sum_payload"] == want["sum_payload"]


@pytest.mark.parametrize("kind", ["dense_offset", "dense_negative", "hashed"])
@pytest.mark.parametrize("jt", TYPES)
def test_join_dense_and_hashed_tables(db, kind, jt):
    """The build picks a direct-addressed table when its keys span fewer values
    than it has slots, else it hashes; both give the oracle's answers, with
    duplicate build keys, NULL keys on both sides, probe keys outside the
    build range and at the int64 extremes."""
    r = np.random.default_rng(11 + jt)
    nb, npr = 20_000, 400_000
    if kind == "dense_offset":
        keys = 10**15 + r.permutation(nb)
    elif kind == "dense_negative":
        keys = -7 * 10**12 + r.integers(0, nb // 2, nb)  # many duplicates
    else:
        keys = r.integers(-(1 << 62), 1 << 62, nb)
    b = {"key": keys.astype(np.int64), "payload": r.integers(-1000, 1000, nb)}
    p = {"key": _edge_probes(r, b["key"], npr).astype(np.int64), "value": r.random(npr)}
    bvalid = F.validity_words(r.random(nb) > 0.05)
    pvalid = F.validity_words(r.random(npr) > 0.05)
    got = agg(db, b, p, jt, bvalid, pvalid, dense=kind != "hashed")
    want = O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt, bvalid=bvalid, pvalid=pvalid)
    check_agg(got, want, jt)


@pytest.mark.parametrize("span_extra,dense", [(0, True), (1, False)])
def test_join_dense_threshold(db, span_extra, dense):
    """Build keys spanning exactly the table's slot count minus one are dense;
    one more value and the table hashes.  Row pairs and aggregates match the
    oracle either way."""
    r = np.random.default_rng(5)
    nb = 1000
    h0 = ops.HashTable(db, dev(np.arange(nb, dtype=np.int64)), None, nb)
    cap = h0.capacity
    h0.free()
    keys = np.arange(nb, dtype=np.int64) - 40
    keys[-1] = keys[0] + cap - 1 + span_extra
    pk = np.concatenate([keys, r.integers(-100, cap + 100, 50_000)]).astype(np.int64)
    b = {"key": keys, "payload": r.integers(0, 50, nb)}
    p = {"key": pk, "value": r.random(len(pk))}
    for jt in TYPES:
        check_agg(agg(db, b, p, jt, dense=dense), O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt), jt)
    h = ops.HashTable(db, dev(keys), None, nb)
    assert h.capacity == cap and h.dense == dense
    want_l, want_r = O.join_pairs(keys, pk, F.JOIN_INNER)
    left, right, cnt = h.probe_pairs(dev(pk), len(pk), F.JOIN_INNER, capacity=len(want_l) + 16)
    c = int(cnt.item())
    assert c == len(want_l)
    got = sorted(zip(left[:c].cpu().numpy().view(np.uint32).tolist(), right[:c].cpu().numpy().view(np.uint32).tolist()))
    assert got == sorted(zip(want_l.tolist(), want_r.tolist()))
    h.free()


@pytest.mark.parametrize("kind", ["bits", "dense_wide", "hashed"])
def test_semi_anti_on_every_table_path(db, kind):
    """SEMI / ANTI with SUM(value) on the three probe paths: a dense table
    whose key range fits a CTA's shared memory as presence bits (bit test
    only), a dense table too wide for that (one 16-byte slot read), and a
    hashed table.  Build keys with NULLs and INT64_MIN; probe keys below,
    inside and above the range, NULL and INT64_MIN; NULL values."""
    r = np.random.default_rng({"bits": 1, "dense_wide": 2, "hashed": 3}[kind])
    # dense_wide: 700K keys get a 2^21-slot table, and a 2M-value range is
    # dense there but wider than the 1.57M presence bits a CTA holds.
    nb = {"bits": 400_000, "dense_wide": 700_000, "hashed": 400_000}[kind]
    span = {"bits": 600_000, "dense_wide": 2_000_000, "hashed": 10**12}[kind]
    keys = np.unique(r.integers(0, span, int(nb * 1.3)))
    r.shuffle(keys)
    keys = keys[:nb].astype(np.int64) - 5_000
    nb = len(keys)
    keys[0], keys[1] = -5_000, span - 5_001  # the range's two ends
    keys[::1000] = I64.min
    bvalid = r.random(nb) > 0.01
    b = {"key": keys, "payload": r.integers(0, 1000, nb)}
    npb = 3_000_001
    pk = r.integers(int(keys[keys != I64.min].min()) - 100, int(keys.max()) + 100, npb)
    pk[::777] = I64.min
    pvalid = r.random(npb) > 0.02
    vals = r.random(npb)
    vvalid = r.random(npb) > 0.05
    p = {"key": pk, "value": vals}
    bvw, pvw = F.validity_words(bvalid), F.validity_words(pvalid)
    h = ops.HashTable(db, (dev(keys), dev(bvw.view(np.int64))), dev(b["payload"]), nb)
    assert h.dense == (kind != "hashed")
    for jt in (F.JOIN_SEMI, F.JOIN_ANTI):
        out = h.probe_agg((dev(pk), dev(pvw.view(np.int64))), npb, jt,
                          value=(dev(vals), dev(F.validity_words(vvalid).view(np.int64))))
        got = ops.to_records(out, F.JOIN_AGG_DTYPE, 1)[0]
        want = O.join_agg(keys, b["payload"], pk, vals, jt, bvalid=bvw, pvalid=pvw,
                          pvvalid=F.validity_words(vvalid))
        assert got["count"] == want["count"]
        assert got["payload_rows"] == want["payload_rows"]
        assert abs(got["sum_value"] - want["sum_value"]) <= 1e-12 * abs(want["sum_value"])
    h.free()


@pytest.mark.parametrize("lo,hi", [(-3_000_000_000, 3_000_000_000), (I64.min + 1, I64.max)])
def test_hashed_table_key_range_filter(db, lo, hi):
    """A hashed table reads nothing for probe keys outside its build keys'
    [min, max]: keys one below the minimum and one above the maximum miss,
    the two ends themselves match, and a build side reaching both int64
    extremes (a range of 2^64 - 1 values) filters nothing.  Aggregates and
    row pairs match the oracle on every join type."""
    r = np.random.default_rng(21)
    nb = 50_000
    keys = r.integers(lo // 2, hi // 2, nb)
    keys[0], keys[1] = lo, hi
    b = {"key": keys.astype(np.int64), "payload": r.integers(0, 1000, nb)}
    edges = [lo, hi, lo + 1, hi - 1, I64.min]
    if lo > I64.min + 1:
        edges += [lo - 1, I64.min + 1]
    if hi < I64.max:
        edges += [hi + 1, I64.max]
    pk = np.concatenate([np.repeat(np.array(edges, dtype=np.int64), 3), r.choice(keys, 20_000),
                         r.integers(lo // 2, hi // 2, 20_000)]).astype(np.int64)
    r.shuffle(pk)
    p = {"key": pk, "value": r.random(len(pk))}
    for jt in TYPES:
        check_agg(agg(db, b, p, jt, dense=False), O.join_agg(b["key"], b["payload"], p["key"], p["value"], jt), jt)
    h = ops.HashTable(db, dev(b["key"]), None, nb)
    assert not h.dense
    for jt in TYPES:
        want_l, want_r = O.join_pairs(b["key"], pk, jt)
        left, right, cnt = h.probe_pairs(dev(pk), len(pk), jt, capacity=len(want_l) + 16)
        c = int(cnt.item())
        assert c == len(want_l), jt
        gl = left[:c].cpu().numpy().view(np.uint32).tolist()
        if jt <= 1:
            gr = right[:c].cpu().numpy().view(np.uint32).tolist()
            assert sorted(zip(gl, gr)) == sorted(zip(want_l.tolist(), want_r.tolist()))
        else:
            assert sorted(gl) == sorted(want_l.tolist())
    h.free()
