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


def agg(db, b, p, jt, bvalid=None, pvalid=None, lf=0.0):
    bk = (dev(b["key"]), dev(bvalid.view(np.int64))) if bvalid is not None else dev(b["key"])
    pk = (dev(p["key"]), dev(pvalid.view(np.int64))) if pvalid is not None else dev(p["key"])
    h = ops.HashTable(db, bk, dev(b["payload"]), len(b["key"]), lf)
    out = h.probe_agg(pk, len(p["key"]), jt, value=dev(p["value"]))
    rec = ops.to_records(out, F.JOIN_AGG_DTYPE, 1)[0]
    h.free()
    return rec


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
