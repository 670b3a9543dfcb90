"""GPU parity of ORDER BY .. LIMIT k against the oracle's restatement of
top_k_ascending + assemble (sort.rs:564-599, 773-791): bit-exact row lists,
ties broken by row ascending, NULLs first/last."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run(db, col, n, k, desc, nulls_last=None):
    rows, cnt = ops.topk(db, col, n, k, desc, nulls_last)
    c = int(cnt.item())
    return rows[:c].cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 5, 10, 11, 1000, 65_537, 1_000_003, 3_000_017])
@pytest.mark.parametrize("desc", [True, False])
def test_topk_f64_random(db, n, desc):
    v = np.random.default_rng(n).random(n) * 100
    got = run(db, dev(v), n, 10, desc)
    assert np.array_equal(got, O.topk(v, 10, desc))


@pytest.mark.parametrize("k", [1, 7, 10, 32, 33, 100, 1000, 4096])
def test_topk_k_range(db, k):
    n = 2_000_003
    v = np.random.default_rng(k).random(n)
    for desc in (True, False):
        assert np.array_equal(run(db, dev(v), n, k, desc), O.topk(v, k, desc)), (k, desc)


@pytest.mark.parametrize("n", [100, 1_048_576, 5_000_000])
def test_topk_ascending_id_desc(db, n):
    """The reference's slow case: an ascending column read DESC (every row is a
    candidate for a running threshold)."""
    v = np.arange(n, dtype=np.int64)
    assert np.array_equal(run(db, dev(v), n, 10, True), O.topk(v, 10, True))
    assert np.array_equal(run(db, dev(v), n, 10, False), O.topk(v, 10, False))


@pytest.mark.parametrize("k", [1, 17, 32])
def test_topk_candidate_floods_with_ties(db, k):
    """Inputs where whole warps hold candidates at once (the batched bitonic
    insertion): ascending runs of equal keys, and a sawtooth whose every tile
    beats the running bound; ties must still break on row ascending."""
    n = 3_000_001
    v = (np.arange(n) // 3).astype(np.int64)
    w = (np.arange(n) % 65_536).astype(np.float64)
    for col in (v, w):
        for desc in (True, False):
            assert np.array_equal(run(db, dev(col), n, k, desc), O.topk(col, k, desc)), (k, desc, col.dtype)


def test_topk_all_equal_ties_on_row(db):
    n = 2_000_000
    v = np.full(n, 42.5)
    assert list(run(db, dev(v), n, 10, True)) == list(range(10))
    v2 = np.zeros(n, dtype=np.int64)
    assert list(run(db, dev(v2), n, 50, False)) == list(range(50))


def test_topk_many_ties_at_boundary(db):
    n = 1_500_000
    v = np.random.default_rng(2).integers(0, 5, n)  # 5 distinct values
    for desc in (True, False):
        assert np.array_equal(run(db, dev(v), n, 100, desc), O.topk(v, 100, desc))


def test_topk_descending_column_and_negatives(db):
    n = 1_200_000
    v = -np.arange(n, dtype=np.float64) * 0.5
    v[::7] = -v[::7]
    for desc in (True, False):
        assert np.array_equal(run(db, dev(v), n, 10, desc), O.topk(v, 10, desc))


def test_topk_nan_and_inf(db):
    n = 100_000
    v = np.random.default_rng(4).random(n)
    v[[3, 77, 500]] = np.nan
    v[[10, 20]] = np.inf
    v[[11]] = -np.inf
    for desc in (True, False):
        assert np.array_equal(run(db, dev(v), n, 10, desc), O.topk(v, 10, desc))


def test_topk_signed_zero_and_negative_nan(db):
    """-0.0 orders below +0.0 and a NaN with the sign bit set below -inf
    (f64_ord_key, sort.rs:451-454); the value-domain prefilter must pass all
    of them on to the exact key test."""
    n = 200_003
    v = np.random.default_rng(8).random(n) - 0.5
    v[::5] = 0.0
    v[1::5] = -0.0
    neg_nan = np.array([0xFFF8000000000001], dtype=np.uint64).view(np.float64)[0]
    v[[7, 70_000]] = neg_nan
    v[9] = np.nan
    v[11] = -np.inf
    for k in (1, 10, 32):
        for desc in (True, False):
            assert np.array_equal(run(db, dev(v), n, k, desc), O.topk(v, k, desc)), (k, desc)
    z = np.where(np.arange(n) % 2 == 0, 0.0, -0.0)  # only signed zeros: ties on the key, then row
    for desc in (True, False):
        assert np.array_equal(run(db, dev(z), n, 10, desc), O.topk(z, 10, desc)), desc


@pytest.mark.parametrize("nulls_last", [True, False])
def test_topk_with_nulls(db, nulls_last):
    n = 1000
    i = np.arange(n)
    v = ((i * 7919) % n).astype(np.float64) + 0.5
    null = i % 97 == 0
    vw = F.validity_words(~null)
    col = (dev(v), dev(vw.view(np.int64)))
    for k in (5, 10, 15):
        for desc in (True, False):
            got = run(db, col, n, k, desc, nulls_last)
            want = O.topk(v, k, desc, nulls_last=nulls_last, validity=vw)
            assert np.array_equal(got, want), (k, desc)
    # all-NULL head: k larger than the number of keyed rows
    vw2 = F.validity_words(i < 3)
    got = run(db, (dev(v), dev(vw2.view(np.int64))), n, 10, True, nulls_last)
    assert np.array_equal(got, O.topk(v, 10, True, nulls_last=nulls_last, validity=vw2))


def test_topk_k_larger_than_n(db):
    v = np.array([3.0, 1.0, 2.0])
    assert list(run(db, dev(v), 3, 10, True)) == [0, 2, 1]
