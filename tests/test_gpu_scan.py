"""GPU parity of the scan kernels (filter mask / COUNT WHERE / aggregates /
COUNT DISTINCT codes / compaction / gather) against the oracle, through the
C ABI.  Integer results are bit-exact; FP64 SUM/AVG within 1e-12 relative of the
serial FP64 oracle (reduction order differs)."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import ops
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-12
SIZES = [0, 1, 3, 63, 64, 65, 4095, 4096, 4097, 100_003, 1_000_003]
OPS = [F.EQ, F.NE, F.LT, F.LE, F.GT, F.GE]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def words_np(t, n):
    w = t.cpu().numpy().view(np.uint64)
    return w[: (n + 63) // 64]


def rng(seed):
    return np.random.default_rng(seed)


@pytest.mark.parametrize("n", SIZES)
def test_count_where_f64(db, n):
    v = rng(n).random(n) * 100.0
    v[: min(n, 5)] = 50.0  # exact ties with the literal
    d = dev(v)
    for op in OPS:
        for lit in (50, 50.0, 12.5):
            got = int(ops.filter_count(db, [d], n, [ops.cmp(0, op, lit)]).item())
            want = O.popcount(O.cmp_mask(v, op, lit))
            assert got == want, (n, op, lit)


@pytest.mark.parametrize("n", [0, 1, 65, 4097, 1_000_003])
def test_count_where_i64_and_widening(db, n):
    v = rng(n + 1).integers(-1000, 1000, n)
    d = dev(v)
    for op in OPS:
        for lit in (7, -3, 7.5, -0.5):  # float literals widen the column (expr.rs:1122-1132)
            got = int(ops.filter_count(db, [d], n, [ops.cmp(0, op, lit)]).item())
            assert got == O.popcount(O.cmp_mask(v, op, lit)), (n, op, lit)


def test_count_where_nan_semantics(db):
    v = np.array([np.nan, 1.0, 50.0, np.nan, 99.0, -np.inf, np.inf], dtype=np.float64)
    d = dev(v)
    for op in OPS:
        got = int(ops.filter_count(db, [d], len(v), [ops.cmp(0, op, 50.0)]).item())
        assert got == O.popcount(O.cmp_mask(v, op, 50.0)), op


@pytest.mark.parametrize("n", [1, 63, 64, 65, 129, 10_000, 250_001])
def test_filter_mask_programs(db, n):
    r = rng(n)
    a = r.random(n) * 100
    b = r.integers(0, 50, n)
    valid = r.random(n) > 0.2
    vw = F.validity_words(valid)
    da, db_, dv = dev(a), dev(b), dev(vw.view(np.int64))
    cols = [da, (db_, dv)]
    progs = {
        "a>50": ([ops.cmp(0, F.GT, 50)], O.cmp_mask(a, F.GT, 50)),
        "a>50 AND b<20": ([ops.cmp(0, F.GT, 50), ops.cmp(1, F.LT, 20), ops.AND()],
                          O.cmp_mask(a, F.GT, 50) & O.cmp_mask(b, F.LT, 20, validity=vw)),
        "a<5 OR b=7": ([ops.cmp(0, F.LT, 5), ops.cmp(1, F.EQ, 7), ops.OR()],
                       O.cmp_mask(a, F.LT, 5) | O.cmp_mask(b, F.EQ, 7, validity=vw)),
        "b IS NULL": ([ops.is_null(1)], None),
    }
    null_words = ~vw
    if n % 64:
        null_words[-1] &= np.uint64((1 << (n % 64)) - 1)
    for name, (prog, want) in progs.items():
        if want is None:
            want = null_words
        got = words_np(ops.filter_mask(db, cols, n, prog), n)
        assert np.array_equal(got, want[: len(got)]), name
        # the popcount fast path must agree with the mask (padding bits zero)
        cnt = int(ops.filter_count(db, cols, n, prog).item())
        assert cnt == O.popcount(want), name


def test_code_set_terms(db):
    n = 10_007
    codes = rng(5).integers(0, 12, n).astype(np.uint32)
    codes[::101] = 0xFFFFFFFF  # NULL codes
    passing = [i % 3 == 0 for i in range(12)]
    term, keep = ops.code_set(0, passing, torch.device("cuda"))
    d = dev(codes.view(np.int32))
    got = words_np(ops.filter_mask(db, [d], n, [term]), n)
    assert np.array_equal(got, O.code_mask(codes, passing))
    null = words_np(ops.filter_mask(db, [d], n, [ops.is_null(0)]), n)
    assert O.popcount(null) == int((codes == 0xFFFFFFFF).sum())


@pytest.mark.parametrize("n", SIZES)
def test_aggregates_f64(db, n):
    v = rng(n + 7).random(n) * 100.0
    d = dev(v)
    out = ops.aggregate(db, [d], n, [], [(F.AGG_SUM, 0), (F.AGG_AVG, 0), (F.AGG_MIN, 0), (F.AGG_MAX, 0)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE, 4)
    for j, func in enumerate([2, 3, 4, 5]):
        want, cnt = O.agg(func, v)
        if want is None:
            assert rec[j]["valid"] == 0
            continue
        assert rec[j]["valid"] == 1 and rec[j]["n"] == cnt
        if func in (4, 5):
            assert rec[j]["f"] == want
        else:
            assert abs(rec[j]["f"] - want) <= RTOL * abs(want), (func, rec[j]["f"], want)


@pytest.mark.parametrize("n", [0, 1, 5, 65, 100_003])
def test_aggregates_i64_exact(db, n):
    v = rng(n + 9).integers(30_000, 200_001, n)
    d = dev(v)
    out = ops.aggregate(db, [d], n, [], [(F.AGG_SUM, 0), (F.AGG_MIN, 0), (F.AGG_MAX, 0), (F.AGG_COUNT_STAR, 0)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE, 4)
    if n:
        assert rec[0]["f"] == float(O.sum_i64_exact(v))  # exact i64 then as f64
        assert rec[1]["f"] == float(v.min()) and rec[2]["f"] == float(v.max())
    assert rec[3]["i"] == n and rec[3]["is_int"] == 1


def test_aggregate_with_filter_and_nulls(db):
    n = 300_001
    r = rng(11)
    a = r.random(n) * 100
    s = r.integers(0, 1000, n)
    valid = r.random(n) > 0.1
    vw = F.validity_words(valid)
    cols = [dev(a), (dev(s), dev(vw.view(np.int64)))]
    prog = [ops.cmp(0, F.GT, 50)]
    out = ops.aggregate(db, cols, n, prog, [(F.AGG_COUNT_STAR, 0), (F.AGG_COUNT, 1), (F.AGG_SUM, 1), (F.AGG_AVG, 0)])
    rec = ops.to_records(out, F.AGG_VALUE_DTYPE, 4)
    mask = O.cmp_mask(a, F.GT, 50)
    assert rec[0]["i"] == O.popcount(mask)
    assert rec[1]["i"] == O.agg(1, s, mask=mask, validity=vw)[1]
    assert rec[2]["f"] == float(O.sum_i64_exact(s, mask=mask, validity=vw))
    want = O.agg(3, a, mask=mask)[0]
    assert abs(rec[3]["f"] - want) <= RTOL * abs(want)


def test_sum_is_repeatable(db):
    v = rng(3).random(2_000_003)
    d = dev(v)
    a = [ops.to_records(ops.aggregate(db, [d], len(v), [], [(F.AGG_SUM, 0)]), F.AGG_VALUE_DTYPE, 1)[0]["f"]
         for _ in range(3)]
    assert a[0] == a[1] == a[2]


@pytest.mark.parametrize("n", [1, 64, 65, 1_000_003])
def test_distinct_codes(db, n):
    codes = rng(n).integers(0, 12, n).astype(np.uint32)
    codes[rng(1).random(n) < 0.01] = 0xFFFFFFFF
    d = dev(codes.view(np.int32))
    bm = ops.distinct_codes(db, [d], n, [], 0, 12).cpu().numpy().view(np.uint64)
    got = [(int(bm[0]) >> i) & 1 for i in range(12)]
    assert got == list(O.present_codes(codes, 12))
    # a dictionary larger than 64 entries (shared-memory bitmap)
    codes2 = rng(n + 1).integers(0, 5000, n).astype(np.uint32)
    bm2 = ops.distinct_codes(db, [dev(codes2.view(np.int32))], n, [], 0, 5000).cpu().numpy().view(np.uint64)
    got2 = [(int(bm2[i >> 6]) >> (i & 63)) & 1 for i in range(5000)]
    assert got2 == list(O.present_codes(codes2, 5000))


@pytest.mark.parametrize("n", [1, 63, 64, 65, 131_073, 1_000_003])
def test_compact_and_gather(db, n):
    v = rng(n).random(n) * 100
    d = dev(v)
    mask = ops.filter_mask(db, [d], n, [ops.cmp(0, F.GT, 70)])
    rows, cnt = ops.compact(db, mask, n)
    k = int(cnt.item())
    want = O.mask_rows(O.cmp_mask(v, F.GT, 70), n)
    got = rows[:k].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, want)
    g, _ = ops.gather(db, d, rows, k)
    assert np.array_equal(g[:k].cpu().numpy(), v[want])


def test_unaligned_views_use_the_plain_path(db):
    """A view starting off a 16-byte boundary cannot be staged by TMA; the
    kernels read it with plain loads and must give the same answers."""
    n = 1_000_001
    v = rng(21).random(n + 1) * 100
    base = dev(v)
    view = base[1:]  # 8-byte offset
    assert view.data_ptr() % 16 == 8
    got = int(ops.filter_count(db, [view], n, [ops.cmp(0, F.GT, 50)]).item())
    assert got == O.popcount(O.cmp_mask(v[1:], F.GT, 50))
    rec = ops.to_records(ops.aggregate(db, [view], n, [], [(F.AGG_SUM, 0)]), F.AGG_VALUE_DTYPE, 1)
    want = O.sum_serial(v[1:])
    assert abs(rec[0]["f"] - want) <= RTOL * want


@pytest.mark.parametrize("n", [0, 1, 31, 257, 1_000_003])
def test_filtered_aggregates_fast_path(db, n):
    """One `col op literal` WHERE over NULL-free columns (the fast filtered
    scan) against the oracle and against the interpreted scan (the same WHERE
    with a second, always-true term)."""
    r = rng(n + 21)
    f = r.random(n) * 100
    if n > 10:
        f[r.integers(0, n, max(1, n // 50))] = np.nan
        f[: min(n, 5)] = 50.0
    i = r.integers(-1000, 1000, n)
    cols = [dev(f), dev(i)]
    aggs = [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_MIN, 0), (F.AGG_MAX, 1)]
    aggs2 = [(F.AGG_AVG, 0), (F.AGG_COUNT, 1), (F.AGG_MAX, 0), (F.AGG_MIN, 1)]
    cases = [(0, op, 50.0) for op in OPS] + [(0, op, 50) for op in (F.LT, F.NE)] + \
            [(1, op, 0) for op in OPS] + [(1, F.GT, 0.5), (1, F.LE, -0.5), (0, F.NE, float("nan")),
                                          (0, F.EQ, float("nan"))]
    for col, op, lit in cases:
        x = f if col == 0 else i
        with np.errstate(invalid="ignore"):
            sel = {F.EQ: x == lit, F.NE: x != lit, F.LT: x < lit, F.LE: x <= lit, F.GT: x > lit,
                   F.GE: x >= lit}[op]
        for spec in (aggs, aggs2):
            fast = ops.to_records(ops.aggregate(db, cols, n, [ops.cmp(col, op, lit)], spec), F.AGG_VALUE_DTYPE, 4)
            slow = ops.to_records(ops.aggregate(db, cols, n, [ops.cmp(col, op, lit), ops.is_not_null(0), ops.AND()],
                                                spec), F.AGG_VALUE_DTYPE, 4)
            for j, (func, c) in enumerate(spec):
                a, b = fast[j], slow[j]
                assert (a["valid"], a["n"], a["is_int"]) == (b["valid"], b["n"], b["is_int"]), (col, op, lit, func)
                if func in (F.AGG_SUM, F.AGG_AVG) and c == 0:   # NaN rows make both NaN
                    assert (a["f"] != a["f"] and b["f"] != b["f"]) or \
                        abs(a["f"] - b["f"]) <= RTOL * max(abs(b["f"]), 1e-300), (col, op, lit, func)
                else:
                    assert (a["f"], a["i"]) == (b["f"], b["i"]) or (a["f"] != a["f"] and b["f"] != b["f"]), \
                        (col, op, lit, func, a, b)
                vals = (f if c == 0 else i)[sel]
                if func == F.AGG_COUNT_STAR:
                    assert a["i"] == int(sel.sum())
                elif func == F.AGG_SUM and c == 1:
                    assert a["f"] == float(vals.sum()) if len(vals) else a["valid"] == 0
                elif func in (F.AGG_MIN, F.AGG_MAX):
                    want, cnt = O.agg(func, vals)
                    assert a["n"] == cnt
                    if want is not None:
                        assert a["f"] == want


@pytest.mark.parametrize("n", [7, 4099, 2_000_011])
def test_filtered_aggregates_fast_path_edge_values(db, n):
    """The fast filtered scan on the values where its accumulator forms could
    differ from the interpreted scan's order-key / 128-bit forms: -0.0 and
    +0.0, +-inf, NaN, and INT64 values near the limits whose sums need more
    than 64 bits.  Values equal the oracle's; the sign of a zero MIN / MAX
    (which f64::min / max leave unspecified) equals the interpreted scan's:
    MAX is +0.0 and MIN -0.0 when both occur."""
    r = rng(n + 5)
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0])
    f = specials[r.integers(0, len(specials), n)]
    big = np.array([np.iinfo(np.int64).max, np.iinfo(np.int64).min, np.iinfo(np.int64).max - 7, -(1 << 62), 1 << 62,
                    -1, 0], dtype=np.int64)
    i = big[r.integers(0, len(big), n)]
    cols = [dev(f), dev(i)]
    spec = [(F.AGG_SUM, 1), (F.AGG_MIN, 0), (F.AGG_MAX, 0), (F.AGG_AVG, 1)]
    for col, op, lit in [(1, F.GE, -(1 << 62)), (1, F.NE, 0), (0, F.NE, 5.0), (0, F.LE, 0.0), (1, F.LT, 1 << 62)]:
        x = f if col == 0 else i
        with np.errstate(invalid="ignore"):
            sel = {F.NE: x != lit, F.LE: x <= lit, F.GE: x >= lit, F.LT: x < lit}[op]
        got = ops.to_records(ops.aggregate(db, cols, n, [ops.cmp(col, op, lit)], spec), F.AGG_VALUE_DTYPE, 4)
        slow = ops.to_records(ops.aggregate(db, cols, n, [ops.cmp(col, op, lit), ops.is_not_null(0), ops.AND()],
                                            spec), F.AGG_VALUE_DTYPE, 4)
        s = int(i[sel].astype(object).sum()) if sel.any() else 0
        assert got[0]["n"] == int(sel.sum())
        # The 128-bit sum is exact; its conversion to FLOAT64 is within an ulp.
        assert abs(got[0]["f"] - float(s)) <= 2.0 ** -52 * abs(float(s)), (col, op, lit)
        if sel.any():
            assert abs(got[3]["f"] - float(s) / int(sel.sum())) <= 2.0 ** -51 * abs(float(s) / int(sel.sum()))
        for j, func in ((1, F.AGG_MIN), (2, F.AGG_MAX)):
            want, cnt = O.agg(func, f[sel])
            assert got[j]["n"] == cnt and bool(got[j]["valid"]) == (want is not None)
            if want is not None:
                assert got[j]["f"] == want, (col, op, lit, func)
        for j in range(4):
            assert got[j].tobytes() == slow[j].tobytes(), (col, op, lit, j, got[j], slow[j])
    # Signed zeros alone.
    zeros = np.where(r.random(n) < 0.5, 0.0, -0.0)
    got = ops.to_records(ops.aggregate(db, [dev(zeros), cols[1]], n, [ops.cmp(1, F.NE, 12345)],
                                       [(F.AGG_MIN, 0), (F.AGG_MAX, 0)]), F.AGG_VALUE_DTYPE, 2)
    assert got[0]["f"] == 0.0 and got[1]["f"] == 0.0
    assert np.signbit(got[0]["f"]) == bool(np.signbit(zeros).any())
    assert np.signbit(got[1]["f"]) == (not (~np.signbit(zeros)).any())
