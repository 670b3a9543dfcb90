"""MIN / MAX over NaN and +-inf on the GPU, through Database::sql: the no-key
scan, the INT64-key hash GROUP BY and the dictionary GROUP BY all follow one
rule (MIN / MAX over the non-NULL, non-NaN values, +-inf included; NULL when
there are none), on the cases whose reference answers
tests/test_minmax_rules.py pins.  Where the reference's batch-dependent rules
give another answer, the case is listed in DIFFERS, so the deviation is
recorded case by case rather than hidden."""
import math

import numpy as np
import pytest

import falcondb_b200 as F
from oracle import oracle as O
from tests.test_minmax_rules import GROUP, NOKEY

pytestmark = pytest.mark.gpu
INF, NAN = float("inf"), float("nan")

# The engine's answer per no-key case: (MIN, MAX); None = NULL.
OURS_NOKEY = {
    "dense_neg_inf": (-INF, 3.0),
    "dense_two_batches": (-INF, 5.0),
    "dense_all_nan": (None, None),
    "dense_pos_inf": (1.0, INF),
    "nullable_nan_only": (None, None),
    "nullable_inf": (-INF, INF),
    "finite": (-1.5, 9.25),
}
# The engine's answer per GROUP BY case: {key: (MIN, MAX)}.
OURS_GROUP = {
    "leading_nan_sticks": {1: (1.0, 1.0), 2: (3.0, 3.0)},
    "later_nan_skipped": {1: (1.0, 1.0)},
    "inf_kept": {7: (-INF, INF)},
    "nan_batch_first": {1: (0.5, 0.5)},
    "nan_batch_second": {1: (0.5, 0.5)},
}
# Cases where the reference, as written, answers otherwise.
DIFFERS = {"dense_neg_inf", "dense_two_batches", "dense_pos_inf", "nullable_nan_only", "leading_nan_sticks",
           "nan_batch_first"}


def typed_rows(res):
    """Rows of typed values (None = NULL)."""
    return [[res.value(r, c) for c in range(len(res.columns))] for r in range(res.row_count())]


def same(a, b):
    if a is None or b is None:
        return a is None and b is None
    return (math.isnan(a) and math.isnan(b)) or a == b


@pytest.mark.parametrize("case", NOKEY, ids=lambda c: c[0])
def test_nokey_min_max(db, case):
    name, vals, valid, rows, ref_min, ref_max = case
    v = np.array(vals, dtype=np.float64)
    col = v if valid is None else np.ma.MaskedArray(v, mask=~np.asarray(valid))
    db.create_table("m", {"v": col})
    got = typed_rows(db.sql("SELECT MIN(v), MAX(v) FROM m"))[0]
    want = OURS_NOKEY[name]
    assert same(got[0], want[0]) and same(got[1], want[1]), (name, got)
    # Our rule is the oracle's value semantics.
    w = None if valid is None else F.validity_words(np.asarray(valid))
    assert same(O.agg(4, v, validity=w)[0], want[0]) and same(O.agg(5, v, validity=w)[0], want[1])
    differs = not (same(ref_min, want[0]) and same(ref_max, want[1]))
    assert differs == (name in DIFFERS), name


@pytest.mark.parametrize("case", GROUP, ids=lambda c: c[0])
def test_group_by_min_max(db, case):
    name, keys, vals, rows, ref_min, ref_max = case
    k = np.array(keys, dtype=np.int64)
    v = np.array(vals, dtype=np.float64)
    labels = sorted({f"k{x}" for x in keys})
    codes = np.array([labels.index(f"k{x}") for x in keys], dtype=np.uint32)
    db.create_table("m", {"k": k, "d": F.Utf8(codes, labels), "v": v})
    want = OURS_GROUP[name]
    by_int = {r[0]: (r[1], r[2]) for r in typed_rows(db.sql("SELECT k, MIN(v), MAX(v) FROM m GROUP BY k"))}
    by_text = {int(r[0][1:]): (r[1], r[2]) for r in typed_rows(db.sql("SELECT d, MIN(v), MAX(v) FROM m GROUP BY d"))}
    for got in (by_int, by_text):
        assert set(got) == set(want), (name, got)
        for key, (mn, mx) in want.items():
            assert same(got[key][0], mn) and same(got[key][1], mx), (name, key, got[key])
    differs = any(not (same(ref_min[key], want[key][0]) and same(ref_max[key], want[key][1])) for key in want)
    assert differs == (name in DIFFERS), name


def test_all_nan_group_is_null(db):
    """A group whose values are all NaN has no MIN / MAX: NULL, in both
    GROUP BY kernels."""
    db.create_table("m", {"k": np.array([1, 1, 2], np.int64), "d": F.Utf8(np.array([0, 0, 1], np.uint32), ["a", "b"]),
                          "v": np.array([NAN, NAN, 4.0])})
    rows = typed_rows(db.sql("SELECT k, MIN(v), MAX(v) FROM m GROUP BY k ORDER BY k"))
    assert rows[0][0] == 1 and rows[0][1] is None and rows[0][2] is None
    assert rows[1] == [2, 4.0, 4.0]
    rows = typed_rows(db.sql("SELECT d, MIN(v), MAX(v) FROM m GROUP BY d ORDER BY d"))
    assert rows[0][0] == "a" and rows[0][1] is None and rows[0][2] is None
