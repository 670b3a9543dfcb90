"""MIN / MAX on NaN and +-inf: the reference's own rules, restated in the
oracle (ref_minmax_nokey, ref_minmax_group), pinned here to answers worked
out by hand from the reference's source, case by case.

The reference's answers on non-finite floats depend on how a table is cut
into batches (65,536 rows):
* no-key MIN/MAX over a NULL-free FLOAT64 batch fold f64::min / f64::max and
  drop the batch when the fold is not finite (aggregate.rs:3308-3320,
  3351-3363), so a batch holding -inf drops out of MIN, finite values and all;
* no-key MIN/MAX over a batch with NULLs (or an integer column) scan with
  `<` / `>` from +-inf, so a batch of NaN and NULL gives +inf / -inf
  (3322-3330, 3365-3373);
* GROUP BY MIN/MAX take a group's first value in a batch as it is, so a
  leading NaN stays (1092-1101, merged by 1369-1380).

The engine uses one batch-independent rule instead: MIN/MAX over the
non-NULL, non-NaN values, +-inf included, NULL when there are none.  On the
configurations' data (finite, no NULLs) both give the same answers, which the
property test below checks; tests/test_gpu_minmax.py holds the engine to its
rule on these same cases and records each difference."""
import math

import numpy as np

from oracle import oracle as O

INF, NAN = float("inf"), float("nan")


def words(valid):
    import falcondb_b200 as F

    return F.validity_words(np.asarray(valid, dtype=bool))


# (name, values, validity or None, batch rows, reference MIN, reference MAX)
NOKEY = [
    # One NULL-free batch holding -inf: its fold is -inf, not finite, dropped.
    ("dense_neg_inf", [3.0, -INF, 1.0], None, 65_536, None, 3.0),
    # Batch 0 = [5, NaN] folds to 5 (f64::min skips NaN); batch 1 = [-inf, 2]
    # folds to -inf and is dropped from MIN; MAX sees 5 and 2.
    ("dense_two_batches", [5.0, NAN, -INF, 2.0], None, 2, 5.0, 5.0),
    # Only NaN: both folds stay infinite, so both are NULL.
    ("dense_all_nan", [NAN, NAN], None, 65_536, None, None),
    # +inf in a NULL-free batch: MAX's fold is +inf and is dropped; MIN is 1.
    ("dense_pos_inf", [1.0, INF], None, 65_536, 1.0, None),
    # With a NULL the batch is scanned with `<` / `>` from +-inf: NaN never
    # replaces the running value, and `any` is set, so MIN is +inf, MAX -inf.
    ("nullable_nan_only", [NAN, 0.0], [True, False], 65_536, INF, -INF),
    # The same scan keeps -inf / +inf.
    ("nullable_inf", [NAN, 2.0, 0.0, -INF, INF], [True, True, False, True, True], 65_536, -INF, INF),
    # Finite values: the plain minimum and maximum.
    ("finite", [4.0, -1.5, 9.25], None, 65_536, -1.5, 9.25),
]

# (name, keys, values, batch rows, {key: reference MIN}, {key: reference MAX})
GROUP = [
    ("leading_nan_sticks", [1, 1, 2], [NAN, 1.0, 3.0], 65_536, {1: NAN, 2: 3.0}, {1: NAN, 2: 3.0}),
    ("later_nan_skipped", [1, 1], [1.0, NAN], 65_536, {1: 1.0}, {1: 1.0}),
    ("inf_kept", [7, 7, 7], [2.0, INF, -INF], 65_536, {7: -INF}, {7: INF}),
    # Batch 0's state for key 1 is NaN; batch 1's 0.5 cannot replace it.
    ("nan_batch_first", [1, 1], [NAN, 0.5], 1, {1: NAN}, {1: NAN}),
    # Batch 0's state is 0.5; batch 1's NaN state cannot replace it.
    ("nan_batch_second", [1, 1], [0.5, NAN], 1, {1: 0.5}, {1: 0.5}),
]


def same(a, b):
    if a is None or b is None:
        return a is None and b is None
    return (math.isnan(a) and math.isnan(b)) or a == b


def test_reference_nokey_rules_pinned():
    for name, vals, valid, rows, want_min, want_max in NOKEY:
        v = np.array(vals, dtype=np.float64)
        w = None if valid is None else words(valid)
        assert same(O.ref_minmax_nokey(v, True, w, rows), want_min), name
        assert same(O.ref_minmax_nokey(v, False, w, rows), want_max), name


def test_reference_group_rules_pinned():
    for name, keys, vals, rows, want_min, want_max in GROUP:
        got_min = O.ref_minmax_group(keys, vals, True, rows)
        got_max = O.ref_minmax_group(keys, vals, False, rows)
        assert set(got_min) == set(want_min) and set(got_max) == set(want_max), name
        for k in want_min:
            assert same(got_min[k], want_min[k]), (name, k)
            assert same(got_max[k], want_max[k]), (name, k)


def test_reference_rules_agree_with_the_oracle_on_finite_data():
    """Finite, NULL-free values over several batches (the configurations'
    kind of data): the reference's rules and the oracle's value semantics
    give the same MIN / MAX, per table and per group."""
    r = np.random.default_rng(5)
    for n, batch in ((1000, 64), (777, 100), (5, 65_536)):
        v = r.random(n) * 200 - 100
        k = r.integers(0, 17, n)
        for is_min, func in ((True, 4), (False, 5)):
            want, _ = O.agg(func, v)
            assert O.ref_minmax_nokey(v, is_min, None, batch) == want
        g = O.group_i64(k, v)
        rmin = O.ref_minmax_group(k, v, True, batch)
        rmax = O.ref_minmax_group(k, v, False, batch)
        for key, mn, mx in zip(g["key"], g["min"], g["max"]):
            assert rmin[int(key)] == mn and rmax[int(key)] == mx
