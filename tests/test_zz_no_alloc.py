"""fdb_aggregate_noalloc: the no-key aggregate scan with its per-CTA partials
and ticket in a fixed device array instead of the context's scratch arena.

Each case calls the entry point twice in a row through the C ABI and compares
both results with fdb_aggregate on the same input: counts, integer sums and
MIN/MAX exactly, FP64 SUM/AVG within 1e-12 relative (fdb_aggregate may take a
specialised kernel whose reduction order differs).  The two no-alloc calls run
the same kernel on the same grid, so they agree bit for bit.  This file is
collected last, so it also runs after every other GPU test."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import check, lib, ops

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def call(db, name, cols, n, prog, aggs):
    c, nc = ops._cols(cols)
    p, npr = ops._prog(prog)
    a, na = ops._aggs(aggs)
    out = torch.zeros(F.AGG_VALUE_DTYPE.itemsize * na, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()  # inputs written on torch's stream are visible to the library's stream
    check(getattr(lib(), name)(db.handle, c, nc, n, p, npr, a, na, out.data_ptr()))
    db.synchronize()  # also returns any deferred device-side error
    return ops.to_records(out, F.AGG_VALUE_DTYPE, na)


def same(got, want, float_sum):
    assert got["valid"] == want["valid"] and got["n"] == want["n"] and got["is_int"] == want["is_int"]
    assert got["i"] == want["i"]
    if not want["valid"]:
        return
    if float_sum:
        assert abs(got["f"] - want["f"]) <= RTOL * abs(want["f"]), (got["f"], want["f"])
    else:
        assert got["f"] == want["f"]


def run_case(db, cols, n, prog, aggs, float_sums):
    ref = call(db, "fdb_aggregate", cols, n, prog, aggs)
    first = call(db, "fdb_aggregate_noalloc", cols, n, prog, aggs)
    second = call(db, "fdb_aggregate_noalloc", cols, n, prog, aggs)
    assert first.tobytes() == second.tobytes()
    for j in range(len(aggs)):
        same(first[j], ref[j], float_sums[j])
        same(second[j], ref[j], float_sums[j])


@pytest.mark.parametrize("n", [0, 1, 4097, 3_000_001])
def test_noalloc_single_f64_column(db, n):
    v = np.random.default_rng(n + 5).random(n) * 100.0
    aggs = [(F.AGG_SUM, 0), (F.AGG_AVG, 0), (F.AGG_MIN, 0), (F.AGG_MAX, 0)]
    run_case(db, [dev(v)], n, [], aggs, [True, True, False, False])


def test_noalloc_where_nulls_and_int_sums(db):
    n = 2_000_003
    r = np.random.default_rng(17)
    score = r.random(n) * 100.0
    salary = r.integers(30_000, 200_001, n)
    valid = r.random(n) > 0.1
    vw = F.validity_words(valid)
    cols = [dev(score), (dev(salary), dev(vw.view(np.int64)))]
    prog = [ops.cmp(0, F.GT, 50.0)]
    aggs = [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_SUM, 0), (F.AGG_MIN, 1)]
    run_case(db, cols, n, prog, aggs, [False, False, True, False])
