"""fdb_aggregate_noalloc: the no-key aggregate scan with its per-CTA partials
and ticket in a fixed device array instead of the context's scratch arena.

Some callers cannot allocate device memory at the moment they aggregate: a
serving loop that has handed its whole budget to resident tables, or a
latency-critical path where a pool allocation could block.  This entry point
serves them, so the tests check two things:

* it allocates nothing: on a fresh context it is the first operator called,
  and the context's budget-counted bytes, its scratch arena, the device pool's
  reserved and used bytes, and the device's free memory are the same after two
  calls as before them (the free memory from after the first call, since the
  first launch of a kernel may load its module);
* its answers equal fdb_aggregate's on the same input, on two calls in a row:
  counts, integer sums and MIN/MAX exactly, FP64 SUM/AVG within 1e-12
  relative (fdb_aggregate may take a specialised kernel whose reduction order
  differs).  The two no-alloc calls run the same kernel on the same grid, so
  they agree bit for bit.

This file is collected last, so it also runs after every other GPU test."""
import numpy as np
import pytest
import torch

import falcondb_b200 as F
from falcondb_b200 import check, lib, ops

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


class Call:
    """One prepared aggregate call: argument structs and output buffer made
    up front, so that issuing it creates no torch allocation."""

    def __init__(self, cols, n, prog, aggs):
        self.c, self.nc = ops._cols(cols)
        self.p, self.npr = ops._prog(prog)
        self.a, self.na = ops._aggs(aggs)
        self.n = n
        self.out = torch.zeros(F.AGG_VALUE_DTYPE.itemsize * self.na, dtype=torch.uint8, device="cuda")

    def issue(self, db, name):
        torch.cuda.synchronize()  # inputs written on torch's stream are visible to the library's stream
        check(getattr(lib(), name)(db.handle, self.c, self.nc, self.n, self.p, self.npr, self.a, self.na,
                                   self.out.data_ptr()))
        db.synchronize()  # also returns any deferred device-side error
        return ops.to_records(self.out, F.AGG_VALUE_DTYPE, self.na).copy()


def same(got, want, float_sum):
    assert got["valid"] == want["valid"] and got["n"] == want["n"] and got["is_int"] == want["is_int"]
    assert got["i"] == want["i"]
    if not want["valid"]:
        return
    if float_sum:
        assert abs(got["f"] - want["f"]) <= RTOL * abs(want["f"]), (got["f"], want["f"])
    else:
        assert got["f"] == want["f"]


def run_case(cols, n, prog, aggs, float_sums):
    with F.Database(0) as db:  # fresh context: the no-alloc call is its first operator
        call = Call(cols, n, prog, aggs)
        torch.cuda.synchronize()
        before = db.memory_stats()
        first = call.issue(db, "fdb_aggregate_noalloc")
        free_after_first = torch.cuda.mem_get_info()[0]
        second = call.issue(db, "fdb_aggregate_noalloc")
        assert torch.cuda.mem_get_info()[0] == free_after_first
        assert db.memory_stats() == before
        ref = call.issue(db, "fdb_aggregate")
    assert first.tobytes() == second.tobytes()
    for j in range(len(aggs)):
        same(first[j], ref[j], float_sums[j])
        same(second[j], ref[j], float_sums[j])


@pytest.mark.parametrize("n", [0, 1, 4097, 3_000_001])
def test_noalloc_single_f64_column(n):
    v = np.random.default_rng(n + 5).random(n) * 100.0
    aggs = [(F.AGG_SUM, 0), (F.AGG_AVG, 0), (F.AGG_MIN, 0), (F.AGG_MAX, 0)]
    run_case([dev(v)], n, [], aggs, [True, True, False, False])


def test_noalloc_where_nulls_and_int_sums():
    n = 2_000_003
    r = np.random.default_rng(17)
    score = r.random(n) * 100.0
    salary = r.integers(30_000, 200_001, n)
    valid = r.random(n) > 0.1
    vw = F.validity_words(valid)
    cols = [dev(score), (dev(salary), dev(vw.view(np.int64)))]
    prog = [ops.cmp(0, F.GT, 50.0)]
    aggs = [(F.AGG_COUNT_STAR, 0), (F.AGG_SUM, 1), (F.AGG_SUM, 0), (F.AGG_MIN, 1)]
    run_case(cols, n, prog, aggs, [False, False, True, False])
