"""The device-side bounded waits: a streamed scan whose input tile never
arrives gives up, reports FDB_E_TIMEOUT at the next fdb_synchronize, and
leaves the context usable.

fdb_test_stall makes the producer warp of one CTA stop before one tile's bulk
copy (every copy it issued before that has been waited for, so none is in
flight when the CTA exits) and shortens the consumers' wait bound, so the
wait runs out within milliseconds.  Nothing faults, traps or spins without a
bound.  The hook is set and cleared in a child process, so it cannot touch
any other test."""
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

CHILD = textwrap.dedent(r"""
    import sys, time
    sys.path.insert(0, sys.argv[1])
    import numpy as np, torch
    import falcondb_b200 as F
    from falcondb_b200 import ops
    from oracle import oracle as O

    n = 10_000_003
    v = np.random.default_rng(4).random(n)
    want = O.sum_serial(v)
    with F.Database(0) as db:
        d = torch.from_numpy(v).cuda()
        aggs = [(F.AGG_SUM, 0), (F.AGG_COUNT_STAR, 0)]
        # A healthy call first: the kernel is loaded and the answer is right.
        rec = ops.to_records(ops.aggregate(db, [d], n, [], aggs), F.AGG_VALUE_DTYPE, 2)
        db.synchronize()
        assert abs(rec[0]["f"] - want) <= 1e-12 * want
        for tile in (0, 5, 1_000):  # the first tile, an early one, one of a later round
            F.check(F.lib().fdb_test_stall(db.handle, tile, 1 << 14))
            t0 = time.perf_counter()
            ops.aggregate(db, [d], n, [], aggs)
            try:
                db.synchronize()
                raise SystemExit("no time-out was reported")
            except F.FalconError as e:
                assert e.code == -8, e  # FDB_E_TIMEOUT
            waited = time.perf_counter() - t0
            assert waited < 10.0, waited
            F.check(F.lib().fdb_test_stall(db.handle, 2**64 - 1, 0))
            # The same context answers correctly again.
            rec = ops.to_records(ops.aggregate(db, [d], n, [], aggs), F.AGG_VALUE_DTYPE, 2)
            db.synchronize()
            assert rec[1]["n"] == n or rec[1]["i"] == n
            assert abs(rec[0]["f"] - want) <= 1e-12 * want
            print("tile", tile, "timed out after", round(waited * 1e3, 2), "ms")
    print("ok")
""")


def test_wait_for_a_tile_that_never_arrives_times_out():
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok"), r.stdout
