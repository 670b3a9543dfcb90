"""Host logic of the push-based operator contract (falcondb_b200.operators):
the pipeline driver, chunking and LimitOp, restated from the reference's own
cases (pipeline.rs tests, operators.rs:339-404) over a host batch type.  The
driver and LimitOp only need row_count() and slice(), so no GPU is involved."""
import numpy as np

from falcondb_b200.operators import LimitOp, OpResult, Operator, Pipeline, into_chunks

CH = 2048  # the reference's CHUNK_ROWS, used here to exercise chunk boundaries


class HostBatch:
    def __init__(self, v):
        self.v = np.asarray(v, dtype=np.int64)

    def row_count(self):
        return len(self.v)

    def slice(self, start, n):
        return HostBatch(self.v[start:start + n])


def values(batches):
    return [int(x) for b in batches for x in b.v]


class Identity(Operator):
    def process(self, chunk):
        return OpResult.Emit(chunk)

    def name(self):
        return "Identity"


class Collect(Operator):
    """A blocking stage: holds everything, emits one batch at flush."""

    def __init__(self):
        self.held = []

    def process(self, chunk):
        self.held.append(chunk.v)
        return OpResult.Empty

    def flush(self):
        if not self.held:
            return []
        out, self.held = HostBatch(np.concatenate(self.held)), []
        return [out]

    def name(self):
        return "Collect"


class TakeN(Operator):
    def __init__(self, n):
        self.left = n

    def process(self, chunk):
        if self.left == 0:
            return OpResult.Done
        k = min(self.left, chunk.row_count())
        self.left -= k
        return OpResult.Emit(chunk.slice(0, k))

    def name(self):
        return "TakeN"


class Filter(Operator):
    def __init__(self, gt):
        self.gt = gt

    def process(self, chunk):
        out = chunk.v[chunk.v > self.gt]
        return OpResult.Emit(HostBatch(out)) if len(out) else OpResult.Empty

    def name(self):
        return "Filter"


def run(ops_, *batches):
    return Pipeline(ops_, chunk_rows=CH).run([HostBatch(b) for b in batches])


def test_chunking_preserves_values_and_order():
    chunks = into_chunks(HostBatch(range(5000)), CH)
    assert len(chunks) > 1 and all(c.row_count() <= CH for c in chunks)
    assert values(chunks) == list(range(5000))
    assert len(into_chunks(HostBatch(range(100)), CH)) == 1


def test_empty_pipeline_returns_its_input():
    assert values(run([], range(3000))) == list(range(3000))


def test_streaming_and_blocking_stages():
    assert values(run([Identity()], range(5000))) == list(range(5000))
    assert values(run([Collect()], range(3000))) == list(range(3000))
    assert values(run([Collect(), TakeN(10)], range(5000))) == list(range(10))
    assert values(run([Collect(), Collect()], range(2500))) == list(range(2500))


def test_done_stops_the_source_early():
    class Counting(Identity):
        seen = 0

        def process(self, chunk):
            Counting.seen += chunk.row_count()
            return OpResult.Emit(chunk)

    got = run([Counting(), TakeN(5)], range(10 * CH))
    assert values(got) == list(range(5))
    assert Counting.seen <= 2 * CH  # the source stopped after the limit was met


def test_multiple_inputs_and_empty_input():
    assert values(run([Identity()], range(100), range(100, 200))) == list(range(200))
    assert Pipeline([Identity()]).run([]) == []
    p = Pipeline([Identity(), Collect()])
    assert p.stage_names() == ["Identity", "Collect"] and not p.is_empty()


def test_limit_semantics():
    assert values(run([LimitOp(0, 7)], range(5000))) == list(range(7))
    assert values(run([LimitOp(3000, 5)], range(5000))) == list(range(3000, 3005))  # offset across chunks
    assert run([LimitOp(10_000, None)], range(5000)) == []
    assert run([LimitOp(0, 0)], range(100)) == []
    assert values(run([Filter(100), LimitOp(0, 3)], range(5000))) == [101, 102, 103]
    assert values(run([Collect(), LimitOp(0, 3)], range(5000))) == [0, 1, 2]
