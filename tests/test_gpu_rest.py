"""The REST front end on the GPU: concurrent POST /sql requests, the serving
templates answered by the continuous-batching loop and everything else by
fdb_sql; each response equals fdb_sql's rows for the same text (FP64 sums
within 1e-12 relative: the two paths add in different orders)."""
import json
import urllib.request
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from falcondb_b200 import rest as R
from falcondb_b200 import workloads as W

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _post(port, sql):
    req = urllib.request.Request(f"http://127.0.0.1:{port}/sql", data=json.dumps({"sql": sql}).encode(),
                                 method="POST", headers={"Content-Type": "application/json"})
    with urllib.request.urlopen(req, timeout=60) as r:
        return json.loads(r.read())


def _same_cell(a, b):
    if a == b:
        return True
    try:
        x, y = float(a), float(b)
    except ValueError:
        return False
    return abs(x - y) <= RTOL * max(abs(x), abs(y))


def test_rest_sql_batches_templates_and_matches_fdb_sql(db):
    db.create_table("t", W.table_t(1_000_000, seed=12))
    b, p = W.join_tables(100_000, 1_000_003, seed=13)
    db.create_table("b", b)
    db.create_table("p", p)
    rng = np.random.default_rng(1)
    served, plain = [], []
    for x in rng.uniform(0, 100, 12):
        x = round(float(x), 2)
        served += [f"SELECT COUNT(*) FROM t WHERE score > {x}",
                   f"SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM t WHERE score > {x} GROUP BY dept",
                   f"SELECT dept, COUNT(*), SUM(score), SUM(salary) FROM t WHERE score > {x} GROUP BY dept",
                   f"SELECT id, score, dept FROM t WHERE score < {x} ORDER BY score DESC LIMIT 10",
                   f"SELECT COUNT(*), SUM(b.payload) FROM p JOIN b ON p.key = b.key WHERE p.value < {x / 100:.4f}"]
    served += ["SELECT COUNT(*), SUM(b.payload) FROM p JOIN b ON p.key = b.key WHERE p.value < 0",
               "SELECT COUNT(*) FROM t WHERE score > 50"]
    plain += ["SELECT id FROM t ORDER BY id DESC LIMIT 5", "SELECT DISTINCT dept FROM t",
              "SELECT COUNT(*) FROM t WHERE score >= 50", "SELECT SUM(score) FROM t"]
    want = {sql: db.sql(sql) for sql in served + plain}
    srv = R.RestServer(db, port=0, batching=True, max_batch=64, slots=2).start()
    try:
        texts = (served + plain) * 3
        with ThreadPoolExecutor(48) as ex:
            got = list(ex.map(lambda s: (s, _post(srv.port, s)), texts))
        batched = 0
        for sql, body in got:
            w = want[sql]
            assert body["path"] == ("serving" if sql in served else "sql"), sql
            assert body["columns"] == list(w.columns), sql
            assert body["row_count"] == w.rows, sql
            rows = w.to_rows()
            assert all(len(a) == len(e) and all(_same_cell(x, y) for x, y in zip(a, e))
                       for a, e in zip(body["rows"], rows)), (sql, body["rows"][:3], rows[:3])
            batched += body.get("batch_size", 0) > 1
        assert batched > 0  # concurrent template requests shared launches
        assert _post(srv.port, "SELECT DISTINCT dept FROM t")["row_count"] == 12
    finally:
        stats = srv.stop()
    assert stats.batches >= 1
