"""The REST front end's host logic on the CPU: routes and JSON shapes of
FalconDB's server (src/bin/server.rs:65-170) over a stand-in database, the
request parsing, and the serving templates' text matching."""
import json
import math
import urllib.error
import urllib.request

import pytest

from falcondb_b200 import FalconError
from falcondb_b200 import rest as R


class _Result:
    def __init__(self):
        self.columns = ["x"]
        self.rows = 2

    def to_rows(self):
        return [["1"], ["2"]]


class _FakeDb:
    """Just what RestServer asks of a Database when batching is off."""

    def __init__(self):
        self.t = {"t": {"name": "t", "row_count": 2, "col_count": 1,
                        "columns": [{"name": "x", "data_type": "Int64", "nullable": False}]}}
        self.dropped = []

    def tables(self):
        return sorted(self.t)

    def table_info(self, name):
        return self.t.get(name)

    def drop_table(self, name):
        self.dropped.append(name)
        del self.t[name]

    def sql(self, text):
        if "SELEKT" in text:
            raise FalconError(-5, "expected 'SELECT' near 'SELEKT'")
        if "BOOM" in text:
            raise RuntimeError("boom")
        return _Result()


def _call(port, method, path, body=None):
    data = None if body is None else (body if isinstance(body, bytes) else json.dumps(body).encode())
    req = urllib.request.Request(f"http://127.0.0.1:{port}{path}", data=data, method=method,
                                 headers={"Content-Type": "application/json"})
    try:
        with urllib.request.urlopen(req, timeout=10) as r:
            return r.status, json.loads(r.read())
    except urllib.error.HTTPError as e:
        return e.code, json.loads(e.read())


@pytest.fixture()
def server():
    db = _FakeDb()
    s = R.RestServer(db, port=0, batching=False).start()
    yield s, db
    s.stop()


def test_routes_and_shapes(server):
    s, db = server
    assert _call(s.port, "GET", "/health") == (200, {"status": "ok", "engine": "falcondb"})
    assert _call(s.port, "GET", "/tables") == (200, {"tables": ["t"]})
    code, info = _call(s.port, "GET", "/tables/t")
    assert code == 200 and info["row_count"] == 2 and info["columns"][0]["data_type"] == "Int64"
    assert _call(s.port, "GET", "/tables/nope")[0] == 404
    code, body = _call(s.port, "POST", "/sql", {"sql": "SELECT x FROM t"})
    assert code == 200
    assert body["columns"] == ["x"] and body["rows"] == [["1"], ["2"]] and body["row_count"] == 2
    assert body["path"] == "sql" and isinstance(body["elapsed_ms"], int)
    assert _call(s.port, "DELETE", "/tables/t") == (200, {"dropped": "t"})
    assert db.dropped == ["t"]
    assert _call(s.port, "DELETE", "/tables/t")[0] == 404


def test_errors_are_400_with_a_message(server):
    s, _ = server
    code, body = _call(s.port, "POST", "/sql", {"sql": "SELEKT 1"})
    assert code == 400 and "SELECT" in body["error"]
    assert _call(s.port, "POST", "/sql", b"not json")[0] == 400
    assert _call(s.port, "POST", "/sql", {"query": "SELECT 1"})[0] == 400
    assert _call(s.port, "POST", "/load/csv", {"path": "a.csv", "table": "t"})[0] == 400
    assert _call(s.port, "POST", "/tables/t/save", {"path": "t.fdb"})[0] == 400
    assert _call(s.port, "GET", "/nowhere")[0] == 404
    code, body = _call(s.port, "POST", "/sql", {"sql": "SELECT BOOM"})
    assert code == 500 and "boom" in body["error"]


def test_concurrent_requests(server):
    """Bursts of clients (the batching loop's use) are all answered."""
    from concurrent.futures import ThreadPoolExecutor

    s, _ = server
    with ThreadPoolExecutor(64) as ex:
        got = list(ex.map(lambda i: _call(s.port, "POST", "/sql", {"sql": f"SELECT x FROM t -- {i}"}), range(256)))
    assert all(code == 200 and body["row_count"] == 2 for code, body in got)


def test_template_text_matching():
    n = R._norm
    assert R._PATTERNS["count"].match(n("select count(*) from t where score > 50;"))
    assert R._PATTERNS["group"].match(n("SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM t "
                                        "WHERE score > 50 GROUP BY dept"))
    m = R._PATTERNS["topk"].match(n("SELECT id,  score FROM t WHERE score < 20.5 ORDER BY score DESC LIMIT 10"))
    assert m and m.groups()[0] == "id, score" and m.groups()[-1] == "10"
    assert R._PATTERNS["join"].match(n("SELECT COUNT(*), SUM(b.payload) FROM p JOIN b ON p.key = b.key "
                                       "WHERE p.value < 0.25"))
    # Other shapes are not templates: they go to fdb_sql.
    assert not R._PATTERNS["count"].match(n("SELECT COUNT(*) FROM t WHERE score >= 50"))
    assert not R._PATTERNS["topk"].match(n("SELECT id FROM t WHERE score < 20 ORDER BY score ASC LIMIT 10"))
    assert R._lit("50") == 50.0 and R._lit("-2.5") == -2.5


class _ColDb:
    """Counts the catalog calls the template matcher makes."""

    def __init__(self):
        self.generation = 0
        self.calls = 0

    def table_info(self, name):
        self.calls += 1
        if name != "t":
            return None
        return {"name": "t", "row_count": 10, "col_count": 1,
                "columns": [{"name": "score", "data_type": "Float64", "nullable": False}]}

    def column(self, table, name):
        self.calls += 1

        class _Dc:
            ptr, validity = 4096, 0
        return _Dc()


def test_catalog_lookups_are_cached_per_generation():
    db = _ColDb()
    cat = R._Catalog(db)
    first = cat.col("t", "score")
    assert first[0] == R.FLOAT64 and first[2] == 10
    n = db.calls
    assert cat.col("t", "score") is first and db.calls == n  # no library call on a hit
    assert cat.col("t", "nope") is None
    db.generation += 1  # a table was created or dropped
    cat.col("t", "score")
    assert db.calls > n + 1
    assert cat.names("t") == ["score"] and cat.names("u") is None


def test_command_line_parsing():
    assert R._parse_bind("127.0.0.1:8080") == ("127.0.0.1", 8080)
    assert R._parse_bind("0.0.0.0:9") == ("0.0.0.0", 9)
    with pytest.raises(ValueError):
        R._parse_bind("8080")
    assert R._parse_loads(["t=/data/t.parquet", "b=b.parquet"]) == [("t", "/data/t.parquet"), ("b", "b.parquet")]
    with pytest.raises(ValueError):
        R._parse_loads(["t.parquet"])


def test_join_threshold_is_exact():
    """x with x / 100 == v in f64, as the serving join compares value < x / 100."""
    for v in [0.0, 0.25, 0.29, 0.1, 0.3, 0.7, 0.99, 1e-9, 0.123456789]:
        x = R.join_threshold(v)
        assert x is not None and x / 100.0 == v
    assert R.join_threshold(math.inf) is None
