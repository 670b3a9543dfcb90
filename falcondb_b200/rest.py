"""REST front end: FalconDB's HTTP server routes (src/bin/server.rs:65-170)
over a :class:`Database`, with ``POST /sql`` feeding the continuous-batching
serving loop.

Routes, with the reference's JSON shapes:

* ``GET /health`` -> ``{"status": "ok", "engine": "falcondb"}``;
* ``GET /tables`` -> ``{"tables": [...]}`` (sorted);
* ``GET /tables/{name}`` -> TableInfo (name, row_count, col_count, columns),
  404 if unknown;
* ``DELETE /tables/{name}`` -> ``{"dropped": name}``, 404 if unknown;
* ``POST /sql`` ``{"sql": "..."}`` -> QueryResponse
  ``{"columns", "rows" (display strings), "row_count", "elapsed_ms"}``, or 400
  ``{"error": "..."}``.

The file loaders and ``save`` (``/load/csv``, ``/load/fdb``,
``/tables/{name}/save``) answer 400: tables reach this engine through the
library (``Database.create_table``), not through files.

``POST /sql`` routing: the reference runs every request through
``Database::sql`` on its own (server.rs:151-169).  Here, a request whose text
is exactly one of the serving templates over columns without NULLs is
submitted to the native serving loop (:class:`serving.Server`).  That loop
batches whatever requests are in flight into shared scans.  Every other
request runs through ``fdb_sql``.  A served request answers with the rows
``fdb_sql`` gives for the same text; FP64 sums may differ in the last place,
because the two paths add in different orders.  The templates:

* ``SELECT COUNT(*) FROM t WHERE c > x`` (c FLOAT64);
* ``SELECT g, COUNT(*), SUM(c), SUM(v) | AVG(v) FROM t WHERE c > x GROUP BY g``
  (g Utf8 with at most 16 values, c FLOAT64, v INT64);
* ``SELECT cols FROM t WHERE c < x ORDER BY c DESC LIMIT k`` (c FLOAT64,
  k <= 32);
* ``SELECT COUNT(*), SUM(b.p) FROM a JOIN b ON a.k = b.k WHERE a.v < x``
  (a.k, b.k, b.p INT64, a.v FLOAT64; the build table of b is kept resident).

Each response carries ``"path"`` (``"serving"`` or ``"sql"``) and, for a
served request, ``"batch_size"``: how many queries shared its launch.
"""
from __future__ import annotations

import json
import math
import re
import threading
import time
from dataclasses import dataclass
from http.server import BaseHTTPRequestHandler, ThreadingHTTPServer
from typing import Any, Callable, Dict, List, Optional, Tuple

import numpy as np
import torch

from . import FLOAT64, INT64, UTF8, Database, FalconError, _fmt, fdb_serve_result
from . import ops, serving
from .operators import _view

__all__ = ["RestServer", "match_template", "join_threshold"]

_ID = r"([A-Za-z_][A-Za-z0-9_]*)"
_NUM = r"(-?\d+(?:\.\d+)?)"
_MAX_GROUPS = 16
_MAX_K = 32


def _norm(sql: str) -> str:
    s = sql.strip()
    if s.endswith(";"):
        s = s[:-1].rstrip()
    return re.sub(r"\s+", " ", s)


def _lit(text: str) -> float:
    """A numeric literal as the SQL front end compares it with a FLOAT64 column:
    an integer literal is widened to f64 (expr.rs:1117), a decimal one is read
    as f64."""
    return float(int(text)) if re.fullmatch(r"-?\d+", text) else float(text)


def join_threshold(v: float) -> Optional[float]:
    """The serving join template compares with x / 100 (in f64 on the device);
    the x for which that quotient is exactly v, or None if none is near v*100."""
    if not math.isfinite(v):
        return None
    t = v * 100.0
    cands = [t]
    up, down = t, t
    for _ in range(4):
        up, down = math.nextafter(up, math.inf), math.nextafter(down, -math.inf)
        cands += [up, down]
    for c in cands:
        if c / 100.0 == v:
            return c
    return None


_PATTERNS = {
    "count": re.compile(rf"SELECT COUNT\(\*\) FROM {_ID} WHERE {_ID} > {_NUM}$", re.I),
    "group": re.compile(rf"SELECT {_ID}, COUNT\(\*\), (SUM)\({_ID}\), (SUM|AVG)\({_ID}\) FROM {_ID} "
                        rf"WHERE {_ID} > {_NUM} GROUP BY {_ID}$", re.I),
    "topk": re.compile(rf"SELECT (\*|{_ID}(?:, {_ID})*) FROM {_ID} WHERE {_ID} < {_NUM} "
                       rf"ORDER BY {_ID} DESC LIMIT (\d+)$", re.I),
    "join": re.compile(rf"SELECT COUNT\(\*\), (SUM)\({_ID}\.{_ID}\) FROM {_ID} (?:INNER )?JOIN {_ID} "
                       rf"ON {_ID}\.{_ID} = {_ID}\.{_ID} WHERE {_ID}\.{_ID} < {_NUM}$", re.I),
}


@dataclass
class Served:
    """A request matched to a serving template: the query to submit and how to
    turn its result into (columns, display rows)."""

    query: serving.Query
    finish: Callable[[fdb_serve_result], Tuple[List[str], List[List[str]]]]


class _Catalog:
    """What the matcher needs to know about a table: its columns' types, NULLs
    and device views.  Lookups are remembered until the database's
    ``generation`` changes (a table created or dropped), so a request that
    matches a template makes no library call that waits on a running query."""

    def __init__(self, db: Database):
        self.db = db
        self._gen = None
        self._cols: Dict[Tuple[str, str], Any] = {}
        self._names: Dict[str, Optional[List[str]]] = {}

    def _fresh(self) -> None:
        gen = getattr(self.db, "generation", None)
        if gen is None or gen != self._gen:
            self._cols.clear()
            self._names.clear()
            self._gen = gen

    def col(self, table: str, name: str):
        self._fresh()
        key = (table, name)
        if key not in self._cols:
            self._cols[key] = self._lookup(table, name)
        return self._cols[key]

    def _lookup(self, table: str, name: str):
        info = self.db.table_info(table)
        if info is None:
            return None
        for c in info["columns"]:
            if c["name"] == name:
                dt = {"Int64": INT64, "Float64": FLOAT64, "Utf8": UTF8}[c["data_type"]]
                dc = self.db.column(table, name)
                if c["nullable"] or dc.validity:
                    return None
                return dt, dc, info["row_count"]
        return None

    def names(self, table: str) -> Optional[List[str]]:
        self._fresh()
        if table not in self._names:
            info = self.db.table_info(table)
            self._names[table] = None if info is None else [c["name"] for c in info["columns"]]
        return self._names[table]


def match_template(db: Database, sql: str, join_tables: Optional[Callable] = None,
                   catalog: Optional[_Catalog] = None) -> Optional[Served]:
    """The serving template `sql` is, bound to `db`'s resident columns; None when
    it is not one (or a column is nullable, of another type, or out of range)."""
    s = _norm(sql)
    cat = catalog if catalog is not None else _Catalog(db)
    m = _PATTERNS["count"].match(s)
    if m:
        t, c, x = m.groups()
        col = cat.col(t, c)
        if not col or col[0] != FLOAT64:
            return None
        q = serving.count_query(col[1].ptr, col[2], _lit(x))
        return Served(q, lambda r: (["COUNT(*)"], [[str(int(r.count))]]))
    m = _PATTERNS["group"].match(s)
    if m:
        g, f1, c0, f2, c2, t, cw, x, gb = m.groups()
        if g != gb or c0 != cw:
            return None
        gc, vc0, vc2 = cat.col(t, g), cat.col(t, c0), cat.col(t, c2)
        if not (gc and vc0 and vc2) or gc[0] != UTF8 or vc0[0] != FLOAT64 or vc2[0] != INT64:
            return None
        d = db.dictionary(t, g)
        if not 0 < len(d) <= _MAX_GROUPS:
            return None
        avg = f2.upper() == "AVG"
        names = [g, "COUNT(*)", f"SUM({c0})", f"{f2.upper()}({c2})"]

        def finish(r, d=d, avg=avg, names=names):
            rows = []
            for k in range(len(d)):
                n = int(r.group_count[k])
                if n <= 0:
                    continue
                v2 = float(r.group_sum2[k])
                rows.append([d[k], str(n), _fmt(float(r.group_sum0[k]), FLOAT64),
                             _fmt(v2 / n if avg else v2, FLOAT64)])
            return names, rows

        q = serving.group_query(vc0[1].ptr, gc[1].ptr, vc2[1].ptr, len(d), vc0[2], _lit(x))
        return Served(q, finish)
    m = _PATTERNS["topk"].match(s)
    if m:
        groups = m.groups()
        sel, t, cw, x, co, k = groups[0], groups[-5], groups[-4], groups[-3], groups[-2], int(groups[-1])
        if cw != co or not 1 <= k <= _MAX_K:
            return None
        key = cat.col(t, cw)
        if not key or key[0] != FLOAT64:
            return None
        names = cat.names(t) if sel == "*" else [c.strip() for c in sel.split(",")]
        if names is None or len(set(names)) != len(names):
            return None  # a repeated column is renamed by fdb_sql's result: let it answer
        outs = [cat.col(t, n) for n in names]
        if any(o is None for o in outs):
            return None
        views = [_view(o[1].ptr, o[2], o[0]) for o in outs]
        dicts = [db.dictionary(t, n) if o[0] == UTF8 else None for n, o in zip(names, outs)]

        def finish(r, names=names, outs=outs, views=views, dicts=dicts):
            n = int(r.count)
            rows_idx = torch.tensor([int(r.rows[i]) for i in range(n)], dtype=torch.int64, device=views[0].device)
            cols = []
            for (dt, _, _), v, dct in zip(outs, views, dicts):
                vals = v[rows_idx].cpu().numpy() if n else np.zeros(0)
                if dt == UTF8:
                    cols.append([dct[int(c) & 0xFFFFFFFF] for c in vals])
                else:
                    cols.append([_fmt(x, dt) for x in vals.tolist()])
            return names, [[c[i] for c in cols] for i in range(n)]

        q = serving.topk_query(key[1].ptr, key[2], _lit(x), k=k)
        return Served(q, finish)
    m = _PATTERNS["join"].match(s)
    if m and join_tables is not None:
        (_, sb, sp, a, b, l1, lk, r1, rk, w1, wv, x) = m.groups()
        if sb != b or w1 != a:
            return None
        if {l1, r1} != {a, b}:
            return None
        ak, bk = (lk, rk) if l1 == a else (rk, lk)
        kcol, vcol = cat.col(a, ak), cat.col(a, wv)
        bkey, bpay = cat.col(b, bk), cat.col(b, sp)
        if not (kcol and vcol and bkey and bpay):
            return None
        if kcol[0] != INT64 or bkey[0] != INT64 or bpay[0] != INT64 or vcol[0] != FLOAT64:
            return None
        thr = join_threshold(_lit(x))
        if thr is None:
            return None
        table = join_tables(b, bk, sp, bkey, bpay)
        names = ["COUNT(*)", f"SUM({sp})"]

        def finish(r, names=names):
            n = int(r.count)
            return names, [[str(n), _fmt(float(r.sum_payload), FLOAT64) if n else "NULL"]]

        return Served(serving.join_query(kcol[1].ptr, vcol[1].ptr, table, kcol[2], thr), finish)
    return None


class _HttpServer(ThreadingHTTPServer):
    # Clients open connections in bursts; the listen queue takes a burst of
    # them (socketserver's default is 5, past which connections are reset).
    request_queue_size = 1024


class RestServer:
    """HTTP server over `db` (one thread per connection).  With ``batching``,
    template requests go through a serving loop of ``max_batch`` queries per
    launch and ``slots`` launches in flight."""

    def __init__(self, db: Database, host: str = "127.0.0.1", port: int = 8080, batching: bool = True,
                 max_batch: int = 128, slots: int = 2):
        self.db = db
        self.batching = batching
        self._server = serving.Server(db, max_batch=max_batch, slots=slots) if batching else None
        self._joins: Dict[Tuple[str, str, str], ops.HashTable] = {}
        self._catalog = _Catalog(db)
        self._join_gen = getattr(db, "generation", None)
        self._lock = threading.Lock()        # join-table cache and the table catalog
        self._inflight = 0                   # served queries not yet answered
        self._idle = threading.Condition(self._lock)
        rest = self

        class Handler(BaseHTTPRequestHandler):
            protocol_version = "HTTP/1.1"

            def log_message(self, *a):  # keep stderr quiet
                pass

            def _send(self, code: int, body: Dict[str, Any]) -> None:
                data = json.dumps(body).encode()
                self.send_response(code)
                self.send_header("Content-Type", "application/json")
                self.send_header("Content-Length", str(len(data)))
                self.end_headers()
                self.wfile.write(data)

            def do_GET(self):
                self._send(*rest.route("GET", self.path, None))

            def do_DELETE(self):
                self._send(*rest.route("DELETE", self.path, None))

            def do_POST(self):
                n = int(self.headers.get("Content-Length") or 0)
                raw = self.rfile.read(n) if n else b""
                self._send(*rest.route("POST", self.path, raw))

        self._http = _HttpServer((host, port), Handler)
        self._http.daemon_threads = True
        self.port = self._http.server_address[1]
        self._thread = threading.Thread(target=self._http.serve_forever, daemon=True)

    # ------------------------------------------------------------------ lifecycle
    def start(self) -> "RestServer":
        self._thread.start()
        return self

    def stop(self):
        """Stop accepting requests, drain the serving loop and free the join
        tables; returns the serving loop's statistics (None without batching)."""
        self._http.shutdown()
        self._http.server_close()
        return self._close()

    def serve_forever(self) -> None:
        """Serve on the calling thread until interrupted, then shut down as stop() does."""
        try:
            self._http.serve_forever()
        except KeyboardInterrupt:
            pass
        finally:
            self._http.server_close()
            self._close()

    def _close(self):
        stats = self._server.stop() if self._server else None
        self._server = None
        for h in self._joins.values():
            h.free()
        self._joins.clear()
        return stats

    # ------------------------------------------------------------------ routing
    def route(self, method: str, path: str, body: Optional[bytes]) -> Tuple[int, Dict[str, Any]]:
        path = path.split("?", 1)[0].rstrip("/") or "/"
        try:
            if method == "GET" and path == "/health":
                return 200, {"status": "ok", "engine": "falcondb"}
            if method == "GET" and path == "/tables":
                return 200, {"tables": self.db.tables()}
            m = re.fullmatch(r"/tables/([^/]+)", path)
            if m and method == "GET":
                info = self.db.table_info(m.group(1))
                if info is None:
                    return 404, {"error": f"table '{m.group(1)}' not found"}
                return 200, info
            if m and method == "DELETE":
                return self._drop(m.group(1))
            if method == "POST" and path == "/sql":
                try:
                    req = json.loads(body or b"")
                    sql = req["sql"]
                    if not isinstance(sql, str):
                        raise TypeError
                except (ValueError, KeyError, TypeError):
                    return 400, {"error": "expected a JSON body {\"sql\": \"...\"}"}
                return self.sql(sql)
            if method == "POST" and (path in ("/load/csv", "/load/fdb") or re.fullmatch(r"/tables/[^/]+/save", path)):
                return 400, {"error": "files are not loaded or saved here: create tables through the library"}
            return 404, {"error": f"no route {method} {path}"}
        except FalconError as e:
            return 400, {"error": str(e)}
        except Exception as e:  # a fault of this server, not of the request: say so rather than drop the connection
            return 500, {"error": f"{type(e).__name__}: {e}"}

    def _drop(self, name: str) -> Tuple[int, Dict[str, Any]]:
        with self._lock:
            if self.db.table_info(name) is None:
                return 404, {"error": f"table '{name}' not found"}
            # Served queries read device columns without a copy: let them finish.
            while self._inflight:
                self._idle.wait()
            for key in [k for k in self._joins if k[0] == name]:
                self._joins.pop(key).free()
            self.db.drop_table(name)
        return 200, {"dropped": name}

    def _join_table(self, b: str, key: str, payload: str, bkey, bpay) -> int:
        """The resident build table of b(key -> payload), built on first use and
        rebuilt after any table is created or dropped (self._lock held)."""
        gen = getattr(self.db, "generation", None)
        if gen != self._join_gen:
            while self._inflight:  # served joins may still read the old tables
                self._idle.wait()
            for h in self._joins.values():
                h.free()
            self._joins.clear()
            self._join_gen = gen
        k = (b, key, payload)
        h = self._joins.get(k)
        if h is None:
            h = ops.HashTable(self.db, bkey[1], bpay[1], bkey[2])
            self._joins[k] = h
        return h._h.value

    def sql(self, sql: str) -> Tuple[int, Dict[str, Any]]:
        """One /sql request: (HTTP status, JSON body)."""
        t0 = time.perf_counter()
        served = None
        if self._server is not None:
            with self._lock:
                try:
                    served = match_template(self.db, sql, self._join_table, self._catalog)
                except FalconError:
                    served = None
                if served is not None:
                    self._inflight += 1
        if served is not None:
            try:
                ticket = self._server.submit(served.query)
                r = self._server.wait(ticket)
                if r.status != 0:
                    return 400, {"error": f"serving loop error {r.status}"}
                cols, rows = served.finish(r)
                batch = int(r.batch_size)
            finally:
                with self._lock:
                    self._inflight -= 1
                    self._idle.notify_all()
            return 200, {"columns": cols, "rows": rows, "row_count": len(rows),
                         "elapsed_ms": int((time.perf_counter() - t0) * 1e3), "path": "serving",
                         "batch_size": batch}
        res = self.db.sql(sql)
        return 200, {"columns": list(res.columns), "rows": res.to_rows(), "row_count": res.rows,
                     "elapsed_ms": int((time.perf_counter() - t0) * 1e3), "path": "sql"}


def _parse_bind(bind: str) -> Tuple[str, int]:
    """host:port as FALCONDB_BIND gives it (server.rs:178, default 127.0.0.1:8080)."""
    host, _, port = bind.rpartition(":")
    if not host or not port.isdigit():
        raise ValueError(f"FALCONDB_BIND must be host:port, got {bind!r}")
    return host, int(port)


def _parse_loads(args: List[str]) -> List[Tuple[str, str]]:
    """`table=path.parquet` arguments: the tables to load before serving."""
    out = []
    for a in args:
        table, sep, path = a.partition("=")
        if not sep or not table or not path:
            raise ValueError(f"expected table=path.parquet, got {a!r}")
        out.append((table, path))
    return out


def main(argv: Optional[List[str]] = None) -> None:
    """Run the server as the reference's binary does: bind from FALCONDB_BIND,
    one database on GPU 0; `table=path.parquet` arguments are loaded first."""
    import os
    import sys

    from .parquet import load_parquet

    host, port = _parse_bind(os.environ.get("FALCONDB_BIND", "127.0.0.1:8080"))
    loads = _parse_loads(list(sys.argv[1:] if argv is None else argv))
    db = Database(0)
    for table, path in loads:
        n = load_parquet(db, path, table)
        print(f"loaded {n} rows into '{table}'")
    srv = RestServer(db, host=host, port=port)
    print(f"falcondb server listening on http://{host}:{srv.port}")
    try:
        srv.serve_forever()
    finally:
        db.close()


if __name__ == "__main__":
    main()
