"""Writes tests/golden/known_answers.json: the known-answer cases of FalconDB's
own test suites on the scan / filter / aggregate / join / top-k path, restated
as data (inputs, SQL, expected answer) with the file:line each comes from.

Expected answers are the reference's assertions; where the reference asserts
"fast path == materialised path" (count_star_filter.rs) the materialised count
is computed here by plain Python over the fixture rows.  Generated fixtures are
described by a small spec that tests/known_answers.py expands (the formulas are
the reference's: e.g. `maybe` is NULL when i % 3 == 0).

Run: python tests/golden/make_known_answers.py
"""
import json
from pathlib import Path

OUT = Path(__file__).with_name("known_answers.json")
cases = []


def case(name, source, tables, sql, **expect):
    cases.append({"name": name, "source": source, "tables": tables, "sql": sql, "expect": expect})


def cols(**kw):
    return {"columns": [{"name": k, "type": t, "values": v} for k, (t, v) in kw.items()]}


# --- tests/count_star_filter.rs:51-90 ------------------------------------------------
PREDS = [
    ("n >= 0", lambda i: i >= 0),
    ("n < 0", lambda i: i < 0),
    ("n >= 0 AND n < 100000", lambda i: 0 <= i < 100000),
    ("n > 10", lambda i: i > 10),
    ("maybe IS NULL", lambda i: i % 3 == 0),
    ("maybe IS NOT NULL", lambda i: i % 3 != 0),
    ("s = 'a'", lambda i: i % 3 == 0),
    ("s <> 'a'", lambda i: i % 3 != 0),
    ("s LIKE 'b%'", lambda i: i % 3 == 1),
    ("n IN (1, 2, 3)", lambda i: i in (1, 2, 3)),
    ("n NOT IN (1, 2, 3)", lambda i: i not in (1, 2, 3)),
    ("n > 5 AND n < 20", lambda i: 5 < i < 20),
    ("n < 2 OR n > 9995", lambda i: i < 2 or i > 9995),
]
for rows in [1, 63, 64, 65, 127, 128, 129, 1000, 4095, 10000]:
    for pred, fn in PREDS:
        materialised = sum(1 for i in range(rows) if fn(i))
        case(f"count_star_filter[{rows}][{pred}]", "tests/count_star_filter.rs:51-90",
             {"t": {"gen": "count_star", "rows": rows}}, f"SELECT COUNT(*) FROM t WHERE {pred}",
             scalar=str(materialised))
case("count_col_counts_non_null", "tests/count_star_filter.rs:92-97",
     {"t": {"gen": "count_star", "rows": 300}}, "SELECT COUNT(maybe) FROM t WHERE n >= 0", scalar="200")

# --- tests/sql_integration.rs:239-310 -------------------------------------------------
case("group_by_count", "tests/sql_integration.rs:239-248",
     {"t": cols(dept=("utf8", ["eng", "hr", "eng", "hr", "eng"]))},
     "SELECT dept, COUNT(*) as n FROM t GROUP BY dept", rows=[["eng", "3"], ["hr", "2"]], sorted=True)
case("group_by_sum", "tests/sql_integration.rs:250-258",
     {"t": cols(dept=("utf8", ["eng", "hr", "eng", "hr"]), salary=("int64", [100, 80, 120, 90]))},
     "SELECT dept, SUM(salary) as total FROM t GROUP BY dept", rows=[["eng", "220"], ["hr", "170"]], sorted=True)
case("group_by_avg", "tests/sql_integration.rs:260-267",
     {"t": cols(dept=("utf8", ["eng", "eng", "hr"]), score=("int64", [10, 20, 30]))},
     "SELECT dept, AVG(score) as avg FROM t GROUP BY dept", rows=[["eng", "15"], ["hr", "30"]], sorted=True)
case("group_by_min_max", "tests/sql_integration.rs:269-277",
     {"t": cols(dept=("utf8", ["eng", "eng", "eng"]), score=("int64", [5, 10, 7]))},
     "SELECT dept, MIN(score) as mn, MAX(score) as mx FROM t GROUP BY dept", rows=[["eng", "5", "10"]])
case("aggregate_without_group_by", "tests/sql_integration.rs:279-285",
     {"t": cols(n=("int64", [1, 2, 3, 4, 5]))}, "SELECT COUNT(*) as cnt FROM t", scalar="5")
case("count_on_empty_table", "tests/sql_integration.rs:287-292",
     {"t": cols(n=("int64", []))}, "SELECT COUNT(*) as cnt FROM t", scalar="0")
case("group_by_single_group", "tests/sql_integration.rs:294-300",
     {"t": cols(dept=("utf8", ["eng", "eng", "eng"]), n=("int64", [1, 2, 3]))},
     "SELECT dept, SUM(n) as total FROM t GROUP BY dept", rows=[["eng", "6"]])
case("group_by_all_unique", "tests/sql_integration.rs:302-307",
     {"t": cols(dept=("utf8", ["eng", "hr", "finance"]), n=("int64", [1, 2, 3]))},
     "SELECT dept, COUNT(*) as cnt FROM t GROUP BY dept", row_count=3)

# --- tests/sql_integration.rs:1343-1380 (JOIN), 1396-1410 (COUNT DISTINCT) -------------
EMP = cols(id=("int64", [1, 2, 3]), name=("utf8", ["alice", "bob", "carol"]))
SCORES = cols(id=("int64", [1, 2]), score=("float64", [9.5, 7.0]))
case("inner_join_basic", "tests/sql_integration.rs:1343-1361", {"emp": EMP, "scores": SCORES},
     "SELECT name, score FROM emp JOIN scores ON emp.id = scores.id",
     rows=[["alice", "9.5"], ["bob", "7"]], sorted=True)
case("left_join_keeps_unmatched", "tests/sql_integration.rs:1363-1380", {"emp": EMP, "scores": SCORES},
     "SELECT name FROM emp LEFT JOIN scores ON emp.id = scores.id", row_count=3)
case("count_distinct_basic", "tests/sql_integration.rs:1396-1400",
     {"t": cols(dept=("utf8", ["eng", "hr", "eng", "hr", "eng"]))},
     "SELECT COUNT(DISTINCT dept) as n FROM t", scalar="2")

# --- src/query/aggregate.rs:3519-3597, 3704-3734 ---------------------------------------
DEPTS5 = ["eng", "sales", "hr", "ops", "legal"]
TOTAL = 700_000
exp = []
for g, d in enumerate(DEPTS5):
    vals = range(g, TOTAL, 5)
    exp.append([d, str(len(vals)), str(sum(vals))])
case("parallel_group_by_matches_a_single_batch", "src/query/aggregate.rs:3519-3597",
     {"t": {"gen": "split_700k"}}, "SELECT dept, COUNT(v) AS cnt, SUM(v) AS total FROM t GROUP BY dept",
     rows=sorted(exp), sorted=True)
MB = cols(dept=("utf8", ["eng", "eng", "hr", "hr", "eng"]), score=("float64", [9.0, 8.0, 7.0, 6.0, 10.0]))
case("agg_only_count_sum", "src/query/aggregate.rs:3704-3718", {"t": MB},
     "SELECT COUNT(score) AS cnt, SUM(score) AS total FROM t", rows=[["5", "40"]])
case("agg_min_max", "src/query/aggregate.rs:3720-3734", {"t": MB},
     "SELECT MIN(score) AS min_s, MAX(score) AS max_s FROM t", rows=[["6", "10"]])

# --- src/query/join.rs:2607-2660: NULL join keys match nothing ------------------------
NL = cols(k=("int64", [1, None, 3, None]))
NR = cols(rk=("int64", [1, None, 4]))
case("null_key_inner", "src/query/join.rs:2633-2634", {"l": NL, "r": NR},
     "SELECT COUNT(*) FROM l JOIN r ON l.k = r.rk", scalar="1")
case("null_key_left", "src/query/join.rs:2635-2636", {"l": NL, "r": NR},
     "SELECT COUNT(*) FROM l LEFT JOIN r ON l.k = r.rk", scalar="4")
case("null_key_semi", "src/query/join.rs:2654-2655", {"l": NL, "r": NR},
     "SELECT COUNT(*) FROM l WHERE EXISTS (SELECT 1 FROM r WHERE r.rk = l.k)", scalar="1")
case("null_key_anti", "src/query/join.rs:2656-2658", {"l": NL, "r": NR},
     "SELECT COUNT(*) FROM l WHERE NOT EXISTS (SELECT 1 FROM r WHERE r.rk = l.k)", scalar="3")

# --- tests/join_and_parquet_paths.rs:47-113 -------------------------------------------
def join_db(l, r, base=0):
    return {"l": {"gen": "join_db_left", "rows": l}, "r": {"gen": "join_db_right", "rows": r, "base": base}}


case("inner_join_keeps_every_match", "tests/join_and_parquet_paths.rs:47-57", join_db(4000, 2000),
     "SELECT lv FROM l JOIN r ON l.k = r.k", row_count=2000)
case("inner_join_below_threshold", "tests/join_and_parquet_paths.rs:59-64", join_db(500, 300),
     "SELECT lv FROM l JOIN r ON l.k = r.k", row_count=300)
case("left_join_keeps_unmatched_rows", "tests/join_and_parquet_paths.rs:66-76", join_db(4000, 2000),
     "SELECT lv FROM l LEFT JOIN r ON l.k = r.k", row_count=4000)
case("join_with_no_overlap", "tests/join_and_parquet_paths.rs:78-101", join_db(2000, 2000, base=100_000),
     "SELECT lv FROM l JOIN r ON l.k = r.k", row_count=0)
case("join_result_matches_a_small_reference", "tests/join_and_parquet_paths.rs:103-113", join_db(2000, 2000),
     "SELECT l.k, lv, rv FROM l JOIN r ON l.k = r.k WHERE l.k < 3", first_col_sorted=["0", "1", "2"])

# --- benches/query_bench.rs assertions (dataset 103-122, lookup 486-500) ---------------
for rows in [100_000, 1_000_000]:
    case(f"bench_sum_score[{rows}]", "benches/query_bench.rs:208-211", {"bench": {"gen": "bench", "rows": rows}},
         "SELECT SUM(score) AS s FROM bench", scalar=str(rows // 100 * 5000))
    case(f"bench_filter_half[{rows}]", "benches/query_bench.rs:272-273", {"bench": {"gen": "bench", "rows": rows}},
         "SELECT COUNT(*) FROM bench WHERE score > 50", scalar=str(rows // 2))
    tabs = {"bench": {"gen": "bench", "rows": rows}, "lookup": {"gen": "lookup", "rows": rows}}
    case(f"bench_inner_join[{rows}]", "benches/query_bench.rs:519-522", tabs,
         "SELECT COUNT(*) AS n FROM bench JOIN lookup ON bench.id = lookup.lid", scalar=str(rows // 10))
    case(f"bench_left_join[{rows}]", "benches/query_bench.rs:630-634", tabs,
         "SELECT COUNT(*) AS n FROM bench LEFT JOIN lookup ON bench.id = lookup.lid", scalar=str(rows))
    case(f"bench_semi_join[{rows}]", "benches/query_bench.rs:635-639", tabs,
         "SELECT COUNT(*) AS n FROM bench WHERE EXISTS (SELECT 1 FROM lookup WHERE lookup.lid = bench.id)",
         scalar=str(rows // 10))
    case(f"bench_anti_join[{rows}]", "benches/query_bench.rs:640-644", tabs,
         "SELECT COUNT(*) AS n FROM bench WHERE NOT EXISTS (SELECT 1 FROM lookup WHERE lookup.lid = bench.id)",
         scalar=str(rows - rows // 10))

# --- ORDER BY several keys / a text key, DISTINCT over whole rows ---------------------
case("order_by_string", "tests/sql_integration.rs:210-216",
     {"t": cols(name=("utf8", ["charlie", "alice", "bob"]))},
     "SELECT * FROM t ORDER BY name ASC", rows=[["alice"], ["bob"], ["charlie"]])
case("order_by_multi_key", "tests/sql_integration.rs:218-226",
     {"t": cols(dept=("utf8", ["eng", "hr", "eng", "hr"]), score=("int64", [8, 9, 9, 7]))},
     "SELECT * FROM t ORDER BY dept ASC, score DESC", head_rows=[["eng", "9"], ["eng", "8"], ["hr", "9"]])
for direction, want in (("ASC", ["apple", "apple", "fig", "pear"]), ("DESC", ["pear", "fig", "apple", "apple"])):
    case(f"sort_text_by_string_not_dictionary_position[{direction}]", "src/query/sort.rs:979-1001",
         {"t": cols(s=("utf8", ["pear", "apple", "fig", "apple"]))},
         f"SELECT s FROM t ORDER BY s {direction}", rows=[[w] for w in want])
for order_by, want in (("s ASC", ["NULL", "NULL", "a", "b"]), ("s ASC NULLS LAST", ["a", "b", "NULL", "NULL"]),
                       ("s DESC", ["b", "a", "NULL", "NULL"])):
    case(f"sort_text_places_nulls[{order_by}]", "src/query/sort.rs:1003-1022",
         {"t": cols(s=("utf8", ["b", None, "a", None]))},
         f"SELECT s FROM t ORDER BY {order_by}", rows=[[w] for w in want])
for direction in ("ASC", "DESC"):
    case(f"sort_equal_strings_keep_row_order[{direction}]", "src/query/sort.rs:1024-1049",
         {"t": cols(s=("utf8", ["x", "x", "x", "x"]), id=("int64", [10, 20, 30, 40]))},
         f"SELECT id FROM t ORDER BY s {direction}", rows=[["10"], ["20"], ["30"], ["40"]])
_distinct64 = ["%03d" % ((i * 37) % 64) for i in range(64)]
case("sort_all_distinct_text_column", "src/query/sort.rs:1051-1060",
     {"t": cols(s=("utf8", _distinct64))}, "SELECT s FROM t ORDER BY s", rows=[[w] for w in sorted(_distinct64)])
case("sort_multi_key", "src/query/sort.rs:1747-1766",
     {"t": cols(dept=("utf8", ["eng", "hr", "eng"]), score=("float64", [8.0, 9.0, 7.0]))},
     "SELECT dept, score FROM t ORDER BY dept ASC, score DESC", rows=[["eng", "8"], ["eng", "7"], ["hr", "9"]])
case("distinct_compares_whole_rows", "tests/sort_and_dedup_paths.rs:162-165",
     {"t": cols(a=("int64", [1, 1, 1]), b=("utf8", ["x", "y", "x"]))},
     "SELECT DISTINCT a, b FROM t", row_count=2)

OUT.write_text(json.dumps({"generated_by": "tests/golden/make_known_answers.py", "cases": cases}, indent=1))
print(f"wrote {len(cases)} cases to {OUT}")
