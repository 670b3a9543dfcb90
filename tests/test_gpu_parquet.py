"""A Parquet file loaded into HBM (falcondb_b200.parquet) answers the config-0
query like the same table created from memory: per-department results by
string value, over row groups that meet the departments in different orders
(the case the reference's per-batch dictionaries get wrong,
aggregate.rs:655-658)."""
import numpy as np
import pytest

import falcondb_b200 as F
from falcondb_b200 import parquet as P
from falcondb_b200 import workloads as W
from oracle import oracle as O

pa = pytest.importorskip("pyarrow")
pq = pytest.importorskip("pyarrow.parquet")

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def test_parquet_load_then_group_by(db, tmp_path):
    n = 300_000
    t = W.table_t(n, seed=31)
    depts = np.array(W.DEPTS, dtype=object)[t["dept"].codes]
    depts[:65_536] = np.where(np.arange(65_536) % 2 == 0, "d11", "d03")  # the first row group: two departments
    path = str(tmp_path / "t.parquet")
    pq.write_table(pa.table({"id": t["id"], "dept": pa.array(depts.tolist()), "score": t["score"],
                             "salary": t["salary"]}), path, row_group_size=65_536)
    assert P.load_parquet(db, path, "pt") == n
    res = db.sql("SELECT dept, COUNT(*), SUM(score), AVG(salary) FROM pt WHERE score > 50 GROUP BY dept")
    codes = np.array([W.DEPTS.index(d) for d in depts], dtype=np.uint32)
    g = O.group_codes(codes, 12, mask=O.cmp_mask(t["score"], F.GT, 50), fvals=t["score"], ivals=t["salary"])
    got = {res.column(0)[i]: (res.column(1)[i], res.column(2)[i], res.column(3)[i]) for i in range(res.rows)}
    want = {W.DEPTS[k]: (g["rows"][k], g["fsum"][k], g["isum"][k] / g["icnt"][k]) for k in range(12) if g["rows"][k]}
    assert set(got) == set(want)
    for d, (cnt, s, avg) in want.items():
        assert got[d][0] == cnt and abs(got[d][1] - s) <= RTOL * s and got[d][2] == avg
    assert db.sql("SELECT COUNT(*) FROM pt WHERE score > 50").column(0)[0] == int((t["score"] > 50).sum())
    db.drop_table("pt")


def test_parquet_text_columns_merged_on_the_gpu(db, tmp_path):
    """Several row groups whose dictionaries list the departments in different
    orders (and one that lacks most of them), NULL text values, and a second
    text column: the loader merges the dictionaries and fdb_dict_remap
    rewrites every row's code on the device; answers by department name equal
    the oracle's, and every row's string equals the file's."""
    n = 200_000
    r = np.random.default_rng(8)
    codes = r.integers(0, 12, n)
    depts = np.array(W.DEPTS, dtype=object)[codes]
    depts[:20_000] = np.where(np.arange(20_000) % 3 == 0, "d07", "d01")  # group 0: two departments
    depts[20_000:40_000] = sorted(depts[20_000:40_000], reverse=True)    # group 1: d11 first
    nulls = r.random(n) < 0.03
    depts_n = [None if nulls[i] else depts[i] for i in range(n)]
    city = np.array(["oslo", "lima", "kyiv", "pune"], dtype=object)[r.integers(0, 4, n)]
    score = r.random(n) * 100
    path = str(tmp_path / "m.parquet")
    pq.write_table(pa.table({"dept": pa.array(depts_n), "city": pa.array(city.tolist()), "score": score}), path,
                   row_group_size=20_000)
    assert pq.ParquetFile(path).num_row_groups == 10
    assert P.load_parquet(db, path, "m") == n
    res = db.sql("SELECT dept, COUNT(*), SUM(score) FROM m WHERE score > 25 GROUP BY dept")
    got = {res.column(0)[i]: (res.column(1)[i], res.column(2)[i]) for i in range(res.rows)}
    sel = score > 25
    dn = np.array(["" if d is None else d for d in depts_n], dtype=object)
    for name in set(d for d in depts_n if d is not None):
        m = sel & (dn == name)
        want_sum = O.sum_serial(score[m])
        assert got[name][0] == int(m.sum()) and abs(got[name][1] - want_sum) <= RTOL * want_sum
    assert got[None][0] == int((sel & nulls).sum())  # the NULL group
    # Row by row: the strings read back are the file's.
    back = db.sql("SELECT dept, city FROM m")
    assert back.column(0) == depts_n and back.column(1) == city.tolist()
    db.drop_table("m")
