"""Zone maps on the CPU: the oracle's restatement against brute force, and
the engine's pruning logic (csrc/zone_prune.cpp, compiled here with g++ and
no CUDA) against the oracle.

The bar for pruning is the reference's own (stats.rs:8-10): a batch may be
ruled out only when no row of it passes.  Every case checks that by
evaluating the predicate on every row, with the filter's semantics (NULL fails
every comparison, NaN passes NE only, an INT64 column against a FLOAT64
literal compares as float)."""
import ctypes as C
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import falcondb_b200 as F
from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "falcondb_b200" / "csrc"

DRIVER = r"""
#include <stdexcept>
#include <string>
#include "zone.h"
namespace fdb {
void fail(int, const std::string& m) { throw std::runtime_error(m); }
}
extern "C" int zr_rule_out(const fdb_zone* zones, const int32_t* dtypes, int ncols, uint64_t nb,
                           const fdb_pred_term* prog, int nterms, const uint64_t* sets,
                           const uint64_t* set_off, uint8_t* out) {
  try {
    std::vector<std::vector<fdb_zone>> z(ncols);
    std::vector<const std::vector<fdb_zone>*> zp;
    std::vector<int32_t> dt;
    for (int c = 0; c < ncols; ++c) {
      z[c].assign(zones + c * nb, zones + (c + 1) * nb);
      zp.push_back(&z[c]);
      dt.push_back(dtypes[c]);
    }
    std::vector<std::vector<uint64_t>> cs(nterms);
    for (int i = 0; i < nterms; ++i) cs[i].assign(sets + set_off[i], sets + set_off[i + 1]);
    const std::vector<uint8_t> r = fdb::zone_rule_out(zp, dt, prog, nterms, cs, nb);
    for (uint64_t b = 0; b < nb; ++b) out[b] = r[b];
    return 0;
  } catch (...) {
    return -1;
  }
}
extern "C" int zr_key_range(const fdb_zone* zones, uint64_t nb, uint64_t first, uint64_t n,
                            int64_t* lo, int64_t* hi) {
  std::vector<fdb_zone> z(zones, zones + nb);
  return fdb::zone_key_range(z, first, n, lo, hi) ? 1 : 0;
}
"""

KIND_DTYPE = {"int": F.INT64, "float": F.FLOAT64, "code": F.UTF8}


@pytest.fixture(scope="module")
def zr():
    d = Path(tempfile.mkdtemp(prefix="zone_host_"))
    (d / "driver.cpp").write_text(DRIVER)
    so = d / "libzr.so"
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", str(CSRC), str(CSRC / "zone_prune.cpp"),
                    str(d / "driver.cpp"), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    lib.zr_rule_out.restype = C.c_int
    lib.zr_key_range.restype = C.c_int
    return lib


def engine_rule_out(lib, zones, kinds, terms, batch_count):
    """Runs zone_prune.cpp's zone_rule_out on the oracle's zone maps."""
    ncols = len(zones)
    flat = np.concatenate([np.asarray(z, dtype=O.ZONE_DTYPE) for z in zones]) if ncols else np.zeros(0, O.ZONE_DTYPE)
    dtypes = np.array([KIND_DTYPE[k] for k in kinds], dtype=np.int32)
    prog = (F.fdb_pred_term * max(1, len(terms)))()
    sets, offs = [], [0]
    for i, t in enumerate(terms):
        prog[i].kind = t["kind"]
        prog[i].col = t.get("col", 0)
        prog[i].op = t.get("op", 0)
        if t["kind"] == O.T_CODE_SET:
            words = np.zeros((t["dict_len"] + 63) // 64 or 1, dtype=np.uint64)
            for c in t["set"]:
                words[c >> 6] |= np.uint64(1) << np.uint64(c & 63)
            prog[i].lit_i = t["dict_len"]
            sets.append(words)
        elif t["kind"] == O.T_CMP:
            if t.get("lit_float"):
                prog[i].lit_type, prog[i].lit_f = F.FLOAT64, float(t["lit"])
            else:
                prog[i].lit_type, prog[i].lit_i = F.INT64, int(t["lit"])
        offs.append(offs[-1] + (len(sets[-1]) if t["kind"] == O.T_CODE_SET else 0))
    allsets = np.concatenate(sets) if sets else np.zeros(1, np.uint64)
    off = np.array(offs, dtype=np.uint64)
    out = np.zeros(max(1, batch_count), dtype=np.uint8)
    rc = lib.zr_rule_out(C.c_void_p(flat.ctypes.data), C.c_void_p(dtypes.ctypes.data), ncols,
                         C.c_uint64(batch_count), prog, len(terms), C.c_void_p(allsets.ctypes.data),
                         C.c_void_p(off.ctypes.data), C.c_void_p(out.ctypes.data))
    assert rc == 0
    return out[:batch_count].astype(bool)


def row_pass(cols, kinds, valids, terms, n):
    """The predicate on every row (eval_leaf / eval_prog semantics)."""
    st = []
    for t in terms:
        k = t["kind"]
        if k in (O.T_AND, O.T_OR):
            a, b = st.pop(), st.pop()
            st.append(a & b if k == O.T_AND else a | b)
            continue
        v, kind, ok = cols[t["col"]], kinds[t["col"]], valids[t["col"]].copy()
        if kind == "code":
            isnull = ~ok | (v == O.NULL_CODE)
        else:
            isnull = ~ok
        if k == O.T_IS_NULL:
            st.append(isnull)
            continue
        if k == O.T_IS_NOT_NULL:
            st.append(~isnull)
            continue
        if k == O.T_CODE_SET:
            inset = np.isin(v, np.array(sorted(t["set"]), dtype=v.dtype)) & (v < t["dict_len"])
            st.append(inset & ~isnull)
            continue
        op = t["op"]
        if kind == "float" or (kind == "int" and t.get("lit_float")):
            a, lit = v.astype(np.float64), float(t["lit"])
        else:
            a, lit = v.astype(np.int64), int(t["lit"])
        with np.errstate(invalid="ignore"):
            r = {O.EQ: a == lit, O.NE: a != lit, O.LT: a < lit, O.LE: a <= lit, O.GT: a > lit, O.GE: a >= lit}[op]
        st.append(r & ~isnull)
    return st.pop()


def random_column(rng, kind, n, sorted_=False, nulls=0.0, nan=0.0):
    if kind == "int":
        v = rng.integers(-1000, 1000, n).astype(np.int64)
    elif kind == "float":
        v = rng.normal(0, 100, n)
        if nan:
            v[rng.random(n) < nan] = np.nan
    else:
        v = rng.integers(0, 40, n).astype(np.uint32)
    if sorted_:
        v = np.sort(v) if kind != "float" else np.sort(v)
    valid = rng.random(n) >= nulls
    return v, valid


def random_terms(rng, kinds, cols, depth=2):
    def leaf():
        c = int(rng.integers(0, len(kinds)))
        kind = kinds[c]
        r = rng.random()
        if r < 0.1:
            return [dict(kind=O.T_IS_NULL, col=c)]
        if r < 0.2:
            return [dict(kind=O.T_IS_NOT_NULL, col=c)]
        if kind == "code":
            s = set(int(x) for x in rng.integers(0, 40, int(rng.integers(0, 4))))
            return [dict(kind=O.T_CODE_SET, col=c, set=s, dict_len=40)]
        x = cols[c][int(rng.integers(0, len(cols[c])))]
        lit_float = kind == "float" or rng.random() < 0.3
        lit = float(x) + (rng.choice([-0.5, 0.0, 0.5]) if lit_float else 0) if lit_float else int(x)
        if lit_float and rng.random() < 0.05:
            lit = float("nan")
        return [dict(kind=O.T_CMP, col=c, op=int(rng.integers(0, 6)), lit=lit, lit_float=lit_float)]

    def tree(d):
        if d == 0 or rng.random() < 0.4:
            return leaf()
        return tree(d - 1) + tree(d - 1) + [dict(kind=O.T_AND if rng.random() < 0.5 else O.T_OR)]

    return tree(depth)


def test_oracle_zone_map_against_brute_force():
    rng = np.random.default_rng(1)
    n = 3 * 1000 + 17
    for kind in ("int", "float", "code"):
        v, valid = random_column(rng, kind, n, nulls=0.1, nan=0.05)
        words = np.packbits(valid, bitorder="little")
        words = np.concatenate([words, np.zeros((-len(words)) % 8, np.uint8)]).view(np.uint64)
        z = O.zone_map(v, kind, words, batch_rows=1000)
        assert len(z) == 4 and list(z["rows"]) == [1000, 1000, 1000, 17]
        for b in range(4):
            s, e = b * 1000, min(n, (b + 1) * 1000)
            ok = valid[s:e] & ((v[s:e] != O.NULL_CODE) if kind == "code" else True)
            assert z["null_count"][b] == (~ok).sum()
            x = v[s:e][ok]
            if kind == "float":
                assert bool(z["flags"][b] & O.ZONE_NAN) == bool(np.isnan(x).any())
                x = x[~np.isnan(x)]
                assert z["min_f"][b] == x.min() and z["max_f"][b] == x.max()
            else:
                assert z["min_i"][b] == x.min() and z["max_i"][b] == x.max()


@pytest.mark.parametrize("seed", range(12))
def test_pruning_is_sound_and_engine_matches_oracle(zr, seed):
    rng = np.random.default_rng(seed)
    br = 512
    n = br * 9 + int(rng.integers(1, br))
    kinds = ["int", "float", "code"]
    cols, valids, zones = [], [], []
    for i, kind in enumerate(kinds):
        v, valid = random_column(rng, kind, n, sorted_=(seed + i) % 2 == 0, nulls=[0.0, 0.05, 0.5][seed % 3],
                                 nan=0.02 if seed % 4 == 0 else 0.0)
        if seed % 5 == 0:  # a batch of nothing but NULLs
            valid[br:2 * br] = False
        cols.append(v)
        valids.append(valid)
        words = np.packbits(valid, bitorder="little")
        words = np.concatenate([words, np.zeros((-len(words)) % 8, np.uint8)]).view(np.uint64)
        zones.append(O.zone_map(v, kind, words, batch_rows=br))
    nb = len(zones[0])
    fired = 0
    for _ in range(40):
        terms = random_terms(rng, kinds, cols)
        want = O.zone_rule_out(zones, kinds, terms)
        got = engine_rule_out(zr, zones, kinds, terms, nb)
        assert np.array_equal(got, want), terms
        passing = row_pass(cols, kinds, valids, terms, n)
        for b in np.flatnonzero(want):
            assert not passing[b * br:(b + 1) * br].any(), (b, terms)
        fired += int(want.sum())
    assert fired > 0


def test_pruning_edge_rules(zr):
    """Rules where the engine's exact pruning and the reference's f64 rule
    (stats.rs:70-113) part: INT64 bounds beyond 2^53, NE over a batch with a
    NaN, and a NaN literal."""
    big = np.array([2**53 + 1] * 10, dtype=np.int64)
    z = O.zone_map(big, "int", batch_rows=16)
    # col > 2^53 passes every row: neither may rule the batch out...
    t = [dict(kind=O.T_CMP, col=0, op=O.GT, lit=2**53)]
    assert not O.zone_rule_out([z], ["int"], t)[0]
    assert not engine_rule_out(zr, [z], ["int"], t, 1)[0]
    # ...but the reference's rule, with bounds rounded through f64, does.
    assert O.ref_can_skip_cmp(big, O.GT, 2**53)
    assert row_pass([big], ["int"], [np.ones(10, bool)], t, 10).all()

    f = np.array([1.0, 1.0, np.nan])
    zf = O.zone_map(f, "float", batch_rows=16)
    t = [dict(kind=O.T_CMP, col=0, op=O.NE, lit=1.0, lit_float=True)]
    assert not O.zone_rule_out([zf], ["float"], t)[0]
    assert not engine_rule_out(zr, [zf], ["float"], t, 1)[0]
    assert O.ref_can_skip_cmp(f, O.NE, 1.0)      # the reference would drop the NaN row
    assert row_pass([f], ["float"], [np.ones(3, bool)], t, 3)[2]

    for op in range(6):
        t = [dict(kind=O.T_CMP, col=0, op=op, lit=float("nan"), lit_float=True)]
        want = op != O.NE
        assert O.zone_rule_out([zf], ["float"], t)[0] == want
        assert engine_rule_out(zr, [zf], ["float"], t, 1)[0] == want


def test_key_range_from_zone_maps(zr):
    v = np.arange(10 * 100, dtype=np.int64)[::-1].copy()
    z = O.zone_map(v, "int", batch_rows=O.ZONE_BATCH_ROWS)
    lo, hi = C.c_int64(), C.c_int64()
    assert zr.zr_key_range(C.c_void_p(z.ctypes.data), C.c_uint64(len(z)), C.c_uint64(0), C.c_uint64(len(v)),
                           C.byref(lo), C.byref(hi)) == 1
    assert (lo.value, hi.value) == (0, 999)
    # INT64_MIN is a NULL key to GROUP BY: no range from the zone map.
    v[3] = np.iinfo(np.int64).min
    z = O.zone_map(v, "int")
    assert zr.zr_key_range(C.c_void_p(z.ctypes.data), C.c_uint64(len(z)), C.c_uint64(0), C.c_uint64(len(v)),
                           C.byref(lo), C.byref(hi)) == 0
    # Rows past the zone map: no range.
    assert zr.zr_key_range(C.c_void_p(z.ctypes.data), C.c_uint64(len(z)), C.c_uint64(0),
                           C.c_uint64(O.ZONE_BATCH_ROWS + 1), C.byref(lo), C.byref(hi)) == 0
