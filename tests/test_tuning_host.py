"""The launch tuning on the CPU: csrc/tuning_json.cpp and tuned_grid
(csrc/tuning.h), compiled here with g++ and no CUDA.

tuned_grid is the GPU form of the reference's par_min_rows (tuning.rs:39-53):
rows per CTA times CTAs instead of rows per thread times threads."""
import ctypes as C
import json
import subprocess
import tempfile
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "falcondb_b200" / "csrc"

DRIVER = r"""
#include <cstring>
#include <string>
#include "tuning.h"
static std::string g_out;
extern "C" int tg(int cps, unsigned long long minrows, int sms, int occ, int cap, unsigned long long want,
                  unsigned long long n) {
  fdb::OpTuning t;
  t.ctas_per_sm = cps;
  t.min_rows_per_cta = minrows;
  return fdb::tuned_grid(t, sms, occ, cap, want, n);
}
extern "C" const char* to_json(const int* cps, const unsigned long long* rows, double lf, int bcps, int btr,
                               const char* dev, int sms) {
  fdb::TuningSet t;
  for (int k = 0; k < FDB_TUNE_KINDS; ++k) {
    t.op[k].ctas_per_sm = cps[k];
    t.op[k].min_rows_per_cta = rows[k];
  }
  t.batch.load_factor = lf;
  t.batch.ctas_per_sm = bcps;
  t.batch.tile_rows = btr;
  g_out = fdb::tuning_to_json(t, dev, sms);
  return g_out.c_str();
}
// Parses text; on success writes the fields and returns "", else the error.
extern "C" const char* from_json(const char* text, int* cps, unsigned long long* rows, double* lf, int* bcps,
                                 int* btr, char* dev, int devcap, int* sms) {
  fdb::TuningSet t;
  std::string d;
  g_out = fdb::tuning_from_json(text, &t, &d, sms);
  if (!g_out.empty()) return g_out.c_str();
  for (int k = 0; k < FDB_TUNE_KINDS; ++k) {
    cps[k] = t.op[k].ctas_per_sm;
    rows[k] = t.op[k].min_rows_per_cta;
  }
  *lf = t.batch.load_factor;
  *bcps = t.batch.ctas_per_sm;
  *btr = t.batch.tile_rows;
  std::strncpy(dev, d.c_str(), devcap - 1);
  dev[devcap - 1] = 0;
  return g_out.c_str();
}
"""

KINDS = 5


@pytest.fixture(scope="module")
def lib():
    d = Path(tempfile.mkdtemp(prefix="tuning_host_"))
    (d / "driver.cpp").write_text(DRIVER)
    so = d / "libtg.so"
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", str(CSRC), str(CSRC / "tuning_json.cpp"),
                    str(d / "driver.cpp"), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    L.tg.restype = C.c_int
    L.tg.argtypes = [C.c_int, C.c_ulonglong, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_ulonglong]
    L.to_json.restype = C.c_char_p
    L.to_json.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_ulonglong), C.c_double, C.c_int, C.c_int, C.c_char_p,
                          C.c_int]
    L.from_json.restype = C.c_char_p
    L.from_json.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_ulonglong), C.POINTER(C.c_double),
                            C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p, C.c_int, C.POINTER(C.c_int)]
    return L


def test_tuned_grid(lib):
    # Defaults: one CTA per unit of work, up to SMs x min(occupancy, cap).
    assert lib.tg(0, 0, 148, 3, 4, 10_000, 10**8) == 148 * 3
    assert lib.tg(0, 0, 148, 6, 4, 10_000, 10**8) == 148 * 4
    assert lib.tg(0, 0, 148, 0, 4, 10_000, 10**8) == 148          # occupancy reported 0: still one per SM
    assert lib.tg(0, 0, 148, 3, 4, 17, 10**8) == 17
    assert lib.tg(0, 0, 148, 3, 4, 0, 0) == 1
    # A cap below occupancy applies; above it changes nothing.
    assert lib.tg(2, 0, 148, 3, 4, 10_000, 10**8) == 296
    assert lib.tg(8, 0, 148, 3, 4, 10_000, 10**8) == 148 * 3
    # Rows per CTA: ceil(n / rows) CTAs, at least 1, never more than the work.
    assert lib.tg(0, 1 << 17, 148, 3, 4, 10_000, 1_000_000) == 8
    assert lib.tg(0, 1 << 17, 148, 3, 4, 5, 1_000_000) == 5
    assert lib.tg(0, 1 << 17, 148, 3, 4, 10_000, 1) == 1
    assert lib.tg(0, 1, 148, 3, 4, 10_000, 10**8) == 148 * 3


def arrays(cps, rows):
    return (C.c_int * KINDS)(*cps), (C.c_ulonglong * KINDS)(*rows)


def test_json_round_trip(lib):
    cps, rows = arrays([4, 0, 3, 8, 1], [0, 1 << 15, 0, 1 << 19, 12345])
    text = lib.to_json(cps, rows, 0.7, 3, 4096, b'NVIDIA B200 "x"\\', 148)
    doc = json.loads(text)                      # valid JSON
    assert doc["device"] == 'NVIDIA B200 "x"\\' and doc["sm_count"] == 148
    assert doc["ops"]["probe"] == {"ctas_per_sm": 8, "min_rows_per_cta": 1 << 19}
    assert doc["gb_batch"] == {"load_factor": 0.7, "ctas_per_sm": 3, "tile_rows": 4096}
    o_cps, o_rows = arrays([9] * KINDS, [9] * KINDS)
    lf, bc, bt, sms = C.c_double(), C.c_int(), C.c_int(), C.c_int()
    dev = C.create_string_buffer(128)
    err = lib.from_json(text, o_cps, o_rows, C.byref(lf), C.byref(bc), C.byref(bt), dev, 128, C.byref(sms))
    assert err == b""
    assert list(o_cps) == [4, 0, 3, 8, 1] and list(o_rows) == [0, 1 << 15, 0, 1 << 19, 12345]
    assert (lf.value, bc.value, bt.value, sms.value) == (0.7, 3, 4096, 148)
    assert dev.value == b'NVIDIA B200 "x"\\'


def parse(lib, text):
    o_cps, o_rows = arrays([9] * KINDS, [9] * KINDS)
    lf, bc, bt, sms = C.c_double(), C.c_int(), C.c_int(), C.c_int()
    dev = C.create_string_buffer(128)
    err = lib.from_json(text.encode(), o_cps, o_rows, C.byref(lf), C.byref(bc), C.byref(bt), dev, 128, C.byref(sms))
    return err.decode(), list(o_cps), list(o_rows)


def test_json_partial_and_bad_files(lib):
    # Kinds a file leaves out keep the defaults; key order does not matter.
    err, cps, rows = parse(lib, '{"ops": {"topk": {"min_rows_per_cta": 5, "ctas_per_sm": 2}}, '
                                '"sm_count": 148, "device": "B"}')
    assert err == "" and cps == [0, 0, 0, 0, 2] and rows == [0, 0, 0, 0, 5]
    for bad in ['', '[]', '{"device": "B"}', '{"device": "B", "sm_count": 148}',
                '{"device": "B", "sm_count": 148, "ops": {"scan": {"ctas_per_sm": -1, "min_rows_per_cta": 0}}}',
                '{"device": "B", "sm_count": 148, "ops": {"scan": {"ctas_per_sm": 1.5, "min_rows_per_cta": 0}}}',
                '{"device": "B", "sm_count": 148, "ops": {}, "gb_batch": {"load_factor": 2, "ctas_per_sm": 1, '
                '"tile_rows": 4096}}',
                '{"device": "B", "sm_count": 148, "ops": {}} trailing',
                '{"device": "B", "sm_count": 148, "ops": {"scan": {"ctas_per_sm": 1}}}']:
        err, _, _ = parse(lib, bad)
        assert err, bad
