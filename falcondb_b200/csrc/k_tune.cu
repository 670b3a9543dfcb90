// Autotuner of the streamed operators' launch shapes: the GPU counterpart of
// the reference's fixed parallel cut-offs (par_min_rows, tuning.rs:39-53).
// Each kind of operator is timed on synthetic columns in device memory, over
// candidate CTAs per SM at the requested size, then candidate rows per CTA on
// a small input, where launching fewer CTAs can pay.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace fdb {
namespace {

// Synthetic columns, the configurations' shapes: score FLOAT64 uniform
// [0, 100), dept codes 0..11, salary INT64 in [30000, 200000], an INT64
// group key uniform over [0, n / 16), and probe keys uniform over [0, 2B).
__global__ void tune_fill_kernel(uint64_t n, uint64_t build, double* score, uint32_t* dept, int64_t* salary,
                                 int64_t* gkey, int64_t* pkey) {
  const uint64_t groups = n / 16 > 0 ? n / 16 : 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t h = mix64(i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull);
    const uint64_t h2 = mix64(h ^ 0xD1B54A32D192ED03ull);
    score[i] = (double)(h >> 11) * 0x1.0p-53 * 100.0;
    dept[i] = (uint32_t)((h & 0xffffffffull) % 12u);
    salary[i] = 30000 + (int64_t)((h2 >> 32) % 170001u);
    gkey[i] = (int64_t)(h2 % groups);
    pkey[i] = (int64_t)((h2 >> 7) % (2 * build));
  }
}

__global__ void tune_build_kernel(uint64_t b, int64_t* key, int64_t* payload) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < b; i += (uint64_t)gridDim.x * blockDim.x) {
    key[i] = (int64_t)i;
    payload[i] = (int64_t)(mix64(i) % 1000000u);
  }
}

struct Synth {
  uint64_t n = 0, build = 0;
  DevBuf score, dept, salary, gkey, pkey, bkey, bpay;
  DevBuf out;  // outputs of every operator (large enough for each)
};

fdb_dev_column dcol(int32_t dtype, const DevBuf& b) {
  fdb_dev_column d;
  std::memset(&d, 0, sizeof(d));
  d.dtype = dtype;
  d.values = b.ptr;
  return d;
}

// Median device time of `reps` calls of f, each bracketed by events on the
// context stream, after one untimed call.
template <class F>
double median_ms(Ctx& c, int reps, F&& f) {
  c.scratch_reset();
  f();
  std::vector<float> t;
  for (int r = 0; r < reps; ++r) {
    c.scratch_reset();
    FDB_CUDA(cudaEventRecord(c.ev0, c.stream));
    f();
    FDB_CUDA(cudaEventRecord(c.ev1, c.stream));
    FDB_CUDA(cudaEventSynchronize(c.ev1));
    float ms = 0.f;
    FDB_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    t.push_back(ms);
  }
  std::sort(t.begin(), t.end());
  const int e = c.check_device_error();
  if (e) fail(e, "an operator failed while being tuned");
  return t.empty() ? 0.0 : (double)t[t.size() / 2];
}

// One call of kind k's workload over the first n synthetic rows.
void run_kind(Ctx& c, int kind, const Synth& s, uint64_t n, HashTable* ht) {
  const fdb_dev_column score = dcol(FDB_FLOAT64, s.score), dept = dcol(FDB_UTF8, s.dept);
  const fdb_dev_column salary = dcol(FDB_INT64, s.salary), gkey = dcol(FDB_INT64, s.gkey);
  const fdb_dev_column pkey = dcol(FDB_INT64, s.pkey);
  fdb_pred_term gt{};
  gt.kind = FDB_TERM_CMP;
  gt.op = FDB_GT;
  gt.lit_type = FDB_FLOAT64;
  gt.lit_f = 50.0;
  char* out = static_cast<char*>(s.out.ptr);
  switch (kind) {
    case FDB_TUNE_SCAN: {  // COUNT(*) WHERE score > 50; SUM(score) WHERE score > 50
      op_filter_count(c, &score, 1, n, &gt, 1, reinterpret_cast<uint64_t*>(out));
      const fdb_agg_spec sum{FDB_AGG_SUM, 0};
      op_aggregate(c, &score, 1, n, &gt, 1, &sum, 1, reinterpret_cast<fdb_agg_value*>(out + 64));
      break;
    }
    case FDB_TUNE_GROUP: {  // config 0's filter -> GROUP BY dept
      const fdb_dev_column cols[3] = {dept, score, salary};
      fdb_pred_term t = gt;
      t.col = 1;
      const fdb_agg_spec aggs[3] = {{FDB_AGG_COUNT_STAR, 0}, {FDB_AGG_SUM, 1}, {FDB_AGG_AVG, 2}};
      op_group_by_codes(c, cols, 3, n, &t, 1, 0, 12, aggs, 3, reinterpret_cast<fdb_agg_value*>(out),
                        reinterpret_cast<int64_t*>(out + 4096));
      break;
    }
    case FDB_TUNE_GROUP_I64: {  // GROUP BY an INT64 key, COUNT/SUM/MIN/MAX of score
      // Every prefix's keys lie in the full column's range [0, s.n / 16).
      const uint64_t groups = s.n / 16 > 0 ? s.n / 16 : 1;
      GbSizing sz;
      sz.groups = groups;
      sz.has_range = true;
      sz.kmin = 0;
      sz.kmax = (int64_t)groups - 1;
      c.ensure_scratch(group_by_i64_scratch(sz, 0.5) + (16u << 20));
      c.scratch_reset();
      op_group_by_i64(c, gkey, score, n, nullptr, 0, nullptr, 0, sz, 0.5,
                      reinterpret_cast<fdb_group_i64*>(out + 8192), groups + 2, reinterpret_cast<uint64_t*>(out));
      break;
    }
    case FDB_TUNE_PROBE:  // INNER join COUNT(*) + SUM(payload)
      op_join_probe_agg(c, *ht, pkey, nullptr, n, FDB_JOIN_INNER, reinterpret_cast<fdb_join_agg*>(out));
      break;
    default:  // ORDER BY score DESC LIMIT 10
      op_topk(c, score, n, 10, true, false, reinterpret_cast<uint32_t*>(out + 64),
              reinterpret_cast<uint64_t*>(out));
      break;
  }
}

}  // namespace

void op_autotune(Ctx& c, uint64_t rows, int reps, fdb_op_tuning* best, double* ms_at_rows) {
  if (rows < (1u << 16)) fail(FDB_E_ARG, "autotune needs at least 65,536 rows");
  if (rows >= (1ull << 32)) fail(FDB_E_ARG, "autotune takes fewer than 2^32 rows");
  if (reps < 1) reps = 5;
  Synth s;
  s.n = rows;
  s.build = std::min<uint64_t>(1u << 20, std::max<uint64_t>(1024, rows / 100));
  const uint64_t out_bytes = 8192 + (rows / 16 + 2) * sizeof(fdb_group_i64);
  HashTable* ht = nullptr;
  auto release = [&] {
    if (ht) join_free(ht);
    ht = nullptr;
    for (DevBuf* b : {&s.score, &s.dept, &s.salary, &s.gkey, &s.pkey, &s.bkey, &s.bpay, &s.out}) c.free_buf(*b);
  };
  const TuningSet saved = c.tune;
  try {
    s.score = c.alloc_buf(rows * 8);
    s.dept = c.alloc_buf(rows * 4);
    s.salary = c.alloc_buf(rows * 8);
    s.gkey = c.alloc_buf(rows * 8);
    s.pkey = c.alloc_buf(rows * 8);
    s.bkey = c.alloc_buf(s.build * 8);
    s.bpay = c.alloc_buf(s.build * 8);
    s.out = c.alloc_buf(out_bytes);
    const unsigned grid = (unsigned)(c.sm_count * 8);
    tune_fill_kernel<<<grid, 256, 0, c.stream>>>(rows, s.build, static_cast<double*>(s.score.ptr),
                                                static_cast<uint32_t*>(s.dept.ptr), static_cast<int64_t*>(s.salary.ptr),
                                                static_cast<int64_t*>(s.gkey.ptr), static_cast<int64_t*>(s.pkey.ptr));
    FDB_CUDA(cudaGetLastError());
    tune_build_kernel<<<grid, 256, 0, c.stream>>>(s.build, static_cast<int64_t*>(s.bkey.ptr),
                                                 static_cast<int64_t*>(s.bpay.ptr));
    FDB_CUDA(cudaGetLastError());
    c.scratch_reset();
    ht = op_join_build(c, dcol(FDB_INT64, s.bkey), dcol(FDB_INT64, s.bpay), s.build, 0.5);

    const uint64_t small = std::max<uint64_t>(1u << 16, rows / 64);
    static const int kCtas[] = {0, 1, 2, 3, 4};
    static const uint64_t kRows[] = {0, 1ull << 15, 1ull << 17, 1ull << 19};
    for (int k = 0; k < FDB_TUNE_KINDS; ++k) {
      OpTuning& t = c.tune.op[k];
      // CTAs per SM at `rows`: keep the occupancy limit unless a cap is
      // faster by more than 2 %.
      t = OpTuning{};
      const double base = median_ms(c, reps, [&] { run_kind(c, k, s, rows, ht); });
      double best_ms = base;
      int best_ctas = 0;
      for (int cand : kCtas) {
        if (cand == 0) continue;
        t.ctas_per_sm = cand;
        const double ms = median_ms(c, reps, [&] { run_kind(c, k, s, rows, ht); });
        if (ms < best_ms && ms < 0.98 * base) {
          best_ms = ms;
          best_ctas = cand;
        }
      }
      t.ctas_per_sm = best_ctas;
      // Rows per CTA on a small input, the same 2 % rule.
      t.min_rows_per_cta = 0;
      const double sbase = median_ms(c, reps, [&] { run_kind(c, k, s, small, ht); });
      double sbest = sbase;
      uint64_t best_rows = 0;
      for (uint64_t cand : kRows) {
        if (cand == 0) continue;
        t.min_rows_per_cta = cand;
        const double ms = median_ms(c, reps, [&] { run_kind(c, k, s, small, ht); });
        if (ms < sbest && ms < 0.98 * sbase) {
          sbest = ms;
          best_rows = cand;
        }
      }
      t.min_rows_per_cta = best_rows;
      if (best) {
        best[k].ctas_per_sm = t.ctas_per_sm;
        best[k]._pad = 0;
        best[k].min_rows_per_cta = t.min_rows_per_cta;
      }
      if (ms_at_rows) ms_at_rows[k] = best_ms;
    }
  } catch (...) {
    c.tune = saved;
    FDB_CUDA(cudaStreamSynchronize(c.stream));
    release();
    throw;
  }
  FDB_CUDA(cudaStreamSynchronize(c.stream));
  release();
}

}  // namespace fdb
