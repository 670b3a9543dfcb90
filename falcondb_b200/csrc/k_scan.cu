// Scan kernels: WHERE mask, COUNT(*) WHERE, no-key aggregates, dictionary-code
// presence (COUNT DISTINCT), selection compaction and gather.
//
// Reference routines replaced (FalconDB, src/):
//   eval_mask_bits / fast_cmp_mask / cmp_f64_avx2 ........ query/expr.rs:635-1175
//   COUNT(*)+WHERE popcount ............................... db.rs:1439-1476
//   execute_agg_only / accumulate_typed / sum_lanes ....... query/aggregate.rs:1394-1590, 3121-3386
//   present_codes (COUNT DISTINCT over a dictionary) ...... query/aggregate.rs:3167-3200
//   gather_by_bitmask / filter_by_bitmask_cols ............ storage/column.rs:1077-1123, table.rs:148-189
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "engine.h"
#include "stream.cuh"

namespace fdb {

// ---------------------------------------------------------------------------
// Shared: predicate + column getter used by the scan ops.
// ---------------------------------------------------------------------------
struct ScanCols {
  DevCol cols[4];
};

template <class Acc>
struct RowGetter {
  const ScanCols& sc;
  const Acc& acc;
  uint32_t i;
  uint64_t row;
  __device__ __forceinline__ int operator()(int c, int64_t& iv, double& fv, uint32_t& code,
                                            bool& valid) const {
    const DevCol& col = sc.cols[c];
    const int dt = col.dtype;
    if (dt == FDB_FLOAT64)
      fv = acc.template get<double>(c, i);
    else if (dt == FDB_INT64)
      iv = acc.template get<int64_t>(c, i);
    else
      code = acc.template get<uint32_t>(c, i);
    valid = col.validity ? col_valid(col, row) : true;
    return dt;
  }
};

// ---------------------------------------------------------------------------
// No-key aggregate op (execute_agg_only).  Per-thread accumulators, a fixed
// block tree, per-CTA partials, and a last-CTA final pass in CTA order: the
// FP64 reduction order depends only on the grid, so results are repeatable.
// ---------------------------------------------------------------------------
struct AggAcc {
  double f;      // FP64 sum
  uint64_t slo;  // exact int sum, low 64 bits (two's complement, 128-bit)
  int64_t shi;   // high 64 bits
  uint64_t n;    // rows / values counted
  uint64_t m;    // MIN / MAX order key
};

__device__ __forceinline__ void i128_add(uint64_t& lo, int64_t& hi, uint64_t blo, int64_t bhi) {
  uint64_t r = lo + blo;
  hi = hi + bhi + (r < lo ? 1 : 0);
  lo = r;
}

__device__ __forceinline__ void agg_combine(AggAcc& a, const AggAcc& b, int func) {
  a.f += b.f;
  i128_add(a.slo, a.shi, b.slo, b.shi);
  a.n += b.n;
  if (func == FDB_AGG_MIN) a.m = b.m < a.m ? b.m : a.m;
  if (func == FDB_AGG_MAX) a.m = b.m > a.m ? b.m : a.m;
}

__device__ __forceinline__ AggAcc agg_identity(int func) {
  AggAcc a;
  a.f = 0.0;
  a.slo = 0;
  a.shi = 0;
  a.n = 0;
  a.m = func == FDB_AGG_MIN ? ~0ull : 0ull;
  return a;
}

__device__ __forceinline__ AggAcc warp_agg(AggAcc a, int func) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    AggAcc b;
    b.f = __shfl_xor_sync(0xffffffffu, a.f, o);
    b.slo = __shfl_xor_sync(0xffffffffu, a.slo, o);
    b.shi = __shfl_xor_sync(0xffffffffu, a.shi, o);
    b.n = __shfl_xor_sync(0xffffffffu, a.n, o);
    b.m = __shfl_xor_sync(0xffffffffu, a.m, o);
    agg_combine(a, b, func);
  }
  return a;
}

__device__ double i128_to_f64(uint64_t lo, int64_t hi) {
  if ((hi == 0 && (int64_t)lo >= 0) || (hi == -1 && (int64_t)lo < 0)) return (double)(int64_t)lo;
  return (double)hi * 18446744073709551616.0 + (double)lo;
}

struct ScanAggParams {
  PredProg prog;
  ScanCols sc;
  int32_t naggs;
  int32_t func[4];
  int32_t acol[4];
  // FilterAggOp's decoded WHERE: one compare of column f_cmp_col (-1: none)
  // against a literal, as double (f_cmp_f64) or as int64; f_cmp_mask holds
  // the accepted outcomes (bit 0 unordered, 1 less, 2 equal, 3 greater).
  int32_t f_cmp_col;
  uint32_t f_cmp_mask;
  int32_t f_cmp_f64;
  uint32_t f_agg_f64;     // bit a: aggregate a's column is FLOAT64
  double f_lit_f;
  int64_t f_lit_i;
  AggAcc* partials;       // [gridDim.x * 4]
  unsigned int* ticket;   // zero on entry; reset by the last CTA
  fdb_agg_value* out;     // [naggs] or nullptr
  uint64_t* out_count;    // receives agg 0's count (COUNT(*) WHERE) or nullptr
};

struct ScanAggOp {
  using Params = ScanAggParams;
  struct Local {
    AggAcc a[4];
  };
  static constexpr int kSmem = 32 * 4 * sizeof(AggAcc) + 16;

  static __device__ void init(Local& st, const Params& p, unsigned char*, int, int) {
#pragma unroll
    for (int a = 0; a < 4; ++a) st.a[a] = agg_identity(a < p.naggs ? p.func[a] : FDB_AGG_COUNT);
  }

  template <class Acc>
  static __device__ __forceinline__ void one_row(Local& st, const Params& p, const Acc& acc,
                                                 uint32_t i) {
    const uint64_t row = acc.row(i);
    RowGetter<Acc> get{p.sc, acc, i, row};
    if (!eval_prog(p.prog, get)) return;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (a >= p.naggs) break;
      const int f = p.func[a];
      if (f == FDB_AGG_COUNT_STAR) {
        st.a[a].n++;
        continue;
      }
      int64_t iv = 0;
      double fv = 0.0;
      uint32_t code = 0;
      bool valid = true;
      const int dt = get(p.acol[a], iv, fv, code, valid);
      if (!valid) continue;
      if (f == FDB_AGG_COUNT) {
        st.a[a].n++;
      } else if (f == FDB_AGG_SUM || f == FDB_AGG_AVG) {
        if (dt == FDB_FLOAT64)
          st.a[a].f += fv;
        else
          i128_add(st.a[a].slo, st.a[a].shi, (uint64_t)iv, iv < 0 ? -1 : 0);
        st.a[a].n++;
      } else if (f == FDB_AGG_MIN || f == FDB_AGG_MAX) {
        uint64_t k;
        if (dt == FDB_FLOAT64) {
          if (isnan(fv)) continue;  // f64::min / f64::max skip NaN
          k = f64_ord_key(fv);
        } else {
          k = i64_ord_key(iv);
        }
        if (f == FDB_AGG_MIN)
          st.a[a].m = k < st.a[a].m ? k : st.a[a].m;
        else
          st.a[a].m = k > st.a[a].m ? k : st.a[a].m;
        st.a[a].n++;
      }
    }
  }

  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char*, const Acc& acc,
                              uint32_t rows, int ctid, int nct) {
    for (uint32_t i = ctid; i < rows; i += nct) one_row(st, p, acc, i);
  }

  // Block-reduce `st` into op_smem slot 0 (returned by thread 0).
  static __device__ void block_reduce(Local& st, const Params& p, AggAcc* sm, int ctid, int nct) {
    const int warp = ctid >> 5, lane = ctid & 31, nw = nct >> 5;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (a >= p.naggs) break;
      AggAcc w = warp_agg(st.a[a], p.func[a]);
      if (lane == 0) sm[warp * 4 + a] = w;
    }
    consumer_bar(nct);
    if (ctid == 0) {
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (a >= p.naggs) break;
        AggAcc t = sm[a];
        for (int w = 1; w < nw; ++w) agg_combine(t, sm[w * 4 + a], p.func[a]);
        st.a[a] = t;
      }
    }
  }

  static __device__ void finish(Local& st, const Params& p, unsigned char* op_smem, int ctid,
                                int nct) {
    AggAcc* sm = reinterpret_cast<AggAcc*>(op_smem);
    unsigned int* s_last = reinterpret_cast<unsigned int*>(op_smem + 32 * 4 * sizeof(AggAcc));
    block_reduce(st, p, sm, ctid, nct);
    if (ctid == 0) {
#pragma unroll
      for (int a = 0; a < 4; ++a)
        if (a < p.naggs) p.partials[blockIdx.x * 4 + a] = st.a[a];
      __threadfence();
      unsigned int t = atomicAdd(p.ticket, 1u);
      *s_last = (t == gridDim.x - 1) ? 1u : 0u;
    }
    consumer_bar(nct);
    if (*s_last == 0) return;
    __threadfence();
    // Last CTA: combine the per-CTA partials in CTA order.
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (a >= p.naggs) break;
      AggAcc t = agg_identity(p.func[a]);
      for (int b = ctid; b < (int)gridDim.x; b += nct) {
        const AggAcc* src = p.partials + b * 4 + a;
        AggAcc v;
        v.f = __ldcg(&src->f);
        v.slo = __ldcg(&src->slo);
        v.shi = __ldcg(&src->shi);
        v.n = __ldcg(&src->n);
        v.m = __ldcg(&src->m);
        agg_combine(t, v, p.func[a]);
      }
      st.a[a] = t;
    }
    consumer_bar(nct);
    block_reduce(st, p, sm, ctid, nct);
    if (ctid == 0) {
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (a >= p.naggs) break;
        const AggAcc& t = st.a[a];
        const int f = p.func[a];
        const int dt = f == FDB_AGG_COUNT_STAR ? FDB_INT64 : p.sc.cols[p.acol[a]].dtype;
        fdb_agg_value v;
        v.f = 0.0;
        v.i = 0;
        v.n = (int64_t)t.n;
        v.is_int = 0;
        v.valid = t.n > 0;
        if (f == FDB_AGG_COUNT_STAR || f == FDB_AGG_COUNT) {
          v.is_int = 1;
          v.i = (int64_t)t.n;
          v.valid = 1;
        } else if (f == FDB_AGG_SUM || f == FDB_AGG_AVG) {
          double s = dt == FDB_FLOAT64 ? t.f : i128_to_f64(t.slo, t.shi);
          v.f = (f == FDB_AGG_AVG && t.n > 0) ? s / (double)t.n : s;
        } else if (f == FDB_AGG_MIN || f == FDB_AGG_MAX) {
          if (t.n > 0)
            v.f = dt == FDB_FLOAT64 ? f64_from_ord_key(t.m) : (double)(int64_t)(t.m ^ (1ull << 63));
        }
        if (p.out) p.out[a] = v;
        if (a == 0 && p.out_count) *p.out_count = t.n;
      }
      *p.ticket = 0u;
    }
  }
};

// ---------------------------------------------------------------------------
// Specialised scans for the two shapes that dominate analytical scans: an
// aggregate over one NULL-free column with no WHERE (SUM(score)), and COUNT(*)
// WHERE `col op literal` over one NULL-free column (the popcount fast path of
// db.rs:1439-1476).  Same partials / final pass as ScanAggOp; the comparison
// and the value type are template parameters so nothing is decided per row.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void fold_value(AggAcc& a, int f, T v) {
  if (f == FDB_AGG_SUM || f == FDB_AGG_AVG) {
    if constexpr (sizeof(T) == 8 && T(0.5) != T(0))
      a.f += v;
    else
      i128_add(a.slo, a.shi, (uint64_t)v, v < 0 ? -1 : 0);
  } else if (f == FDB_AGG_MIN || f == FDB_AGG_MAX) {
    uint64_t k;
    if constexpr (T(0.5) != T(0)) {
      if (isnan(v)) return;
      k = f64_ord_key(v);
    } else {
      k = i64_ord_key(v);
    }
    if (f == FDB_AGG_MIN)
      a.m = k < a.m ? k : a.m;
    else
      a.m = k > a.m ? k : a.m;
  }
  a.n++;
}

// Aggregates with at most one `col op literal` WHERE, every column NULL-free
// and numeric (SELECT SUM(score), AVG(salary) ... WHERE score > 50).  A thread
// takes its rows of the tile four at a time (ctid, ctid + nct, ...): it
// compares them into a 4-bit mask, branch-free, and then each aggregate folds
// the four rows under the mask with selects, not branches, so the aggregate
// function and the column type are decided once per four rows (a uniform
// branch), not per row as ScanAggOp's interpreter does.  Groups of four rows
// that lie wholly inside the tile (all but at most one per tile) load without
// bounds checks.
//
// While rows are folded, two accumulators hold other forms than ScanAggOp's,
// which finish() converts back before the shared partials / final pass:
//   * an INT64 SUM / AVG keeps the sum of the values' low 32-bit halves
//     (unsigned) in slo and of their high halves (signed) in shi, so that
//     the value is shi * 2^32 + slo; exact while a thread folds fewer than
//     2^32 rows (the host only takes this path below 2^40 rows);
//   * a FLOAT64 MIN / MAX keeps the running value in f (+inf / -inf before the
//     first row) and compares doubles: NaN compares false and never takes
//     part (f64::min / max), and on equal values the sign bits are combined
//     so that +0.0 wins a MAX and -0.0 a MIN, as their order keys do.
// FilterAggOp's launch shape: 2048-row tiles, two stages, and registers held
// to three resident CTAs per SM (72, no spills).  On COUNT, SUM(score),
// AVG(salary), MAX(score) WHERE score > 50 over 100M rows this took the query
// from 0.443 ms (1024-row tiles, four stages, two CTAs per SM) to 0.362 ms;
// 2048 x 3 stages: 0.386; 1024 x 3 stages at 3 CTAs: 0.390.
#ifndef FDB_FA_TR
#define FDB_FA_TR 2048
#endif
#ifndef FDB_FA_STAGES
#define FDB_FA_STAGES 2
#endif
#ifndef FDB_FA_MINB
#define FDB_FA_MINB 3
#endif
struct FilterAggOp : ScanAggOp {
  static constexpr int R = 4;

  static __device__ bool f64_minmax(const Params& p, int a) {
    return ((p.f_agg_f64 >> a) & 1u) && (p.func[a] == FDB_AGG_MIN || p.func[a] == FDB_AGG_MAX);
  }
  static __device__ bool i64_sum(const Params& p, int a) {
    return !((p.f_agg_f64 >> a) & 1u) && (p.func[a] == FDB_AGG_SUM || p.func[a] == FDB_AGG_AVG);
  }

  static __device__ void init(Local& st, const Params& p, unsigned char* sm, int ctid, int nct) {
    ScanAggOp::init(st, p, sm, ctid, nct);
    const double inf = __longlong_as_double(0x7FF0000000000000ll);
#pragma unroll
    for (int a = 0; a < 4; ++a)
      if (a < p.naggs && f64_minmax(p, a)) st.a[a].f = p.func[a] == FDB_AGG_MIN ? inf : -inf;
  }

  template <bool kFull, typename T, class Acc>
  static __device__ __forceinline__ void load_r(T (&x)[R], const Acc& acc, int col, const uint32_t (&i)[R],
                                                uint32_t ok) {
#pragma unroll
    for (int j = 0; j < R; ++j)
      x[j] = (kFull || ((ok >> j) & 1u)) ? acc.template get<T>(col, i[j]) : T(0);
  }

  template <bool kFull, class Acc>
  static __device__ __forceinline__ uint32_t pass_mask(const Params& p, const Acc& acc, const uint32_t (&i)[R],
                                                       uint32_t ok) {
    const int pc = p.f_cmp_col;
    if (pc < 0) return ok;
    const uint32_t amask = p.f_cmp_mask;
    const bool a_un = amask & 1u, a_lt = (amask >> 1) & 1u, a_eq = (amask >> 2) & 1u, a_gt = (amask >> 3) & 1u;
    uint32_t m = 0;
    if (p.f_cmp_f64) {
      const double lit = p.f_lit_f;
      const bool lit_nan = lit != lit;  // every outcome is then unordered
      double x[R];
      if (p.sc.cols[pc].dtype == FDB_FLOAT64) {
        load_r<kFull, double>(x, acc, pc, i, ok);
      } else {
        int64_t y[R];
        load_r<kFull, int64_t>(y, acc, pc, i, ok);
#pragma unroll
        for (int j = 0; j < R; ++j) x[j] = (double)y[j];
      }
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const bool pass = (a_lt && x[j] < lit) || (a_eq && x[j] == lit) || (a_gt && x[j] > lit) ||
                          (a_un && (lit_nan || x[j] != x[j]));
        m |= (pass ? 1u : 0u) << j;
      }
    } else {
      const int64_t lit = p.f_lit_i;
      int64_t x[R];
      load_r<kFull, int64_t>(x, acc, pc, i, ok);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const bool pass = (a_lt && x[j] < lit) || (a_eq && x[j] == lit) || (a_gt && x[j] > lit);
        m |= (pass ? 1u : 0u) << j;
      }
    }
    return kFull ? m : m & ok;
  }

  template <bool kFull, typename T, class Acc>
  static __device__ __forceinline__ void fold_r(AggAcc& a, int f, const Acc& acc, int col, const uint32_t (&i)[R],
                                                uint32_t ok, uint32_t m) {
    T x[R];
    load_r<kFull, T>(x, acc, col, i, ok);
    if (f == FDB_AGG_SUM || f == FDB_AGG_AVG) {
      if constexpr (T(0.5) != T(0)) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < R; ++j) s += ((m >> j) & 1u) ? x[j] : 0.0;
        a.f += s;
      } else {
        uint64_t lo = 0;
        int64_t hi = 0;
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const int64_t v = ((m >> j) & 1u) ? x[j] : 0;
          lo += (uint32_t)v;
          hi += (int32_t)(v >> 32);
        }
        a.slo += lo;
        a.shi += hi;
      }
      a.n += (uint64_t)__popc(m);
      return;
    }
    if constexpr (T(0.5) != T(0)) {
      const bool is_max = f == FDB_AGG_MAX;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const bool in = (m >> j) & 1u;
        const double v = x[j];
        if (in && (is_max ? v > a.f : v < a.f)) {
          a.f = v;
        } else if (in && v == a.f) {
          const uint64_t fb = (uint64_t)__double_as_longlong(a.f), vb = (uint64_t)__double_as_longlong(v);
          a.f = __longlong_as_double((long long)(is_max ? (fb & vb) : (fb | vb)));
        }
        a.n += (in && v == v) ? 1u : 0u;
      }
    } else {
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const bool in = (m >> j) & 1u;
        const uint64_t k = i64_ord_key(x[j]);
        if (f == FDB_AGG_MIN)
          a.m = (in && k < a.m) ? k : a.m;
        else
          a.m = (in && k > a.m) ? k : a.m;
        a.n += in ? 1u : 0u;
      }
    }
  }

  template <bool kFull, class Acc>
  static __device__ __forceinline__ void group(Local& st, const Params& p, const Acc& acc, uint32_t b,
                                               uint32_t rows, int ctid, int nct) {
    uint32_t i[R];
    uint32_t ok = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      i[j] = b + (uint32_t)j * (uint32_t)nct + (uint32_t)ctid;
      ok |= (kFull || i[j] < rows ? 1u : 0u) << j;
    }
    const uint32_t m = pass_mask<kFull>(p, acc, i, ok);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (a >= p.naggs) break;
      const int f = p.func[a];
      if (f == FDB_AGG_COUNT_STAR || f == FDB_AGG_COUNT)
        st.a[a].n += (uint64_t)__popc(m);
      else if ((p.f_agg_f64 >> a) & 1u)
        fold_r<kFull, double>(st.a[a], f, acc, p.acol[a], i, ok, m);
      else
        fold_r<kFull, int64_t>(st.a[a], f, acc, p.acol[a], i, ok, m);
    }
  }

  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char*, const Acc& acc, uint32_t rows, int ctid,
                              int nct) {
    const uint32_t g = R * (uint32_t)nct;
    uint32_t b = 0;
    for (; b + g <= rows; b += g) group<true>(st, p, acc, b, rows, ctid, nct);
    if (b < rows) group<false>(st, p, acc, b, rows, ctid, nct);
  }

  // Back to ScanAggOp's accumulator forms, then its reduction and final pass.
  static __device__ void finish(Local& st, const Params& p, unsigned char* op_smem, int ctid, int nct) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (a >= p.naggs) break;
      AggAcc& x = st.a[a];
      if (i64_sum(p, a)) {
        // shi * 2^32 + slo as a 128-bit integer.
        uint64_t lo = (uint64_t)x.shi << 32;
        int64_t hi = x.shi >> 32;
        i128_add(lo, hi, x.slo, 0);
        x.slo = lo;
        x.shi = hi;
      } else if (f64_minmax(p, a)) {
        x.m = x.n ? f64_ord_key(x.f) : agg_identity(p.func[a]).m;
        x.f = 0.0;
      }
    }
    ScanAggOp::finish(st, p, op_smem, ctid, nct);
  }
};

// Aggregates over column 0 only, no predicate, no NULLs.
template <typename T>
struct ColAggOp : ScanAggOp {
  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char*, const Acc& acc,
                              uint32_t rows, int ctid, int nct) {
    if constexpr (Acc::kSmemTile && T(0.5) != T(0)) {
      // SUM alone over a FLOAT64 tile: two rows per 16-byte load, two chains.
      if (p.naggs == 1 && p.func[0] == FDB_AGG_SUM && (rows & 1u) == 0) {
        const double2* v = reinterpret_cast<const double2*>(acc.template col_ptr<double>(0));
        double s0 = 0.0, s1 = 0.0;
        for (uint32_t i = ctid; i < (rows >> 1); i += nct) {
          const double2 x = v[i];
          s0 += x.x;
          s1 += x.y;
        }
        st.a[0].f += s0 + s1;
        st.a[0].n += rows / nct + ((uint32_t)ctid < rows % nct ? 1 : 0);
        return;
      }
    }
    uint32_t i = ctid;
    for (; i + nct < rows; i += 2 * nct) {
      const T v0 = acc.template get<T>(0, i);
      const T v1 = acc.template get<T>(0, i + nct);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (a >= p.naggs) break;
        fold_value<T>(st.a[a], p.func[a], v0);
        fold_value<T>(st.a[a], p.func[a], v1);
      }
    }
    for (; i < rows; i += nct) {
      const T v = acc.template get<T>(0, i);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (a >= p.naggs) break;
        fold_value<T>(st.a[a], p.func[a], v);
      }
    }
  }
};

template <int OP, typename T>
__device__ __forceinline__ bool cmp_fixed(T a, T b) {
  if constexpr (OP == FDB_EQ) return a == b;
  else if constexpr (OP == FDB_NE) return a != b;
  else if constexpr (OP == FDB_LT) return a < b;
  else if constexpr (OP == FDB_LE) return a <= b;
  else if constexpr (OP == FDB_GT) return a > b;
  else return a >= b;
}

// COUNT(*) WHERE col OP literal; T is the comparison type (double for a
// FLOAT64 column or a widened INT64 one), S the stored type.
template <typename S, typename T, int OP>
struct CmpCountOp : ScanAggOp {
  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char*, const Acc& acc,
                              uint32_t rows, int ctid, int nct) {
    const T lit = sizeof(T) == 8 && T(0.5) != T(0)
                      ? (T)(p.prog.t[0].lit_type == FDB_FLOAT64 ? p.prog.t[0].lit_f : (double)p.prog.t[0].lit_i)
                      : (T)p.prog.t[0].lit_i;
    uint32_t cnt = 0;
    uint32_t i = ctid;
    for (; i + 3 * nct < rows; i += 4 * nct) {
      cnt += cmp_fixed<OP, T>((T)acc.template get<S>(0, i), lit);
      cnt += cmp_fixed<OP, T>((T)acc.template get<S>(0, i + nct), lit);
      cnt += cmp_fixed<OP, T>((T)acc.template get<S>(0, i + 2 * nct), lit);
      cnt += cmp_fixed<OP, T>((T)acc.template get<S>(0, i + 3 * nct), lit);
    }
    for (; i < rows; i += nct) cnt += cmp_fixed<OP, T>((T)acc.template get<S>(0, i), lit);
    st.a[0].n += cnt;
  }
};

// ---------------------------------------------------------------------------
// Dictionary-code presence (COUNT DISTINCT over a Utf8 column).
// ---------------------------------------------------------------------------
struct DistinctParams {
  PredProg prog;
  ScanCols sc;
  int32_t code_col;
  uint32_t dict_len;
  uint64_t* bitmap;  // global, zeroed before launch
};

struct DistinctOp {
  using Params = DistinctParams;
  struct Local {
    uint64_t bits;   // dict_len <= 64: codes seen by this thread
  };
  static constexpr int kSmemMaxCodes = 32768;
  static constexpr int kSmem = kSmemMaxCodes / 8;

  static __device__ void init(Local& st, const Params& p, unsigned char* sm, int ctid, int nct) {
    st.bits = 0;
    if (p.dict_len > 64 && p.dict_len <= kSmemMaxCodes) {
      uint32_t* w = reinterpret_cast<uint32_t*>(sm);
      for (int i = ctid; i < kSmemMaxCodes / 32; i += nct) w[i] = 0;
    }
  }
  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char* sm, const Acc& acc,
                              uint32_t rows, int ctid, int nct) {
    if constexpr (Acc::kSmemTile) {
      // Fast path: one code column, no WHERE, no NULLs, <= 64 codes: four
      // codes per 16-byte shared-memory load into a register bitmask.
      if (p.prog.n == 0 && p.dict_len <= 64 && p.sc.cols[p.code_col].validity == nullptr && (rows & 3u) == 0) {
        const uint4* v = reinterpret_cast<const uint4*>(acc.template col_ptr<uint32_t>(p.code_col));
        uint64_t bits = 0;
        const uint32_t dl = p.dict_len;
        for (uint32_t i = ctid; i < (rows >> 2); i += nct) {
          const uint4 c = v[i];
          bits |= (c.x < dl ? 1ull << c.x : 0ull) | (c.y < dl ? 1ull << c.y : 0ull) |
                  (c.z < dl ? 1ull << c.z : 0ull) | (c.w < dl ? 1ull << c.w : 0ull);
        }
        st.bits |= bits;
        return;
      }
    }
    const bool small = p.dict_len <= 64;
    const bool in_smem = !small && p.dict_len <= kSmemMaxCodes;
    uint32_t* w = reinterpret_cast<uint32_t*>(sm);
    for (uint32_t i = ctid; i < rows; i += nct) {
      const uint64_t row = acc.row(i);
      if (p.prog.n) {
        RowGetter<Acc> get{p.sc, acc, i, row};
        if (!eval_prog(p.prog, get)) continue;
      }
      const uint32_t code = acc.template get<uint32_t>(p.code_col, i);
      if (code == kNullCode || code >= p.dict_len) continue;
      const DevCol& c = p.sc.cols[p.code_col];
      if (c.validity && !col_valid(c, row)) continue;
      if (small) {
        st.bits |= 1ull << code;
      } else if (in_smem) {
        const uint32_t m = 1u << (code & 31);
        if (!(w[code >> 5] & m)) atomicOr(&w[code >> 5], m);
      } else {
        const unsigned long long m = 1ull << (code & 63);
        if (!(p.bitmap[code >> 6] & m)) atomicOr((unsigned long long*)&p.bitmap[code >> 6], m);
      }
    }
  }
  static __device__ void finish(Local& st, const Params& p, unsigned char* sm, int ctid, int nct) {
    if (p.dict_len <= 64) {
      uint64_t b = st.bits;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) b |= __shfl_xor_sync(0xffffffffu, b, o);
      if ((ctid & 31) == 0 && b) atomicOr((unsigned long long*)&p.bitmap[0], (unsigned long long)b);
      return;
    }
    if (p.dict_len <= kSmemMaxCodes) {
      consumer_bar(nct);
      const uint32_t* w = reinterpret_cast<const uint32_t*>(sm);
      const uint32_t nw = (p.dict_len + 31) / 32;
      for (uint32_t i = ctid; i < nw; i += nct)
        if (w[i]) atomicOr((unsigned int*)p.bitmap + i, w[i]);  // little-endian u64 halves
    }
  }
};

// ---------------------------------------------------------------------------
// Launch helpers for the streamer.
// ---------------------------------------------------------------------------
// Tile rows per column and ring depth: ~64 KB of staging per CTA so that three
// CTAs (24 consumer warps) fit on one SM.
template <int NC>
struct TileShape {
  static constexpr int TR = NC == 1 ? 2048 : 1024;
  static constexpr int STAGES = NC <= 2 ? 4 : 3;
  static constexpr int NCW = 8;
};
template <int NC, int TRo, int STo = 0>
struct TileShapeO {
  static constexpr int TR = TRo ? TRo : TileShape<NC>::TR;
  static constexpr int STAGES = STo ? STo : TileShape<NC>::STAGES;
  static constexpr int NCW = TileShape<NC>::NCW;
};

// TRo / CBo / STo override the tile rows, the bytes reserved per row per
// column (a scan of one 4-byte column uses 4096-row, 16 KB tiles) and the
// stages; MINB is the kernel's minimum of resident CTAs per SM (0: none).
template <class Op, int NC, int TRo = 0, int CBo = 8, int STo = 0, int MINB = 1>
static void launch_stream(Ctx& c, const fdb_dev_column* cols, uint64_t n, const typename Op::Params& p,
                          size_t op_smem_bytes) {
  using S = TileShapeO<NC, TRo, STo>;
  StreamSrc<NC> src;
  const void* bases[NC];
  for (int i = 0; i < NC; ++i) {
    src.base[i] = static_cast<const unsigned char*>(cols[i].values);
    src.esize[i] = dtype_size(cols[i].dtype);
    if (src.esize[i] > CBo) fail(FDB_E_ARG, "column wider than the tile layout");
    bases[i] = cols[i].values;
  }
  src.n = n;
  src.m_end = stream_m_end(bases, NC, n);
  const int op_off = (int)stream_smem_bytes<NC, S::TR, S::STAGES, CBo>();
  const size_t smem = op_off + op_smem_bytes;
  auto kern = stream_kernel<Op, NC, S::TR, S::STAGES, S::NCW, CBo, MINB>;
  static PerDeviceOnce attr_done;  // per instantiation and device
  attr_done(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)); });
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (S::NCW + 1) * 32, smem));
  const uint64_t ntiles = (src.m_end + S::TR - 1) / S::TR;
  const uint64_t want = ntiles ? ntiles : (n + S::NCW * 32 * 8 - 1) / (S::NCW * 32 * 8);
  // At most 4 CTAs per SM: the per-CTA partials are sized for that.
  const int grid = tuned_grid(c.tune.op[FDB_TUNE_SCAN], c.sm_count, per_sm, 4, want, n);
  kern<<<grid, (S::NCW + 1) * 32, smem, c.stream>>>(src, p, c.d_err, op_off);
  FDB_CUDA(cudaGetLastError());
}

template <class Op, int TRo = 0, int STo = 0, int MINB = 1>
static void launch_stream_nc(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                             const typename Op::Params& p, size_t op_smem) {
  switch (ncols) {
    case 1: launch_stream<Op, 1, TRo, 8, STo, MINB>(c, cols, n, p, op_smem); break;
    case 2: launch_stream<Op, 2, TRo, 8, STo, MINB>(c, cols, n, p, op_smem); break;
    case 3: launch_stream<Op, 3, TRo, 8, STo, MINB>(c, cols, n, p, op_smem); break;
    case 4: launch_stream<Op, 4, TRo, 8, STo, MINB>(c, cols, n, p, op_smem); break;
    default: fail(FDB_E_ARG, "between 1 and 4 input columns are supported per scan");
  }
}

// Grid upper bound used to size per-CTA partials.
static int max_stream_grid(Ctx& c) { return c.sm_count * 4; }

static void fill_prog(PredProg& pp, const fdb_pred_term* prog, int nterms, int ncols) {
  if (nterms < 0 || nterms > FDB_MAX_TERMS) fail(FDB_E_ARG, "predicate has too many terms");
  std::memset(&pp, 0, sizeof(pp));
  pp.n = nterms;
  int depth = 0;
  for (int i = 0; i < nterms; ++i) {
    pp.t[i] = prog[i];
    const int k = prog[i].kind;
    if (k == FDB_TERM_AND || k == FDB_TERM_OR) {
      if (depth < 2) fail(FDB_E_ARG, "malformed predicate program (AND/OR needs two operands)");
      depth -= 1;
    } else if (k == FDB_TERM_CMP || k == FDB_TERM_IS_NULL || k == FDB_TERM_IS_NOT_NULL ||
               k == FDB_TERM_CODE_SET) {
      if (prog[i].col < 0 || prog[i].col >= ncols) fail(FDB_E_ARG, "predicate column out of range");
      if (k == FDB_TERM_CMP && (prog[i].op < FDB_EQ || prog[i].op > FDB_GE))
        fail(FDB_E_ARG, "bad comparison operator");
      if (k == FDB_TERM_CODE_SET && prog[i].code_set == nullptr)
        fail(FDB_E_ARG, "CODE_SET term without a code set");
      depth += 1;
    } else {
      fail(FDB_E_ARG, "unknown predicate term kind");
    }
  }
  if (nterms > 0 && depth != 1) fail(FDB_E_ARG, "malformed predicate program");
}

static void fill_cols(ScanCols& sc, const fdb_dev_column* cols, int ncols, uint64_t n) {
  if (ncols < 1 || ncols > 4) fail(FDB_E_ARG, "between 1 and 4 input columns are supported per scan");
  std::memset(&sc, 0, sizeof(sc));
  for (int i = 0; i < ncols; ++i) {
    if (cols[i].values == nullptr && n > 0) fail(FDB_E_ARG, "column without values");
    if (cols[i].dtype != FDB_INT64 && cols[i].dtype != FDB_FLOAT64 && cols[i].dtype != FDB_UTF8)
      fail(FDB_E_TYPE, "unsupported column type");
    sc.cols[i] = DevCol{cols[i].dtype, cols[i].values, cols[i].validity, cols[i].validity_offset};
  }
}

void op_aggregate(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                  const fdb_pred_term* prog, int nterms, const fdb_agg_spec* aggs, int naggs,
                  fdb_agg_value* d_out) {
  if (naggs < 1 || naggs > 4) fail(FDB_E_ARG, "between 1 and 4 aggregates per scan");
  ScanAggParams p;
  std::memset(&p, 0, sizeof(p));
  fill_cols(p.sc, cols, ncols, n);
  fill_prog(p.prog, prog, nterms, ncols);
  p.naggs = naggs;
  for (int a = 0; a < naggs; ++a) {
    const int f = aggs[a].func;
    if (f < FDB_AGG_COUNT_STAR || f > FDB_AGG_MAX)
      fail(FDB_E_ARG, "aggregate not supported by fdb_aggregate (COUNT DISTINCT: fdb_distinct_codes)");
    if (f != FDB_AGG_COUNT_STAR) {
      if (aggs[a].col < 0 || aggs[a].col >= ncols) fail(FDB_E_ARG, "aggregate column out of range");
      if (f != FDB_AGG_COUNT && cols[aggs[a].col].dtype == FDB_UTF8)
        fail(FDB_E_TYPE, "SUM/AVG/MIN/MAX need a numeric column");
    }
    p.func[a] = f;
    p.acol[a] = aggs[a].col;
  }
  p.partials = static_cast<AggAcc*>(c.scratch_take(sizeof(AggAcc) * 4 * max_stream_grid(c)));
  p.ticket = c.d_ticket;
  p.out = d_out;
  p.out_count = nullptr;
  // One NULL-free numeric column, no WHERE, every aggregate over it.
  bool single = ncols == 1 && nterms == 0 && cols[0].validity == nullptr && cols[0].dtype != FDB_UTF8;
  for (int a = 0; a < naggs && single; ++a)
    single = aggs[a].func == FDB_AGG_COUNT_STAR || aggs[a].col == 0;
  if (single) {
    if (cols[0].dtype == FDB_FLOAT64)
      launch_stream<ColAggOp<double>, 1>(c, cols, n, p, ScanAggOp::kSmem);
    else
      launch_stream<ColAggOp<int64_t>, 1>(c, cols, n, p, ScanAggOp::kSmem);
    return;
  }
  // At most one `col op literal` and NULL-free numeric columns: FilterAggOp
  // (whose split INT64 sums are exact below 2^32 rows per thread).
  bool fast = (nterms == 0 || (nterms == 1 && prog[0].kind == FDB_TERM_CMP)) && n < (1ull << 40);
  for (int i = 0; i < ncols && fast; ++i) fast = cols[i].validity == nullptr && cols[i].dtype != FDB_UTF8;
  if (fast) {
    p.f_cmp_col = -1;
    if (nterms == 1) {
      const fdb_pred_term& t = prog[0];
      p.f_cmp_col = t.col;
      // Accepted outcomes of x op lit (bit 0 unordered, 1 less, 2 equal, 3
      // greater): NaN passes != only, as cmp_op does.
      static const uint32_t kAccept[6] = {0x4u, 0xBu, 0x2u, 0x6u, 0x8u, 0xCu};
      p.f_cmp_mask = kAccept[t.op];
      p.f_cmp_f64 = cols[t.col].dtype == FDB_FLOAT64 || t.lit_type == FDB_FLOAT64;
      p.f_lit_f = t.lit_type == FDB_FLOAT64 ? t.lit_f : (double)t.lit_i;
      p.f_lit_i = t.lit_i;
    }
    for (int a = 0; a < naggs; ++a)
      if (aggs[a].func != FDB_AGG_COUNT_STAR && cols[aggs[a].col].dtype == FDB_FLOAT64) p.f_agg_f64 |= 1u << a;
    launch_stream_nc<FilterAggOp, FDB_FA_TR, FDB_FA_STAGES, FDB_FA_MINB>(c, cols, ncols, n, p, ScanAggOp::kSmem);
    return;
  }
  launch_stream_nc<ScanAggOp>(c, cols, ncols, n, p, ScanAggOp::kSmem);
}

// ---------------------------------------------------------------------------
// Aggregate scan that allocates nothing: its per-CTA partials and its ticket
// live in a fixed module-scope device array instead of the context's scratch
// arena (which may grow, i.e. allocate, on any call).  The array's device
// address is looked up once per device with cudaGetSymbolAddress, by the first
// call made on that device.  All calls on one device share the array, so two
// calls whose kernels overlap in time race on it.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = 128 * 1024;  // ticket (256 B) + partials
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[kNoAllocMaxDevices];

// Device address of g_noalloc_scratch on the current device (c.device).
static unsigned char* noalloc_scratch(Ctx& c) {
  if (c.device < 0 || c.device >= kNoAllocMaxDevices) fail(FDB_E_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (g_noalloc_ptr[c.device] == nullptr) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr)
      fail(FDB_E_CUDA, std::string("cudaGetSymbolAddress of the fixed aggregate scratch failed: ") +
                           cudaGetErrorString(e));
    g_noalloc_ptr[c.device] = ptr;
  }
  return static_cast<unsigned char*>(g_noalloc_ptr[c.device]);
}

void op_aggregate_noalloc(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                          const fdb_pred_term* prog, int nterms, const fdb_agg_spec* aggs, int naggs,
                          fdb_agg_value* d_out) {
  if (naggs < 1 || naggs > 4) fail(FDB_E_ARG, "between 1 and 4 aggregates per scan");
  const size_t need = 256 + sizeof(AggAcc) * 4 * (size_t)max_stream_grid(c);
  if (need > kNoAllocScratchBytes)
    fail(FDB_E_CAPACITY, "fdb_aggregate_noalloc: this device needs " + std::to_string(need) +
                             " bytes of partials, above the fixed " + std::to_string(kNoAllocScratchBytes));
  ScanAggParams p;
  std::memset(&p, 0, sizeof(p));
  fill_cols(p.sc, cols, ncols, n);
  fill_prog(p.prog, prog, nterms, ncols);
  p.naggs = naggs;
  for (int a = 0; a < naggs; ++a) {
    const int f = aggs[a].func;
    if (f < FDB_AGG_COUNT_STAR || f > FDB_AGG_MAX)
      fail(FDB_E_ARG, "aggregate not supported by fdb_aggregate_noalloc");
    if (f != FDB_AGG_COUNT_STAR) {
      if (aggs[a].col < 0 || aggs[a].col >= ncols) fail(FDB_E_ARG, "aggregate column out of range");
      if (f != FDB_AGG_COUNT && cols[aggs[a].col].dtype == FDB_UTF8)
        fail(FDB_E_TYPE, "SUM/AVG/MIN/MAX need a numeric column");
    }
    p.func[a] = f;
    p.acol[a] = aggs[a].col;
  }
  unsigned char* scratch = noalloc_scratch(c);
  p.ticket = reinterpret_cast<unsigned int*>(scratch);
  p.partials = reinterpret_cast<AggAcc*>(scratch + 256);
  p.out = d_out;
  p.out_count = nullptr;
  // The ticket must start at zero (the last CTA resets it, but a launch that
  // timed out may have left it set).  The partials are written before read.
  FDB_CUDA(cudaMemsetAsync(p.ticket, 0, sizeof(unsigned int), c.stream));
  launch_stream_nc<ScanAggOp>(c, cols, ncols, n, p, ScanAggOp::kSmem);
}

// The bounded-wait test hook of this file's streamed scans (fdb_aggregate,
// fdb_filter_count, ...): see StreamHook.  tile = ~0 clears it.
void stream_test_stall(Ctx& c, uint64_t tile, uint32_t spin_limit) {
  StreamHook h{};
  h.withhold_tile1 = tile == ~0ull ? 0 : tile + 1;
  h.spin_limit = spin_limit;
  FDB_CUDA(cudaMemcpyToSymbolAsync(g_stream_hook, &h, sizeof(h), 0, cudaMemcpyHostToDevice, c.stream));
  FDB_CUDA(cudaStreamSynchronize(c.stream));
}

template <typename S, typename T>
static void launch_cmp_count(Ctx& c, const fdb_dev_column* cols, uint64_t n, const ScanAggParams& p, int op) {
  switch (op) {
    case FDB_EQ: launch_stream<CmpCountOp<S, T, FDB_EQ>, 1>(c, cols, n, p, ScanAggOp::kSmem); break;
    case FDB_NE: launch_stream<CmpCountOp<S, T, FDB_NE>, 1>(c, cols, n, p, ScanAggOp::kSmem); break;
    case FDB_LT: launch_stream<CmpCountOp<S, T, FDB_LT>, 1>(c, cols, n, p, ScanAggOp::kSmem); break;
    case FDB_LE: launch_stream<CmpCountOp<S, T, FDB_LE>, 1>(c, cols, n, p, ScanAggOp::kSmem); break;
    case FDB_GT: launch_stream<CmpCountOp<S, T, FDB_GT>, 1>(c, cols, n, p, ScanAggOp::kSmem); break;
    default: launch_stream<CmpCountOp<S, T, FDB_GE>, 1>(c, cols, n, p, ScanAggOp::kSmem); break;
  }
}

void op_filter_count(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                     const fdb_pred_term* prog, int nterms, uint64_t* d_count) {
  ScanAggParams p;
  std::memset(&p, 0, sizeof(p));
  fill_cols(p.sc, cols, ncols, n);
  fill_prog(p.prog, prog, nterms, ncols);
  p.naggs = 1;
  p.func[0] = FDB_AGG_COUNT_STAR;
  p.acol[0] = 0;
  p.partials = static_cast<AggAcc*>(c.scratch_take(sizeof(AggAcc) * 4 * max_stream_grid(c)));
  p.ticket = c.d_ticket;
  p.out = nullptr;
  p.out_count = d_count;
  // `col op literal` over one NULL-free numeric column.
  if (ncols == 1 && nterms == 1 && prog[0].kind == FDB_TERM_CMP && prog[0].col == 0 &&
      cols[0].validity == nullptr && cols[0].dtype != FDB_UTF8) {
    if (cols[0].dtype == FDB_FLOAT64)
      launch_cmp_count<double, double>(c, cols, n, p, prog[0].op);
    else if (prog[0].lit_type == FDB_FLOAT64)
      launch_cmp_count<int64_t, double>(c, cols, n, p, prog[0].op);  // widened (expr.rs:1122-1132)
    else
      launch_cmp_count<int64_t, int64_t>(c, cols, n, p, prog[0].op);
    return;
  }
  launch_stream_nc<ScanAggOp>(c, cols, ncols, n, p, ScanAggOp::kSmem);
}

void op_distinct_codes(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                       const fdb_pred_term* prog, int nterms, int code_col, uint32_t dict_len,
                       uint64_t* d_bitmap) {
  DistinctParams p;
  std::memset(&p, 0, sizeof(p));
  fill_cols(p.sc, cols, ncols, n);
  fill_prog(p.prog, prog, nterms, ncols);
  if (code_col < 0 || code_col >= ncols || cols[code_col].dtype != FDB_UTF8)
    fail(FDB_E_TYPE, "COUNT DISTINCT over codes needs a Utf8 column");
  p.code_col = code_col;
  p.dict_len = dict_len;
  p.bitmap = d_bitmap;
  const size_t words = (dict_len + 63) / 64;
  if (words) FDB_CUDA(cudaMemsetAsync(d_bitmap, 0, words * 8, c.stream));
  if (n == 0 || dict_len == 0) return;
  if (ncols == 1)
    launch_stream<DistinctOp, 1, 4096, 4>(c, cols, n, p, DistinctOp::kSmem);
  else
    launch_stream_nc<DistinctOp>(c, cols, ncols, n, p, DistinctOp::kSmem);
}

// ---------------------------------------------------------------------------
// WHERE mask: one warp per 64-row word, two ballots per word; padding bits zero.
// ---------------------------------------------------------------------------
struct MaskParams {
  PredProg prog;
  ScanCols sc;
};

__device__ __forceinline__ bool row_passes(const MaskParams& p, uint64_t row) {
  auto get = [&](int c, int64_t& iv, double& fv, uint32_t& code, bool& valid) -> int {
    const DevCol& col = p.sc.cols[c];
    const int dt = col.dtype;
    if (dt == FDB_FLOAT64)
      fv = static_cast<const double*>(col.values)[row];
    else if (dt == FDB_INT64)
      iv = static_cast<const int64_t*>(col.values)[row];
    else
      code = static_cast<const uint32_t*>(col.values)[row];
    valid = col.validity ? col_valid(col, row) : true;
    return dt;
  };
  return eval_prog(p.prog, get);
}

__global__ void filter_mask_kernel(MaskParams p, uint64_t n, uint64_t* mask) {
  const uint64_t nwords = (n + 63) / 64;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = gw; w < nwords; w += nwarps) {
    const uint64_t r0 = w * 64 + lane, r1 = r0 + 32;
    const bool a = r0 < n && row_passes(p, r0);
    const bool b = r1 < n && row_passes(p, r1);
    const uint32_t lo = __ballot_sync(0xffffffffu, a);
    const uint32_t hi = __ballot_sync(0xffffffffu, b);
    if (lane == 0) mask[w] = (uint64_t)lo | ((uint64_t)hi << 32);
  }
}

void op_filter_mask(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                    const fdb_pred_term* prog, int nterms, uint64_t* d_mask) {
  MaskParams p;
  std::memset(&p, 0, sizeof(p));
  fill_cols(p.sc, cols, ncols, n);
  fill_prog(p.prog, prog, nterms, ncols);
  const uint64_t nwords = (n + 63) / 64;
  if (nwords == 0) return;
  const int threads = 256;
  const uint64_t blocks = umin64((nwords + 7) / 8, (uint64_t)c.sm_count * 8);
  filter_mask_kernel<<<(unsigned)blocks, threads, 0, c.stream>>>(p, n, d_mask);
  FDB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Stable compaction of a mask into row numbers: chunk popcounts, one-block
// exclusive scan of the chunk counts, then each chunk writes its rows.
// ---------------------------------------------------------------------------
constexpr int kCompactThreads = 256;
constexpr int kWordsPerThread = 8;
constexpr int kChunkWords = kCompactThreads * kWordsPerThread;  // 2048 words = 131072 rows

template <typename T>
__device__ T block_exclusive_scan(T v, T* sm_warp, T* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T s = lane < nw ? sm_warp[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) sm_warp[lane] = s;  // inclusive prefix of warp totals
  }
  __syncthreads();
  T warp_base = warp ? sm_warp[warp - 1] : T(0);
  if (total) *total = sm_warp[nw - 1];
  __syncthreads();
  return warp_base + x - v;
}

__global__ void compact_count_kernel(const uint64_t* mask, uint64_t nwords, uint64_t* counts) {
  __shared__ uint64_t sm[32];
  const uint64_t w0 = (uint64_t)blockIdx.x * kChunkWords + threadIdx.x * kWordsPerThread;
  uint64_t cnt = 0;
#pragma unroll
  for (int j = 0; j < kWordsPerThread; ++j)
    if (w0 + j < nwords) cnt += __popcll(mask[w0 + j]);
  uint64_t total;
  block_exclusive_scan<uint64_t>(cnt, sm, &total);
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

__global__ void compact_scan_kernel(uint64_t* counts, uint64_t nchunks, uint64_t* d_count,
                                    uint64_t capacity, int* err) {
  __shared__ uint64_t sm[32];
  // Each thread owns a contiguous run of chunks.
  const uint64_t per = (nchunks + blockDim.x - 1) / blockDim.x;
  const uint64_t b0 = threadIdx.x * per;
  uint64_t local = 0;
  for (uint64_t i = b0; i < b0 + per && i < nchunks; ++i) local += counts[i];
  uint64_t total;
  uint64_t base = block_exclusive_scan<uint64_t>(local, sm, &total);
  for (uint64_t i = b0; i < b0 + per && i < nchunks; ++i) {
    uint64_t v = counts[i];
    counts[i] = base;
    base += v;
  }
  if (threadIdx.x == 0) {
    *d_count = total;
    if (total > capacity) atomicExch(err, kErrCapacity);
  }
}

__global__ void compact_write_kernel(const uint64_t* mask, uint64_t nwords, const uint64_t* offsets,
                                     uint32_t* rows, uint64_t capacity) {
  __shared__ uint64_t sm[32];
  const uint64_t w0 = (uint64_t)blockIdx.x * kChunkWords + threadIdx.x * kWordsPerThread;
  uint64_t words[kWordsPerThread];
  uint64_t cnt = 0;
#pragma unroll
  for (int j = 0; j < kWordsPerThread; ++j) {
    words[j] = (w0 + j < nwords) ? mask[w0 + j] : 0ull;
    cnt += __popcll(words[j]);
  }
  uint64_t off = offsets[blockIdx.x] + block_exclusive_scan<uint64_t>(cnt, sm, nullptr);
#pragma unroll
  for (int j = 0; j < kWordsPerThread; ++j) {
    uint64_t w = words[j];
    while (w) {
      const int b = __ffsll((long long)w) - 1;
      w &= w - 1;
      if (off < capacity) rows[off] = (uint32_t)((w0 + j) * 64 + b);
      ++off;
    }
  }
}

void op_compact_mask(Ctx& c, const uint64_t* d_mask, uint64_t n, uint32_t* d_rows,
                     uint64_t capacity, uint64_t* d_count) {
  const uint64_t nwords = (n + 63) / 64;
  if (nwords == 0) {
    FDB_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), c.stream));
    return;
  }
  const uint64_t nchunks = (nwords + kChunkWords - 1) / kChunkWords;
  uint64_t* counts = static_cast<uint64_t*>(c.scratch_take(nchunks * sizeof(uint64_t)));
  compact_count_kernel<<<(unsigned)nchunks, kCompactThreads, 0, c.stream>>>(d_mask, nwords, counts);
  compact_scan_kernel<<<1, 1024, 0, c.stream>>>(counts, nchunks, d_count, capacity, c.d_err);
  compact_write_kernel<<<(unsigned)nchunks, kCompactThreads, 0, c.stream>>>(d_mask, nwords, counts,
                                                                            d_rows, capacity);
  FDB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Gather rows of one column.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void gather_kernel(const T* __restrict__ in, const uint32_t* __restrict__ rows, uint64_t n,
                              T* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[rows[i]];
}

__global__ void gather_validity_kernel(const uint64_t* __restrict__ validity, uint64_t voff,
                                       const uint32_t* __restrict__ rows, uint64_t n,
                                       uint64_t* __restrict__ out) {
  const uint64_t nwords = (n + 63) / 64;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = gw; w < nwords; w += nwarps) {
    bool a = false, b = false;
    const uint64_t i0 = w * 64 + lane, i1 = i0 + 32;
    if (i0 < n) {
      const uint64_t bit = voff + rows[i0];
      a = (validity[bit >> 6] >> (bit & 63)) & 1ull;
    }
    if (i1 < n) {
      const uint64_t bit = voff + rows[i1];
      b = (validity[bit >> 6] >> (bit & 63)) & 1ull;
    }
    const uint32_t lo = __ballot_sync(0xffffffffu, a), hi = __ballot_sync(0xffffffffu, b);
    if (lane == 0) out[w] = (uint64_t)lo | ((uint64_t)hi << 32);
  }
}

template <typename T>
__global__ void gather_opt_kernel(const T* __restrict__ in, const uint64_t* validity, uint64_t voff,
                                  const uint32_t* __restrict__ rows, uint64_t n, T* __restrict__ out,
                                  uint64_t* __restrict__ out_valid) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (n + 31) / 32;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = gw; w < nw; w += nwarps) {  // 32 outputs per warp step
    const uint64_t i = w * 32 + lane;
    bool ok = false;
    if (i < n) {
      const uint32_t r = rows[i];
      if (r != FDB_NO_ROW) {
        ok = true;
        if (validity) {
          const uint64_t b = voff + r;
          ok = (validity[b >> 6] >> (b & 63)) & 1ull;
        }
        out[i] = in[r];
      } else {
        out[i] = T(0);
      }
    }
    const uint32_t m = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) reinterpret_cast<uint32_t*>(out_valid)[w] = m;
  }
}

void op_gather_opt(Ctx& c, const fdb_dev_column& col, const uint32_t* d_rows, uint64_t n, void* d_out,
                   uint64_t* d_out_validity) {
  if (n == 0) return;
  FDB_CUDA(cudaMemsetAsync(d_out_validity, 0, ((n + 63) / 64) * 8, c.stream));
  const unsigned blocks = (unsigned)umin64((n + 255) / 256, (uint64_t)c.sm_count * 16);
  if (dtype_size(col.dtype) == 8)
    gather_opt_kernel<uint64_t><<<blocks, 256, 0, c.stream>>>(
        static_cast<const uint64_t*>(col.values), col.validity, col.validity_offset, d_rows, n,
        static_cast<uint64_t*>(d_out), d_out_validity);
  else
    gather_opt_kernel<uint32_t><<<blocks, 256, 0, c.stream>>>(
        static_cast<const uint32_t*>(col.values), col.validity, col.validity_offset, d_rows, n,
        static_cast<uint32_t*>(d_out), d_out_validity);
  FDB_CUDA(cudaGetLastError());
}

void op_gather(Ctx& c, const fdb_dev_column& col, const uint32_t* d_rows, uint64_t n, void* d_out,
               uint64_t* d_out_validity) {
  if (n == 0) return;
  const int threads = 256;
  const unsigned blocks = (unsigned)umin64((n + threads - 1) / threads, (uint64_t)c.sm_count * 16);
  if (dtype_size(col.dtype) == 8)
    gather_kernel<uint64_t><<<blocks, threads, 0, c.stream>>>(
        static_cast<const uint64_t*>(col.values), d_rows, n, static_cast<uint64_t*>(d_out));
  else
    gather_kernel<uint32_t><<<blocks, threads, 0, c.stream>>>(
        static_cast<const uint32_t*>(col.values), d_rows, n, static_cast<uint32_t*>(d_out));
  if (col.validity && d_out_validity) {
    const uint64_t nwords = (n + 63) / 64;
    const unsigned vb = (unsigned)umin64((nwords + 7) / 8, (uint64_t)c.sm_count * 8);
    gather_validity_kernel<<<vb, 256, 0, c.stream>>>(col.validity, col.validity_offset, d_rows, n,
                                                     d_out_validity);
  }
  FDB_CUDA(cudaGetLastError());
}

}  // namespace fdb
