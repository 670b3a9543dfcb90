// GROUP BY kernels.
//
// 1. Dictionary-code GROUP BY (fast_utf8_gb, FalconDB src/query/aggregate.rs:619-836,
//    accumulate_batch 916-1169, merge_state_entry 1351-1390).  The group id of a
//    row is its dictionary code (value semantics: one dictionary per column, so
//    the multi-batch dictionary hazard of the reference cannot arise).  Rows are
//    combined inside a warp first: __match_any_sync groups the lanes that share a
//    code, the lowest lane of each group folds its peers' contributions in lane
//    order and updates the warp's private table in shared memory.  Warp tables,
//    CTA partials and the final merge are combined in fixed order, so FP64 sums
//    are repeatable for a given grid.
//
// 2. int64-key hash GROUP BY (fast_i64_gb, aggregate.rs:840-912) with COUNT(*),
//    SUM, MIN, MAX of one value column.  Each CTA keeps an open-addressing table
//    in shared memory that absorbs the frequent keys (Zipf heavy hitters); rows
//    whose key finds no room there go straight to a global open-addressing table
//    with atomics; the CTA table is flushed to the global one at the end.  Keys
//    are stored XOR 2^63 so that an all-zero slot is empty (cudaMemset clears the
//    table); MIN is kept as the bitwise NOT of the order key so both MIN and MAX
//    are atomicMax from a zero identity.  SUM is FP64 atomicAdd (order varies run
//    to run; tests hold it to 1e-12 relative).
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "common.cuh"
#include "engine.h"
#include "gtable.cuh"
#include "stream.cuh"

namespace fdb {

// ===========================================================================
// 1. Dictionary-code GROUP BY
// ===========================================================================
enum SlotKind : int32_t { kAddU64 = 0, kAddF64 = 1, kMaxU64 = 2 };
constexpr int kMaxSlots = 9;            // rows + 4 aggregates x (value, count)
constexpr int kGbWarpTableEntries = 512;  // (groups) x (slots) per warp

struct GbCodesParams {
  PredProg prog;
  DevCol cols[4];
  int32_t key_col;
  uint32_t ngroups;        // dict_len + 1 (last = NULL key)
  int32_t nslots;
  int32_t naggs;
  int32_t func[4];
  int32_t acol[4];
  int32_t vslot[4];        // value slot of each aggregate (-1: none)
  int32_t cslot[4];        // count slot of each aggregate (-1: uses the row slot)
  int32_t kind[kMaxSlots];
  // Specialised lane path (GbLaneFastOp): WHERE is absent or one FP64
  // column compare, the key column and every value column have no NULLs, and
  // every aggregate is COUNT(*), SUM or AVG.  Slot 0 counts rows; slot s >= 1
  // sums column f_vcol[s-1].
  int32_t f_cmp_col;       // WHERE column (-1: no WHERE)
  uint32_t f_cmp_mask;     // accepted outcomes: bit 0 unordered, 1 less, 2 equal, 3 greater
  double f_lit;
  int32_t f_vcol[4];
  uint32_t f_f64;          // bit s-1: slot s sums an FP64 column (else int64, wrapping)
  uint64_t* partials;      // [grid][ngroups][nslots]
  unsigned int* ticket;
  fdb_agg_value* out;      // [ngroups][naggs]
  int64_t* group_rows;     // [ngroups]
};

__device__ __forceinline__ uint64_t slot_combine(int kind, uint64_t a, uint64_t b) {
  if (kind == kAddF64)
    return (uint64_t)__double_as_longlong(__longlong_as_double((long long)a) +
                                          __longlong_as_double((long long)b));
  if (kind == kMaxU64) return a > b ? a : b;
  return a + b;
}

template <class Acc>
struct GbGetter {
  const DevCol* cols;
  const Acc& acc;
  uint32_t i;
  uint64_t row;
  __device__ __forceinline__ int operator()(int c, int64_t& iv, double& fv, uint32_t& code,
                                            bool& valid) const {
    const DevCol& col = cols[c];
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

// Row i of `acc`: false when it fails the WHERE program; otherwise its group
// id (dictionary code; ngroups-1 for the NULL key) and the value each table
// slot adds (slot 0: the row count).
template <class Acc>
__device__ __forceinline__ bool gb_row_values(const GbCodesParams& p, const Acc& acc, uint32_t i, uint32_t& gid,
                                              uint64_t (&v)[kMaxSlots]) {
#pragma unroll
  for (int s = 0; s < kMaxSlots; ++s) v[s] = 0;
  const uint64_t row = acc.row(i);
  GbGetter<Acc> get{p.cols, acc, i, row};
  if (!eval_prog(p.prog, get)) return false;
  int64_t iv;
  double fv;
  uint32_t code;
  bool valid;
  get(p.key_col, iv, fv, code, valid);
  gid = (!valid || code == kNullCode || code >= p.ngroups - 1) ? p.ngroups - 1 : code;
  v[0] = 1;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    if (a >= p.naggs) break;
    const int f = p.func[a];
    if (f == FDB_AGG_COUNT_STAR) continue;
    const int dt = get(p.acol[a], iv, fv, code, valid);
    if (!valid) continue;
    if ((f == FDB_AGG_MIN || f == FDB_AGG_MAX) && dt == FDB_FLOAT64 && isnan(fv)) continue;
    const int cs = p.cslot[a];
    const int vs = p.vslot[a];
#pragma unroll
    for (int s = 1; s < kMaxSlots; ++s)
      if (s == cs) v[s] = 1;
    uint64_t x = 0;
    if (f == FDB_AGG_SUM || f == FDB_AGG_AVG) {
      x = dt == FDB_FLOAT64 ? (uint64_t)__double_as_longlong(fv) : (uint64_t)iv;
    } else if (f == FDB_AGG_MIN) {
      x = ~(dt == FDB_FLOAT64 ? f64_ord_key(fv) : i64_ord_key(iv));
    } else if (f == FDB_AGG_MAX) {
      x = dt == FDB_FLOAT64 ? f64_ord_key(fv) : i64_ord_key(iv);
    }
#pragma unroll
    for (int s = 1; s < kMaxSlots; ++s)
      if (s == vs) v[s] = x;
  }
  return true;
}

__device__ void gb_codes_merge(const GbCodesParams& p, uint64_t* tab, unsigned int* s_last, int ctid, int nct);

struct GbCodesOp {
  using Params = GbCodesParams;
  struct Local {};
  // smem: per-warp tables [NW][kGbWarpTableEntries] + staging [NW][32][kMaxSlots] + flag
  static constexpr int kNW = 8;
  static constexpr size_t kSmem =
      (size_t)kNW * kGbWarpTableEntries * 8 + (size_t)kNW * 32 * kMaxSlots * 8 + 16;

  static __device__ void init(Local&, const Params& p, unsigned char* sm, int ctid, int nct) {
    uint64_t* tab = reinterpret_cast<uint64_t*>(sm);
    for (int i = ctid; i < kNW * kGbWarpTableEntries; i += nct) tab[i] = 0;
  }

  template <class Acc>
  static __device__ void step(Local&, const Params& p, unsigned char* sm, const Acc& acc,
                              uint32_t rows, int ctid, int nct) {
    const int warp = ctid >> 5, lane = ctid & 31;
    uint64_t* tab = reinterpret_cast<uint64_t*>(sm) + (size_t)warp * kGbWarpTableEntries;
    uint64_t* stage = reinterpret_cast<uint64_t*>(sm) + (size_t)kNW * kGbWarpTableEntries +
                      (size_t)warp * 32 * kMaxSlots;
    const int ns = p.nslots;
    for (uint32_t b = 0; b < rows; b += nct) {
      const uint32_t i = b + ctid;
      uint32_t gid = 0xFFFFFFFFu;
      uint64_t v[kMaxSlots];
      if (!(i < rows && gb_row_values(p, acc, i, gid, v))) {
        gid = 0xFFFFFFFFu;
#pragma unroll
        for (int s = 0; s < kMaxSlots; ++s) v[s] = 0;
      }
      // Warp-level combine of the lanes that share a group.
      const unsigned peers = __match_any_sync(0xffffffffu, gid);
      const int leader = __ffs(peers) - 1;
#pragma unroll
      for (int s = 0; s < kMaxSlots; ++s)
        if (s < ns) stage[lane * kMaxSlots + s] = v[s];
      __syncwarp();
      if (lane == leader && gid != 0xFFFFFFFFu) {
        unsigned rest = peers & ~(1u << lane);
        while (rest) {
          const int q = __ffs(rest) - 1;
          rest &= rest - 1;
#pragma unroll
          for (int s = 0; s < kMaxSlots; ++s)
            if (s < ns) v[s] = slot_combine(p.kind[s], v[s], stage[q * kMaxSlots + s]);
        }
        uint64_t* t = tab + (size_t)gid * ns;
#pragma unroll
        for (int s = 0; s < kMaxSlots; ++s)
          if (s < ns) t[s] = slot_combine(p.kind[s], t[s], v[s]);
      }
      __syncwarp();
    }
  }

  static __device__ void finish(Local&, const Params& p, unsigned char* sm, int ctid, int nct) {
    uint64_t* tab = reinterpret_cast<uint64_t*>(sm);
    unsigned int* s_last = reinterpret_cast<unsigned int*>(
        sm + (size_t)kNW * kGbWarpTableEntries * 8 + (size_t)kNW * 32 * kMaxSlots * 8);
    const int ns = p.nslots;
    const uint32_t entries = p.ngroups * ns;
    consumer_bar(nct);
    // Fold warp tables in warp order into the CTA partial.
    for (uint32_t e = ctid; e < entries; e += nct) {
      const int kind = p.kind[e % ns];
      uint64_t acc = tab[e];
      for (int w = 1; w < kNW; ++w) acc = slot_combine(kind, acc, tab[(size_t)w * kGbWarpTableEntries + e]);
      p.partials[(size_t)blockIdx.x * entries + e] = acc;
    }
    gb_codes_merge(p, tab, s_last, ctid, nct);
  }
};

// Publish this CTA's partial (already in p.partials) and, in the last CTA,
// fold all partials in CTA order and write the per-group results.  `tab` is
// shared memory of at least ngroups * nslots words.
__device__ void gb_codes_merge(const GbCodesParams& p, uint64_t* tab, unsigned int* s_last, int ctid, int nct) {
    const int ns = p.nslots;
    const uint32_t entries = p.ngroups * ns;
    __threadfence();
    consumer_bar(nct);
    if (ctid == 0) {
      const unsigned int t = atomicAdd(p.ticket, 1u);
      *s_last = (t == gridDim.x - 1) ? 1u : 0u;
    }
    consumer_bar(nct);
    if (*s_last == 0) return;
    __threadfence();
    // Last CTA: fold the CTA partials of each table entry in CTA order.  The
    // CTAs are cut into nseg contiguous ranges, each folded by its own thread
    // with 8 loads in flight, and the range results are folded in range order:
    // a fixed tree for a given grid, so FP64 sums repeat run to run.
    const uint32_t G = gridDim.x;
    uint32_t nseg = (uint32_t)nct / entries;
    nseg = nseg < 1 ? 1 : (nseg > 16 ? 16 : nseg);
    uint64_t* part = tab + entries;  // [entries][nseg], after the final entries
    for (uint32_t w = ctid; w < entries * nseg; w += nct) {
      const uint32_t e = w / nseg, sg = w % nseg;
      const uint32_t b0 = (uint32_t)((uint64_t)G * sg / nseg), b1 = (uint32_t)((uint64_t)G * (sg + 1) / nseg);
      const int kind = p.kind[e % ns];
      uint64_t acc = 0;
      bool first = true;
      for (uint32_t b = b0; b < b1; b += 8) {
        uint64_t v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = b + j < b1 ? __ldcg(&p.partials[(size_t)(b + j) * entries + e]) : 0;
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (b + j < b1) {
            acc = first ? v[j] : slot_combine(kind, acc, v[j]);
            first = false;
          }
      }
      part[(size_t)e * nseg + sg] = acc;
    }
    consumer_bar(nct);
    for (uint32_t e = ctid; e < entries; e += nct) {
      const int kind = p.kind[e % ns];
      uint64_t acc = 0;
      bool first = true;
      for (uint32_t sg = 0; sg < nseg; ++sg) {
        if ((uint64_t)G * sg / nseg == (uint64_t)G * (sg + 1) / nseg) continue;  // an empty range
        acc = first ? part[(size_t)e * nseg + sg] : slot_combine(kind, acc, part[(size_t)e * nseg + sg]);
        first = false;
      }
      tab[e] = acc;
    }
    consumer_bar(nct);
    for (uint32_t g = ctid; g < p.ngroups; g += nct) {
      const uint64_t* t = tab + (size_t)g * ns;
      p.group_rows[g] = (int64_t)t[0];
      for (int a = 0; a < p.naggs; ++a) {
        const int f = p.func[a];
        const int dt = f == FDB_AGG_COUNT_STAR ? FDB_INT64 : p.cols[p.acol[a]].dtype;
        const uint64_t cnt = p.cslot[a] >= 0 ? t[p.cslot[a]] : t[0];
        fdb_agg_value v;
        v.f = 0.0;
        v.i = 0;
        v.n = (int64_t)cnt;
        v.is_int = 0;
        v.valid = cnt > 0;
        if (f == FDB_AGG_COUNT_STAR || f == FDB_AGG_COUNT) {
          v.is_int = 1;
          v.i = (int64_t)cnt;
          v.valid = 1;
        } else if (f == FDB_AGG_SUM || f == FDB_AGG_AVG) {
          const uint64_t x = t[p.vslot[a]];
          const double s = dt == FDB_FLOAT64 ? __longlong_as_double((long long)x) : (double)(int64_t)x;
          v.f = (f == FDB_AGG_AVG && cnt) ? s / (double)cnt : s;
        } else if (cnt) {
          uint64_t key = t[p.vslot[a]];
          if (f == FDB_AGG_MIN) key = ~key;
          v.f = dt == FDB_FLOAT64 ? f64_from_ord_key(key) : (double)(int64_t)(key ^ (1ull << 63));
        }
        p.out[(size_t)g * p.naggs + a] = v;
      }
    }
    if (ctid == 0) *p.ticket = 0u;
}

// Lane-private variant for small tables ((groups x slots) <= kLaneEntries):
// every consumer thread owns one column of a shared-memory table laid out
// [entry][thread], so a row updates its thread's own words — no atomics, no
// warp combine, bank-conflict free (a warp's 32 threads touch 32 consecutive
// 8-byte words whatever groups they hit).  Each thread folds its rows in row
// order; the CTA then folds the 256 columns in thread order: FP64 sums are
// repeatable for a given grid.
constexpr int kLaneEntries = 48;
// Tile rows and ring stages of the three-column lane GROUP BY (config 0's shape).
#ifndef FDB_LANE_TR3
#define FDB_LANE_TR3 512
#endif
#ifndef FDB_LANE_ST3
#define FDB_LANE_ST3 2
#endif
#ifndef FDB_LANE_NCW3
#define FDB_LANE_NCW3 8
#endif

struct GbLaneOp {
  using Params = GbCodesParams;
  struct Local {};

  static __device__ void init(Local&, const Params& p, unsigned char* sm, int ctid, int nct) {
    uint64_t* tab = reinterpret_cast<uint64_t*>(sm);
    const uint32_t entries = p.ngroups * p.nslots;
    for (uint32_t e = 0; e < entries; ++e) tab[(size_t)e * nct + ctid] = 0;  // every kind's identity is 0
  }

  // Column-at-a-time inside the tile: first the WHERE result and group id of
  // this thread's (up to kR) rows, then one tight loop per aggregate whose
  // (function, type) dispatch is decided once per tile, not per row.
  static constexpr int kR = 8;

  template <class Acc>
  static __device__ void step(Local&, const Params& p, unsigned char* sm, const Acc& acc, uint32_t rows,
                              int ctid, int nct) {
    uint64_t* tab = reinterpret_cast<uint64_t*>(sm);
    const int ns = p.nslots;
    for (uint32_t b = 0; b < rows; b += kR * nct) {
      uint32_t off[kR];  // table word offset of (group, slot 0) for this thread
      uint32_t pm = 0;
      // Phase 1: WHERE + group id.
      const bool one_cmp = p.prog.n == 1 && p.prog.t[0].kind == FDB_TERM_CMP &&
                           p.cols[p.prog.t[0].col].dtype == FDB_FLOAT64 && !p.cols[p.prog.t[0].col].validity;
      const int pc = p.prog.t[0].col, pop = p.prog.t[0].op;
      const double plit = p.prog.t[0].lit_type == FDB_FLOAT64 ? p.prog.t[0].lit_f : (double)p.prog.t[0].lit_i;
      const DevCol& kc = p.cols[p.key_col];
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        const uint32_t i = b + j * nct + ctid;
        off[j] = 0;
        if (i >= rows) continue;
        bool pass;
        if (p.prog.n == 0) {
          pass = true;
        } else if (one_cmp) {
          pass = cmp_op<double>(pop, acc.template get<double>(pc, i), plit);
        } else {
          GbGetter<Acc> get{p.cols, acc, i, acc.row(i)};
          pass = eval_prog(p.prog, get);
        }
        if (!pass) continue;
        const uint32_t code = acc.template get<uint32_t>(p.key_col, i);
        const bool kvalid = !kc.validity || col_valid(kc, acc.row(i));
        const uint32_t gid = (!kvalid || code >= p.ngroups - 1) ? p.ngroups - 1 : code;
        off[j] = gid * ns * nct + ctid;
        pm |= 1u << j;
      }
      if (pm == 0) continue;
      // Phase 2: the row count (slot 0).
#pragma unroll
      for (int j = 0; j < kR; ++j)
        if ((pm >> j) & 1u) tab[off[j]] += 1;
      // Phase 3: one loop per aggregate.
      for (int a = 0; a < p.naggs; ++a) {
        const int f = p.func[a];
        if (f == FDB_AGG_COUNT_STAR) continue;
        const int c = p.acol[a];
        const DevCol& col = p.cols[c];
        const int dt = col.dtype;
        const uint32_t cs = p.cslot[a] >= 0 ? (uint32_t)p.cslot[a] * nct : 0xFFFFFFFFu;
        const uint32_t vs = p.vslot[a] >= 0 ? (uint32_t)p.vslot[a] * nct : 0u;
        const bool sum = f == FDB_AGG_SUM || f == FDB_AGG_AVG;
        if (sum && dt == FDB_FLOAT64 && !col.validity && cs == 0xFFFFFFFFu) {
#pragma unroll
          for (int j = 0; j < kR; ++j)
            if ((pm >> j) & 1u) {
              double* w = reinterpret_cast<double*>(tab + off[j] + vs);
              *w += acc.template get<double>(c, b + j * nct + ctid);
            }
        } else if (sum && dt == FDB_INT64 && !col.validity && cs == 0xFFFFFFFFu) {
#pragma unroll
          for (int j = 0; j < kR; ++j)
            if ((pm >> j) & 1u) tab[off[j] + vs] += (uint64_t)acc.template get<int64_t>(c, b + j * nct + ctid);
        } else {
          // General: validity, counts, MIN / MAX.
#pragma unroll
          for (int j = 0; j < kR; ++j) {
            if (!((pm >> j) & 1u)) continue;
            const uint32_t i = b + j * nct + ctid;
            if (col.validity && !col_valid(col, acc.row(i))) continue;
            uint64_t x = 0;
            double fv = 0.0;
            int64_t iv = 0;
            if (dt == FDB_FLOAT64)
              fv = acc.template get<double>(c, i);
            else if (dt == FDB_INT64)
              iv = acc.template get<int64_t>(c, i);
            if ((f == FDB_AGG_MIN || f == FDB_AGG_MAX) && dt == FDB_FLOAT64 && isnan(fv)) continue;
            if (cs != 0xFFFFFFFFu) tab[off[j] + cs] += 1;
            if (f == FDB_AGG_COUNT) continue;
            if (sum) {
              if (dt == FDB_FLOAT64) {
                double* w = reinterpret_cast<double*>(tab + off[j] + vs);
                *w += fv;
              } else {
                tab[off[j] + vs] += (uint64_t)iv;
              }
              continue;
            }
            const uint64_t k = dt == FDB_FLOAT64 ? f64_ord_key(fv) : i64_ord_key(iv);
            x = f == FDB_AGG_MIN ? ~k : k;
            uint64_t& w = tab[off[j] + vs];
            w = x > w ? x : w;
          }
        }
      }
    }
  }

  static __device__ void finish(Local&, const Params& p, unsigned char* sm, int ctid, int nct) {
    uint64_t* tab = reinterpret_cast<uint64_t*>(sm);
    const int ns = p.nslots;
    const uint32_t entries = p.ngroups * ns;
    unsigned int* s_last = reinterpret_cast<unsigned int*>(sm + (size_t)entries * nct * 8);
    const int warp = ctid >> 5, lane = ctid & 31, nw = nct >> 5;
    consumer_bar(nct);
    // Fold each entry's thread columns: lanes read 32 consecutive words per
    // step, then a fixed shuffle tree.
    for (uint32_t e = warp; e < entries; e += nw) {
      const int kind = p.kind[e % ns];
      uint64_t a = tab[(size_t)e * nct + lane];
      for (int j = lane + 32; j < nct; j += 32) a = slot_combine(kind, a, tab[(size_t)e * nct + j]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a = slot_combine(kind, a, __shfl_xor_sync(0xffffffffu, a, o));
      if (lane == 0) p.partials[(size_t)blockIdx.x * entries + e] = a;
    }
    consumer_bar(nct);
    gb_codes_merge(p, tab, s_last, ctid, nct);
  }
};

// The lane-private table for the common shape (GbCodesParams::f_*): NV summed
// value slots, NCT = consumer threads.  Same table layout, init and fold as
// GbLaneOp; the row loop differs:
//   * every slot offset is a compile-time constant (slot s of a group is
//     s * NCT words after slot 0), so a row's 1 + NV table words load
//     together, independent of one another;
//   * a thread first loads its kR rows' WHERE value, code and NV values
//     (shared-memory loads only), then applies them to the table one row at a
//     time: each row's read-modify-write chain is one load latency long;
//   * the WHERE compare is branch-free: the outcome (unordered / less / equal
//     / greater) indexes the accepted-outcome mask the host derived from the
//     operator, with C++ semantics for NaN (only != accepts it).
// Launch shapes (consumer warps, rows per thread per tile, ring stages),
// measured on 100M and 1M rows of the three-column shape: large inputs run
// 3 CTAs of 4 consumer warps per SM with 512-row tiles (0.39 ms at 100M rows);
// small ones, where the launch and the final fold dominate, 8 consumer warps.
#ifndef FDB_LF_BIG_NCW
#define FDB_LF_BIG_NCW 4
#endif
#ifndef FDB_LF_BIG_R
#define FDB_LF_BIG_R 4
#endif
#ifndef FDB_LF_BIG_ST
#define FDB_LF_BIG_ST 2
#endif
#ifndef FDB_LF_SMALL_NCW
#define FDB_LF_SMALL_NCW 8
#endif
#ifndef FDB_LF_SMALL_R
#define FDB_LF_SMALL_R 2
#endif
#ifndef FDB_LF_SMALL_ST
#define FDB_LF_SMALL_ST 3
#endif
constexpr uint64_t kLaneFastBigRows = 1ull << 24;
template <int NV, int NCW, int R>
struct GbLaneFastOp {
  using Params = GbCodesParams;
  struct Local {};
  static constexpr int NCT = NCW * 32;
  static constexpr int kR = R;
  static constexpr int kTileRows = kR * NCT;

  static __device__ void init(Local& l, const Params& p, unsigned char* sm, int ctid, int nct) {
    GbLaneOp::Local g;
    GbLaneOp::init(g, p, sm, ctid, nct);
  }

  template <class Acc>
  static __device__ void step(Local&, const Params& p, unsigned char* sm, const Acc& acc, uint32_t rows,
                              int ctid, int) {
    uint64_t* tab = reinterpret_cast<uint64_t*>(sm) + ctid;
    const int pc = p.f_cmp_col, kc = p.key_col;
    const uint32_t pmask = p.f_cmp_mask;
    const double plit = p.f_lit;
    const uint32_t glast = p.ngroups - 1;
    const uint32_t f64 = p.f_f64;
    int vc[NV > 0 ? NV : 1];
#pragma unroll
    for (int s = 0; s < NV; ++s) vc[s] = p.f_vcol[s];
    for (uint32_t b = 0; b < rows; b += kTileRows) {
      uint32_t off[kR];
      uint64_t val[kR][NV > 0 ? NV : 1];
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        const uint32_t i = b + j * NCT + ctid;
        off[j] = 0xFFFFFFFFu;
#pragma unroll
        for (int s = 0; s < NV; ++s) val[j][s] = 0;
        if (i < rows) {
          bool pass = true;
          if (pc >= 0) {
            const double x = acc.template get<double>(pc, i);
            const uint32_t o = (x < plit ? 1u : 0u) + (x == plit ? 2u : 0u) + (x > plit ? 3u : 0u);
            pass = (pmask >> o) & 1u;
          }
          const uint32_t code = acc.template get<uint32_t>(kc, i);
          const uint32_t gid = code >= glast ? glast : code;  // the NULL code is above every group
          if (pass) off[j] = gid * (uint32_t)((1 + NV) * NCT);
#pragma unroll
          for (int s = 0; s < NV; ++s) val[j][s] = acc.template get<uint64_t>(vc[s], i);
        }
      }
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        if (off[j] == 0xFFFFFFFFu) continue;
        uint64_t* t = tab + off[j];
        uint64_t w[1 + NV];
#pragma unroll
        for (int s = 0; s <= NV; ++s) w[s] = t[s * NCT];
        t[0] = w[0] + 1;
#pragma unroll
        for (int s = 0; s < NV; ++s) {
          const uint64_t sum_f = (uint64_t)__double_as_longlong(__longlong_as_double((long long)w[s + 1]) +
                                                                __longlong_as_double((long long)val[j][s]));
          t[(s + 1) * NCT] = ((f64 >> s) & 1u) ? sum_f : w[s + 1] + val[j][s];
        }
      }
    }
  }

  static __device__ void finish(Local&, const Params& p, unsigned char* sm, int ctid, int nct) {
    GbLaneOp::Local g;
    GbLaneOp::finish(g, p, sm, ctid, nct);
  }
};

// ===========================================================================
// 2. int64-key hash GROUP BY
// ===========================================================================
struct GbHashParams {
  PredProg prog;
  DevCol cols[4];          // 0 = key, 1 = value, 2.. = predicate columns
  GSlot* table;            // global, capacity pow2, zeroed
  uint64_t mask;           // capacity - 1
  GSlot* null_slot;        // accumulator of the NULL key group (zeroed)
  int* err;
};

// Find or claim the slot of `skey` (key ^ 2^63, nonzero) in the global table.
__device__ __forceinline__ GSlot* gtable_slot(const GbHashParams& p, uint64_t skey) {
  return gtable_find(p.table, p.mask, skey, p.err);
}

// Rows whose key finds no room in the CTA table do not probe the global table
// where they stand (a third of a warp's lanes, each waiting on a DRAM round
// trip while the others idle).  The warp queues them in a ring in shared
// memory and drains them 64 at a time: every lane takes two queued rows and
// has both home-slot loads in flight before it resolves either.
#ifndef FDB_GB_DRAIN
#define FDB_GB_DRAIN 64
#endif
struct GbHashOp {
  using Params = GbHashParams;
  struct Local {
    uint32_t head, tail;  // the warp's ring: entries [head, tail), warp-uniform
  };
  static constexpr int kNW = 8;             // consumer warps of every GbHashOp launch
  static constexpr uint32_t kRing = 128;    // ring entries per warp (holds 63 + 32)
  static constexpr uint32_t kDrain = FDB_GB_DRAIN;  // 32 or 64
  static_assert(kDrain == 32 || kDrain == 64, "a drain takes one or two rows per lane");
  static constexpr size_t kTabBytes = (size_t)(kSmemSlots + 1) * sizeof(GSlot);
  static constexpr size_t kRingOff = kTabBytes + 16;
  static constexpr size_t kSmem = kRingOff + (size_t)kNW * kRing * (8 + 8 + 1);
  static_assert(kRingOff % 8 == 0, "ring alignment");

  struct Ring {
    uint64_t* key;
    double* val;
    unsigned char* has;
  };
  static __device__ __forceinline__ Ring ring(unsigned char* sm, int warp) {
    Ring r;
    r.key = reinterpret_cast<uint64_t*>(sm + kRingOff) + (size_t)warp * kRing;
    r.val = reinterpret_cast<double*>(sm + kRingOff + (size_t)kNW * kRing * 8) + (size_t)warp * kRing;
    r.has = sm + kRingOff + (size_t)kNW * kRing * 16 + (size_t)warp * kRing;
    return r;
  }

  static __device__ void init(Local& l, const Params&, unsigned char* sm, int ctid, int nct) {
    uint64_t* w = reinterpret_cast<uint64_t*>(sm);
    const size_t words = kTabBytes / 8;
    for (size_t i = ctid; i < words; i += nct) w[i] = 0;
    l.head = l.tail = 0;
  }

  // Apply the first `count` (<= kDrain) queued rows to the global table.
  static __device__ void drain(Local& l, const Params& p, const Ring& r, int lane, uint32_t count) {
    __syncwarp();
    const uint32_t e0 = (l.head + lane) & (kRing - 1), e1 = (l.head + 32 + lane) & (kRing - 1);
    const bool live0 = (uint32_t)lane < count, live1 = (uint32_t)lane + 32 < count;
    const uint64_t k0 = r.key[e0], k1 = r.key[e1];
    const double v0 = r.val[e0], v1 = r.val[e1];
    const bool h0 = r.has[e0], h1 = r.has[e1];
    __syncwarp();
    l.head += count;
    if (*reinterpret_cast<volatile int*>(p.err) != 0) return;
    const uint64_t a0 = mix64(k0) & p.mask, a1 = mix64(k1) & p.mask;
    const uint64_t c0 = live0 ? *reinterpret_cast<volatile uint64_t*>(&p.table[a0].key) : 0;
    const uint64_t c1 = live1 ? *reinterpret_cast<volatile uint64_t*>(&p.table[a1].key) : 0;
    if (live0) {
      GSlot* d = gtable_find_from(p.table, p.mask, k0, a0, c0, p.err);
      if (d) gslot_accum(d, v0, h0);
    }
    if (live1) {
      GSlot* d = gtable_find_from(p.table, p.mask, k1, a1, c1, p.err);
      if (d) gslot_accum(d, v1, h1);
    }
  }

  template <class Acc>
  static __device__ void step(Local& l, const Params& p, unsigned char* sm, const Acc& acc,
                              uint32_t rows, int ctid, int nct) {
    GSlot* tab = reinterpret_cast<GSlot*>(sm);
    const int lane = ctid & 31;
    const Ring r = ring(sm, ctid >> 5);
    for (uint32_t b = 0; b < rows; b += nct) {  // uniform trip count: the ballot below sees whole warps
      const uint32_t i = b + ctid;
      int j = -1;  // CTA slot of the row (kSmemSlots: the NULL group); -1: none
      bool spill = false;
      uint64_t skey = 0;
      double v = 0.0;
      bool has_v = false;
      if (i < rows) {
        const uint64_t row = acc.row(i);
        bool pass = true;
        if (p.prog.n) {
          GbGetter<Acc> get{p.cols, acc, i, row};
          pass = eval_prog(p.prog, get);
        }
        if (pass) {
          const int64_t key = acc.template get<int64_t>(0, i);
          const bool kvalid = p.cols[0].validity ? col_valid(p.cols[0], row) : true;
          has_v = p.cols[1].validity ? col_valid(p.cols[1], row) : true;
          if (has_v)
            v = p.cols[1].dtype == FDB_FLOAT64 ? acc.template get<double>(1, i)
                                               : (double)acc.template get<int64_t>(1, i);
          if (!kvalid || key == INT64_MIN) {  // NULL group (i64::MIN reads as NULL)
            j = (int)kSmemSlots;
          } else {
            skey = (uint64_t)key ^ (1ull << 63);
            GSlot* dst = smem_table_slot(tab, skey);
            if (dst)
              j = (int)(dst - tab);
            else
              spill = true;
          }
        }
      }
      if (j >= 0) sslot_accum(tab + j, v, has_v);
      const unsigned m = __ballot_sync(0xffffffffu, spill);
      if (m) {
        if (spill) {
          const uint32_t pos = (l.tail + __popc(m & ((1u << lane) - 1u))) & (kRing - 1);
          r.key[pos] = skey;
          r.val[pos] = v;
          r.has[pos] = has_v ? 1 : 0;
        }
        l.tail += __popc(m);
        if (l.tail - l.head >= kDrain) drain(l, p, r, lane, kDrain);
      }
    }
  }

  static __device__ void finish(Local& l, const Params& p, unsigned char* sm, int ctid, int nct) {
    const Ring r = ring(sm, ctid >> 5);
    if (l.tail != l.head) drain(l, p, r, ctid & 31, l.tail - l.head);
    GSlot* tab = reinterpret_cast<GSlot*>(sm);
    consumer_bar(nct);
    for (uint32_t i = ctid; i < kSmemSlots; i += nct) {
      const GSlot s = tab[i];
      if (s.key == 0) continue;
      GSlot* g = gtable_slot(p, s.key);
      if (g) gslot_merge(g, s);
    }
    if (ctid == 0) {
      const GSlot s = tab[kSmemSlots];
      if (s.count) gslot_merge(p.null_slot, s);
    }
  }
};

__global__ void gb_hash_compact_kernel(const GSlot* __restrict__ table, uint64_t capacity,
                                       const GSlot* null_slot, fdb_group_i64* out, uint64_t cap_out,
                                       unsigned long long* counter, int* err) {
  const int lane = threadIdx.x & 31;
  for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x; i0 < capacity + 32;
       i0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = i0 + threadIdx.x;
    GSlot s;
    bool live = false;
    if (i < capacity) {
      s = table[i];
      live = s.key != 0;
    } else if (i == capacity && null_slot->count) {
      s = *null_slot;
      s.key = 0;  // key INT64_MIN after the XOR below
      live = true;
    }
    const unsigned m = __ballot_sync(0xffffffffu, live);
    if (!m) continue;
    unsigned long long base = 0;
    const int leader = __ffs(m) - 1;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (live) {
      const uint64_t pos = base + __popc(m & ((1u << lane) - 1u));
      if (pos < cap_out) {
        out[pos] = gslot_group(s.key, s);
      } else {
        atomicExch(err, kErrCapacity);
      }
    }
  }
}

// ===========================================================================
// 3. int64-key GROUP BY on a direct-addressed table
// ===========================================================================
// When the non-NULL keys span a range not much wider than the number of
// groups (surrogate keys, dense id domains: the 100M-row Zipf workload's keys
// span 0..10M-1 with 4.85M groups), the global table holds one 32-byte slot
// per key value: slot k - kmin.  A row then needs no hash, no probe and no key
// compare-and-swap, and its update is four fire-and-forget atomics into one
// aligned 32-byte sector.  Each CTA still absorbs the frequent keys in a
// shared-memory table first (the Zipf head), keyed by the slot index.  The
// output comes out in key order, from an ordered compaction of the slots.
struct DSlot {                 // 32 bytes, 32-byte aligned; all-zero = no row yet
  unsigned long long count;
  double sum;
  unsigned long long nmin;     // ~order key of MIN (atomicMax)
  unsigned long long max;      // order key of MAX
};
static_assert(sizeof(DSlot) == 32, "one sector per slot");

// The CTA table, structure of arrays: field f of slot j is element j of
// array f, so the lanes of a warp touching random slots spread over all 32
// banks (32-byte array-of-structs slots put every field of every slot on 4
// of them).  Slot kDenseSmemSlots (the last) is the NULL key group.
struct SDTab {
  double* sum;
  unsigned long long* nmin;    // ~order key of MIN (atomicMax)
  unsigned long long* max;     // order key of MAX
  unsigned int* mmhi;          // [2j] high 32 bits of nmin[j], [2j + 1] of max[j] (lower bounds)
  unsigned int* k1;            // slot index + 1 (0 = empty)
  unsigned int* count;         // a CTA sees fewer than 2^32 rows
};

#ifndef FDB_GBD_SLOTS
#define FDB_GBD_SLOTS 1024
#endif
constexpr uint32_t kDenseSmemSlots = FDB_GBD_SLOTS;  // power of two
constexpr int kDenseSmemLog = __builtin_ctz(kDenseSmemSlots);
static_assert((kDenseSmemSlots & (kDenseSmemSlots - 1)) == 0, "CTA table slots: a power of two");
constexpr uint64_t kDenseMaxSlots = 1ull << 31;  // slot indices (and index + 1) fit 32 bits
// Probes into the CTA table before a row goes to the global table.
#ifndef FDB_GBD_PROBE
#define FDB_GBD_PROBE 4
#endif
constexpr uint32_t kDenseProbe = FDB_GBD_PROBE;
// Copies of each CTA slot's SUM, picked by lane: lanes of one warp that add to
// the same hot slot then contend on up to kDenseSumCopies addresses, not one.
#ifndef FDB_GBD_SUMSPLIT
#define FDB_GBD_SUMSPLIT 1
#endif
constexpr uint32_t kDenseSumCopies = FDB_GBD_SUMSPLIT;
static_assert((kDenseSumCopies & (kDenseSumCopies - 1)) == 0, "SUM copies: a power of two");
// Launch shape of the two-column instance (key, value): tile rows, stages,
// consumer warps.
#ifndef FDB_GBD_TR
#define FDB_GBD_TR 1024
#endif
#ifndef FDB_GBD_ST
#define FDB_GBD_ST 2
#endif
#ifndef FDB_GBD_NCW
#define FDB_GBD_NCW 8
#endif
// Rows a consumer thread decodes together: their tile reads and first CTA
// table probes are all issued before any of them is applied.
#ifndef FDB_GBD_ROWS
#define FDB_GBD_ROWS 4
#endif
constexpr uint32_t kDenseRows = FDB_GBD_ROWS;

struct GbDenseParams {
  PredProg prog;
  DevCol cols[4];              // 0 = key, 1 = value, 2.. = predicate columns
  DSlot* table;                // [slots], zeroed
  uint64_t slots;              // kmax - kmin + 1
  int64_t kmin;
  DSlot* null_slot;            // the NULL key group (zeroed)
  int* err;
};

// MIN / MAX checked first against one 8-byte word holding the high halves of
// both order keys (1), or against the two 64-bit keys (0).
#ifndef FDB_GBD_MMHI
#define FDB_GBD_MMHI 1
#endif

// Shared-memory bytes of the CTA table: kDenseSumCopies SUM arrays, then
// nmin, max, the packed high halves, k1, count (slot kDenseSmemSlots is the
// NULL group).
constexpr size_t kDenseSmemBytes = (size_t)(kDenseSmemSlots + 1) * (8 * kDenseSumCopies + 32);

__device__ __forceinline__ SDTab sdtab(unsigned char* sm) {
  constexpr uint32_t S = kDenseSmemSlots + 1;
  constexpr size_t kSums = (size_t)8 * S * kDenseSumCopies;
  SDTab t;
  t.sum = reinterpret_cast<double*>(sm);  // copy c of slot j: sum[c * S + j]
  t.nmin = reinterpret_cast<unsigned long long*>(sm + kSums);
  t.max = reinterpret_cast<unsigned long long*>(sm + kSums + 8 * S);
  t.mmhi = reinterpret_cast<unsigned int*>(sm + kSums + 16 * S);
  t.k1 = reinterpret_cast<unsigned int*>(sm + kSums + 24 * S);
  t.count = reinterpret_cast<unsigned int*>(sm + kSums + 28 * S);
  return t;
}

// A value into CTA slot j.  MIN / MAX take the 64-bit atomic only when the
// value improves on the slot, which after a frequent key's first few hundred
// rows is rare, so its rows do not queue on two 64-bit shared atomics.  The
// first test reads one 8-byte word holding lower bounds of the high halves of
// both keys (mmhi, raised after the 64-bit keys): a value whose high half is
// below the bound cannot improve the slot, so most rows read 8 bytes of the
// table for MIN and MAX together instead of 16.
__device__ __forceinline__ void sdslot_accum(const SDTab& t, uint32_t j, double v, bool has_v) {
  atomicAdd(&t.count[j], 1u);
  if (!has_v) return;
  const uint32_t copy = kDenseSumCopies > 1 ? (threadIdx.x & (kDenseSumCopies - 1)) : 0;
  atomicAdd(&t.sum[copy * (kDenseSmemSlots + 1) + j], v);
  if (isnan(v)) return;
  const unsigned long long k = f64_ord_key(v);
#if FDB_GBD_MMHI
  const unsigned long long w = *reinterpret_cast<volatile unsigned long long*>(&t.mmhi[2 * j]);
  const uint32_t nhi = (uint32_t)(~k >> 32), khi = (uint32_t)(k >> 32);
  const uint32_t nb = (uint32_t)w, kb = (uint32_t)(w >> 32);
  if (nhi >= nb && ~k > *reinterpret_cast<volatile unsigned long long*>(&t.nmin[j])) {
    atomicMax(&t.nmin[j], ~k);
    if (nhi > nb) atomicMax(&t.mmhi[2 * j], nhi);
  }
  if (khi >= kb && k > *reinterpret_cast<volatile unsigned long long*>(&t.max[j])) {
    atomicMax(&t.max[j], k);
    if (khi > kb) atomicMax(&t.mmhi[2 * j + 1], khi);
  }
#else
  if (~k > *reinterpret_cast<volatile unsigned long long*>(&t.nmin[j])) atomicMax(&t.nmin[j], ~k);
  if (k > *reinterpret_cast<volatile unsigned long long*>(&t.max[j])) atomicMax(&t.max[j], k);
#endif
}

// A value straight into its global slot (no result is used: RED operations).
__device__ __forceinline__ void dslot_accum(DSlot* d, double v, bool has_v) {
  atomicAdd(&d->count, 1ull);
  if (!has_v) return;
  atomicAdd(&d->sum, v);
  if (isnan(v)) return;
  const unsigned long long k = f64_ord_key(v);
  atomicMax(&d->nmin, ~k);
  atomicMax(&d->max, k);
}

__device__ __forceinline__ void dslot_merge(DSlot* d, const SDTab& t, uint32_t j) {
  atomicAdd(&d->count, (unsigned long long)t.count[j]);
  double sum = t.sum[j];
#pragma unroll
  for (uint32_t c = 1; c < kDenseSumCopies; ++c) sum += t.sum[c * (kDenseSmemSlots + 1) + j];
  if (__double_as_longlong(sum) != 0) atomicAdd(&d->sum, sum);
  if (t.nmin[j]) atomicMax(&d->nmin, t.nmin[j]);
  if (t.max[j]) atomicMax(&d->max, t.max[j]);
}

// The CTA home slot of slot index k.
__device__ __forceinline__ uint32_t smem_dense_home(uint32_t k) {
  return (k * 0x9E3779B1u) >> (32 - kDenseSmemLog);
}

// The CTA slot of slot index k, claiming one if free within kDenseProbe
// probes from its home slot h; -1 when it has no room there.  cur0 is a read
// of slot h's key taken earlier.  A CTA slot's key only ever goes from 0 to
// a slot index, so an early read can only be stale as 0, and the
// compare-and-swap then returns the key that is really there.
__device__ __forceinline__ int smem_dense_slot_from(const SDTab& t, uint32_t k, uint32_t h, unsigned int cur0) {
  const unsigned int k1 = k + 1u;
  unsigned int cur = cur0;
  for (uint32_t probe = 0; probe < kDenseProbe; ++probe) {
    if (probe) cur = *reinterpret_cast<volatile unsigned int*>(&t.k1[h]);
    if (cur == k1) return (int)h;
    if (cur == 0) {
      const unsigned int prev = atomicCAS(&t.k1[h], 0u, k1);
      if (prev == 0 || prev == k1) return (int)h;
    }
    h = (h + 1) & (kDenseSmemSlots - 1);
  }
  return -1;
}

struct GbDenseOp {
  using Params = GbDenseParams;
  struct Local {};
  static constexpr size_t kSmem = kDenseSmemBytes;

  static __device__ void init(Local&, const Params&, unsigned char* sm, int ctid, int nct) {
    uint64_t* w = reinterpret_cast<uint64_t*>(sm);
    for (size_t i = ctid; i < kSmem / 8; i += nct) w[i] = 0;
  }

  template <class Acc>
  static __device__ void step(Local&, const Params& p, unsigned char* sm, const Acc& acc, uint32_t rows, int ctid,
                              int nct) {
    const SDTab tab = sdtab(sm);
    constexpr uint32_t R = kDenseRows;
    enum : uint8_t { kSkip, kNull, kSlot };
    for (uint32_t i0 = ctid; i0 < rows; i0 += (uint32_t)nct * R) {
      uint32_t k[R], h[R];
      unsigned int cur[R];
      double v[R];
      uint8_t kind[R];
      bool has_v[R];
      // Decode every row first: key, value, its kind and its CTA home slot.
#pragma unroll
      for (uint32_t r = 0; r < R; ++r) {
        const uint32_t i = i0 + r * (uint32_t)nct;
        kind[r] = kSkip;
        has_v[r] = false;
        v[r] = 0.0;
        k[r] = 0;
        if (i >= rows) continue;
        const uint64_t row = acc.row(i);
        if (p.prog.n) {
          GbGetter<Acc> get{p.cols, acc, i, row};
          if (!eval_prog(p.prog, get)) continue;
        }
        const int64_t key = acc.template get<int64_t>(0, i);
        has_v[r] = p.cols[1].validity ? col_valid(p.cols[1], row) : true;
        if (has_v[r])
          v[r] = p.cols[1].dtype == FDB_FLOAT64 ? acc.template get<double>(1, i)
                                                : (double)acc.template get<int64_t>(1, i);
        const bool kvalid = (p.cols[0].validity ? col_valid(p.cols[0], row) : true) && key != INT64_MIN;
        if (!kvalid) {  // NULL group (i64::MIN reads as NULL)
          kind[r] = kNull;
          continue;
        }
        const uint64_t kk = (uint64_t)key - (uint64_t)p.kmin;
        if (kk >= p.slots) {  // outside the sized range: the sizing did not see this column
          atomicExch(p.err, kErrCapacity);
          continue;
        }
        k[r] = (uint32_t)kk;
        kind[r] = kSlot;
      }
      // Every row's first probe in flight together.
#pragma unroll
      for (uint32_t r = 0; r < R; ++r) {
        h[r] = smem_dense_home(k[r]);
        cur[r] = kind[r] == kSlot ? tab.k1[h[r]] : 0u;
      }
#pragma unroll
      for (uint32_t r = 0; r < R; ++r) {
        if (kind[r] == kNull) {
          sdslot_accum(tab, kDenseSmemSlots, v[r], has_v[r]);
        } else if (kind[r] == kSlot) {
          const int j = smem_dense_slot_from(tab, k[r], h[r], cur[r]);
          if (j >= 0)
            sdslot_accum(tab, (uint32_t)j, v[r], has_v[r]);
          else
            dslot_accum(p.table + k[r], v[r], has_v[r]);
        }
      }
    }
  }

  static __device__ void finish(Local&, const Params& p, unsigned char* sm, int ctid, int nct) {
    const SDTab tab = sdtab(sm);
    consumer_bar(nct);
    for (uint32_t j = ctid; j < kDenseSmemSlots; j += nct) {
      const unsigned int k1 = tab.k1[j];
      if (k1) dslot_merge(p.table + (k1 - 1), tab, j);
    }
    if (ctid == 0 && tab.count[kDenseSmemSlots]) dslot_merge(p.null_slot, tab, kDenseSmemSlots);
  }
};

// Ordered compaction of the dense table.  Slots are cut into chunks of
// kDenseChunk; pass 1 counts each chunk's live slots, one CTA turns the counts
// into output offsets (and writes the NULL group after the last key), pass 2
// writes each chunk's groups at its offset in slot (= key) order.
constexpr uint32_t kDenseChunk = 4096;
constexpr uint32_t kDenseCompactThreads = 256;

__global__ void __launch_bounds__(kDenseCompactThreads)
    dense_chunk_count_kernel(const DSlot* __restrict__ t, uint64_t slots, unsigned long long* chunk_off) {
  __shared__ unsigned int wsum[kDenseCompactThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kDenseChunk;
  unsigned int live = 0;
#pragma unroll 4
  for (uint32_t j = threadIdx.x; j < kDenseChunk; j += kDenseCompactThreads) {
    const uint64_t i = base + j;
    if (i < slots) live += __ldcs(&t[i].count) != 0;
  }
  live = __reduce_add_sync(0xffffffffu, live);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = live;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    for (int w = 0; w < kDenseCompactThreads / 32; ++w) tot += wsum[w];
    chunk_off[blockIdx.x] = tot;
  }
}

// One CTA: exclusive scan of the chunk counts in place, then the group count
// and the NULL group (written last, after every key).
__global__ void __launch_bounds__(1024)
    dense_chunk_scan_kernel(unsigned long long* chunk_off, uint64_t nchunks, const DSlot* null_slot,
                            fdb_group_i64* out, uint64_t cap_out, uint64_t* d_ngroups, int* err) {
  __shared__ unsigned long long wsum[32];
  __shared__ unsigned long long carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint64_t b = 0; b < nchunks; b += 1024) {
    const uint64_t i = b + threadIdx.x;
    const unsigned long long v = i < nchunks ? chunk_off[i] : 0;
    unsigned long long x = v;  // inclusive warp scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned long long w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const unsigned long long before = carry + (warp ? wsum[warp - 1] : 0) + x - v;
    if (i < nchunks) chunk_off[i] = before;
    __syncthreads();
    if (threadIdx.x == 1023) carry = before + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    unsigned long long total = carry;
    const DSlot ns = *null_slot;
    if (ns.count) {
      if (total < cap_out) {
        GSlot g{0, ns.count, ns.sum, ns.nmin, ns.max};
        out[total] = gslot_group(0, g);  // key INT64_MIN
      } else {
        atomicExch(err, kErrCapacity);
      }
      ++total;
    }
    *d_ngroups = total;
  }
}

__global__ void __launch_bounds__(kDenseCompactThreads)
    dense_emit_kernel(const DSlot* __restrict__ t, uint64_t slots, int64_t kmin,
                      const unsigned long long* __restrict__ chunk_off, fdb_group_i64* out, uint64_t cap_out,
                      int* err) {
  __shared__ unsigned int wcnt[kDenseCompactThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kDenseChunk;
  unsigned long long pos = chunk_off[blockIdx.x];
  for (uint32_t j = 0; j < kDenseChunk; j += kDenseCompactThreads) {
    const uint64_t i = base + j + threadIdx.x;
    DSlot s{0, 0.0, 0, 0};
    if (i < slots) s = t[i];
    const bool live = s.count != 0;
    const unsigned m = __ballot_sync(0xffffffffu, live);
    if (lane == 0) wcnt[warp] = __popc(m);
    __syncthreads();
    unsigned int before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kDenseCompactThreads / 32; ++w) {
      before += w < warp ? wcnt[w] : 0;
      total += wcnt[w];
    }
    if (live) {
      const unsigned long long o = pos + before + __popc(m & ((1u << lane) - 1u));
      if (o < cap_out) {
        GSlot g{0, s.count, s.sum, s.nmin, s.max};
        out[o] = gslot_group(((uint64_t)kmin + i) ^ (1ull << 63), g);
      } else {
        atomicExch(err, kErrCapacity);
      }
    }
    pos += total;
    __syncthreads();
  }
}

// ===========================================================================
// Launchers
// ===========================================================================
constexpr uint64_t kGbTilesPerCta = 8;

template <class Op, int NC, int TR, int STAGES, int NCW>
static void launch_stream_gb(Ctx& c, const fdb_dev_column* cols, uint64_t n,
                             const typename Op::Params& p, size_t op_smem) {
  StreamSrc<NC> src;
  const void* bases[NC];
  for (int i = 0; i < NC; ++i) {
    src.base[i] = static_cast<const unsigned char*>(cols[i].values);
    src.esize[i] = dtype_size(cols[i].dtype);
    bases[i] = cols[i].values;
  }
  src.n = n;
  src.m_end = stream_m_end(bases, NC, n);
  const int op_off = (int)stream_smem_bytes<NC, TR, STAGES>();
  const size_t smem = op_off + op_smem;
  auto kern = stream_kernel<Op, NC, TR, STAGES, NCW>;
  static PerDeviceOnce attr;  // per instantiation and device
  attr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024)); });
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (NCW + 1) * 32, smem));
  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  // At least kGbTilesPerCta tiles per CTA: on small inputs fewer CTAs means
  // fewer partials for the last CTA to fold.
  const uint64_t want =
      ntiles ? (ntiles + kGbTilesPerCta - 1) / kGbTilesPerCta : (n + NCW * 32 * 8 - 1) / (NCW * 32 * 8);
  constexpr int kKind =
      std::is_same<Op, GbDenseOp>::value || std::is_same<Op, GbHashOp>::value ? FDB_TUNE_GROUP_I64 : FDB_TUNE_GROUP;
  const int grid = tuned_grid(c.tune.op[kKind], c.sm_count, per_sm, 4, want, n);
  kern<<<grid, (NCW + 1) * 32, smem, c.stream>>>(src, p, c.d_err, op_off);
  FDB_CUDA(cudaGetLastError());
}

static void gb_fill_prog(PredProg& pp, const fdb_pred_term* prog, int nterms, int ncols, int col_shift) {
  if (nterms < 0 || nterms > FDB_MAX_TERMS) fail(FDB_E_ARG, "predicate has too many terms");
  std::memset(&pp, 0, sizeof(pp));
  pp.n = nterms;
  int depth = 0;
  for (int i = 0; i < nterms; ++i) {
    pp.t[i] = prog[i];
    const int k = prog[i].kind;
    if (k == FDB_TERM_AND || k == FDB_TERM_OR) {
      if (depth < 2) fail(FDB_E_ARG, "malformed predicate program");
      --depth;
    } else if (k == FDB_TERM_CMP || k == FDB_TERM_IS_NULL || k == FDB_TERM_IS_NOT_NULL ||
               k == FDB_TERM_CODE_SET) {
      if (prog[i].col < 0 || prog[i].col >= ncols) fail(FDB_E_ARG, "predicate column out of range");
      if (k == FDB_TERM_CODE_SET && !prog[i].code_set) fail(FDB_E_ARG, "CODE_SET without a set");
      pp.t[i].col += col_shift;
      ++depth;
    } else {
      fail(FDB_E_ARG, "unknown predicate term kind");
    }
  }
  if (nterms > 0 && depth != 1) fail(FDB_E_ARG, "malformed predicate program");
}

template <int NC, int NV, int NCW, int R, int ST>
static void launch_lane_fast_shape(Ctx& c, const fdb_dev_column* cols, uint64_t n, const GbCodesParams& p) {
  using Op = GbLaneFastOp<NV, NCW, R>;
  const size_t smem = (size_t)p.ngroups * (1 + NV) * Op::NCT * 8 + 16;
  launch_stream_gb<Op, NC, Op::kTileRows, ST, NCW>(c, cols, n, p, smem);
}

template <int NC, int NV>
static void launch_lane_fast(Ctx& c, const fdb_dev_column* cols, uint64_t n, const GbCodesParams& p) {
  if (n >= kLaneFastBigRows)
    launch_lane_fast_shape<NC, NV, FDB_LF_BIG_NCW, FDB_LF_BIG_R, FDB_LF_BIG_ST>(c, cols, n, p);
  else
    launch_lane_fast_shape<NC, NV, FDB_LF_SMALL_NCW, FDB_LF_SMALL_R, FDB_LF_SMALL_ST>(c, cols, n, p);
}

// Launch GbLaneFastOp when the query has its shape; false otherwise.
static bool gb_lane_fast(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n, const fdb_pred_term* prog,
                         int nterms, int key_col, const fdb_agg_spec* aggs, int naggs, GbCodesParams& p) {
  if (cols[key_col].validity) return false;
  p.f_cmp_col = -1;
  if (nterms == 1) {
    const fdb_pred_term& t = prog[0];
    if (t.kind != FDB_TERM_CMP || cols[t.col].dtype != FDB_FLOAT64 || cols[t.col].validity) return false;
    static const uint32_t kAccept[6] = {
        1u << 2,                       // ==
        (1u << 0) | (1u << 1) | (1u << 3),  // != (true for NaN)
        1u << 1,                       // <
        (1u << 1) | (1u << 2),         // <=
        1u << 3,                       // >
        (1u << 3) | (1u << 2)};        // >=
    if (t.op < FDB_EQ || t.op > FDB_GE) return false;
    p.f_cmp_col = t.col;
    p.f_cmp_mask = kAccept[t.op];
    p.f_lit = t.lit_type == FDB_FLOAT64 ? t.lit_f : (double)t.lit_i;
  } else if (nterms != 0) {
    return false;
  }
  p.f_f64 = 0;
  for (int a = 0; a < naggs; ++a) {
    const int f = aggs[a].func;
    if (f == FDB_AGG_COUNT_STAR) continue;
    if (f != FDB_AGG_SUM && f != FDB_AGG_AVG) return false;
    const fdb_dev_column& col = cols[aggs[a].col];
    if (col.validity || (col.dtype != FDB_FLOAT64 && col.dtype != FDB_INT64)) return false;
    const int s = p.vslot[a];
    if (s < 1 || s > 4 || p.cslot[a] >= 0) return false;
    p.f_vcol[s - 1] = aggs[a].col;
    if (col.dtype == FDB_FLOAT64) p.f_f64 |= 1u << (s - 1);
  }
  const int nv = p.nslots - 1;
  switch (ncols * 8 + nv) {
#define FDB_LF_CASE(NC, NV) \
  case NC * 8 + NV: launch_lane_fast<NC, NV>(c, cols, n, p); return true;
    FDB_LF_CASE(1, 0)
    FDB_LF_CASE(2, 0) FDB_LF_CASE(2, 1) FDB_LF_CASE(2, 2) FDB_LF_CASE(2, 3)
    FDB_LF_CASE(3, 0) FDB_LF_CASE(3, 1) FDB_LF_CASE(3, 2) FDB_LF_CASE(3, 3)
    FDB_LF_CASE(4, 0) FDB_LF_CASE(4, 1) FDB_LF_CASE(4, 2) FDB_LF_CASE(4, 3)
#undef FDB_LF_CASE
    default: return false;
  }
}

void op_group_by_codes(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                       const fdb_pred_term* prog, int nterms, int key_col, uint32_t dict_len,
                       const fdb_agg_spec* aggs, int naggs, fdb_agg_value* d_out,
                       int64_t* d_group_rows) {
  if (ncols < 1 || ncols > 4) fail(FDB_E_ARG, "between 1 and 4 input columns per GROUP BY scan");
  if (naggs < 1 || naggs > 4) fail(FDB_E_ARG, "between 1 and 4 aggregates per GROUP BY");
  if (key_col < 0 || key_col >= ncols || cols[key_col].dtype != FDB_UTF8)
    fail(FDB_E_TYPE, "dictionary GROUP BY needs a Utf8 key column");
  GbCodesParams p;
  std::memset(&p, 0, sizeof(p));
  for (int i = 0; i < ncols; ++i) {
    if (!cols[i].values && n > 0) fail(FDB_E_ARG, "column without values");
    p.cols[i] = DevCol{cols[i].dtype, cols[i].values, cols[i].validity, cols[i].validity_offset};
  }
  gb_fill_prog(p.prog, prog, nterms, ncols, 0);
  p.key_col = key_col;
  p.ngroups = dict_len + 1;
  p.naggs = naggs;
  int ns = 1;
  p.kind[0] = kAddU64;
  for (int a = 0; a < naggs; ++a) {
    const int f = aggs[a].func;
    p.func[a] = f;
    p.acol[a] = aggs[a].col;
    p.vslot[a] = -1;
    p.cslot[a] = -1;
    if (f == FDB_AGG_COUNT_STAR) continue;
    if (f < FDB_AGG_COUNT || f > FDB_AGG_MAX) fail(FDB_E_ARG, "aggregate not supported in GROUP BY");
    if (aggs[a].col < 0 || aggs[a].col >= ncols) fail(FDB_E_ARG, "aggregate column out of range");
    const int dt = cols[aggs[a].col].dtype;
    if (f != FDB_AGG_COUNT && dt == FDB_UTF8) fail(FDB_E_TYPE, "SUM/AVG/MIN/MAX need a numeric column");
    // A value count equals the group's row count when the column has no NULLs
    // (and, for MIN/MAX, no NaN to skip: integers), so it needs no slot.
    const bool own_count = cols[aggs[a].col].validity != nullptr || f == FDB_AGG_COUNT ||
                           ((f == FDB_AGG_MIN || f == FDB_AGG_MAX) && dt == FDB_FLOAT64);
    if (own_count) {
      p.cslot[a] = ns;
      p.kind[ns++] = kAddU64;
    }
    if (f == FDB_AGG_COUNT) continue;
    p.vslot[a] = ns;
    p.kind[ns++] = (f == FDB_AGG_SUM || f == FDB_AGG_AVG) ? (dt == FDB_FLOAT64 ? kAddF64 : kAddU64)
                                                          : kMaxU64;
  }
  p.nslots = ns;
  if ((uint64_t)p.ngroups * ns > kGbWarpTableEntries)
    fail(FDB_E_ARG, "dictionary too large for the code GROUP BY ((dict_len+1) x slots > 512)");
  const int max_grid = c.sm_count * 4;
  p.partials = static_cast<uint64_t*>(c.scratch_take((size_t)max_grid * p.ngroups * ns * 8));
  p.ticket = c.d_ticket;
  p.out = d_out;
  p.group_rows = d_group_rows;
  if ((uint64_t)p.ngroups * ns <= kLaneEntries && gb_lane_fast(c, cols, ncols, n, prog, nterms, key_col, aggs,
                                                               naggs, p))
    return;
  if ((uint64_t)p.ngroups * ns <= kLaneEntries) {
    // Lane-private tables: one table column per consumer thread.
    const size_t sm4 = (size_t)p.ngroups * ns * 128 * 8 + 16;
    const size_t smw = (size_t)p.ngroups * ns * (FDB_LANE_NCW3 * 32) * 8 + 16;
    switch (ncols) {
      case 1: launch_stream_gb<GbLaneOp, 1, 2048, 3, 4>(c, cols, n, p, sm4); break;
      case 2: launch_stream_gb<GbLaneOp, 2, 1024, 3, 4>(c, cols, n, p, sm4); break;
      case 3: launch_stream_gb<GbLaneOp, 3, FDB_LANE_TR3, FDB_LANE_ST3, FDB_LANE_NCW3>(c, cols, n, p, smw); break;
      default: launch_stream_gb<GbLaneOp, 4, 1024, 2, 4>(c, cols, n, p, sm4); break;
    }
    return;
  }
  switch (ncols) {
    case 1: launch_stream_gb<GbCodesOp, 1, 2048, 4, 8>(c, cols, n, p, GbCodesOp::kSmem); break;
    case 2: launch_stream_gb<GbCodesOp, 2, 1024, 4, 8>(c, cols, n, p, GbCodesOp::kSmem); break;
    case 3: launch_stream_gb<GbCodesOp, 3, 1024, 3, 8>(c, cols, n, p, GbCodesOp::kSmem); break;
    default: launch_stream_gb<GbCodesOp, 4, 1024, 3, 8>(c, cols, n, p, GbCodesOp::kSmem); break;
  }
}

static uint64_t gb_table_capacity(uint64_t expected_groups, double load_factor) {
  uint64_t cap = 1024;
  while ((double)cap * load_factor < (double)expected_groups) cap <<= 1;
  return cap;
}

GbSizing group_by_i64_sizing(Ctx& c, const fdb_dev_column& key, uint64_t n, uint64_t expected_groups) {
  GbSizing s;
  if (expected_groups) {
    s.groups = expected_groups;
    return s;
  }
  if (n == 0) {
    s.groups = 1;
    return s;
  }
  if (key.dtype != FDB_INT64) fail(FDB_E_TYPE, "hash GROUP BY needs an INT64 key");
  // A resident column's zone map bounds its keys without a pass over them.
  // The direct-addressed table is then taken when it has at most one slot per
  // two rows: its zeroing and compaction cost no more than the rows' reads.
  uint64_t table_rows = 0, first_row = 0;
  Column* col = c.zone_maps ? column_by_values(c, key.values, &table_rows, &first_row) : nullptr;
  int64_t zmin = 0, zmax = 0;
  if (col && col->dtype == FDB_INT64 && first_row + n <= table_rows &&
      zone_key_range(column_zones(c, *col), first_row, n, &zmin, &zmax)) {
    const uint64_t span = (uint64_t)zmax - (uint64_t)zmin;
    if (span < kDenseMaxSlots && span + 1 <= n / 2) {
      s.groups = span + 1;
      s.has_range = true;
      s.kmin = zmin;
      s.kmax = zmax;
      return s;
    }
  }
  const KeyStats k = key_stats_i64(c, key, n);
  // 15 % headroom over the sketch (about nine standard errors).
  s.groups = std::min<uint64_t>(n, k.distinct * 115 / 100 + 64);
  s.has_range = k.has_range;
  s.kmin = k.kmin;
  s.kmax = k.kmax;
  return s;
}

// Slots of a direct-addressed table for `s` (one per key value), or 0 when the
// hash table is the better choice: the range must be known and its table no
// more than twice the bytes of the hash table that the same groups would get.
static uint64_t gb_dense_slots(const GbSizing& s, double load_factor) {
  if (!s.has_range) return 0;
  const uint64_t span = (uint64_t)s.kmax - (uint64_t)s.kmin;
  if (span >= kDenseMaxSlots) return 0;
  const uint64_t slots = span + 1;
  const uint64_t hash_bytes = (gb_table_capacity(s.groups ? s.groups : 1, load_factor) + 1) * sizeof(GSlot);
  return slots * sizeof(DSlot) <= 2 * hash_bytes ? slots : 0;
}

static double gb_load_factor(double lf) { return (lf <= 0.0 || lf >= 1.0) ? 0.5 : lf; }

size_t group_by_i64_scratch(const GbSizing& s, double load_factor) {
  load_factor = gb_load_factor(load_factor);
  // Each scratch_take rounds up to 256 bytes.
  if (const uint64_t slots = gb_dense_slots(s, load_factor))
    return (slots + 1) * sizeof(DSlot) + (slots / kDenseChunk + 1) * 8 + 3 * 256;
  const uint64_t cap = gb_table_capacity(s.groups ? s.groups : 1, load_factor);
  return (cap + 1) * sizeof(GSlot) + 2 * 256;
}

void op_group_by_i64(Ctx& c, const fdb_dev_column& key, const fdb_dev_column& value, uint64_t n,
                     const fdb_pred_term* prog, int nterms, const fdb_dev_column* pred_cols,
                     int npred, const GbSizing& sz, double load_factor,
                     fdb_group_i64* d_groups, uint64_t capacity, uint64_t* d_ngroups) {
  if (key.dtype != FDB_INT64) fail(FDB_E_TYPE, "hash GROUP BY needs an INT64 key");
  if (value.dtype != FDB_FLOAT64 && value.dtype != FDB_INT64)
    fail(FDB_E_TYPE, "hash GROUP BY value must be FLOAT64 or INT64");
  if (npred < 0 || npred > 2) fail(FDB_E_ARG, "at most 2 predicate columns");
  // The CTA tables count rows in 32 bits; a CTA sees about n / grid rows.
  if (n / (uint64_t)c.sm_count >= (1ull << 31)) fail(FDB_E_ARG, "more than 2^31 rows per SM in one GROUP BY");
  load_factor = gb_load_factor(load_factor);
  fdb_dev_column all[4];
  all[0] = key;
  all[1] = value;
  for (int i = 0; i < npred; ++i) all[2 + i] = pred_cols[i];
  const int nc = 2 + npred;
  DevCol dcols[4];
  for (int i = 0; i < nc; ++i) {
    if (!all[i].values && n > 0) fail(FDB_E_ARG, "column without values");
    dcols[i] = DevCol{all[i].dtype, all[i].values, all[i].validity, all[i].validity_offset};
  }

  if (const uint64_t slots = gb_dense_slots(sz, load_factor)) {
    // Direct-addressed table: slot k - kmin per key value, NULL group after it.
    DSlot* table = static_cast<DSlot*>(c.scratch_take((slots + 1) * sizeof(DSlot)));
    const uint64_t nchunks = (slots + kDenseChunk - 1) / kDenseChunk;
    unsigned long long* chunk_off = static_cast<unsigned long long*>(c.scratch_take(nchunks * 8));
    FDB_CUDA(cudaMemsetAsync(table, 0, (slots + 1) * sizeof(DSlot), c.stream));
    GbDenseParams p;
    std::memset(&p, 0, sizeof(p));
    for (int i = 0; i < nc; ++i) p.cols[i] = dcols[i];
    gb_fill_prog(p.prog, prog, nterms, npred, 2);
    p.table = table;
    p.slots = slots;
    p.kmin = sz.kmin;
    p.null_slot = table + slots;
    p.err = c.d_err;
    if (n > 0) {
      switch (nc) {
        case 2: launch_stream_gb<GbDenseOp, 2, FDB_GBD_TR, FDB_GBD_ST, FDB_GBD_NCW>(c, all, n, p, GbDenseOp::kSmem); break;
        case 3: launch_stream_gb<GbDenseOp, 3, 1024, 2, FDB_GBD_NCW>(c, all, n, p, GbDenseOp::kSmem); break;
        default: launch_stream_gb<GbDenseOp, 4, 512, 3, FDB_GBD_NCW>(c, all, n, p, GbDenseOp::kSmem); break;
      }
    }
    dense_chunk_count_kernel<<<(unsigned)nchunks, kDenseCompactThreads, 0, c.stream>>>(table, slots, chunk_off);
    FDB_CUDA(cudaGetLastError());
    dense_chunk_scan_kernel<<<1, 1024, 0, c.stream>>>(chunk_off, nchunks, table + slots, d_groups, capacity,
                                                      d_ngroups, c.d_err);
    FDB_CUDA(cudaGetLastError());
    dense_emit_kernel<<<(unsigned)nchunks, kDenseCompactThreads, 0, c.stream>>>(table, slots, sz.kmin, chunk_off,
                                                                               d_groups, capacity, c.d_err);
    FDB_CUDA(cudaGetLastError());
    return;
  }

  const uint64_t cap = gb_table_capacity(sz.groups ? sz.groups : (n ? n : 1), load_factor);
  const size_t tbytes = cap * sizeof(GSlot);
  GSlot* table = static_cast<GSlot*>(c.scratch_take(tbytes + sizeof(GSlot)));
  GSlot* null_slot = table + cap;
  FDB_CUDA(cudaMemsetAsync(table, 0, tbytes + sizeof(GSlot), c.stream));
  unsigned long long* counter = static_cast<unsigned long long*>(c.scratch_take(8));
  FDB_CUDA(cudaMemsetAsync(counter, 0, 8, c.stream));

  GbHashParams p;
  std::memset(&p, 0, sizeof(p));
  for (int i = 0; i < nc; ++i) p.cols[i] = dcols[i];
  gb_fill_prog(p.prog, prog, nterms, npred, 2);
  p.table = table;
  p.mask = cap - 1;
  p.null_slot = null_slot;
  p.err = c.d_err;
  if (n > 0) {
    switch (nc) {
      // NCW = GbHashOp::kNW: the operator keeps one spill ring per consumer warp.
      case 2: launch_stream_gb<GbHashOp, 2, 1024, 3, 8>(c, all, n, p, GbHashOp::kSmem); break;
      case 3: launch_stream_gb<GbHashOp, 3, 1024, 2, 8>(c, all, n, p, GbHashOp::kSmem); break;
      default: launch_stream_gb<GbHashOp, 4, 512, 3, 8>(c, all, n, p, GbHashOp::kSmem); break;
    }
  }
  const unsigned blocks = (unsigned)umin64((cap + 255) / 256 + 1, (uint64_t)c.sm_count * 8);
  gb_hash_compact_kernel<<<blocks, 256, 0, c.stream>>>(table, cap, null_slot, d_groups, capacity,
                                                       counter, c.d_err);
  FDB_CUDA(cudaGetLastError());
  FDB_CUDA(cudaMemcpyAsync(d_ngroups, counter, 8, cudaMemcpyDeviceToDevice, c.stream));
}

}  // namespace fdb
