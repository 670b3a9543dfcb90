// Serving loop: continuous batching of queries over device-resident tables.
//
// A scheduler thread owns `slots` launch slots.  Each slot has a stream, a
// pinned input buffer (a batch header and one descriptor per query), a pinned
// output buffer (one result per query) and a CUDA graph captured once:
//   H2D descriptors -> zero results -> serve_kernel -> serve_topk_kernel ->
//   serve_finish_kernel -> D2H results (+ the slot's error word).
// Whenever a slot is free and queries are waiting, the scheduler admits them
// in arrival order while the device-memory budget allows (resident tables plus
// what admitted queries hold) up to max_batch, writes their descriptors and
// replays the slot's graph; batches on different slots overlap on the GPU.  A
// slot's results are handed out when its completion event fires.
//
// serve_kernel is persistent and scans shared: the batch's COUNT, GROUP and
// JOIN queries are grouped by the table they read, and each group's rows are
// cut into units that fill one pipeline stage (22 KB: 2816 rows of one 8-byte
// column, 1024 rows of a GROUP or JOIN group's columns).  A
// CTA's producer warp claims units from one counter and stages their columns
// into a ring of shared-memory buffers with bulk copies; its consumer warps
// then probe a join group's rows once (whether a build row matches does not
// depend on the query) and evaluate every query of the group that covers the
// unit from shared memory, each with its own predicate.  HBM therefore sees
// each table once per batch, not once per query.  A CTA folds its partial
// results in shared memory and adds them to the global results when it ends.
// serve_topk_kernel then runs the top-k queries over their own rows in
// kServeTile-row units from a second counter: a CTA keeps a list per warp while
// its consecutive units belong to one query and publishes its k best (below
// the query's running bound) as candidates when it moves on;
// serve_finish_kernel reduces them, one CTA per query.  Top-k lives in its own
// kernel so that each kernel gets the registers and CTAs per SM it needs.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "join_table.cuh"
#include "topk_warp.cuh"

namespace fdb {

constexpr int kServeThreads = 256;                 // consumer threads (8 warps)
constexpr int kServeWarps = kServeThreads / 32;
constexpr int kServeBlock = kServeThreads + 32;    // + the producer warp
constexpr uint32_t kServeTile = 8192;
constexpr int kServeMaxBatch = 256;
#ifndef FDB_SERVE_CTAS
#define FDB_SERVE_CTAS 3
#endif
// A batch's join, scan and top-k kernels run side by side (1) or one after
// another (0).
#ifndef FDB_SERVE_FORK
#define FDB_SERVE_FORK 1
#endif
// Long-scan batches leave SM slots to the other launch slots under load (1).
#ifndef FDB_SERVE_YIELD
#define FDB_SERVE_YIELD 0
#endif
// Queries waiting at which the short-scan slots hold off while a long-scan
// batch runs (0: never).
#ifndef FDB_SERVE_HOLD
#define FDB_SERVE_HOLD 4
#endif
constexpr int kServeHoldBacklog = FDB_SERVE_HOLD;
constexpr int kServeCtasPerSm = FDB_SERVE_CTAS;
#ifndef FDB_SERVE_JOIN_CTAS
#define FDB_SERVE_JOIN_CTAS 2
#endif
constexpr int kServeJoinCtasPerSm = FDB_SERVE_JOIN_CTAS;
constexpr int kServeTopkCtasPerSm = 2;
#ifndef FDB_SERVE_STAGES
#define FDB_SERVE_STAGES 2
#endif
constexpr int kServeStages = FDB_SERVE_STAGES;
// A stage holds one unit of a shared group: its columns c0 (8 B/row), c1 (0,
// 4 or 8 B/row), c2 (0 or 8 B/row) and, for a join, the match counts (4 B/row),
// one after another; a unit is as many rows (a multiple of 256) as fit.
#ifndef FDB_SERVE_STAGE_KB
#define FDB_SERVE_STAGE_KB 22
#endif
constexpr size_t kShareStage = FDB_SERVE_STAGE_KB * 1024;
// The join instance's stages are larger: a join unit is one probe pass (each
// thread kProbeIlp rows, all their L2 reads in flight together), and each
// unit costs a CTA one L2 round trip, so more rows per unit means more rows
// per round trip.
#ifndef FDB_SERVE_JOIN_STAGE_KB
#define FDB_SERVE_JOIN_STAGE_KB 40
#endif
constexpr size_t kShareStageJoin = FDB_SERVE_JOIN_STAGE_KB * 1024;
template <bool JOIN>
__host__ __device__ constexpr size_t share_stage() { return JOIN ? kShareStageJoin : kShareStage; }
// Barrier block: full[stages], empty[stages], the unit of each stage, and the
// columns each stage's consumers must load themselves (bit c: column c).
constexpr size_t kServeBar = 128;
constexpr size_t kShareSmem = kServeBar + kServeStages * kShareStage;
constexpr size_t kShareSmemJoin = kServeBar + kServeStages * kShareStageJoin;
static_assert(kServeStages * (8 + 8 + 8 + 4) <= kServeBar, "barrier block");

struct ServeQ {            // device descriptor of one query
  int32_t kind, k;
  uint64_t n, tile0;
  double thr;
  const void* c0;
  const void* c1;
  const void* c2;
  uint32_t dict_len, _pad;
  const JSlot* slots;
  const unsigned int* cnt;
  uint64_t cap;
  int32_t unique, _pad2;
};

struct ServeRes {          // device result of one query (and its host copy)
  unsigned long long count;
  long long sum;
  unsigned long long nbound;   // TOPK: ~(best published k-th order key); 0 = none
  unsigned int ncand, _pad;
  unsigned long long gcount[FDB_SERVE_MAX_GROUPS];
  double gsum0[FDB_SERVE_MAX_GROUPS];
  long long gsum2[FDB_SERVE_MAX_GROUPS];
  uint32_t rows[FDB_SERVE_MAX_K];
};

struct ServeG {             // a group of queries that read the same table
  const void* c0;
  const void* c1;
  const void* c2;
  uint32_t q0, nq;          // its queries, by rows descending
  uint64_t max_n, unit0;
  uint32_t unit_rows;       // rows per unit
  uint32_t off1, off2, offm;  // stage byte offsets of c1, c2 and the join match counts
  int32_t c1_bytes;         // 0 (not read), 4 (dictionary codes) or 8
  int32_t load_c2;
  int32_t join;             // c0 holds probe keys for the table below
  int32_t unique;
  const JSlot* slots;
  const unsigned int* cnt;
  uint64_t cap;
  int64_t dmin;             // smallest build key (dense table: key k lives in slot k - dmin)
  int32_t dense;
  int32_t ngroupq;          // GROUP queries in the group
  int32_t ncountq, njoinq;  // COUNT and JOIN queries in the group
  int32_t _pad4;
  uint64_t span;            // keys outside [dmin, dmin + span) have no slot (0: no range)
};

struct ServeHeader {
  int32_t nq, ngroups;
  int32_t topk0, _pad;      // top-k queries are descriptors [topk0, nq)
  uint64_t shared_units, total_units;
  uint64_t join_units;      // join groups come first: units [0, join_units) are theirs
  int32_t join_groups, _pad2;
  // CTAs of the join, scan and top-k instances that take part (0: all).  The
  // others end at once, leaving their SM slots to another slot's batch.
  int32_t cta_limit[3], _pad3;
};

struct ServeArgs {
  const ServeHeader* hdr;
  const ServeQ* q;
  const ServeG* g;
  ServeRes* res;
  unsigned int* claim;       // zero at launch (after res in the same memset)
  uint64_t* cand_k;          // [kServeMaxBatch][cand_cap]
  uint32_t* cand_r;
  uint32_t cand_cap;
  int* err;
};

// Shared queries whose partial results a CTA keeps in shared memory (the
// first ones of a batch; later ones add theirs per unit).
#ifndef FDB_SERVE_CACHE_Q
#define FDB_SERVE_CACHE_Q 24
#endif
constexpr int kServeCacheQ = FDB_SERVE_CACHE_Q;
// GROUP queries one unit evaluates together, and the fewest worth it (with
// fewer, the per-query fold is faster than the binned atomics).
constexpr int kShareGroupQ = 32;
constexpr int kShareGroupMin = 4;

struct ServeSmem {                      // the shared-scan kernel
  uint64_t gstart[kServeMaxBatch + 1];  // unit0 of each shared group
  // The CTA's partial results of the first kServeCacheQ queries, added to the
  // global results once, when the CTA ends (per-unit global atomics would all
  // meet on the few words of a query's result).
  unsigned long long acount[kServeCacheQ];
  unsigned long long asum[kServeCacheQ];
  unsigned long long agcount[kServeCacheQ][FDB_SERVE_MAX_GROUPS];
  double agsum0[kServeCacheQ][FDB_SERVE_MAX_GROUPS];
  long long agsum2[kServeCacheQ][FDB_SERVE_MAX_GROUPS];
  // GROUP BY partials of one unit, per warp (written by one lane at a time).
  unsigned long long gcount[kServeWarps][FDB_SERVE_MAX_GROUPS];
  double gsum0[kServeWarps][FDB_SERVE_MAX_GROUPS];
  long long gsum2[kServeWarps][FDB_SERVE_MAX_GROUPS];
  // GROUP queries evaluated together over one unit (serve_group_shared):
  // their thresholds ascending, their indices, which queries those are, and
  // the unit's rows binned by (code, number of thresholds below the score).
  double sthr[kShareGroupQ];
  uint32_t sqid[kShareGroupQ];
  uint32_t taken[kServeMaxBatch / 32];
  int32_t sna;
  unsigned int wcnt[kServeWarps][kShareGroupQ];        // COUNT bins, per warp
  unsigned long long wjc[kServeWarps][kShareGroupQ];   // JOIN bins, per warp: matches
  unsigned long long wjp[kServeWarps][kShareGroupQ];   //   and payload sums
  unsigned int dcount[FDB_SERVE_MAX_GROUPS * kShareGroupQ];
  double dsum0[FDB_SERVE_MAX_GROUPS * kShareGroupQ];
  unsigned long long dsum2[FDB_SERVE_MAX_GROUPS * kShareGroupQ];
};

struct TopkSmem {                       // the top-k and finish kernels
  uint64_t start[kServeMaxBatch + 1];   // unit0 of each top-k query
  uint64_t tkeys[kServeWarps][32];
  uint32_t trows[kServeWarps][32];
  unsigned int t;
};

// Barriers among the consumer warps only (named barrier 1): the producer warp
// never joins them.
__device__ __forceinline__ void serve_bar() {
  asm volatile("bar.sync 1, %0;" ::"r"(kServeThreads) : "memory");
}
// True on every consumer thread when `x` holds on any of them.
__device__ __forceinline__ bool serve_bar_any(bool x) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)x), "r"(kServeThreads)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ int serve_find(const uint64_t* start, int nq, uint64_t t) {
  int lo = 0, hi = nq;  // start[lo] <= t < start[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (start[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

// Merge every warp's list into warp 0 (sorted-list merges, log2(warps) levels).
__device__ void serve_tree_merge(TopkSmem& sm, RTLocal& s, uint32_t k, int warp, int lane) {
  for (int half = kServeWarps / 2; half >= 1; half >>= 1) {
    serve_bar();
    if (warp >= half && warp < 2 * half) {
      const bool in = (uint32_t)lane < k;
      sm.tkeys[warp][lane] = in ? s.lk : ~0ull;
      sm.trows[warp][lane] = in ? s.lr : 0xFFFFFFFFu;
    }
    serve_bar();
    if (warp < half) rt_merge_sorted(s, k, sm.tkeys[warp + half][lane], sm.trows[warp + half][lane], lane);
  }
  serve_bar();
}

__device__ __forceinline__ void rt_reset(RTLocal& s) {
  s.lk = ~0ull;
  s.lr = 0xFFFFFFFFu;
  s.tk = ~0ull;
  s.tr = 0xFFFFFFFFu;
  s.steps = 0;
}

// Publish this CTA's top-k state for query qi (all consumer threads call; ends with a barrier).
__device__ void serve_publish(const ServeArgs& a, const ServeQ q, int qi, TopkSmem& sm, RTLocal& tl) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  ServeRes& r = a.res[qi];
  const uint32_t k = (uint32_t)q.k;
  serve_tree_merge(sm, tl, k, warp, lane);
  if (warp == 0) {
    const uint64_t kk = __shfl_sync(0xffffffffu, tl.lk, k - 1);
    const uint32_t kr = __shfl_sync(0xffffffffu, tl.lr, k - 1);
    if (lane == 0 && !(kk == ~0ull && kr == 0xFFFFFFFFu)) atomicMax(&r.nbound, ~kk);
    const uint64_t bound = ~*reinterpret_cast<volatile unsigned long long*>(&r.nbound);
    const bool emit = (uint32_t)lane < k && !(tl.lk == ~0ull && tl.lr == 0xFFFFFFFFu) && tl.lk <= bound;
    const unsigned m = __ballot_sync(0xffffffffu, emit);
    if (m) {
      unsigned int base = 0;
      if (lane == 0) base = atomicAdd(&r.ncand, (unsigned int)__popc(m));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (emit) {
        const uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
        if (pos < a.cand_cap) {
          a.cand_k[(size_t)qi * a.cand_cap + pos] = tl.lk;
          a.cand_r[(size_t)qi * a.cand_cap + pos] = tl.lr;
        } else {
          atomicExch(a.err, kErrCapacity);
        }
      }
    }
  }
  rt_reset(tl);
  serve_bar();
}

// Rows [r0, r1) of a top-k query: WHERE c0 < thr ORDER BY c0 DESC into the warp lists.
__device__ __forceinline__ void serve_topk_tile(const ServeQ q, uint64_t r0, uint64_t r1, RTLocal& tl) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t* c0 = static_cast<const uint64_t*>(q.c0);
  const uint32_t k = (uint32_t)q.k;
  for (uint64_t b = r0 + (uint64_t)warp * 256; b < r1; b += 256 * kServeWarps) {
    uint64_t v[8];
    uint32_t vm = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint64_t i = b + j * 32 + lane;
      v[j] = 0;
      if (i < r1) {
        v[j] = __ldcs(c0 + i);
        vm |= 1u << j;
      }
    }
    const double tv = f64_from_ord_key(~tl.tk);  // the threshold's value (DESC keys)
    uint32_t pm = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double x = __longlong_as_double((long long)v[j]);
      if (x < q.thr && !(x < tv)) pm |= 1u << j;
    }
    pm &= vm;
    if (!__any_sync(0xffffffffu, pm != 0u)) continue;
    uint64_t key[8];
    uint32_t row[8];
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      key[j] = wt_key<FDB_FLOAT64, true>(v[j]);
      row[j] = (uint32_t)(b + j * 32 + lane);
      if (((pm >> j) & 1u) && kr_le(key[j], row[j], tl.tk, tl.tr)) m |= 1u << j;
    }
    if (__any_sync(0xffffffffu, m != 0u)) rt_offer<8>(tl, k, key, row, m, lane);
  }
}

// Copy rows [r0, r0 + rows) of a column (esize 4 or 8) into shared memory
// with plain loads (consumer threads; columns the bulk copies cannot take).
__device__ __forceinline__ void share_load(unsigned char* dst, const void* src, uint64_t r0, uint32_t rows, int esize) {
  const unsigned char* s = static_cast<const unsigned char*>(src) + r0 * esize;
  const uint32_t bytes = rows * (uint32_t)esize;
  uint32_t done = 0;
  if (((uintptr_t)s & 15u) == 0) {
    const uint32_t nv = bytes / 16;
    for (uint32_t i = threadIdx.x; i < nv; i += kServeThreads)
      reinterpret_cast<uint4*>(dst)[i] = __ldcs(reinterpret_cast<const uint4*>(s) + i);
    done = nv * 16;
  }
  if (esize == 8) {
    for (uint32_t i = done / 8 + threadIdx.x; i < rows; i += kServeThreads)
      reinterpret_cast<uint64_t*>(dst)[i] = __ldcs(reinterpret_cast<const unsigned long long*>(s) + i);
  } else {
    for (uint32_t i = done / 4 + threadIdx.x; i < rows; i += kServeThreads)
      reinterpret_cast<uint32_t*>(dst)[i] = __ldcs(reinterpret_cast<const unsigned int*>(s) + i);
  }
}

// Probe every staged row of a join group once: row i's build matches go to
// m[i] and their payload sum replaces its key in s0[i].  A direct-addressed
// table is read with kProbeIlp rows per thread in flight together (a join
// unit is one such pass); a hashed table with kHashIlp rows at a time, one
// 32-byte slot pair (one L2 sector) per row per round, so their L2 round
// trips overlap.
#ifndef FDB_SERVE_PROBE_ILP
#define FDB_SERVE_PROBE_ILP 8
#endif
constexpr int kProbeIlp = FDB_SERVE_PROBE_ILP;
constexpr int kHashIlp = 4;
static_assert(kProbeIlp % kHashIlp == 0, "a probe pass is whole hashed passes");
#ifndef FDB_SERVE_PAIR_ILP
#define FDB_SERVE_PAIR_ILP 2
#endif

// The direct-addressed probe of serve_probe_rows: per row only its slot index
// and the slot read are kept across the loads (the key is read again from
// shared memory to compare), so kProbeIlp reads fit in registers.
__device__ __forceinline__ void serve_probe_dense(const ServeG& g, const JoinMode& mode, uint64_t* s0, uint32_t* m,
                                                  uint32_t rows, bool fused, const double* v, double lim,
                                                  unsigned long long* c, unsigned long long* psum) {
  const uint64_t pol = l2_evict_last_policy();
  for (uint32_t base = 0; base < rows; base += kProbeIlp * kServeThreads) {
    uint32_t hs[kProbeIlp];
    uint32_t todo = 0;
#pragma unroll
    for (int j = 0; j < kProbeIlp; ++j) {
      const uint32_t i = base + j * kServeThreads + threadIdx.x;
      hs[j] = 0;
      if (i >= rows || !(v[i] < lim)) continue;
      const int64_t key = (int64_t)s0[i];
      if (key == INT64_MIN) continue;  // resolved below
      const uint64_t h = join_home(mode, key, (uint64_t)key ^ (1ull << 63));
      if (h < g.cap) {  // keys outside the build keys' span read nothing
        hs[j] = (uint32_t)h;
        todo |= 1u << j;
      }
    }
    JSlot sl[kProbeIlp];
#pragma unroll
    for (int j = 0; j < kProbeIlp; ++j) {
      sl[j].key = 0;
      sl[j].psum = 0;
      if ((todo >> j) & 1u)
        asm volatile("ld.global.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
                     : "=l"(sl[j].key), "=l"(sl[j].psum)
                     : "l"(g.slots + hs[j]), "l"(pol));
    }
#pragma unroll
    for (int j = 0; j < kProbeIlp; ++j) {
      const uint32_t i = base + j * kServeThreads + threadIdx.x;
      if (i >= rows) continue;
      uint32_t mc = 0;
      uint64_t ps = 0;
      if ((todo >> j) & 1u) {
        if (sl[j].key == (s0[i] ^ (1ull << 63))) {
          mc = g.unique ? 1u : g.cnt[hs[j]];
          ps = sl[j].psum;
        }
      } else if (v[i] < lim && (int64_t)s0[i] == INT64_MIN && g.cnt[g.cap] != 0u) {
        mc = g.cnt[g.cap];  // the NULL-group slot after the table
        ps = g.slots[g.cap].psum;
      }
      if (fused) {
        *c += mc;
        *psum += mc ? ps : 0ull;
      } else {
        m[i] = mc;
        s0[i] = ps;
      }
    }
  }
  if (!fused) serve_bar();
}

// Only rows with v[i] < lim are probed (lim: the largest value limit of the
// queries that read the unit; a row at or above it counts for none of them,
// so its match count and payload sum are left 0).  fused (a join group with
// one query): the matches and payload sums are added to *c / *psum instead of
// being written back for the queries to read.
__device__ void serve_probe_rows(const ServeG g, uint64_t* s0, uint32_t* m, uint32_t rows, bool fused,
                                 const double* v, double lim, unsigned long long* c, unsigned long long* psum) {
  JoinMode mode;
  mode.dmin = g.dmin;
  mode.dense = g.dense;
  mode.shift = join_shift(g.cap);
  mode.span = g.span;
  if (mode.dense) {
    serve_probe_dense(g, mode, s0, m, rows, fused, v, lim, c, psum);
    return;
  }
  const uint64_t mask = g.cap - 1;
  const uint64_t pol = l2_evict_last_policy();
  for (uint32_t base = 0; base < rows; base += kHashIlp * kServeThreads) {
    uint64_t sk[kHashIlp], h[kHashIlp], ps[kHashIlp];
    uint32_t at[kHashIlp];
    uint32_t todo = 0;
#pragma unroll
    for (int j = 0; j < kHashIlp; ++j) {
      const uint32_t i = base + j * kServeThreads + threadIdx.x;
      at[j] = kNoSlot;
      ps[j] = 0;
      sk[j] = 0;
      h[j] = 0;
      if (i >= rows) continue;
      if (!(v[i] < lim)) continue;
      const int64_t key = (int64_t)s0[i];
      if (key == INT64_MIN) {
        if (g.cnt[g.cap] != 0u) {
          at[j] = (uint32_t)g.cap;
          ps[j] = g.slots[g.cap].psum;
        }
        continue;
      }
      sk[j] = (uint64_t)key ^ (1ull << 63);
      h[j] = join_home(mode, key, sk[j]);
      if (h[j] <= mask) todo |= 1u << j;  // keys outside the build keys' range read nothing
    }
    // Hashed table: rounds over slot pairs, kPairIlp rows' pairs in flight at a
    // time (fewer than kHashIlp, to keep the registers of the pairs down).
    constexpr int kPairIlp = FDB_SERVE_PAIR_ILP;
#pragma unroll
    for (int j0 = 0; j0 < kHashIlp; j0 += kPairIlp)
    for (uint64_t round = 0; ((todo >> j0) & ((1u << kPairIlp) - 1u)) && round <= mask; ++round) {
      JSlot lo[kPairIlp], hi[kPairIlp];
#pragma unroll
      for (int jj = 0; jj < kPairIlp; ++jj) {
        const int j = j0 + jj;
        if ((todo >> j) & 1u)
          asm volatile("ld.global.L2::cache_hint.v4.u64 {%0, %1, %2, %3}, [%4], %5;"
                       : "=l"(lo[jj].key), "=l"(lo[jj].psum), "=l"(hi[jj].key), "=l"(hi[jj].psum)
                       : "l"(g.slots + (h[j] & ~1ull)), "l"(pol));
      }
#pragma unroll
      for (int jj = 0; jj < kPairIlp; ++jj) {
        const int j = j0 + jj;
        if (!((todo >> j) & 1u)) continue;
        const bool even = (h[j] & 1ull) == 0;
        const bool hit0 = even && lo[jj].key == sk[j];
        const bool stop0 = even && (lo[jj].key == sk[j] || lo[jj].key == 0ull);
        const bool hit1 = !stop0 && hi[jj].key == sk[j];
        if (hit0 || hit1) {
          at[j] = (uint32_t)((h[j] & ~1ull) + (hit1 ? 1 : 0));
          ps[j] = hit1 ? hi[jj].psum : lo[jj].psum;
          todo &= ~(1u << j);
        } else if (stop0 || hi[jj].key == 0ull) {
          todo &= ~(1u << j);
        } else {
          h[j] = ((h[j] & ~1ull) + 2) & mask;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < kHashIlp; ++j) {
      const uint32_t i = base + j * kServeThreads + threadIdx.x;
      if (i >= rows) continue;
      const uint32_t mc = at[j] == kNoSlot ? 0u : (g.unique ? 1u : g.cnt[at[j]]);
      if (fused) {
        *c += mc;
        *psum += mc ? ps[j] : 0ull;
      } else {
        m[i] = mc;
        s0[i] = ps[j];
      }
    }
  }
  if (!fused) serve_bar();
}

// The staged columns of a shared group's unit: column c at stage byte off[c].
struct ShareCols {
  const void* src[3];
  int esize[3];  // 0: not read
  uint32_t off[3];
};

__device__ __forceinline__ ShareCols share_cols(const ServeG& g) {
  ShareCols c;
  c.src[0] = g.c0;
  c.esize[0] = 8;
  c.off[0] = 0;
  c.src[1] = g.c1;
  c.esize[1] = g.c1_bytes;
  c.off[1] = g.off1;
  c.src[2] = g.c2;
  c.esize[2] = g.load_c2 ? 8 : 0;
  c.off[2] = g.off2;
  return c;
}

// Queries of kind `kind` in group g that cover all `rows` rows of this unit
// (up to kShareGroupQ, in list order) are evaluated together in one pass over
// the rows: their keys (the threshold; a JOIN's value limit, threshold / 100)
// go to sm.sthr ascending and their indices to sm.sqid, sm.sna is their number
// (0 when fewer than kShareGroupMin qualify) and sm.taken marks them.  Ends
// with a consumer barrier.
__device__ void serve_pick(const ServeArgs& a, const ServeG& g, uint64_t r0, uint32_t rows, int kind, ServeSmem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  if (warp == 0) {
    int na = 0;
    for (uint32_t c0 = 0; c0 < g.nq && na < kShareGroupQ; c0 += 32) {
      const uint32_t qi = g.q0 + c0 + lane;
      bool el = false;
      double key = 0.0;
      if (c0 + lane < g.nq) {
        const ServeQ& q = a.q[qi];
        el = q.kind == kind && q.n >= r0 + rows;
        key = kind == FDB_SERVE_JOIN ? q.thr / 100.0 : q.thr;
      }
      const unsigned m = __ballot_sync(0xffffffffu, el);
      const int pos = na + __popc(m & below);
      if (el && pos < kShareGroupQ) {
        sm.sthr[pos] = key;
        sm.sqid[pos] = qi;
      }
      na += __popc(m);
    }
    if (na > kShareGroupQ) na = kShareGroupQ;
    if (na < kShareGroupMin) na = 0;
    __syncwarp();
    // Rank the keys (ties by position) and store them ascending.
    const double t = lane < na ? sm.sthr[lane] : 0.0;
    const uint32_t q = lane < na ? sm.sqid[lane] : 0u;
    int rank = 0;
    for (int j = 0; j < na; ++j) {
      const double tj = __shfl_sync(0xffffffffu, t, j);
      rank += (tj < t || (tj == t && j < lane)) ? 1 : 0;
    }
    __syncwarp();
    if (lane < na) {
      sm.sthr[rank] = t;
      sm.sqid[rank] = q;
      atomicOr(&sm.taken[(q - g.q0) >> 5], 1u << ((q - g.q0) & 31));
    }
    if (lane == 0) sm.sna = na;
  }
  serve_bar();
}

// Number of the na ascending keys below v (strict: none for NaN).
__device__ __forceinline__ int serve_rank_below(const double* keys, int na, double v) {
  int lo = 0, hi = na;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Adds a shared query's partial result: to the CTA's copy when the query's
// partials are kept in shared memory, else to the global result.
__device__ __forceinline__ void serve_add_count(const ServeArgs& a, ServeSmem& sm, uint32_t qi, unsigned long long c,
                                                unsigned long long ps, bool with_sum) {
  if (qi < (uint32_t)kServeCacheQ) {
    sm.acount[qi] += c;
    if (with_sum) sm.asum[qi] += ps;
  } else {
    if (c) atomicAdd(&a.res[qi].count, c);
    if (with_sum && ps) atomicAdd(reinterpret_cast<unsigned long long*>(&a.res[qi].sum), ps);
  }
}

// COUNT(*) WHERE score > t for the picked COUNT queries: a row above exactly k
// thresholds counts for queries 0..k-1, so it goes to bin k-1 and query j's
// count is the sum of bins j..na-1.  Bins are per warp; the lowest lane of the
// lanes that share a bin adds their number.
__device__ void serve_count_shared(const ServeArgs& a, uint32_t rows, const uint64_t* s0, ServeSmem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int na = sm.sna;
  sm.wcnt[warp][lane] = 0;
  __syncwarp();
  for (uint32_t b = (uint32_t)warp * 32; b < rows; b += kServeThreads) {
    const uint32_t i = b + lane;
    int k = 0;
    if (i < rows) k = serve_rank_below(sm.sthr, na, __longlong_as_double((long long)s0[i]));
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    if (k > 0 && lane == __ffs(peers) - 1) sm.wcnt[warp][k - 1] += (unsigned)__popc(peers);
    __syncwarp();
  }
  serve_bar();
  if (warp == 0) {
    unsigned long long c = 0;
    if (lane < na)
      for (int w = 0; w < kServeWarps; ++w) c += sm.wcnt[w][lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {  // suffix sums: lane j gets bins j..31
      const unsigned long long x = __shfl_down_sync(0xffffffffu, c, o);
      if (lane + o < 32) c += x;
    }
    if (lane < na) serve_add_count(a, sm, sm.sqid[lane], c, 0, false);
  }
  serve_bar();
}

// The picked JOIN queries (WHERE value < limit, limits ascending): a row whose
// value is at or above exactly k limits counts for queries k..na-1, so its
// matches and payload sum go to bin k and query j's result is the sum of bins
// 0..j.  Bins are per warp; lanes that share a bin add their row in rank
// rounds with plain stores.  A NaN value is under no limit.
__device__ void serve_join_shared(const ServeArgs& a, uint32_t rows, const uint64_t* s0, const double* v,
                                  const uint32_t* smm, ServeSmem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int na = sm.sna;
  sm.wjc[warp][lane] = 0;
  sm.wjp[warp][lane] = 0;
  __syncwarp();
  for (uint32_t b = (uint32_t)warp * 32; b < rows; b += kServeThreads) {
    const uint32_t i = b + lane;
    int k = na;  // na: in no query
    if (i < rows) {
      const double x = v[i];
      if (!isnan(x)) {
        int lo = 0, hi = na;  // limits at or below x
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (sm.sthr[mid] <= x)
            lo = mid + 1;
          else
            hi = mid;
        }
        k = lo;
      }
    }
    const bool in = k < na;
    const unsigned peers = __match_any_sync(0xffffffffu, in ? k : -1);
    const unsigned rank = __popc(peers & below);
    const unsigned rounds = __reduce_max_sync(0xffffffffu, in ? (unsigned)__popc(peers) : 0u);
    unsigned long long mc = 0, ps = 0;
    if (in) {
      mc = smm[i];
      ps = s0[i];
    }
    for (unsigned r = 0; r < rounds; ++r) {
      if (in && rank == r) {
        sm.wjc[warp][k] += mc;
        sm.wjp[warp][k] += ps;
      }
      __syncwarp();
    }
  }
  serve_bar();
  if (warp == 0) {
    unsigned long long c = 0, ps = 0;
    if (lane < na)
      for (int w = 0; w < kServeWarps; ++w) {
        c += sm.wjc[w][lane];
        ps += sm.wjp[w][lane];
      }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {  // prefix sums: lane j gets bins 0..j
      const unsigned long long xc = __shfl_up_sync(0xffffffffu, c, o);
      const unsigned long long xp = __shfl_up_sync(0xffffffffu, ps, o);
      if (lane >= o) {
        c += xc;
        ps += xp;
      }
    }
    if (lane < na) serve_add_count(a, sm, sm.sqid[lane], c, ps, true);
  }
  serve_bar();
}

// The GROUP queries of a group that cover all `rows` rows of this unit, up
// to kShareGroupQ of them, in one pass over the rows.  Query j (thresholds
// t_0 <= t_1 <= ...) takes a row when t_j < score, so a row whose score is
// above exactly k thresholds belongs to queries 0..k-1: it is added once, to
// bin (code, k-1), and query j's group total is the sum of bins j..na-1.  The
// per-row work does not grow with the number of queries.
__device__ void serve_group_shared(const ServeArgs& a, const ServeG& g, uint64_t r0, uint32_t rows,
                                   const uint64_t* s0, const uint32_t* codes, const int64_t* s2, ServeSmem& sm) {
  serve_pick(a, g, r0, rows, FDB_SERVE_GROUP, sm);
  const int na = sm.sna;
  if (na == 0) return;
  for (int i = threadIdx.x; i < FDB_SERVE_MAX_GROUPS * kShareGroupQ; i += kServeThreads) {
    sm.dcount[i] = 0;
    sm.dsum0[i] = 0.0;
    sm.dsum2[i] = 0;
  }
  serve_bar();
  for (uint32_t i = threadIdx.x; i < rows; i += kServeThreads) {
    const uint32_t code = codes[i];
    if (code >= FDB_SERVE_MAX_GROUPS) continue;  // beyond every query's dictionary
    const double v = __longlong_as_double((long long)s0[i]);
    int lo = 0, hi = na;  // k = number of thresholds below v (none for NaN)
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (sm.sthr[mid] < v)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo == 0) continue;
    const int cell = (int)code * kShareGroupQ + lo - 1;
    atomicAdd(&sm.dcount[cell], 1u);
    atomicAdd(&sm.dsum0[cell], v);
    atomicAdd(&sm.dsum2[cell], (unsigned long long)s2[i]);
  }
  serve_bar();
  if (threadIdx.x < FDB_SERVE_MAX_GROUPS) {  // thread gc: the only writer of group gc's totals
    const uint32_t gc = threadIdx.x;
    unsigned long long c = 0;
    double v0 = 0.0;
    long long v2 = 0;
    for (int k = na - 1; k >= 0; --k) {
      const int cell = (int)gc * kShareGroupQ + k;
      c += sm.dcount[cell];
      v0 += sm.dsum0[cell];
      v2 += (long long)sm.dsum2[cell];
      const uint32_t qi = sm.sqid[k];
      if (c == 0 || gc >= a.q[qi].dict_len) continue;
      if (qi < (uint32_t)kServeCacheQ) {
        sm.agcount[qi][gc] += c;
        sm.agsum0[qi][gc] += v0;
        sm.agsum2[qi][gc] += v2;
      } else {
        ServeRes& r = a.res[qi];
        atomicAdd(&r.gcount[gc], c);
        atomicAdd(&r.gsum0[gc], v0);
        atomicAdd(reinterpret_cast<unsigned long long*>(&r.gsum2[gc]), (unsigned long long)v2);
      }
    }
  }
  serve_bar();
}

// One shared unit whose rows are staged at `st` (the columns in `plain` are
// loaded here by the consumers): probe them once for a join group, then
// evaluate every query of the group that reaches this unit.
// `g` is taken by value: the loops below store to shared memory, where a
// cached descriptor may live, so fields read through a reference would be
// reloaded after every store.
template <bool JOIN>
__device__ void serve_shared_unit(const ServeArgs& a, const ServeG g, uint64_t tile, unsigned char* st,
                                  uint32_t plain, ServeSmem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t r0 = tile * g.unit_rows;
  const uint32_t rows = (uint32_t)umin64(g.unit_rows, g.max_n - r0);
  uint64_t* s0 = reinterpret_cast<uint64_t*>(st);
  unsigned char* s1 = st + g.off1;
  const int64_t* s2 = reinterpret_cast<const int64_t*>(st + g.off2);
  uint32_t* smm = reinterpret_cast<uint32_t*>(st + g.offm);
  if (plain) {
    const ShareCols cols = share_cols(g);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if ((plain >> c) & 1u) share_load(st + cols.off[c], cols.src[c], r0, rows, cols.esize[c]);
    serve_bar();
  }
  bool fused = false;
  if constexpr (JOIN) {
    // A join group with one query: filter, probe and count in one pass.
    fused = g.nq == 1;
    unsigned long long c = 0, ps = 0;
    double lim = 0.0;
    uint32_t prows = rows;
    if (fused) {
      const ServeQ& q = a.q[g.q0];
      lim = q.thr / 100.0;
      prows = q.n > r0 ? (uint32_t)umin64(rows, q.n - r0) : 0u;
    } else {
      // The largest limit among the queries that read this unit, found by
      // each warp with its lanes reading the group's descriptors in parallel.
      for (uint32_t k = (uint32_t)lane; k < g.nq; k += 32) {
        const ServeQ& q = a.q[g.q0 + k];
        if (q.n > r0) lim = fmax(lim, q.thr / 100.0);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) lim = fmax(lim, __shfl_xor_sync(0xffffffffu, lim, o));
    }
    serve_probe_rows(g, s0, smm, prows, fused, reinterpret_cast<const double*>(s1), lim, &c, &ps);
    if (fused) {
      c = warp_sum_u64(c);
      ps = warp_sum_u64(ps);
      if (lane == 0 && c) {
        const bool local = g.q0 < (uint32_t)kServeCacheQ;
        atomicAdd(local ? &sm.acount[g.q0] : &a.res[g.q0].count, c);
        atomicAdd(local ? &sm.asum[g.q0] : reinterpret_cast<unsigned long long*>(&a.res[g.q0].sum), ps);
      }
    }
  }
  // Kinds with enough queries in the group are evaluated together, once per
  // row (serve_pick); the loop below skips the queries they answered.
  const bool share = JOIN ? g.njoinq >= kShareGroupMin : (g.ngroupq >= kShareGroupMin || g.ncountq >= kShareGroupMin);
  if (share) {
    if (threadIdx.x < kServeMaxBatch / 32) sm.taken[threadIdx.x] = 0;  // ordered by serve_pick's barrier
    if constexpr (JOIN) {
      serve_pick(a, g, r0, rows, FDB_SERVE_JOIN, sm);
      if (sm.sna) serve_join_shared(a, rows, s0, reinterpret_cast<const double*>(s1), smm, sm);
    } else {
      if (g.ngroupq >= kShareGroupMin)
        serve_group_shared(a, g, r0, rows, s0, reinterpret_cast<const uint32_t*>(s1), s2, sm);
      if (g.ncountq >= kShareGroupMin) {
        serve_pick(a, g, r0, rows, FDB_SERVE_COUNT, sm);
        if (sm.sna) serve_count_shared(a, rows, s0, sm);
      }
    }
  }
  for (uint32_t qi = g.q0; !fused && qi < g.q0 + g.nq; ++qi) {
    const ServeQ& qref = a.q[qi];
    const uint64_t qn = qref.n;
    if (qn <= r0) break;  // queries are by rows descending
    const int qkind = qref.kind;
    if (share && ((sm.taken[(qi - g.q0) >> 5] >> ((qi - g.q0) & 31)) & 1u)) continue;  // answered together
    const double qthr = qref.thr;
    const uint32_t qdict = qref.dict_len;
    const uint32_t re = (uint32_t)umin64(rows, qn - r0);
    ServeRes& r = a.res[qi];
    if (!JOIN && qkind == FDB_SERVE_COUNT) {
      unsigned long long c = 0;
      for (uint32_t i = threadIdx.x; i < re; i += kServeThreads) c += __longlong_as_double((long long)s0[i]) > qthr;
      c = warp_sum_u64(c);
      if (lane == 0 && c) atomicAdd(qi < (uint32_t)kServeCacheQ ? &sm.acount[qi] : &r.count, c);
    } else if (JOIN) {
      const double lim = qthr / 100.0;
      const double* v = reinterpret_cast<const double*>(s1);
      unsigned long long c = 0, ps = 0;
      for (uint32_t i = threadIdx.x; i < re; i += kServeThreads)
        if (v[i] < lim) {
          c += smm[i];
          ps += s0[i];
        }
      c = warp_sum_u64(c);
      ps = warp_sum_u64(ps);
      if (lane == 0 && c) {
        const bool local = qi < (uint32_t)kServeCacheQ;
        atomicAdd(local ? &sm.acount[qi] : &r.count, c);
        atomicAdd(local ? &sm.asum[qi] : reinterpret_cast<unsigned long long*>(&r.sum), ps);
      }
    } else {  // GROUP
      if (lane < FDB_SERVE_MAX_GROUPS) {
        sm.gcount[warp][lane] = 0;
        sm.gsum0[warp][lane] = 0.0;
        sm.gsum2[warp][lane] = 0;
      }
      __syncwarp();
      // 32 rows at a time: the lanes whose rows pass and share a group find
      // one another (__match_any_sync on the code) and take their rank among
      // them.  Round r then lets every lane of rank r add its row to its
      // group's words of the warp's table with plain stores: lanes of one
      // rank never share a group, and no other warp writes these words.  Each
      // lane keeps its own row's values in registers.
      const uint32_t* codes = reinterpret_cast<const uint32_t*>(s1);
      const unsigned below = (1u << lane) - 1u;
      for (uint32_t b = (uint32_t)warp * 32; b < re; b += kServeThreads) {
        const uint32_t i = b + lane;
        uint32_t gc = 0xFFFFFFFFu;
        double v = 0.0;
        long long v2 = 0;
        if (i < re) {
          const uint32_t c = codes[i];
          v = __longlong_as_double((long long)s0[i]);
          if (v > qthr && c < qdict) {
            gc = c;
            v2 = s2[i];
          }
        }
        const unsigned peers = __match_any_sync(0xffffffffu, gc);
        const bool in = gc != 0xFFFFFFFFu;
        const unsigned rank = __popc(peers & below);
        const unsigned rounds = __reduce_max_sync(0xffffffffu, in ? (unsigned)__popc(peers) : 0u);
        if (in && rank == 0) sm.gcount[warp][gc] += (unsigned long long)__popc(peers);
        for (unsigned r = 0; r < rounds; ++r) {
          if (in && rank == r) {
            sm.gsum0[warp][gc] += v;
            sm.gsum2[warp][gc] += v2;
          }
          __syncwarp();  // the next rank's lane reads these words
        }
      }
      serve_bar();
      if (threadIdx.x < qdict) {
        const uint32_t gc = threadIdx.x;
        unsigned long long c = 0;
        double v0 = 0.0;
        long long v2 = 0;
        for (int w = 0; w < kServeWarps; ++w) {
          c += sm.gcount[w][gc];
          v0 += sm.gsum0[w][gc];
          v2 += sm.gsum2[w][gc];
        }
        if (c) {
          if (qi < (uint32_t)kServeCacheQ) {  // thread gc is the only writer of group gc
            sm.agcount[qi][gc] += c;
            sm.agsum0[qi][gc] += v0;
            sm.agsum2[qi][gc] += v2;
          } else {
            atomicAdd(&r.gcount[gc], c);
            atomicAdd(&r.gsum0[gc], v0);
            atomicAdd(reinterpret_cast<unsigned long long*>(&r.gsum2[gc]), (unsigned long long)v2);
          }
        }
      }
      serve_bar();
    }
  }
}

// Persistent: the producer warp claims units one at a time (one global
// counter) and stages each shared unit's columns into a ring of kServeStages
// buffers with bulk copies; the consumer warps evaluate the units in claim
// order.  A column the bulk copy cannot take (its rows do not start on a
// 16-byte boundary, or its byte count is not a multiple of 16) is flagged for
// the consumers to load with plain loads.
template <bool JOIN>
__global__ void __launch_bounds__(kServeBlock, JOIN ? kServeJoinCtasPerSm : kServeCtasPerSm) serve_kernel(ServeArgs a) {
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ ServeSmem sm;
  uint64_t* full = reinterpret_cast<uint64_t*>(tsm);
  uint64_t* empty = full + kServeStages;
  uint64_t* unit = empty + kServeStages;
  uint32_t* plain = reinterpret_cast<uint32_t*>(unit + kServeStages);
  unsigned char* stages = tsm + kServeBar;
  // This instance's groups and units: the join groups come first.
  const int topk0 = a.hdr->topk0;
  const int njg = a.hdr->join_groups;
  const int g0 = JOIN ? 0 : njg;
  const int ng = JOIN ? njg : a.hdr->ngroups - njg;
  const uint64_t lo = JOIN ? 0 : a.hdr->join_units;
  const uint64_t shared = JOIN ? a.hdr->join_units : a.hdr->shared_units;  // end of this instance's units
  if (lo == shared) return;  // no group of this kind in the batch
  const int32_t limit = a.hdr->cta_limit[JOIN ? 0 : 1];
  if (limit > 0 && (int32_t)blockIdx.x >= limit) return;  // units are claimed, so fewer CTAs cover them all
  unsigned int* claim = a.claim + (JOIN ? 0 : 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < ng; i += kServeBlock) sm.gstart[i] = a.g[g0 + i].unit0;
  {
    for (int i = threadIdx.x; i < kServeCacheQ; i += kServeBlock) sm.acount[i] = sm.asum[i] = 0;
    for (int i = threadIdx.x; i < kServeCacheQ * FDB_SERVE_MAX_GROUPS; i += kServeBlock) {
      (&sm.agcount[0][0])[i] = 0;
      (&sm.agsum0[0][0])[i] = 0.0;
      (&sm.agsum2[0][0])[i] = 0;
    }
  }
  if (threadIdx.x == 0) {
    sm.gstart[ng] = shared;
    for (int s = 0; s < kServeStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kServeWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == kServeWarps) {
    // ---------------- producer warp ----------------
    if (lane == 0) {
      const uint64_t policy = l2_evict_first_policy();
      // The next unit is claimed while the stage for the current one drains,
      // so the counter's round trip overlaps the wait.
      uint64_t next = lo + atomicAdd(claim, 1u);
      for (uint32_t it = 0;; ++it) {
        const int s = it % kServeStages;
        const uint32_t ph = (it / kServeStages) & 1u;
        if (it >= kServeStages && !mbar_wait_backoff(&empty[s], ph ^ 1u, a.err, 64)) break;
        const uint64_t t = next;
        if (t < shared) next = lo + atomicAdd(claim, 1u);
        unit[s] = t;
        plain[s] = 0;
        if (t >= shared) {  // the end mark: no rows to stage
          mbar_arrive(&full[s]);
          break;
        }
        const int gi = serve_find(sm.gstart, ng, t);
        const ServeG g = a.g[g0 + gi];
        const ShareCols cols = share_cols(g);
        const uint64_t r0 = (t - sm.gstart[gi]) * g.unit_rows;
        const uint32_t rows = (uint32_t)umin64(g.unit_rows, g.max_n - r0);
        uint32_t bytes = 0, pm = 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (!cols.esize[c]) continue;
          const unsigned char* src = static_cast<const unsigned char*>(cols.src[c]) + r0 * cols.esize[c];
          const uint32_t nb = rows * (uint32_t)cols.esize[c];
          if ((((uintptr_t)src) & 15u) == 0 && (nb & 15u) == 0)
            bytes += nb;
          else
            pm |= 1u << c;
        }
        plain[s] = pm;
        if (bytes == 0) {
          mbar_arrive(&full[s]);
          continue;
        }
        mbar_arrive_expect_tx(&full[s], bytes);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (!cols.esize[c] || ((pm >> c) & 1u)) continue;
          const unsigned char* src = static_cast<const unsigned char*>(cols.src[c]) + r0 * cols.esize[c];
          bulk_g2s(stages + (size_t)s * share_stage<JOIN>() + cols.off[c], src, rows * (uint32_t)cols.esize[c], &full[s],
                   policy);
        }
      }
    }
    return;
  }

  // ---------------- consumer warps ----------------
  for (uint32_t it = 0;; ++it) {
    const int s = it % kServeStages;
    const uint32_t ph = (it / kServeStages) & 1u;
    // A wait that runs out has recorded the error; every consumer leaves
    // together so that the named barriers stay uniform.
    if (serve_bar_any(!mbar_wait(&full[s], ph, a.err))) break;
    const uint64_t t = unit[s];
    const uint32_t pm = plain[s];
    if (t >= shared) break;
    const int gi = serve_find(sm.gstart, ng, t);
    serve_shared_unit<JOIN>(a, a.g[g0 + gi], t - sm.gstart[gi], stages + (size_t)s * share_stage<JOIN>(), pm, sm);
    // The consumers wrote the stage (probe results, plain loads): order those
    // writes before the producer's next bulk copy into it.
    fence_proxy_async_smem();
    serve_bar();  // every consumer is done with the stage (and with sm's per-unit state)
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  // Flush the CTA's partials of the cached shared queries.
  const int nqc = topk0 < kServeCacheQ ? topk0 : kServeCacheQ;  // shared queries come first
  for (int i = threadIdx.x; i < nqc; i += kServeThreads) {
    if (sm.acount[i]) atomicAdd(&a.res[i].count, sm.acount[i]);
    if (sm.asum[i]) atomicAdd(reinterpret_cast<unsigned long long*>(&a.res[i].sum), sm.asum[i]);
  }
  for (int i = threadIdx.x; i < nqc * FDB_SERVE_MAX_GROUPS; i += kServeThreads) {
    const int qi = i / FDB_SERVE_MAX_GROUPS, gc = i % FDB_SERVE_MAX_GROUPS;
    if (sm.agcount[qi][gc]) {
      atomicAdd(&a.res[qi].gcount[gc], sm.agcount[qi][gc]);
      atomicAdd(&a.res[qi].gsum0[gc], sm.agsum0[qi][gc]);
      atomicAdd(reinterpret_cast<unsigned long long*>(&a.res[qi].gsum2[gc]), (unsigned long long)sm.agsum2[qi][gc]);
    }
  }
}

// Top-k queries scan their own rows in kServeTile-row units, claimed from
// their own counter after the shared scan: a CTA keeps a list per warp while
// its consecutive units belong to one query and publishes its k best (below
// the query's running bound) as candidates when it moves on.
__global__ void __launch_bounds__(kServeThreads, kServeTopkCtasPerSm) serve_topk_kernel(ServeArgs a) {
  __shared__ TopkSmem sm;
  const int nq = a.hdr->nq, topk0 = a.hdr->topk0;
  const int ntopk = nq - topk0;
  if (ntopk == 0) return;
  const int32_t limit = a.hdr->cta_limit[2];
  if (limit > 0 && (int32_t)blockIdx.x >= limit) return;
  const uint64_t shared = a.hdr->shared_units, total = a.hdr->total_units;
  for (int i = threadIdx.x; i < ntopk; i += kServeThreads) sm.start[i] = a.q[topk0 + i].tile0;
  if (threadIdx.x == 0) sm.start[ntopk] = total;
  __syncthreads();
  RTLocal tl;
  rt_reset(tl);
  int cur = -1;
  for (;;) {
    if (threadIdx.x == 0) sm.t = atomicAdd(a.claim + 1, 1u);
    __syncthreads();
    const uint64_t t = shared + sm.t;
    if (t >= total) break;
    const int qi = topk0 + serve_find(sm.start, ntopk, t);
    if (qi != cur) {
      if (cur >= 0) serve_publish(a, a.q[cur], cur, sm, tl);
      cur = qi;
    }
    const ServeQ q = a.q[qi];
    rt_bound(tl, ~*reinterpret_cast<volatile unsigned long long*>(&a.res[qi].nbound));
    const uint64_t r0 = (t - q.tile0) * kServeTile;
    serve_topk_tile(q, r0, umin64(r0 + kServeTile, q.n), tl);
    __syncthreads();  // the unit is done before sm.t is rewritten
  }
  if (cur >= 0) serve_publish(a, a.q[cur], cur, sm, tl);
}

// Top-k queries: the k best of the CTAs' candidates, one CTA per query.
__global__ void __launch_bounds__(kServeThreads) serve_finish_kernel(ServeArgs a) {
  __shared__ TopkSmem sm;
  const int qi = blockIdx.x;
  if (qi >= a.hdr->nq) return;
  const ServeQ& q = a.q[qi];
  if (q.kind != FDB_SERVE_TOPK) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t k = (uint32_t)q.k;
  ServeRes& r = a.res[qi];
  const uint32_t nc = min(r.ncand, a.cand_cap);
  RTLocal tl;
  rt_reset(tl);
  rt_bound(tl, ~r.nbound);
  const uint64_t* ck = a.cand_k + (size_t)qi * a.cand_cap;
  const uint32_t* cr = a.cand_r + (size_t)qi * a.cand_cap;
  for (uint32_t b = warp * 256; b < nc; b += 256 * kServeWarps) {
    uint64_t key[8];
    uint32_t row[8];
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t i = b + j * 32 + lane;
      key[j] = ~0ull;
      row[j] = 0xFFFFFFFFu;
      if (i < nc) {
        key[j] = ck[i];
        row[j] = cr[i];
        if (kr_le(key[j], row[j], tl.tk, tl.tr)) m |= 1u << j;
      }
    }
    if (__any_sync(0xffffffffu, m != 0u)) rt_offer<8>(tl, k, key, row, m, lane);
  }
  serve_tree_merge(sm, tl, k, warp, lane);
  if (warp == 0) {
    const bool real = (uint32_t)lane < k && !(tl.lk == ~0ull && tl.lr == 0xFFFFFFFFu);
    const unsigned vb = __ballot_sync(0xffffffffu, real);
    if (real) r.rows[lane] = tl.lr;
    if (lane == 0) r.count = (unsigned long long)__popc(vb);
  }
}

// ---------------------------------------------------------------------------
// Host: slots, scheduler, trace driver
// ---------------------------------------------------------------------------
using Clock = std::chrono::steady_clock;

struct ServeSlot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  unsigned char* h_in = nullptr;   // ServeHeader + ServeQ[kServeMaxBatch] (pinned)
  ServeRes* h_out = nullptr;       // [kServeMaxBatch] (pinned)
  int* h_err = nullptr;            // (pinned)
  DevBuf d_in, d_res, d_cand_k, d_cand_r, d_err;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> tickets;
  bool busy = false;
  bool big = false;                // the batch in flight is of the long-scan class
};

struct ServeJob {
  fdb_serve_query q;
  fdb_serve_result r;
  uint64_t bytes = 0;
  bool done = false;
};

struct Server {
  fdb_db* db = nullptr;
  Ctx* c = nullptr;
  fdb_serve_config cfg{};
  std::vector<ServeSlot> slots;
  std::thread thr;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, ServeJob> jobs;
  uint64_t next_ticket = 1;
  bool stopping = false;
  uint64_t budget = 0, resident = 0, reserved = 0, peak_reserved = 0;
  int64_t batches = 0, batched_queries = 0;
  std::vector<double> latencies;
  double first_arrival = 1e300, last_done = 0.0;
  Clock::time_point t0;
  uint32_t cand_cap = 0;
  int grid = 0, grid_join = 0, grid_topk = 0;
  uint64_t split_rows = 1ull << 22;  // size classes of batches: fewer / at least this many rows
  std::string error;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

static constexpr size_t kServeQOff = sizeof(ServeHeader);
static constexpr size_t kServeGOff = kServeQOff + sizeof(ServeQ) * kServeMaxBatch;
static constexpr size_t kServeInBytes = kServeGOff + sizeof(ServeG) * kServeMaxBatch;
static constexpr size_t kServeResBytes = sizeof(ServeRes) * kServeMaxBatch;

static uint64_t serve_query_bytes(const fdb_serve_query& q, uint32_t cand_cap) {
  return sizeof(ServeQ) + sizeof(ServeRes) + (q.kind == FDB_SERVE_TOPK ? (uint64_t)cand_cap * 12 : 0);
}

static void serve_check(const fdb_serve_query& q) {
  if (q.kind < FDB_SERVE_COUNT || q.kind > FDB_SERVE_TOPK) fail(FDB_E_ARG, "unknown serving template");
  if (q.nrows >= 0xFFFFFFFFull) fail(FDB_E_ARG, "a served query addresses rows as uint32");
  if (q.nrows && !q.c0) fail(FDB_E_ARG, "query without its column");
  if (q.kind == FDB_SERVE_GROUP && (q.dict_len == 0 || q.dict_len > FDB_SERVE_MAX_GROUPS || (q.nrows && (!q.c1 || !q.c2))))
    fail(FDB_E_ARG, "GROUP needs codes (dict_len 1..16) and an INT64 column");
  if (q.kind == FDB_SERVE_JOIN && (!q.table || (q.nrows && !q.c1)))
    fail(FDB_E_ARG, "JOIN needs a build table and a value column");
  if (q.kind == FDB_SERVE_TOPK && (q.k < 1 || q.k > FDB_SERVE_MAX_K)) fail(FDB_E_ARG, "TOPK needs 1 <= k <= 32");
}

static void slot_capture(Server& s, ServeSlot& sl) {
  Ctx& c = *s.c;
  ServeArgs a;
  a.hdr = static_cast<const ServeHeader*>(sl.d_in.ptr);
  a.q = reinterpret_cast<const ServeQ*>(static_cast<unsigned char*>(sl.d_in.ptr) + kServeQOff);
  a.g = reinterpret_cast<const ServeG*>(static_cast<unsigned char*>(sl.d_in.ptr) + kServeGOff);
  a.res = static_cast<ServeRes*>(sl.d_res.ptr);
  a.claim = reinterpret_cast<unsigned int*>(static_cast<unsigned char*>(sl.d_res.ptr) + kServeResBytes);
  a.cand_k = static_cast<uint64_t*>(sl.d_cand_k.ptr);
  a.cand_r = static_cast<uint32_t*>(sl.d_cand_r.ptr);
  a.cand_cap = s.cand_cap;
  a.err = static_cast<int*>(sl.d_err.ptr);
#if FDB_SERVE_FORK
  // The join, scan and top-k instances read their own units and write their
  // own queries' results, so the graph runs them side by side: when one runs
  // out of units, its SMs go to the others instead of idling until it ends.
  cudaStream_t side[2];
  cudaEvent_t fork, joined[2];
  for (int i = 0; i < 2; ++i) FDB_CUDA(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking));
  FDB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  for (int i = 0; i < 2; ++i) FDB_CUDA(cudaEventCreateWithFlags(&joined[i], cudaEventDisableTiming));
#endif
  FDB_CUDA(cudaStreamBeginCapture(sl.stream, cudaStreamCaptureModeThreadLocal));
  cudaMemcpyAsync(sl.d_in.ptr, sl.h_in, kServeInBytes, cudaMemcpyHostToDevice, sl.stream);
  cudaMemsetAsync(sl.d_res.ptr, 0, kServeResBytes + 256, sl.stream);
#if FDB_SERVE_FORK
  cudaEventRecord(fork, sl.stream);
  for (int i = 0; i < 2; ++i) cudaStreamWaitEvent(side[i], fork, 0);
  serve_kernel<true><<<s.grid_join, kServeBlock, kShareSmemJoin, side[0]>>>(a);
  serve_topk_kernel<<<s.grid_topk, kServeThreads, 0, side[1]>>>(a);
  serve_kernel<false><<<s.grid, kServeBlock, kShareSmem, sl.stream>>>(a);
  for (int i = 0; i < 2; ++i) {
    cudaEventRecord(joined[i], side[i]);
    cudaStreamWaitEvent(sl.stream, joined[i], 0);
  }
#else
  serve_kernel<true><<<s.grid_join, kServeBlock, kShareSmemJoin, sl.stream>>>(a);
  serve_kernel<false><<<s.grid, kServeBlock, kShareSmem, sl.stream>>>(a);
  serve_topk_kernel<<<s.grid_topk, kServeThreads, 0, sl.stream>>>(a);
#endif
  serve_finish_kernel<<<kServeMaxBatch, kServeThreads, 0, sl.stream>>>(a);
  cudaMemcpyAsync(sl.h_out, sl.d_res.ptr, kServeResBytes, cudaMemcpyDeviceToHost, sl.stream);
  cudaMemcpyAsync(sl.h_err, sl.d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, sl.stream);
  cudaMemsetAsync(sl.d_err.ptr, 0, sizeof(int), sl.stream);
  FDB_CUDA(cudaStreamEndCapture(sl.stream, &sl.graph));
#if FDB_SERVE_FORK
  for (int i = 0; i < 2; ++i) {
    cudaEventDestroy(joined[i]);
    cudaStreamDestroy(side[i]);
  }
  cudaEventDestroy(fork);
#endif
  FDB_CUDA(cudaGraphInstantiate(&sl.exec, sl.graph, 0));
}

static void server_destroy(Server* s) {
  if (!s) return;
  for (ServeSlot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.exec) cudaGraphExecDestroy(sl.exec);
    if (sl.graph) cudaGraphDestroy(sl.graph);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.h_in) cudaFreeHost(sl.h_in);
    if (sl.h_out) cudaFreeHost(sl.h_out);
    if (sl.h_err) cudaFreeHost(sl.h_err);
    s->c->free_buf(sl.d_in);
    s->c->free_buf(sl.d_res);
    s->c->free_buf(sl.d_cand_k);
    s->c->free_buf(sl.d_cand_r);
    s->c->free_buf(sl.d_err);
  }
  delete s;
}

// Hand out a finished slot's results (scheduler thread, s.mu held).
static void slot_complete(Server& s, ServeSlot& sl) {
  const double t = s.now();
  const int err = *sl.h_err;
  const int n = (int)sl.tickets.size();
  for (int i = 0; i < n; ++i) {
    ServeJob& j = s.jobs[sl.tickets[i]];
    const ServeRes& d = sl.h_out[i];
    fdb_serve_result& r = j.r;
    r.count = (int64_t)d.count;
    r.sum_payload = d.sum;
    for (int g = 0; g < FDB_SERVE_MAX_GROUPS; ++g) {
      r.group_count[g] = (int64_t)d.gcount[g];
      r.group_sum0[g] = d.gsum0[g];
      r.group_sum2[g] = d.gsum2[g];
    }
    std::memcpy(r.rows, d.rows, sizeof(r.rows));
    r.done_s = t;
    r.batch_size = n;
    r.status = err ? (err == kErrCapacity ? FDB_E_CAPACITY : FDB_E_TIMEOUT) : FDB_OK;
    j.done = true;
    s.reserved -= j.bytes;
    s.latencies.push_back(t - r.arrival_s);
    s.first_arrival = std::min(s.first_arrival, r.arrival_s);
    s.last_done = std::max(s.last_done, t);
  }
  sl.tickets.clear();
  sl.busy = false;
}

// Admit queued queries into a free slot and launch it (s.mu held).  The
// admitted queries are laid out group by group (queries reading the same
// table, by rows descending), then the top-k queries.
constexpr int kBigBatchBacklog = 3;  // long scans waiting before they are batched together

// small_only: this slot runs only batches of the small size class.  Slot 0
// runs any batch and the others only small ones, so at most one long scan is
// on the GPU at a time and short queries never wait behind one.
static bool slot_launch(Server& s, ServeSlot& sl, bool small_only) {
  const uint64_t room = s.budget > s.resident ? s.budget - s.resident : 0;
  const double t = s.now();
  // A batch holds queries of one size class, the class of the oldest waiting
  // query: a query that reads few rows never waits for a long scan that
  // happened to be admitted with it.  Within the class, arrival order.
  std::vector<uint64_t> admitted;
  bool big = s.jobs[s.queue.front()].q.nrows >= s.split_rows;
  if (small_only && big) {
    bool any = false;
    for (uint64_t tk : s.queue)
      if (s.jobs[tk].q.nrows < s.split_rows) {
        any = true;
        break;
      }
    if (!any) return false;
    big = false;
  }
  // Long scans are batched only under a backlog.  Two long scans in one batch
  // both finish when the batch does, while one at a time the first finishes
  // early; so at light load each runs alone, and once kBigBatchBacklog of them
  // are waiting, batching them shares their reads and raises throughput.
  int cap = s.cfg.max_batch;
  if (big) {
    int waiting = 0;
    for (auto it = s.queue.begin(); it != s.queue.end() && waiting < kBigBatchBacklog; ++it)
      waiting += s.jobs[*it].q.nrows >= s.split_rows ? 1 : 0;
    if (waiting < kBigBatchBacklog) cap = 1;
  }
  for (auto it = s.queue.begin(); it != s.queue.end() && (int)admitted.size() < cap;) {
    ServeJob& j = s.jobs[*it];
    if ((j.q.nrows >= s.split_rows) != big) {
      ++it;
      continue;
    }
    if (s.reserved + j.bytes > room && !admitted.empty()) break;  // wait for memory (a lone query always runs)
    s.reserved += j.bytes;
    s.peak_reserved = std::max(s.peak_reserved, s.reserved);
    j.r.start_s = t;
    admitted.push_back(*it);
    it = s.queue.erase(it);
  }
  if (admitted.empty()) return false;

  // Groups: COUNT joins any non-join group on the same c0; GROUP needs the same
  // (c0, c1, c2) or a COUNT-only group on c0; JOIN needs the same (c0, c1, table).
  struct G {
    const void *c0, *c1, *c2;
    const fdb_hash* table;
    bool join, has_group;
    std::vector<uint64_t> tickets;
  };
  std::vector<G> groups;
  std::vector<uint64_t> topk;
  for (uint64_t tk : admitted) {
    const fdb_serve_query& q = s.jobs[tk].q;
    if (q.kind == FDB_SERVE_TOPK) {
      topk.push_back(tk);
      continue;
    }
    G* home = nullptr;
    for (G& g : groups) {
      if (g.c0 != q.c0) continue;
      if (q.kind == FDB_SERVE_JOIN) {
        if (g.join && g.c1 == q.c1 && g.table == q.table) home = &g;
      } else if (!g.join) {
        if (q.kind == FDB_SERVE_COUNT) home = &g;
        else if (!g.has_group || (g.c1 == q.c1 && g.c2 == q.c2)) home = &g;
      }
      if (home) break;
    }
    if (!home) {
      groups.push_back(G{q.c0, nullptr, nullptr, nullptr, q.kind == FDB_SERVE_JOIN, false, {}});
      home = &groups.back();
      if (home->join) {
        home->c1 = q.c1;
        home->table = q.table;
      }
    }
    if (q.kind == FDB_SERVE_GROUP && !home->has_group) {
      home->has_group = true;
      home->c1 = q.c1;
      home->c2 = q.c2;
    }
    home->tickets.push_back(tk);
  }
  // Join groups first: serve_kernel<true> takes units [0, join_units).
  std::stable_partition(groups.begin(), groups.end(), [](const G& g) { return g.join; });

  ServeHeader* hdr = reinterpret_cast<ServeHeader*>(sl.h_in);
  ServeQ* dq = reinterpret_cast<ServeQ*>(sl.h_in + kServeQOff);
  ServeG* dg = reinterpret_cast<ServeG*>(sl.h_in + kServeGOff);
  sl.tickets.clear();
  uint64_t units = 0;
  auto put = [&](uint64_t tk) -> ServeQ& {
    const fdb_serve_query& q = s.jobs[tk].q;
    ServeQ& d = dq[sl.tickets.size()];
    std::memset(&d, 0, sizeof(d));
    d.kind = q.kind;
    d.k = q.k;
    d.n = q.nrows;
    d.thr = q.threshold;
    d.c0 = q.c0;
    d.c1 = q.c1;
    d.c2 = q.c2;
    d.dict_len = q.dict_len;
    sl.tickets.push_back(tk);
    return d;
  };
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    G& g = groups[gi];
    std::stable_sort(g.tickets.begin(), g.tickets.end(),
                     [&](uint64_t x, uint64_t y) { return s.jobs[x].q.nrows > s.jobs[y].q.nrows; });
    ServeG& d = dg[gi];
    std::memset(&d, 0, sizeof(d));
    d.c0 = g.c0;
    d.c1 = g.c1;
    d.c2 = g.c2;
    d.q0 = (uint32_t)sl.tickets.size();
    d.nq = (uint32_t)g.tickets.size();
    d.max_n = s.jobs[g.tickets.front()].q.nrows;
    d.c1_bytes = g.join ? 8 : (g.has_group ? 4 : 0);
    d.load_c2 = g.has_group ? 1 : 0;
    {
      const uint32_t row_bytes = 8u + (uint32_t)d.c1_bytes + (d.load_c2 ? 8u : 0u) + (g.join ? 4u : 0u);
      // A join unit is a whole number of probe passes (kProbeIlp rows per thread).
      const uint32_t quantum = g.join ? (uint32_t)(kProbeIlp * kServeThreads) : 256u;
      d.unit_rows = (uint32_t)((g.join ? kShareStageJoin : kShareStage) / row_bytes) / quantum * quantum;
      d.off1 = 8u * d.unit_rows;
      d.off2 = d.off1 + (uint32_t)d.c1_bytes * d.unit_rows;
      d.offm = d.off2 + (d.load_c2 ? 8u : 0u) * d.unit_rows;
    }
    d.unit0 = units;
    units += (d.max_n + d.unit_rows - 1) / d.unit_rows;
    d.ngroupq = d.ncountq = d.njoinq = 0;
    for (uint64_t tk : g.tickets) {
      const int kind = s.jobs[tk].q.kind;
      d.ngroupq += kind == FDB_SERVE_GROUP ? 1 : 0;
      d.ncountq += kind == FDB_SERVE_COUNT ? 1 : 0;
      d.njoinq += kind == FDB_SERVE_JOIN ? 1 : 0;
    }
    d.join = g.join ? 1 : 0;
    if (g.join) {
      const JoinView v = join_view(hash_of(g.table));
      d.slots = static_cast<const JSlot*>(v.slots);
      d.cnt = v.cnt;
      d.cap = v.cap;
      d.unique = v.unique;
      d.dmin = v.dmin;
      d.dense = v.dense;
      d.span = v.span;
    }
    for (uint64_t tk : g.tickets) put(tk);
  }
  hdr->nq = (int32_t)admitted.size();
  hdr->ngroups = (int32_t)groups.size();
  {
    int32_t njg = 0;
    while (njg < (int32_t)groups.size() && groups[njg].join) ++njg;
    hdr->join_groups = njg;
    hdr->join_units = njg ? dg[njg - 1].unit0 + (dg[njg - 1].max_n + dg[njg - 1].unit_rows - 1) / dg[njg - 1].unit_rows : 0;
  }
  hdr->topk0 = (int32_t)sl.tickets.size();
  hdr->shared_units = units;
  // A long-scan batch launched while short queries wait, or while another
  // slot runs, leaves one CTA slot per SM to the other slots' batches: its
  // persistent CTAs would otherwise hold every SM until its last unit.
  hdr->cta_limit[0] = hdr->cta_limit[1] = hdr->cta_limit[2] = 0;
#if FDB_SERVE_YIELD
  if (big && s.slots.size() > 1) {
    bool other_busy = false;
    for (const ServeSlot& o : s.slots) other_busy |= (&o != &sl) && o.busy;
    if (other_busy || !s.queue.empty()) {
      const int sms = s.c->sm_count;
      hdr->cta_limit[0] = std::max(sms, s.grid_join - sms);
      hdr->cta_limit[1] = std::max(sms, s.grid - sms);
      hdr->cta_limit[2] = std::max(sms, s.grid_topk - sms);
    }
  }
#endif
  for (uint64_t tk : topk) {
    ServeQ& d = put(tk);
    d.tile0 = units;
    units += (d.n + kServeTile - 1) / kServeTile;
  }
  hdr->total_units = units;
  FDB_CUDA(cudaGraphLaunch(sl.exec, sl.stream));
  FDB_CUDA(cudaEventRecord(sl.done, sl.stream));
  sl.busy = true;
  sl.big = big;
  ++s.batches;
  s.batched_queries += (int64_t)admitted.size();
  return true;
}

static void server_loop(Server* s) {
  cudaSetDevice(s->c->device);
  for (;;) {
    bool progress = false, idle = true;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (ServeSlot& sl : s->slots) {
        if (!sl.busy) continue;
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaSuccess) {
          slot_complete(*s, sl);
          progress = true;
        } else if (q != cudaErrorNotReady) {
          s->error = cudaGetErrorString(q);
          slot_complete(*s, sl);
          progress = true;
        }
      }
      try {
        for (size_t i = 0; i < s->slots.size(); ++i) {
          if (s->slots[i].busy || s->queue.empty()) continue;
          // Under a backlog, short-scan slots wait while a long scan runs: its
          // persistent CTAs hold the SMs, so a batch launched beside it only
          // queues behind it on the GPU, and the long scan itself slows down.
          if (i > 0 && kServeHoldBacklog > 0 && s->slots[0].busy && s->slots[0].big &&
              s->queue.size() >= (size_t)kServeHoldBacklog)
            continue;
          progress |= slot_launch(*s, s->slots[i], i > 0);
        }
      } catch (const Error& e) {
        s->error = e.what();
      }
      for (ServeSlot& sl : s->slots) idle &= !sl.busy;
      if (progress) s->cv.notify_all();
      if (s->stopping && idle && s->queue.empty()) break;
    }
    if (!progress) std::this_thread::yield();
  }
}

Server* server_start(fdb_db* db, Ctx& c, const fdb_serve_config* cfg) {
  std::unique_ptr<Server, void (*)(Server*)> s(new Server(), server_destroy);
  s->db = db;
  s->c = &c;
  s->cfg.max_batch = cfg && cfg->max_batch > 0 ? std::min(cfg->max_batch, kServeMaxBatch) : 128;
  s->cfg.slots = cfg && cfg->slots > 0 ? std::min(cfg->slots, 8) : 4;
  s->budget = cfg && cfg->mem_budget ? cfg->mem_budget : c.budget;
  s->cfg.mem_budget = s->budget;
  s->resident = c.in_use.load();
  FDB_CUDA(cudaFuncSetAttribute(serve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kShareSmemJoin));
  FDB_CUDA(cudaFuncSetAttribute(serve_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kShareSmem));
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel<false>, kServeBlock, kShareSmem));
  s->grid = c.sm_count * std::max(1, std::min(per_sm, kServeCtasPerSm));
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel<true>, kServeBlock, kShareSmemJoin));
  s->grid_join = c.sm_count * std::max(1, std::min(per_sm, kServeJoinCtasPerSm));
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_topk_kernel, kServeThreads, 0));
  s->grid_topk = c.sm_count * std::max(1, std::min(per_sm, kServeTopkCtasPerSm));
  // A top-k CTA publishes at most once per query (its claims only grow).
  s->cand_cap = (uint32_t)s->grid_topk * FDB_SERVE_MAX_K;
  s->slots.resize(s->cfg.slots);
  for (ServeSlot& sl : s->slots) {
    FDB_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
    FDB_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    FDB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&sl.h_in), kServeInBytes, cudaHostAllocDefault));
    FDB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&sl.h_out), kServeResBytes, cudaHostAllocDefault));
    FDB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&sl.h_err), sizeof(int), cudaHostAllocDefault));
    std::memset(sl.h_in, 0, kServeInBytes);
    *sl.h_err = 0;
    sl.d_in = c.alloc_buf(kServeInBytes);
    sl.d_res = c.alloc_buf(kServeResBytes + 256);
    sl.d_cand_k = c.alloc_buf((size_t)kServeMaxBatch * s->cand_cap * 8);
    sl.d_cand_r = c.alloc_buf((size_t)kServeMaxBatch * s->cand_cap * 4);
    sl.d_err = c.alloc_buf(256);
    FDB_CUDA(cudaMemset(sl.d_err.ptr, 0, 256));
    slot_capture(*s, sl);
  }
  s->t0 = Clock::now();
  Server* raw = s.release();
  raw->thr = std::thread(server_loop, raw);
  return raw;
}

uint64_t server_submit(Server& s, const fdb_serve_query& q, double arrival_s) {
  serve_check(q);
  std::lock_guard<std::mutex> lk(s.mu);
  if (s.stopping) fail(FDB_E_ARG, "the server is stopping");
  const uint64_t t = s.next_ticket++;
  ServeJob& j = s.jobs[t];
  j.q = q;
  std::memset(&j.r, 0, sizeof(j.r));
  j.r.arrival_s = arrival_s >= 0 ? arrival_s : s.now();
  j.bytes = serve_query_bytes(q, s.cand_cap);
  s.queue.push_back(t);
  return t;
}

bool server_wait(Server& s, uint64_t ticket, int64_t timeout_ns, fdb_serve_result* out) {
  std::unique_lock<std::mutex> lk(s.mu);
  auto it = s.jobs.find(ticket);
  if (it == s.jobs.end()) fail(FDB_E_ARG, "unknown ticket");
  const auto until = Clock::now() + std::chrono::nanoseconds(timeout_ns < 0 ? 0 : timeout_ns);
  while (!it->second.done) {
    if (timeout_ns >= 0 && Clock::now() >= until) return false;
    if (timeout_ns >= 0)
      s.cv.wait_until(lk, until);
    else
      s.cv.wait(lk);
  }
  if (out) *out = it->second.r;
  s.jobs.erase(it);
  return true;
}

double server_now(Server& s) { return s.now(); }

void server_stop(Server* s, fdb_serve_stats* st) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  if (s->thr.joinable()) s->thr.join();
  if (st) {
    std::memset(st, 0, sizeof(*st));
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
    st->wall_s = l.empty() ? 0.0 : s->last_done - s->first_arrival;
    st->qps = st->wall_s > 0 ? (double)l.size() / st->wall_s : 0.0;
    st->p50_ms = pct(0.50) * 1e3;
    st->p99_ms = pct(0.99) * 1e3;
    st->max_ms = l.empty() ? 0.0 : l.back() * 1e3;
    st->batches = s->batches;
    st->mean_batch = s->batches ? (double)s->batched_queries / (double)s->batches : 0.0;
    st->peak_reserved = s->peak_reserved;
    st->resident_bytes = s->resident;
  }
  const std::string err = s->error;
  server_destroy(s);
  if (!err.empty()) fail(FDB_E_CUDA, "serving loop: " + err);
}

// Submit the trace's queries at their arrival times (this thread spins for
// the last 100 us before each), then collect every result.
void serve_trace(fdb_db* db, Ctx& c, const fdb_serve_query* qs, int nq, const fdb_serve_config* cfg,
                 fdb_serve_result* out, fdb_serve_stats* st) {
  for (int i = 0; i < nq; ++i) serve_check(qs[i]);
  Server* s = server_start(db, c, cfg);
  std::vector<uint64_t> tickets(nq);
  try {
    for (int i = 0; i < nq; ++i) {
      const double at = qs[i].arrival_s;
      for (;;) {
        const double wait = at - s->now();
        if (wait <= 0) break;
        if (wait > 2e-4) std::this_thread::sleep_for(std::chrono::duration<double>(wait - 1e-4));
      }
      tickets[i] = server_submit(*s, qs[i], at);
    }
    for (int i = 0; i < nq; ++i) server_wait(*s, tickets[i], -1, out ? out + i : nullptr);
  } catch (...) {
    server_stop(s, nullptr);
    throw;
  }
  server_stop(s, st);
}

}  // namespace fdb
