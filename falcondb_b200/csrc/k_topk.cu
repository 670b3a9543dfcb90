// ORDER BY col [DESC] LIMIT k over one FLOAT64 / INT64 column.
//
// Replaces execute_sort_limit / try_typed_sort / top_k_ascending / assemble
// (FalconDB src/query/sort.rs:59-115, 209-445, 564-620, 773-791).  As in the
// reference, values become order keys on which ascending is the wanted order
// (f64_ord_key, sort.rs:451-454; sign-flipped two's complement for integers;
// bitwise NOT for DESC), and the k smallest (key, row) pairs are kept, so ties
// break on row ascending — the order the reference's (key,row) tuples give.
//
// GPU shape (two launches):
//  1. sample: a strided sample of the column (one row in kSampleStride) goes
//     through the block top-k below; its k-th best pair T0 is a valid bound — k
//     distinct rows are at or above it — so the true top-k lies in {x <= T0}.
//  2. main: the TMA streamer feeds every row; each CTA appends the rows with
//     (key,row) <= T to a shared-memory buffer (warp-aggregated), and when the
//     buffer could overflow it bitonic-sorts it, keeps k and tightens T.  Each
//     CTA writes its k best; the last CTA to finish merges them the same way.
// On random data T0 admits about k*kSampleStride rows in total; on an ascending
// column read DESC (the reference's slow case, FINDINGS.md) it admits the same.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "stream.cuh"
#include "topk_warp.cuh"

namespace fdb {

constexpr uint64_t kSampleStride = 256;
constexpr int kTopkR = 4;  // rows per consumer thread per sub-step

// Shared-memory state of one CTA's running top-k.
struct TopkSmem {
  uint64_t* keys;   // [cap]
  uint32_t* rows;   // [cap]
  uint32_t* count;  // number of live entries
  uint64_t* tk;     // threshold key (inclusive)
  uint32_t* tr;     // threshold row
  uint32_t* last;   // last-CTA flag
  uint32_t cap;
};

__host__ __device__ inline uint32_t topk_cap(uint32_t k, int nct) {
  uint32_t need = k + (uint32_t)nct * kTopkR;
  uint32_t c = 1;
  while (c < need) c <<= 1;
  return c;
}
__host__ __device__ inline size_t topk_smem_bytes(uint32_t cap) {
  return (size_t)cap * 12 + 64;
}
__device__ inline TopkSmem topk_smem(unsigned char* base, uint32_t cap) {
  TopkSmem s;
  s.keys = reinterpret_cast<uint64_t*>(base);
  s.rows = reinterpret_cast<uint32_t*>(base + (size_t)cap * 8);
  unsigned char* tail = base + (size_t)cap * 12;
  s.tk = reinterpret_cast<uint64_t*>(tail);
  s.count = reinterpret_cast<uint32_t*>(tail + 8);
  s.tr = reinterpret_cast<uint32_t*>(tail + 12);
  s.last = reinterpret_cast<uint32_t*>(tail + 16);
  s.cap = cap;
  return s;
}

// Sort the buffer ascending by (key,row) and keep the first k; tighten T when
// k entries are kept.  All nct consumer threads call it with the same `cnt`
// (the live count, read between two barriers) and get the same new count back.
__device__ uint32_t topk_reduce(TopkSmem& s, uint32_t k, uint32_t cnt, int ctid, int nct) {
  uint32_t n2 = 1;
  while (n2 < cnt) n2 <<= 1;  // sort the smallest power of two covering cnt
  for (uint32_t i = cnt + ctid; i < n2; i += nct) {
    s.keys[i] = ~0ull;
    s.rows[i] = 0xFFFFFFFFu;
  }
  consumer_bar(nct);
  for (uint32_t k2 = 2; k2 <= n2; k2 <<= 1) {
    for (uint32_t j = k2 >> 1; j > 0; j >>= 1) {
      for (uint32_t i = ctid; i < n2; i += nct) {
        const uint32_t ixj = i ^ j;
        if (ixj > i) {
          const uint64_t a = s.keys[i], b = s.keys[ixj];
          const uint32_t ra = s.rows[i], rb = s.rows[ixj];
          const bool up = (i & k2) == 0;
          if (kr_gt(a, ra, b, rb) == up) {
            s.keys[i] = b;
            s.keys[ixj] = a;
            s.rows[i] = rb;
            s.rows[ixj] = ra;
          }
        }
      }
      consumer_bar(nct);
    }
  }
  const uint32_t out = cnt < k ? cnt : k;
  if (ctid == 0) {
    *s.count = out;
    if (cnt >= k) {
      const uint64_t nk = s.keys[k - 1];
      const uint32_t nr = s.rows[k - 1];
      if (kr_le(nk, nr, *s.tk, *s.tr)) {
        *s.tk = nk;
        *s.tr = nr;
      }
    }
  }
  consumer_bar(nct);
  return out;
}

// Offer one candidate per thread (valid = has one); warp-aggregated append.
// Positions come from an atomic counter, so appends need no barrier.
__device__ __forceinline__ void topk_offer(TopkSmem& s, bool valid, uint64_t key, uint32_t row,
                                           uint64_t tk, uint32_t tr) {
  const bool cand = valid && kr_le(key, row, tk, tr);
  const unsigned m = __ballot_sync(0xffffffffu, cand);
  if (m == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(s.count, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (cand) {
    const uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
    s.keys[pos] = key;
    s.rows[pos] = row;
  }
}

__device__ __forceinline__ uint64_t topk_key(int dtype, bool desc, uint64_t bits) {
  const uint64_t k = dtype == FDB_FLOAT64 ? f64_ord_key(__longlong_as_double((long long)bits))
                                          : i64_ord_key((int64_t)bits);
  return desc ? ~k : k;
}

struct TopkParams {
  DevCol col;
  uint32_t k;
  int32_t desc;
  uint64_t row_stride;      // 1 for the main pass, kSampleStride for the sample
  const uint64_t* t0;       // [key, row, valid] bound from the sample pass, or nullptr
  uint64_t* partials_k;     // [grid * k]
  uint32_t* partials_r;     // [grid * k]
  unsigned int* ticket;
  uint32_t* out_rows;       // [k] final rows, or nullptr
  uint64_t* out_count;      // final count, or nullptr
  uint64_t* out_t0;         // [3]: k-th best pair of this pass (sample pass), or nullptr
};

struct TopkOp {
  using Params = TopkParams;
  // Register state, identical in every consumer thread: how many more
  // sub-steps fit in the buffer before the next check, and the threshold.
  struct Local {
    uint32_t allow;
    uint64_t tk;
    uint32_t tr;
  };

  static __device__ void init(Local& st, const Params& p, unsigned char* sm, int ctid, int nct) {
    TopkSmem s = topk_smem(sm, topk_cap(p.k, nct));
    st.allow = 0;  // forces a check (and a threshold read) before the first append
    st.tk = ~0ull;
    st.tr = 0xFFFFFFFFu;
    if (ctid == 0) {
      *s.count = 0;
      *s.last = 0;
      if (p.t0 && p.t0[2]) {
        *s.tk = p.t0[0];
        *s.tr = (uint32_t)p.t0[1];
      } else {
        *s.tk = ~0ull;
        *s.tr = 0xFFFFFFFFu;
      }
    }
  }

  // Room check: read the live count between two barriers (so no append races
  // the read), sort-reduce when one more sub-step might not fit, then refresh
  // the allowance and the threshold.
  static __device__ void check(Local& st, TopkSmem& s, uint32_t k, int ctid, int nct) {
    const uint32_t sub = (uint32_t)nct * kTopkR;
    consumer_bar(nct);
    uint32_t cnt = *s.count;
    consumer_bar(nct);
    if (s.cap - cnt < sub) cnt = topk_reduce(s, k, cnt, ctid, nct);
    st.allow = (s.cap - cnt) / sub;
    st.tk = *s.tk;
    st.tr = *s.tr;
  }

  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char* sm, const Acc& acc,
                              uint32_t rows, int ctid, int nct) {
    TopkSmem s = topk_smem(sm, topk_cap(p.k, nct));
    const uint32_t sub = (uint32_t)nct * kTopkR;
    for (uint32_t b = 0; b < rows; b += sub) {
      if (st.allow == 0) check(st, s, p.k, ctid, nct);
      --st.allow;
#pragma unroll
      for (int j = 0; j < kTopkR; ++j) {
        const uint32_t i = b + j * nct + ctid;
        uint64_t key = 0;
        uint32_t row = 0;
        bool valid = false;
        if (i < rows) {
          const uint64_t grow = acc.row(i) * p.row_stride;
          row = (uint32_t)grow;
          valid = p.col.validity ? col_valid(p.col, grow) : true;
          key = topk_key(p.col.dtype, p.desc, acc.template get<uint64_t>(0, i));
        }
        topk_offer(s, valid, key, row, st.tk, st.tr);
      }
    }
  }

  static __device__ void finish(Local& st, const Params& p, unsigned char* sm, int ctid, int nct) {
    TopkSmem s = topk_smem(sm, topk_cap(p.k, nct));
    const uint32_t k = p.k;
    consumer_bar(nct);
    uint32_t cnt = *s.count;
    consumer_bar(nct);
    cnt = topk_reduce(s, k, cnt, ctid, nct);  // sorted, cnt <= k
    for (uint32_t i = ctid; i < k; i += nct) {
      p.partials_k[(size_t)blockIdx.x * k + i] = i < cnt ? s.keys[i] : ~0ull;
      p.partials_r[(size_t)blockIdx.x * k + i] = i < cnt ? s.rows[i] : 0xFFFFFFFFu;
    }
    __threadfence();
    consumer_bar(nct);
    if (ctid == 0) {
      const unsigned int t = atomicAdd(p.ticket, 1u);
      *s.last = (t == gridDim.x - 1) ? 1u : 0u;
    }
    consumer_bar(nct);
    if (*s.last == 0) return;
    __threadfence();
    // Last CTA: merge every other CTA's k best through the same buffer (its own
    // are already there).  The sentinel pair (~0, 0xFFFFFFFF) is never a real
    // row (rows < 2^32-1) and is skipped.
    const uint32_t total = gridDim.x * k;
    const uint32_t sub = (uint32_t)nct * kTopkR;
    st.allow = 0;
    for (uint32_t b = 0; b < total; b += sub) {
      if (st.allow == 0) check(st, s, k, ctid, nct);
      --st.allow;
#pragma unroll
      for (int j = 0; j < kTopkR; ++j) {
        const uint32_t i = b + j * nct + ctid;
        bool valid = false;
        uint64_t key = 0;
        uint32_t row = 0;
        if (i < total && i / k != blockIdx.x) {
          key = __ldcg(&p.partials_k[i]);
          row = __ldcg(&p.partials_r[i]);
          valid = !(key == ~0ull && row == 0xFFFFFFFFu);
        }
        topk_offer(s, valid, key, row, st.tk, st.tr);
      }
    }
    consumer_bar(nct);
    cnt = *s.count;
    consumer_bar(nct);
    const uint32_t fin = topk_reduce(s, k, cnt, ctid, nct);
    if (p.out_rows)
      for (uint32_t i = ctid; i < fin; i += nct) p.out_rows[i] = s.rows[i];
    if (ctid == 0) {
      if (p.out_count) *p.out_count = fin;
      if (p.out_t0) {
        const bool ok = fin >= k;
        p.out_t0[0] = ok ? s.keys[k - 1] : ~0ull;
        p.out_t0[1] = ok ? s.rows[k - 1] : 0xFFFFFFFFu;
        p.out_t0[2] = ok ? 1 : 0;
      }
      *p.ticket = 0u;
    }
  }
};

// Sample pass: plain strided loads, all threads are consumers.
struct StridedAcc {
  const uint64_t* base;
  uint64_t row0;   // sample index of local row 0
  uint64_t stride;
  template <typename T>
  __device__ __forceinline__ T get(int, uint32_t i) const {
    return (T)base[(row0 + i) * stride];
  }
  __device__ __forceinline__ uint64_t row(uint32_t i) const { return row0 + i; }
};

__global__ void __launch_bounds__(256) topk_sample_kernel(TopkParams p, uint64_t nsamples) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int nct = blockDim.x, ctid = threadIdx.x;
  TopkOp::Local st;
  TopkOp::init(st, p, smem, ctid, nct);
  consumer_bar(nct);
  const uint64_t per = (nsamples + gridDim.x - 1) / gridDim.x;
  const uint64_t s0 = blockIdx.x * per;
  const uint64_t s1 = umin64(nsamples, s0 + per);
  const uint32_t CH = nct * 16;
  for (uint64_t c0 = s0; c0 < s1; c0 += CH) {
    StridedAcc acc{static_cast<const uint64_t*>(p.col.values), c0, p.row_stride};
    TopkOp::step(st, p, smem, acc, (uint32_t)umin64(CH, s1 - c0), ctid, nct);
  }
  TopkOp::finish(st, p, smem, ctid, nct);
}

// ===========================================================================
// Warp-level top-k (k <= 256): the hot path.
//
// Each warp owns a candidate buffer of kWCap (key,row) pairs in shared memory
// and keeps its count and threshold in registers (identical in every lane, so
// no atomics and no block barrier are needed while streaming).  A warp step
// covers 256 rows (8 per lane, read as 16-byte shared-memory vectors from the
// TMA tile); rows with (key,row) <= T are appended at positions from a lane
// prefix sum of their popcounts.  When the buffer could overflow the warp
// bitonic-sorts it, keeps k and tightens T.  At the end the CTA's warps merge
// pairwise into warp 0, the CTA writes its k best, and the last CTA merges all.
// ===========================================================================
constexpr uint32_t kWCap = 512;
constexpr int kWRows = 8;
constexpr uint32_t kMaxWarpK = kWCap - 32 * kWRows;  // 256

struct WTSmem {
  uint64_t keys[8][kWCap];
  uint32_t rows[8][kWCap];
  uint32_t cnt[8];
  uint32_t last;
};

struct WTState {  // warp-uniform
  uint32_t count;
  uint64_t tk;
  uint32_t tr;
};

__device__ void wt_sort(uint64_t* keys, uint32_t* rows, uint32_t n2, int lane) {
  for (uint32_t k2 = 2; k2 <= n2; k2 <<= 1) {
    for (uint32_t j = k2 >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < n2; i += 32) {
        const uint32_t ixj = i ^ j;
        if (ixj > i) {
          const uint64_t a = keys[i], b = keys[ixj];
          const uint32_t ra = rows[i], rb = rows[ixj];
          if (kr_gt(a, ra, b, rb) == ((i & k2) == 0)) {
            keys[i] = b;
            keys[ixj] = a;
            rows[i] = rb;
            rows[ixj] = ra;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Sort the warp's buffer, keep the best k, tighten the threshold.
__device__ void wt_reduce(uint64_t* keys, uint32_t* rows, WTState& st, uint32_t k, int lane) {
  if (st.count == 0) return;
  uint32_t n2 = 1;
  while (n2 < st.count) n2 <<= 1;
  for (uint32_t i = st.count + lane; i < n2; i += 32) {
    keys[i] = ~0ull;
    rows[i] = 0xFFFFFFFFu;
  }
  __syncwarp();
  wt_sort(keys, rows, n2, lane);
  if (st.count >= k) {
    const uint64_t nk = keys[k - 1];
    const uint32_t nr = rows[k - 1];
    if (kr_le(nk, nr, st.tk, st.tr)) {
      st.tk = nk;
      st.tr = nr;
    }
    st.count = k;
  }
  __syncwarp();
}

// Offer this lane's (up to kWRows) rows; vm marks the real ones.
__device__ __forceinline__ void wt_offer(uint64_t* keys, uint32_t* rows, WTState& st, uint32_t k,
                                         const uint64_t (&key)[kWRows], const uint32_t (&row)[kWRows],
                                         uint32_t vm, int lane) {
  uint32_t m = 0;
#pragma unroll
  for (int j = 0; j < kWRows; ++j)
    if (((vm >> j) & 1u) && kr_le(key[j], row[j], st.tk, st.tr)) m |= 1u << j;
  if (!__any_sync(0xffffffffu, m)) return;
  if (st.count + 32 * kWRows > kWCap) {
    wt_reduce(keys, rows, st, k, lane);
    m = 0;
#pragma unroll
    for (int j = 0; j < kWRows; ++j)
      if (((vm >> j) & 1u) && kr_le(key[j], row[j], st.tk, st.tr)) m |= 1u << j;
  }
  const uint32_t c = __popc(m);
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  uint32_t pos = st.count + incl - c;
#pragma unroll
  for (int j = 0; j < kWRows; ++j)
    if ((m >> j) & 1u) {
      keys[pos] = key[j];
      rows[pos] = row[j];
      ++pos;
    }
  st.count += total;
  __syncwarp();
}

// Merge the CTA's warp buffers pairwise into warp 0 (consumers only).
__device__ void wt_tree_merge(WTSmem& s, WTState& st, uint32_t k, int warp, int lane, int nct) {
  if (lane == 0) s.cnt[warp] = st.count;
  for (int half = 4; half >= 1; half >>= 1) {
    consumer_bar(nct);
    if (warp < half) {
      const uint32_t oc = s.cnt[warp + half];
      for (uint32_t i = lane; i < oc; i += 32) {
        s.keys[warp][st.count + i] = s.keys[warp + half][i];
        s.rows[warp][st.count + i] = s.rows[warp + half][i];
      }
      st.count += oc;
      __syncwarp();
      wt_reduce(s.keys[warp], s.rows[warp], st, k, lane);
      if (lane == 0) s.cnt[warp] = st.count;
    }
  }
  consumer_bar(nct);
}

// The CTA's k best -> partials; the last CTA merges every CTA's and writes the
// result (rows in order, count, and the k-th pair for the sample pass).
__device__ void wt_finish(WTSmem& s, WTState& st, const TopkParams& p, int ctid, int nct) {
  const int warp = ctid >> 5, lane = ctid & 31;
  const uint32_t k = p.k;
  wt_reduce(s.keys[warp], s.rows[warp], st, k, lane);
  wt_tree_merge(s, st, k, warp, lane, nct);
  if (warp == 0) {
    for (uint32_t i = lane; i < k; i += 32) {
      p.partials_k[(size_t)blockIdx.x * k + i] = i < st.count ? s.keys[0][i] : ~0ull;
      p.partials_r[(size_t)blockIdx.x * k + i] = i < st.count ? s.rows[0][i] : 0xFFFFFFFFu;
    }
  }
  __threadfence();
  consumer_bar(nct);
  if (ctid == 0) s.last = (atomicAdd(p.ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
  consumer_bar(nct);
  if (s.last == 0) return;
  __threadfence();
  // Last CTA: warp 0 keeps this CTA's k best; warps 1..7 start empty (their
  // thresholds remain valid bounds) and every warp takes a share of the other
  // CTAs' partials, 256 entries per warp step.
  if (warp != 0) st.count = 0;
  const uint32_t total = gridDim.x * k;
  const uint32_t nchunks = (total + 255) / 256;
  for (uint32_t ch = warp; ch < nchunks; ch += nct / 32) {
    uint64_t key[kWRows];
    uint32_t row[kWRows];
    uint32_t vm = 0;
#pragma unroll
    for (int j = 0; j < kWRows; ++j) {
      const uint32_t i = ch * 256 + j * 32 + lane;
      key[j] = ~0ull;
      row[j] = 0xFFFFFFFFu;
      if (i < total && i / k != blockIdx.x) {
        key[j] = __ldcg(&p.partials_k[i]);
        row[j] = __ldcg(&p.partials_r[i]);
        if (!(key[j] == ~0ull && row[j] == 0xFFFFFFFFu)) vm |= 1u << j;
      }
    }
    wt_offer(s.keys[warp], s.rows[warp], st, k, key, row, vm, lane);
  }
  wt_reduce(s.keys[warp], s.rows[warp], st, k, lane);
  wt_tree_merge(s, st, k, warp, lane, nct);
  if (warp == 0) {
    const uint32_t fin = st.count;
    if (p.out_rows)
      for (uint32_t i = lane; i < fin; i += 32) p.out_rows[i] = s.rows[0][i];
    if (lane == 0) {
      if (p.out_count) *p.out_count = fin;
      if (p.out_t0) {
        const bool ok = fin >= k;
        p.out_t0[0] = ok ? s.keys[0][k - 1] : ~0ull;
        p.out_t0[1] = ok ? s.rows[0][k - 1] : 0xFFFFFFFFu;
        p.out_t0[2] = ok ? 1 : 0;
      }
      *p.ticket = 0u;
    }
  }
}

__device__ __forceinline__ void wt_init(WTState& st, const TopkParams& p) {
  st.count = 0;
  if (p.t0 && p.t0[2]) {
    st.tk = p.t0[0];
    st.tr = (uint32_t)p.t0[1];
  } else {
    st.tk = ~0ull;
    st.tr = 0xFFFFFFFFu;
  }
}

template <int DT, bool DESC>
struct WarpTopkOp {
  using Params = TopkParams;
  using Local = WTState;

  static __device__ void init(Local& st, const Params& p, unsigned char*, int, int) { wt_init(st, p); }

  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char* sm, const Acc& acc, uint32_t rows,
                              int ctid, int nct) {
    WTSmem& s = *reinterpret_cast<WTSmem*>(sm);
    const int warp = ctid >> 5, lane = ctid & 31;
    for (uint32_t b = 0; b < rows; b += 32 * kWRows * (nct / 32)) {
      const uint32_t base = b + warp * 32 * kWRows;
      uint64_t key[kWRows];
      uint32_t row[kWRows];
      uint32_t vm = 0;
#pragma unroll
      for (int q = 0; q < kWRows / 2; ++q) {
        const uint32_t i = base + q * 64 + 2 * lane;  // rows i, i+1
        uint64_t v0 = 0, v1 = 0;
        if constexpr (Acc::kSmemTile) {
          if (i + 1 < rows) {
            const ulonglong2 v = reinterpret_cast<const ulonglong2*>(acc.template col_ptr<uint64_t>(0))[i >> 1];
            v0 = v.x;
            v1 = v.y;
            vm |= 3u << (2 * q);
          } else if (i < rows) {
            v0 = acc.template get<uint64_t>(0, i);
            vm |= 1u << (2 * q);
          }
        } else {
          if (i < rows) {
            v0 = acc.template get<uint64_t>(0, i);
            vm |= 1u << (2 * q);
          }
          if (i + 1 < rows) {
            v1 = acc.template get<uint64_t>(0, i + 1);
            vm |= 2u << (2 * q);
          }
        }
        key[2 * q] = wt_key<DT, DESC>(v0);
        key[2 * q + 1] = wt_key<DT, DESC>(v1);
        row[2 * q] = (uint32_t)acc.row(i);
        row[2 * q + 1] = (uint32_t)acc.row(i + 1);
      }
      if (p.col.validity) {
#pragma unroll
        for (int j = 0; j < kWRows; ++j)
          if (((vm >> j) & 1u) && !col_valid(p.col, row[j])) vm &= ~(1u << j);
      }
      wt_offer(s.keys[warp], s.rows[warp], st, p.k, key, row, vm, lane);
    }
  }

  static __device__ void finish(Local& st, const Params& p, unsigned char* sm, int ctid, int nct) {
    wt_finish(*reinterpret_cast<WTSmem*>(sm), st, p, ctid, nct);
  }
};

// Sample pass for the warp top-k: every load of a warp step is issued before
// any is used, so the strided reads overlap.
template <int DT, bool DESC>
__global__ void __launch_bounds__(256) wt_sample_kernel(TopkParams p, uint64_t nsamples) {
  extern __shared__ __align__(128) unsigned char smem[];
  WTSmem& s = *reinterpret_cast<WTSmem*>(smem);
  const int ctid = threadIdx.x, nct = blockDim.x, warp = ctid >> 5, lane = ctid & 31;
  WTState st;
  wt_init(st, p);
  const uint64_t* col = static_cast<const uint64_t*>(p.col.values);
  const uint64_t per_block = 32 * kWRows * (nct / 32);
  for (uint64_t b = (uint64_t)blockIdx.x * per_block; b < nsamples; b += (uint64_t)gridDim.x * per_block) {
    uint64_t key[kWRows];
    uint32_t row[kWRows];
    uint32_t vm = 0;
    uint64_t v[kWRows];
#pragma unroll
    for (int j = 0; j < kWRows; ++j) {
      const uint64_t i = b + warp * 32 * kWRows + j * 32 + lane;
      row[j] = (uint32_t)(i * p.row_stride);
      v[j] = 0;
      if (i < nsamples) {
        v[j] = __ldg(col + i * p.row_stride);
        vm |= 1u << j;
      }
    }
#pragma unroll
    for (int j = 0; j < kWRows; ++j) {
      key[j] = wt_key<DT, DESC>(v[j]);
      if (((vm >> j) & 1u) && p.col.validity && !col_valid(p.col, row[j])) vm &= ~(1u << j);
    }
    wt_offer(s.keys[warp], s.rows[warp], st, p.k, key, row, vm, lane);
  }
  wt_finish(s, st, p, ctid, nct);
}

// ===========================================================================
// Register top-k (k <= 32): the fast path, one launch.
//
// Every warp holds its best k (key,row) pairs in registers, lane j holding the
// j-th best, and a threshold T: the k-th best it holds, or a tighter bound
// shared across CTAs.  A row is a candidate when (key,row) <= T; a candidate
// is inserted with one ballot (the first lane whose entry is worse) and a
// shuffle that shifts the tail one lane right — no buffer and no sort.
//
// Bounds: before streaming, each CTA reads a strided sample of its own tiles
// (8 rows per 2048-row tile, spread over all its tiles), finds the sample's k-th
// best key, and publishes it with atomicMin to a global bound (k distinct rows
// have keys <= it, so every row of the true top-k does too).  Warps filter with
// min(own k-th best, global bound) and refresh the global bound every 16
// tiles.  An ascending column read DESC — every row beats the rows before it —
// then admits only the rows above the sampled bound.  At the end each CTA
// merges its warps, publishes its k-th key, writes its k best, and the last
// CTA merges the partials that are <= the final global bound.
// ===========================================================================
constexpr uint32_t kRegMaxK = 32;
constexpr uint64_t kRegSamples = 32768;  // sample budget of the register top-k's bound
// Tiles between exchanges of a CTA's bound with the global one (0: never
// during the scan; the CTAs' final bounds still meet in gbound).
#ifndef FDB_TOPK_GLOBAL_EVERY
#define FDB_TOPK_GLOBAL_EVERY 0
#endif
constexpr uint32_t kRtGlobalEvery = FDB_TOPK_GLOBAL_EVERY;

struct RTParams {
  DevCol col;
  uint64_t m_end;                 // rows staged by TMA (multiple of the tile size, or n)
  uint64_t n;
  uint32_t k;
  uint32_t tile_rows;
  unsigned long long* gbound;     // best k-th key seen by any CTA (init ~0)
  uint64_t* partials_k;           // [grid * k]
  uint32_t* partials_r;
  unsigned int* ticket;
  uint32_t* out_rows;
  uint64_t* out_count;
};

struct RTSmem {
  uint64_t keys[8][32];
  uint32_t rows[8][32];
  unsigned long long bound;  // this CTA's view of the best k-th key (key-only bound)
  uint32_t last;
};

// Publish a warp's k-th best key into the CTA bound and refresh the warp's
// threshold from it; warp 0 also exchanges the CTA bound with the global one.
__device__ __forceinline__ void rt_share(RTSmem& sm, RTLocal& s, const RTParams& p, int warp, int lane,
                                         bool with_global) {
  const uint64_t kk = __shfl_sync(0xffffffffu, s.lk, p.k - 1);
  const uint32_t kr = __shfl_sync(0xffffffffu, s.lr, p.k - 1);
  unsigned long long nb = 0;
  if (lane == 0) {
    volatile unsigned long long* vb = &sm.bound;
    if (!(kk == ~0ull && kr == 0xFFFFFFFFu) && kk < *vb) atomicMin(&sm.bound, (unsigned long long)kk);
    if (with_global && warp == 0) {
      const unsigned long long g = *reinterpret_cast<volatile unsigned long long*>(p.gbound);
      const unsigned long long b = *vb;
      if (b < g)
        atomicMin(p.gbound, b);
      else if (g < b)
        atomicMin(&sm.bound, g);
    }
    nb = *vb;
  }
  rt_bound(s, __shfl_sync(0xffffffffu, nb, 0));
}

// Merge the warps' lists into warp 0 (consumer threads only): log2(warps)
// levels, each a sorted-list merge of the upper half's lists into the lower's.
__device__ void rt_tree_merge(RTSmem& sm, RTLocal& s, uint32_t k, int warp, int lane, int nct) {
  for (int half = (nct >> 5) / 2; half >= 1; half >>= 1) {
    consumer_bar(nct);
    if (warp >= half && warp < 2 * half) {
      const bool in = (uint32_t)lane < k;
      sm.keys[warp][lane] = in ? s.lk : ~0ull;
      sm.rows[warp][lane] = in ? s.lr : 0xFFFFFFFFu;
    }
    consumer_bar(nct);
    if (warp < half) rt_merge_sorted(s, k, sm.keys[warp + half][lane], sm.rows[warp + half][lane], lane);
  }
  consumer_bar(nct);
}

template <int DT, bool DESC>
struct RegTopkOp {
  using Params = RTParams;
  using Local = RTLocal;

  static __device__ void init(Local& s, const Params& p, unsigned char* smraw, int ctid, int nct) {
    RTSmem& sm = *reinterpret_cast<RTSmem*>(smraw);
    const int warp = ctid >> 5, lane = ctid & 31;
    rt_clear(s);
    s.tk = ~0ull;
    s.tr = 0xFFFFFFFFu;
    s.steps = 0;
    // Start from the bound the sample pass leaves in gbound.  This grid may be
    // launched while the sample pass still runs (programmatic dependent
    // launch: the producer warp is already streaming tiles); consumers wait
    // here until it has completed and its writes are visible.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (ctid == 0) sm.bound = *reinterpret_cast<volatile unsigned long long*>(p.gbound);
    consumer_bar(nct);
    rt_bound(s, sm.bound);
    (void)warp;
    (void)lane;
  }

  template <class Acc>
  static __device__ void step(Local& s, const Params& p, unsigned char* smraw, const Acc& acc, uint32_t rows, int ctid,
                              int nct) {
    const int warp = ctid >> 5, lane = ctid & 31;
    for (uint32_t b = 0; b < rows; b += 256 * (nct / 32)) {
      const uint32_t base = b + warp * 256;
      uint64_t v[8];
      uint32_t vm = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t i = base + q * 64 + 2 * lane;
        v[2 * q] = 0;
        v[2 * q + 1] = 0;
        if constexpr (Acc::kSmemTile) {
          if (i + 1 < rows) {
            const ulonglong2 x = reinterpret_cast<const ulonglong2*>(acc.template col_ptr<uint64_t>(0))[i >> 1];
            v[2 * q] = x.x;
            v[2 * q + 1] = x.y;
            vm |= 3u << (2 * q);
          } else if (i < rows) {
            v[2 * q] = acc.template get<uint64_t>(0, i);
            vm |= 1u << (2 * q);
          }
        } else {
          if (i < rows) {
            v[2 * q] = acc.template get<uint64_t>(0, i);
            vm |= 1u << (2 * q);
          }
          if (i + 1 < rows) {
            v[2 * q + 1] = acc.template get<uint64_t>(0, i + 1);
            vm |= 2u << (2 * q);
          }
        }
      }
      // Prefilter in the value domain against the threshold's value: a row is
      // dropped only when its value is strictly worse (an ordered compare, so a
      // NaN on either side passes on to the exact test; so does -0.0 against
      // +0.0).  Every dropped row has an order key above T's key.  Order keys
      // and the row tie-break are only computed for rows that pass.
      uint32_t pm = 0;
      const uint64_t tkey = DESC ? ~s.tk : s.tk;
      if constexpr (DT == FDB_FLOAT64) {
        const double tv = f64_from_ord_key(tkey);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const double x = __longlong_as_double((long long)v[j]);
          if (!(DESC ? x < tv : x > tv)) pm |= 1u << j;
        }
      } else {
        const int64_t tv = (int64_t)(tkey ^ (1ull << 63));
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int64_t x = (int64_t)v[j];
          if (DESC ? x >= tv : x <= tv) pm |= 1u << j;
        }
      }
      pm &= vm;
      if (!__any_sync(0xffffffffu, pm != 0u)) continue;
      uint64_t key[8];
      uint32_t row[8];
      uint32_t m = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t i = base + (j >> 1) * 64 + 2 * lane + (j & 1);
        key[j] = wt_key<DT, DESC>(v[j]);
        row[j] = (uint32_t)acc.row(i);
        if (((pm >> j) & 1u) && kr_le(key[j], row[j], s.tk, s.tr)) m |= 1u << j;
      }
      if (p.col.validity) {
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (((m >> j) & 1u) && !col_valid(p.col, row[j])) m &= ~(1u << j);
      }
      if (__any_sync(0xffffffffu, m != 0u)) rt_offer<8>(s, p.k, key, row, m, lane);
    }
    // Every 4 tiles: publish to the CTA bound and refresh from it; every 16
    // tiles warp 0 also exchanges it with the global bound.
    ++s.steps;
    if ((s.steps & 3u) == 0u)
      rt_share(*reinterpret_cast<RTSmem*>(smraw), s, p, warp, lane,
               kRtGlobalEvery != 0u && (s.steps % kRtGlobalEvery) == 0u);
  }

  static __device__ void finish(Local& s, const Params& p, unsigned char* smraw, int ctid, int nct) {
    RTSmem& sm = *reinterpret_cast<RTSmem*>(smraw);
    const int warp = ctid >> 5, lane = ctid & 31;
    const uint32_t k = p.k;
    rt_tree_merge(sm, s, k, warp, lane, nct);
    if (warp == 0) {
      const uint64_t kk = __shfl_sync(0xffffffffu, s.lk, k - 1);
      const uint32_t kr = __shfl_sync(0xffffffffu, s.lr, k - 1);
      if (lane == 0 && !(kk == ~0ull && kr == 0xFFFFFFFFu)) atomicMin(p.gbound, (unsigned long long)kk);
      if ((uint32_t)lane < k) {
        p.partials_k[(size_t)blockIdx.x * k + lane] = s.lk;
        p.partials_r[(size_t)blockIdx.x * k + lane] = s.lr;
      }
    }
    __threadfence();
    consumer_bar(nct);
    if (ctid == 0) sm.last = (atomicAdd(p.ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
    consumer_bar(nct);
    if (sm.last == 0) return;
    __threadfence();
    // Last CTA: only partials at or under the final global bound can matter.
    const uint64_t gb = *reinterpret_cast<volatile unsigned long long*>(p.gbound);
    rt_bound(s, gb);
    if (warp != 0) rt_clear(s);
    // One thread per CTA list: each list is sorted, so only a prefix of it can
    // be at or under the bound, and most lists stop at their first entry.
    // Up to 8 entries per list per pass; a list with more qualifying entries
    // (possible only while the bound is loose) is walked in further passes.
    for (uint32_t c0 = 0; c0 < gridDim.x; c0 += nct) {
      const uint32_t c = c0 + ctid;
      uint32_t from = 0;
      for (;;) {
        uint64_t key[8];
        uint32_t row[8];
        uint32_t m = 0;
        bool more = false;
        if (c < gridDim.x && c != blockIdx.x) {
          const uint64_t* lk = p.partials_k + (size_t)c * k;
          const uint32_t* lr = p.partials_r + (size_t)c * k;
#pragma unroll
          for (int j = 0; j < 8; ++j) {  // independent loads: one L2 round trip per pass
            key[j] = ~0ull;
            row[j] = 0xFFFFFFFFu;
            if (from + j < k) {
              key[j] = __ldcg(lk + from + j);
              row[j] = __ldcg(lr + from + j);
            }
          }
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (!(key[j] == ~0ull && row[j] == 0xFFFFFFFFu) && kr_le(key[j], row[j], s.tk, s.tr)) m |= 1u << j;
          more = ((m >> 7) & 1u) && from + 8 < k;
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            key[j] = ~0ull;
            row[j] = 0xFFFFFFFFu;
          }
        }
        if (__any_sync(0xffffffffu, m != 0u)) rt_offer<8>(s, k, key, row, m, lane);
        if (!__any_sync(0xffffffffu, more)) break;
        from = more ? from + 8 : k;  // a finished list offers nothing on later passes
      }
    }
    rt_tree_merge(sm, s, k, warp, lane, nct);
    if (warp == 0) {
      const bool real = (uint32_t)lane < k && !(s.lk == ~0ull && s.lr == 0xFFFFFFFFu);
      const unsigned vb = __ballot_sync(0xffffffffu, real);
      if (real && p.out_rows) p.out_rows[lane] = s.lr;
      if (lane == 0) {
        if (p.out_count) *p.out_count = (uint64_t)__popc(vb);
        *p.ticket = 0u;
      }
    }
  }
};

// Sample pass of the register top-k: each warp reads 256 rows at a stride of
// kSampleStride (every load issued before any is used), finds its k-th best by
// k rounds of warp-wide min extraction, and the CTA publishes the best of its
// warps' bounds with one atomicMin on gbound.  k distinct rows have keys <=
// any warp's k-th best, so gbound bounds the true top-k.
template <int DT, bool DESC>
__global__ void __launch_bounds__(256) rt_sample_kernel(RTParams p, uint64_t nsamples, uint64_t stride) {
  __shared__ unsigned long long cta_bound;
  const int ctid = threadIdx.x, warp = ctid >> 5, lane = ctid & 31;
  // Let the main pass launch now; it waits for this grid before reading gbound.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (ctid == 0) cta_bound = ~0ull;
  __syncthreads();
  const uint64_t* col = static_cast<const uint64_t*>(p.col.values);
  for (uint64_t b = (uint64_t)blockIdx.x * 2048; b < nsamples; b += (uint64_t)gridDim.x * 2048) {
    uint64_t key[8];
    uint32_t row[8];
    uint64_t v[8];
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint64_t q = b + warp * 256 + j * 32 + lane;
      row[j] = (uint32_t)(q * stride);
      v[j] = 0;
      if (q < nsamples) {
        v[j] = __ldg(col + q * stride);
        m |= 1u << j;
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      key[j] = wt_key<DT, DESC>(v[j]);
      if (((m >> j) & 1u) && p.col.validity && !col_valid(p.col, row[j])) m &= ~(1u << j);
    }
    uint64_t kk = ~0ull;
    uint32_t got = 0;
    for (uint32_t r = 0; r < p.k; ++r) {
      uint64_t bk = ~0ull;
      uint32_t br = 0xFFFFFFFFu;
      int bj = -1;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (((m >> j) & 1u) && kr_gt(bk, br, key[j], row[j])) {
          bk = key[j];
          br = row[j];
          bj = j;
        }
      uint64_t wk = bk;
      uint32_t wr = br;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t ok = __shfl_xor_sync(0xffffffffu, wk, o);
        const uint32_t orow = __shfl_xor_sync(0xffffffffu, wr, o);
        if (kr_gt(wk, wr, ok, orow)) {
          wk = ok;
          wr = orow;
        }
      }
      if (wk == ~0ull && wr == 0xFFFFFFFFu) break;  // no samples left in this warp
      if (bj >= 0 && bk == wk && br == wr) m &= ~(1u << bj);
      kk = wk;
      ++got;
    }
    if (lane == 0 && got == p.k) atomicMin(&cta_bound, (unsigned long long)kk);
  }
  __syncthreads();
  if (ctid == 0 && cta_bound != ~0ull) atomicMin(p.gbound, cta_bound);
}

// Launch shape of the register top-k: tile rows, stages, consumer warps and
// the CTAs per SM its registers must allow.  Two CTAs per SM with six 16 KB
// stages each hold as many bytes in flight as three CTAs with four, and the
// final merge then walks 296 CTA lists instead of 444: 100M rows, score /
// id DESC LIMIT 10, 0.145 / 0.142 ms against 0.150 / 0.152 ms (5 stages: the
// same; 4096-row tiles x 3 stages at 2 CTAs: 0.144 / 0.151 ms).
#ifndef FDB_RT_TR
#define FDB_RT_TR 2048
#endif
#ifndef FDB_RT_STAGES
#define FDB_RT_STAGES 6
#endif
#ifndef FDB_RT_NCW
#define FDB_RT_NCW 8
#endif
#ifndef FDB_RT_MINB
#define FDB_RT_MINB 2
#endif
template <int DT, bool DESC>
static void launch_reg_topk(Ctx& c, const fdb_dev_column& col, uint64_t n, uint32_t k, uint64_t* partials_k,
                            uint32_t* partials_r, uint32_t* out_rows, uint64_t* out_count) {
  constexpr int TR = FDB_RT_TR, STAGES = FDB_RT_STAGES, NCW = FDB_RT_NCW;
  StreamSrc<1> src;
  src.base[0] = static_cast<const unsigned char*>(col.values);
  src.esize[0] = 8;
  src.n = n;
  const void* b = col.values;
  src.m_end = stream_m_end(&b, 1, n);
  RTParams p;
  std::memset(&p, 0, sizeof(p));
  p.col = DevCol{col.dtype, col.values, col.validity, col.validity_offset};
  p.m_end = src.m_end;
  p.n = n;
  p.k = k;
  p.tile_rows = TR;
  // gbound (8 bytes, ~0 = no bound yet) and the dynamic tile counter (4 bytes,
  // 0xFFFFFFFF on entry) share one memset.
  p.gbound = static_cast<unsigned long long*>(c.scratch_take(16));
  FDB_CUDA(cudaMemsetAsync(p.gbound, 0xFF, 16, c.stream));
  src.tile_ctr = reinterpret_cast<unsigned int*>(p.gbound + 1);
  if ((src.m_end + TR - 1) / TR >= 0xFFFFFFFFull) fail(FDB_E_ARG, "too many tiles for the tile counter");
  // At most kRegSamples samples: their loads are scattered (one DRAM burst
  // each), and the batched insertion absorbs the k * stride rows a coarser
  // bound admits.
  const uint64_t stride = std::max<uint64_t>(kSampleStride, n / kRegSamples);
  const uint64_t nsamples = (n + stride - 1) / stride;
  if (nsamples >= 2ull * k) {
    const unsigned sgrid = (unsigned)umin64((nsamples + 2047) / 2048, (uint64_t)c.sm_count * 8);
    rt_sample_kernel<DT, DESC><<<sgrid, 256, 0, c.stream>>>(p, nsamples, stride);
    FDB_CUDA(cudaGetLastError());
  }
  p.partials_k = partials_k;
  p.partials_r = partials_r;
  p.ticket = c.d_ticket;
  p.out_rows = out_rows;
  p.out_count = out_count;
  const int op_off = (int)stream_smem_bytes<1, TR, STAGES>();
  const size_t smem = op_off + sizeof(RTSmem);
  auto kern = stream_kernel<RegTopkOp<DT, DESC>, 1, TR, STAGES, NCW, 8, FDB_RT_MINB, true>;  // dynamic tiles
  static PerDeviceOnce attr;  // per instantiation and device
  attr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); });
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (NCW + 1) * 32, smem));
  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  const int grid = tuned_grid(c.tune.op[FDB_TUNE_TOPK], c.sm_count, per_sm, 4, ntiles, n);
  // Programmatic dependent launch: the grid may start (its producer warps
  // streaming tiles) while the sample pass finishes; consumers wait for it.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((NCW + 1) * 32);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c.stream;
  cudaLaunchAttribute lattr[1];
  lattr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  lattr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = lattr;
  cfg.numAttrs = 1;
  FDB_CUDA(cudaLaunchKernelEx(&cfg, kern, src, p, c.d_err, op_off));
}

// Assemble NULL rows with the keyed result (assemble, sort.rs:773-791).
__global__ void topk_assemble_kernel(const uint32_t* keyed, const uint64_t* keyed_count,
                                     const uint32_t* nulls, const uint64_t* null_count, uint32_t k,
                                     int nulls_last, uint32_t* out_rows, uint64_t* out_count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint64_t kc = *keyed_count, nc = *null_count;
  const uint64_t nn = nc < k ? nc : k;
  uint64_t o = 0;
  if (!nulls_last)
    for (uint64_t i = 0; i < nn && o < k; ++i) out_rows[o++] = nulls[i];
  for (uint64_t i = 0; i < kc && o < k; ++i) out_rows[o++] = keyed[i];
  if (nulls_last)
    for (uint64_t i = 0; i < nn && o < k; ++i) out_rows[o++] = nulls[i];
  *out_count = o;
}

// Mask of the NULL rows of a column view: bit i = row i is NULL.
__global__ void null_mask_kernel(const uint64_t* validity, uint64_t voff, uint64_t n, uint64_t* out) {
  const uint64_t nwords = (n + 63) / 64;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = voff + w * 64;
    const uint64_t q = b >> 6, r = b & 63;
    uint64_t v = validity[q] >> r;
    if (r && (w * 64 + (64 - r)) < n) v |= validity[q + 1] << (64 - r);
    uint64_t m = ~v;
    const uint64_t rem = n - w * 64;
    if (rem < 64) m &= (1ull << rem) - 1;
    out[w] = m;
  }
}

template <int NCW_>
static void launch_topk_main(Ctx& c, const fdb_dev_column& col, uint64_t n, const TopkParams& p) {
  constexpr int TR = 2048, STAGES = 4, NCW = NCW_;
  StreamSrc<1> src;
  src.base[0] = static_cast<const unsigned char*>(col.values);
  src.esize[0] = 8;
  src.n = n;
  const void* b = col.values;
  src.m_end = stream_m_end(&b, 1, n);
  const uint32_t cap = topk_cap(p.k, NCW * 32);
  const int op_off = (int)stream_smem_bytes<1, TR, STAGES>();
  const size_t smem = op_off + topk_smem_bytes(cap);
  auto kern = stream_kernel<TopkOp, 1, TR, STAGES, NCW>;
  static PerDeviceOnce attr;  // per instantiation and device
  attr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024)); });
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (NCW + 1) * 32, smem));
  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  // At most 4 CTAs per SM: the partials are sized for that.
  const int grid = tuned_grid(c.tune.op[FDB_TUNE_TOPK], c.sm_count, per_sm, 4, ntiles, n);
  kern<<<grid, (NCW + 1) * 32, smem, c.stream>>>(src, p, c.d_err, op_off);
  FDB_CUDA(cudaGetLastError());
}

// Warp top-k: optional sample pass, then the streamed main pass.
template <int DT, bool DESC>
static void launch_warp_topk(Ctx& c, const fdb_dev_column& col, uint64_t n, TopkParams p, bool sample,
                             uint64_t nsamples, uint64_t* t0) {
  const size_t wsm = sizeof(WTSmem);
  if (sample) {
    TopkParams ps = p;
    ps.row_stride = kSampleStride;
    ps.t0 = nullptr;
    ps.out_rows = nullptr;
    ps.out_count = nullptr;
    ps.out_t0 = t0;
    auto sk = wt_sample_kernel<DT, DESC>;
    static PerDeviceOnce sattr;  // per instantiation and device
    sattr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(sk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm)); });
    const int grid = (int)umin64((nsamples + 2047) / 2048, (uint64_t)c.sm_count * 4);
    sk<<<grid, 256, wsm, c.stream>>>(ps, nsamples);
    FDB_CUDA(cudaGetLastError());
  }
  constexpr int TR = 2048, STAGES = 4, NCW = 8;
  StreamSrc<1> src;
  src.base[0] = static_cast<const unsigned char*>(col.values);
  src.esize[0] = 8;
  src.n = n;
  const void* b = col.values;
  src.m_end = stream_m_end(&b, 1, n);
  p.row_stride = 1;
  p.t0 = sample ? t0 : nullptr;
  p.out_t0 = nullptr;
  const int op_off = (int)stream_smem_bytes<1, TR, STAGES>();
  const size_t smem = op_off + wsm;
  auto kern = stream_kernel<WarpTopkOp<DT, DESC>, 1, TR, STAGES, NCW>;
  static PerDeviceOnce attr;  // per instantiation and device
  attr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); });
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (NCW + 1) * 32, smem));
  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  const int grid = tuned_grid(c.tune.op[FDB_TUNE_TOPK], c.sm_count, per_sm, 4, ntiles, n);
  kern<<<grid, (NCW + 1) * 32, smem, c.stream>>>(src, p, c.d_err, op_off);
  FDB_CUDA(cudaGetLastError());
}

void op_topk(Ctx& c, const fdb_dev_column& col, uint64_t n, uint32_t k, bool desc, bool nulls_last,
             uint32_t* d_rows, uint64_t* d_count) {
  if (k < 1 || k > 4096) fail(FDB_E_ARG, "top-k supports 1 <= k <= 4096");
  if (col.dtype != FDB_FLOAT64 && col.dtype != FDB_INT64)
    fail(FDB_E_TYPE, "top-k needs a FLOAT64 or INT64 column");
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "top-k addresses rows as uint32");
  if (n == 0) {
    FDB_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), c.stream));
    return;
  }
  constexpr int NCW = 8;
  const int max_grid = c.sm_count * 4;
  TopkParams p;
  std::memset(&p, 0, sizeof(p));
  p.col = DevCol{col.dtype, col.values, col.validity, col.validity_offset};
  p.k = k;
  p.desc = desc ? 1 : 0;
  p.ticket = c.d_ticket;
  p.partials_k = static_cast<uint64_t*>(c.scratch_take(sizeof(uint64_t) * (size_t)max_grid * k));
  p.partials_r = static_cast<uint32_t*>(c.scratch_take(sizeof(uint32_t) * (size_t)max_grid * k));
  uint64_t* t0 = static_cast<uint64_t*>(c.scratch_take(3 * sizeof(uint64_t)));

  // 1. sample pass (only when the sample holds enough rows to bound the top-k)
  const uint64_t nsamples = (n + kSampleStride - 1) / kSampleStride;
  const bool sample = nsamples >= 8ull * k && n >= (1ull << 20);
  uint32_t* keyed_rows0 = d_rows;
  uint64_t* keyed_count0 = d_count;
  if (col.validity != nullptr) {
    keyed_rows0 = static_cast<uint32_t*>(c.scratch_take(sizeof(uint32_t) * k));
    keyed_count0 = static_cast<uint64_t*>(c.scratch_take(sizeof(uint64_t)));
  }
  if (k <= kRegMaxK) {
    const bool f64 = col.dtype == FDB_FLOAT64;
    if (f64 && desc)
      launch_reg_topk<FDB_FLOAT64, true>(c, col, n, k, p.partials_k, p.partials_r, keyed_rows0, keyed_count0);
    else if (f64)
      launch_reg_topk<FDB_FLOAT64, false>(c, col, n, k, p.partials_k, p.partials_r, keyed_rows0, keyed_count0);
    else if (desc)
      launch_reg_topk<FDB_INT64, true>(c, col, n, k, p.partials_k, p.partials_r, keyed_rows0, keyed_count0);
    else
      launch_reg_topk<FDB_INT64, false>(c, col, n, k, p.partials_k, p.partials_r, keyed_rows0, keyed_count0);
  } else if (k <= kMaxWarpK) {
    p.out_rows = keyed_rows0;
    p.out_count = keyed_count0;
    const bool f64 = col.dtype == FDB_FLOAT64;
    if (f64 && desc) launch_warp_topk<FDB_FLOAT64, true>(c, col, n, p, sample, nsamples, t0);
    else if (f64) launch_warp_topk<FDB_FLOAT64, false>(c, col, n, p, sample, nsamples, t0);
    else if (desc) launch_warp_topk<FDB_INT64, true>(c, col, n, p, sample, nsamples, t0);
    else launch_warp_topk<FDB_INT64, false>(c, col, n, p, sample, nsamples, t0);
  } else if (sample) {
    TopkParams ps = p;
    ps.row_stride = kSampleStride;
    ps.t0 = nullptr;
    ps.out_rows = nullptr;
    ps.out_count = nullptr;
    ps.out_t0 = t0;
    const uint32_t cap = topk_cap(k, 256);
    const size_t smem = topk_smem_bytes(cap);
    static PerDeviceOnce attr;  // per instantiation and device
    attr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(topk_sample_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)); });
    const int grid = (int)umin64((uint64_t)c.sm_count, (nsamples + 4095) / 4096);
    topk_sample_kernel<<<grid, 256, smem, c.stream>>>(ps, nsamples);
    FDB_CUDA(cudaGetLastError());
  }

  // 2. main pass (block-buffer path for k > 256)
  uint32_t* keyed_rows = keyed_rows0;
  uint64_t* keyed_count = keyed_count0;
  const bool has_nulls = col.validity != nullptr;
  if (k > kMaxWarpK) {
    p.row_stride = 1;
    p.t0 = sample ? t0 : nullptr;
    p.out_rows = keyed_rows;
    p.out_count = keyed_count;
    p.out_t0 = nullptr;
    launch_topk_main<NCW>(c, col, n, p);
  }

  // 3. NULL rows (first k in row order) and assembly.
  if (has_nulls) {
    const uint64_t nwords = (n + 63) / 64;
    uint64_t* nmask = static_cast<uint64_t*>(c.scratch_take(nwords * 8));
    uint32_t* nrows = static_cast<uint32_t*>(c.scratch_take(sizeof(uint32_t) * k));
    uint64_t* ncount = static_cast<uint64_t*>(c.scratch_take(sizeof(uint64_t)));
    const unsigned nb = (unsigned)umin64((nwords + 255) / 256, (uint64_t)c.sm_count * 4);
    null_mask_kernel<<<nb, 256, 0, c.stream>>>(col.validity, col.validity_offset, n, nmask);
    // Capacity k: the compaction counts every NULL row but writes the first k.
    // Its capacity error flag is not an error here, so use a private error word.
    int* priv_err = static_cast<int*>(c.scratch_take(sizeof(int)));
    FDB_CUDA(cudaMemsetAsync(priv_err, 0, sizeof(int), c.stream));
    int* saved = c.d_err;
    c.d_err = priv_err;
    op_compact_mask(c, nmask, n, nrows, k, ncount);
    c.d_err = saved;
    topk_assemble_kernel<<<1, 32, 0, c.stream>>>(keyed_rows, keyed_count, nrows, ncount, k,
                                                 nulls_last ? 1 : 0, d_rows, d_count);
    FDB_CUDA(cudaGetLastError());
  }
}

}  // namespace fdb
