// Warp-level top-k building blocks shared by the top-k kernels (k_topk.cu)
// and the serving kernel (serve.cu): (order key, row) comparisons, order-key
// transforms, and a warp-held sorted list of up to 32 entries (lane i holds
// the i-th best) with single, batched (bitonic) and sorted-list insertion.
#pragma once
#include "common.cuh"

namespace fdb {

struct KR {
  uint64_t k;
  uint32_t r;
};
__device__ __forceinline__ bool kr_le(uint64_t ak, uint32_t ar, uint64_t bk, uint32_t br) {
  return ak < bk || (ak == bk && ar <= br);
}
__device__ __forceinline__ bool kr_gt(uint64_t ak, uint32_t ar, uint64_t bk, uint32_t br) {
  return ak > bk || (ak == bk && ar > br);
}

// Order key of a raw 8-byte value for ORDER BY (sort.rs:243-268, 451-454):
// ascending key order = the SQL order; DESC flips every bit.
template <int DT, bool DESC>
__device__ __forceinline__ uint64_t wt_key(uint64_t bits) {
  uint64_t k;
  if constexpr (DT == FDB_FLOAT64)
    k = (bits >> 63) ? ~bits : (bits ^ (1ull << 63));
  else
    k = bits ^ (1ull << 63);
  return DESC ? ~k : k;
}

struct RTLocal {
  uint64_t lk;  // this lane's list entry
  uint32_t lr;
  uint64_t tk;  // warp threshold (inclusive)
  uint32_t tr;
  uint32_t steps;
};

__device__ __forceinline__ void rt_insert(RTLocal& s, uint32_t k, uint64_t ck, uint32_t cr, int lane) {
  const bool worse = (uint32_t)lane < k && kr_gt(s.lk, s.lr, ck, cr);
  const unsigned b = __ballot_sync(0xffffffffu, worse);
  if (!b) return;
  const int pos = __ffs(b) - 1;
  const uint64_t pk = __shfl_up_sync(0xffffffffu, s.lk, 1);
  const uint32_t pr = __shfl_up_sync(0xffffffffu, s.lr, 1);
  if (lane > pos) {
    s.lk = pk;
    s.lr = pr;
  } else if (lane == pos) {
    s.lk = ck;
    s.lr = cr;
  }
  const uint64_t kk = __shfl_sync(0xffffffffu, s.lk, k - 1);
  const uint32_t kr = __shfl_sync(0xffffffffu, s.lr, k - 1);
  if (kr_le(kk, kr, s.tk, s.tr)) {
    s.tk = kk;
    s.tr = kr;
  }
}

// One compare-exchange of a bitonic network across lanes: this lane keeps the
// smaller (key,row) of itself and lane ^ stride when keep_min, else the larger.
__device__ __forceinline__ void rt_cx(uint64_t& k, uint32_t& r, int stride, bool keep_min) {
  const uint64_t ok = __shfl_xor_sync(0xffffffffu, k, stride);
  const uint32_t orow = __shfl_xor_sync(0xffffffffu, r, stride);
  if (keep_min == kr_gt(k, r, ok, orow)) {
    k = ok;
    r = orow;
  }
}

// Merge a sorted list held across the warp (lane i: i-th smallest, sentinel
// ~0 past its end) into the warp list: the k best of the two are
// min(list[i], other[31-i]), put in order by a bitonic merge.
__device__ __forceinline__ void rt_merge_sorted(RTLocal& s, uint32_t k, uint64_t ok, uint32_t orow, int lane) {
  const uint64_t rk = __shfl_sync(0xffffffffu, ok, 31 - lane);
  const uint32_t rr = __shfl_sync(0xffffffffu, orow, 31 - lane);
  uint64_t lk = (uint32_t)lane < k ? s.lk : ~0ull;
  uint32_t lr = (uint32_t)lane < k ? s.lr : 0xFFFFFFFFu;
  if (kr_gt(lk, lr, rk, rr)) {
    lk = rk;
    lr = rr;
  }
#pragma unroll
  for (int stride = 16; stride > 0; stride >>= 1) rt_cx(lk, lr, stride, (lane & stride) == 0);
  s.lk = lk;
  s.lr = lr;
  const uint64_t kk = __shfl_sync(0xffffffffu, lk, k - 1);
  const uint32_t kr = __shfl_sync(0xffffffffu, lr, k - 1);
  if (!(kk == ~0ull && kr == 0xFFFFFFFFu) && kr_le(kk, kr, s.tk, s.tr)) {
    s.tk = kk;
    s.tr = kr;
  }
}

// Batched insertion: one candidate per lane (sentinel ~0 where none) is
// bitonic-sorted across the warp, then merged with the list.  ~20 exchange
// steps for 32 candidates, against one ballot/shuffle round per candidate in
// rt_insert; used when many lanes hold candidates at once (rows in key order,
// e.g. ORDER BY id DESC over ascending ids).
__device__ __forceinline__ void rt_insert32(RTLocal& s, uint32_t k, uint64_t ck, uint32_t cr, int lane) {
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
    const bool up = (lane & size) == 0 || size == 32;
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) rt_cx(ck, cr, stride, ((lane & stride) == 0) == up);
  }
  rt_merge_sorted(s, k, ck, cr, lane);
}

constexpr int kRtBulkLanes = 8;  // lanes with candidates from which rt_insert32 pays

// Insert this lane's masked candidates (m: bit j set = key[j]/row[j]) into the
// warp list, re-testing each against the threshold as it tightens.
template <int R>
__device__ __forceinline__ void rt_offer(RTLocal& s, uint32_t k, const uint64_t (&key)[R], const uint32_t (&row)[R],
                                         uint32_t m, int lane) {
  for (;;) {
    const unsigned lanes = __ballot_sync(0xffffffffu, m != 0u);
    if (__popc(lanes) < kRtBulkLanes) break;
    const int j = m ? __ffs(m) - 1 : 0;
    uint64_t ck = ~0ull;
    uint32_t cr = 0xFFFFFFFFu;
    if (m) {
#pragma unroll
      for (int jj = 0; jj < R; ++jj)
        if (jj == j) {
          ck = key[jj];
          cr = row[jj];
        }
      m &= m - 1u;
    }
    rt_insert32(s, k, ck, cr, lane);
    // Drop what the tightened threshold now excludes.
#pragma unroll
    for (int jj = 0; jj < R; ++jj)
      if (((m >> jj) & 1u) && !kr_le(key[jj], row[jj], s.tk, s.tr)) m &= ~(1u << jj);
  }
  for (;;) {
    const unsigned lanes = __ballot_sync(0xffffffffu, m != 0u);
    if (!lanes) break;
    const int src = __ffs(lanes) - 1;
    const int j = m ? __ffs(m) - 1 : 0;
    uint64_t mk = 0;
    uint32_t mr = 0;
#pragma unroll
    for (int jj = 0; jj < R; ++jj)
      if (jj == j) {
        mk = key[jj];
        mr = row[jj];
      }
    const uint64_t ck = __shfl_sync(0xffffffffu, mk, src);
    const uint32_t cr = __shfl_sync(0xffffffffu, mr, src);
    if (lane == src) m &= m - 1u;
    if (kr_le(ck, cr, s.tk, s.tr)) rt_insert(s, k, ck, cr, lane);
  }
}

__device__ __forceinline__ void rt_clear(RTLocal& s) {
  s.lk = ~0ull;
  s.lr = 0xFFFFFFFFu;
}

// Tighten the threshold with a key-only bound b (inclusive: any row).
__device__ __forceinline__ void rt_bound(RTLocal& s, uint64_t b) {
  if (b < s.tk) {
    s.tk = b;
    s.tr = 0xFFFFFFFFu;
  }
}

}  // namespace fdb
