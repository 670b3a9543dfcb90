// Sizing pass over an INT64 key column, for hash and direct-addressed tables:
// a distinct-count estimate from a HyperLogLog sketch (Flajolet, Fusy,
// Gandouet, Meunier, "HyperLogLog: the analysis of a near-optimal cardinality
// estimation algorithm", 2007; 2^12 registers, standard error about 1.6 %),
// and in the same pass the smallest and largest non-NULL key (NULL = a clear
// validity bit, or INT64_MIN, which GROUP BY reads as NULL).  One pass over the
// keys plus a 16 KB device-to-host copy; synchronises the context stream.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace fdb {

constexpr int kHllBits = 12;
constexpr int kHllRegs = 1 << kHllBits;

// regs[0..kHllRegs) then range[0] = min order key (atomicMin from ~0),
// range[1] = max order key (atomicMax from 0) of the non-NULL keys.
struct KeyStatsOut {
  unsigned int regs[kHllRegs];
  unsigned long long range[2];
};

__device__ __forceinline__ void hll_add(unsigned int* r, int64_t key) {
  const uint64_t h = mix64((uint64_t)key ^ (1ull << 63));
  const uint32_t idx = (uint32_t)(h >> (64 - kHllBits));
  const uint64_t w = (h << kHllBits) | (1ull << (kHllBits - 1));  // bounds the run of zeros
  atomicMax(&r[idx], (unsigned int)__clzll((long long)w) + 1u);
}

// Each thread takes 4 aligned pairs of keys per round (4 x 16-byte loads in
// flight), so the pass runs near HBM speed; keys before the first 16-byte
// boundary and after the last full pair are read one by one by thread 0 of
// block 0 and the grid's tail.
__global__ void __launch_bounds__(256) key_stats_kernel(const int64_t* __restrict__ keys, const uint64_t* validity,
                                                        uint64_t voff, uint64_t n, KeyStatsOut* out) {
  __shared__ unsigned int r[kHllRegs];
  for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x) r[i] = 0;
  __syncthreads();
  uint64_t lo = ~0ull, hi = 0;
  auto take = [&](int64_t k, uint64_t row) {
    hll_add(r, k);
    bool valid = k != INT64_MIN;
    if (validity) {
      const uint64_t b = voff + row;
      valid = valid && ((validity[b >> 6] >> (b & 63)) & 1ull);
    }
    if (valid) {
      const uint64_t o = i64_ord_key(k);
      lo = o < lo ? o : lo;
      hi = o > hi ? o : hi;
    }
  };
  // Head: rows before the first 16-byte aligned key.
  const uint64_t head = umin64(n, (uint64_t)((16 - ((uintptr_t)keys & 15)) & 15) / 8);
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (uint64_t i = 0; i < head; ++i) take(keys[i], i);
  const longlong2* pairs = reinterpret_cast<const longlong2*>(keys + head);
  const uint64_t np = (n - head) / 2;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  for (; p + 3 * stride < np; p += 4 * stride) {
    longlong2 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = __ldcs(pairs + p + u * stride);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint64_t row = head + 2 * (p + u * stride);
      take(v[u].x, row);
      take(v[u].y, row + 1);
    }
  }
  for (; p < np; p += stride) {
    const longlong2 v = __ldcs(pairs + p);
    take(v.x, head + 2 * p);
    take(v.y, head + 2 * p + 1);
  }
  // Tail: the last key when n - head is odd.
  if (blockIdx.x == 0 && threadIdx.x == 0 && ((n - head) & 1)) take(keys[n - 1], n - 1);
  lo = warp_min_u64(lo);
  hi = warp_max_u64(hi);
  if ((threadIdx.x & 31) == 0) {
    if (lo != ~0ull) atomicMin(&out->range[0], (unsigned long long)lo);
    if (hi != 0) atomicMax(&out->range[1], (unsigned long long)hi);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x)
    if (r[i]) atomicMax(&out->regs[i], r[i]);
}

static uint64_t hll_estimate(const unsigned int* h, uint64_t n) {
  double z = 0.0;
  int zeros = 0;
  for (int i = 0; i < kHllRegs; ++i) {
    z += std::ldexp(1.0, -(int)h[i]);
    zeros += h[i] == 0;
  }
  const double m = kHllRegs, alpha = 0.7213 / (1.0 + 1.079 / m);
  double e = alpha * m * m / z;
  if (e <= 2.5 * m && zeros > 0) e = m * std::log(m / zeros);  // small-range correction
  return std::min<uint64_t>(n, (uint64_t)std::ceil(e));
}

KeyStats key_stats_i64(Ctx& c, const fdb_dev_column& key, uint64_t n) {
  KeyStats s;
  if (n == 0) {
    s.distinct = 1;
    return s;
  }
  if (!key.values) fail(FDB_E_ARG, "column without values");
  KeyStatsOut* d = static_cast<KeyStatsOut*>(c.scratch_take(sizeof(KeyStatsOut)));
  FDB_CUDA(cudaMemsetAsync(d, 0, sizeof(KeyStatsOut), c.stream));
  FDB_CUDA(cudaMemsetAsync(&d->range[0], 0xFF, 8, c.stream));
  const unsigned grid = (unsigned)umin64((n / 2 + 255) / 256 + 1, (uint64_t)c.sm_count * 8);
  key_stats_kernel<<<grid, 256, 0, c.stream>>>(static_cast<const int64_t*>(key.values), key.validity,
                                               key.validity_offset, n, d);
  FDB_CUDA(cudaGetLastError());
  KeyStatsOut h;
  FDB_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  FDB_CUDA(cudaStreamSynchronize(c.stream));
  s.distinct = n <= 4096 ? n : hll_estimate(h.regs, n);
  if (h.range[0] <= h.range[1]) {
    s.has_range = true;
    s.kmin = (int64_t)(h.range[0] ^ (1ull << 63));
    s.kmax = (int64_t)(h.range[1] ^ (1ull << 63));
  }
  return s;
}

uint64_t estimate_distinct_i64(Ctx& c, const void* keys, uint64_t n) {
  if (n <= 4096) return n ? n : 1;
  fdb_dev_column k{};
  k.dtype = FDB_INT64;
  k.values = keys;
  return key_stats_i64(c, k, n).distinct;
}

}  // namespace fdb
