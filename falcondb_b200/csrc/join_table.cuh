// Device layout of a join build table (built in k_join.cu), shared with the
// serving kernel (serve.cu) that probes resident tables in batched launches.
#pragma once
#include "common.cuh"

namespace fdb {

struct JSlot {
  unsigned long long key;   // key ^ 2^63; 0 = empty
  unsigned long long psum;  // SUM of non-NULL payloads (two's complement)
};

constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

// Home slot of a stored key in a table of 2^(64-shift) slots: multiplicative
// (Fibonacci) hashing, the top bits of key * 2^64/phi.  One 64-bit multiply
// and a shift; consecutive keys land far apart, so linear probing stays
// short on the dense integer keys joins usually have.  The choice of hash is
// not observable in any result (the reference mixes with int_key_hash,
// join.rs:1368-1374).
__host__ __device__ __forceinline__ uint64_t join_hash(uint64_t sk, int shift) {
  return (sk * 0x9E3779B97F4A7C15ull) >> shift;
}
__device__ __forceinline__ int join_shift(uint64_t cap) { return __clzll((long long)cap) + 1; }  // cap = 2^b

// How keys map to home slots.  A table whose build keys span fewer values than
// it has slots (max - min < cap: surrogate keys, dense id ranges) is dense:
// key k lives in slot k - min, so a probe is one slot read and keys outside
// [min, min + cap) read nothing.  Otherwise keys hash (join_hash) with linear
// probing, and a probe key outside the build keys' [min, max] still reads
// nothing: the range read back at build time doubles as a min/max filter, so
// probe keys that run past the build side's (half of uniform [0, 2M) probe
// keys against the 1M build keys 0..1M-1, say) skip the walk to an empty
// slot that each would otherwise take.  The NULL-group slot (key INT64_MIN)
// is slot cap either way.
struct JoinMode {
  int64_t dmin;   // the smallest build key
  int32_t dense;
  int32_t shift;  // join_shift(cap)
  uint64_t span;  // largest build key - dmin + 1 (dense: <= cap); 0 = no range
                  // (an empty build side, or keys over all 2^64 values)
};

// Home slot of key k (stored form sk), or a value >= cap when the table holds
// no key there: outside [dmin, dmin + span), where no build key lies.  A
// dense table's slots past the span are empty; a hashed table is not read.
__device__ __forceinline__ uint64_t join_home(const JoinMode& m, int64_t k, uint64_t sk) {
  const uint64_t d = (uint64_t)k - (uint64_t)m.dmin;
  if (m.dense) return d < m.span ? d : ~0ull;
  if (m.span != 0 && d >= m.span) return ~0ull;
  return join_hash(sk, m.shift);
}

// Slot of probe key k, or kNoSlot.
__device__ __forceinline__ uint32_t join_find(const JSlot* __restrict__ slots, const unsigned int* cnt,
                                              uint64_t cap, const JoinMode& mode, int64_t k, JSlot* out) {
  if (k == INT64_MIN) {
    if (cnt[cap] == 0u) return kNoSlot;
    *out = slots[cap];
    return (uint32_t)cap;
  }
  const unsigned long long sk = (unsigned long long)k ^ (1ull << 63);
  const uint64_t mask = cap - 1;
  uint64_t h = join_home(mode, k, sk);
  if (h >= cap) return kNoSlot;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const JSlot s = slots[h];
    if (s.key == sk) {
      *out = s;
      return (uint32_t)h;
    }
    if (s.key == 0ull) return kNoSlot;
    h = (h + 1) & mask;
  }
  return kNoSlot;
}

}  // namespace fdb
