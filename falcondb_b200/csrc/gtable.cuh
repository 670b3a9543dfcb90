// Open-addressing aggregate table shared by the int64-key GROUP BY kernels
// (one query: k_groupby.cu; many queries in one launch: k_batch.cu).
//
// A slot holds one group: key ^ 2^63 (so the all-zero slot is empty and a
// table is cleared with cudaMemset), COUNT(*), SUM and the MIN / MAX order
// keys of the value.  MIN is kept as the bitwise NOT of its order key so that
// both MIN and MAX are atomicMax from a zero identity.  The key INT64_MIN reads
// as NULL (aggregate.rs:867, 1207) and has a slot of its own outside the table.
#pragma once
#include "common.cuh"

namespace fdb {

struct GSlot {          // 40 bytes; all-zero = empty
  uint64_t key;         // key ^ 2^63
  unsigned long long count;
  double sum;
  unsigned long long nmin;  // ~order key of MIN (atomicMax)
  unsigned long long max;   // order key of MAX
};

constexpr uint32_t kSmemSlots = 1024;      // CTA table slots (power of two)
#ifndef FDB_GB_SMEM_PROBE
#define FDB_GB_SMEM_PROBE 4
#endif
constexpr uint32_t kSmemProbe = FDB_GB_SMEM_PROBE;  // probes before a row spills to global
constexpr uint32_t kGlobalProbeLimit = 1u << 16;

__device__ __forceinline__ void gslot_accum(GSlot* s, double v, bool has_v) {
  atomicAdd(&s->count, 1ull);
  if (has_v) {
    atomicAdd(&s->sum, v);
    if (!isnan(v)) {
      const uint64_t k = f64_ord_key(v);
      atomicMax(&s->nmin, (unsigned long long)~k);
      atomicMax(&s->max, (unsigned long long)k);
    }
  }
}

// Shared-memory (CTA table) slots count rows with a 32-bit atomic on the low
// word of `count`: shared memory has a native 32-bit atomic add, while its
// 64-bit integer and FP64 adds are compare-and-swap loops that serialise on a
// hot slot.  A CTA sees fewer than 2^32 rows of one query, and readers take
// the whole 64-bit word (high word zero).
__device__ __forceinline__ void sslot_accum(GSlot* s, double v, bool has_v) {
  atomicAdd(reinterpret_cast<unsigned int*>(&s->count), 1u);
  if (has_v) {
    atomicAdd(&s->sum, v);
    if (!isnan(v)) {
      const uint64_t k = f64_ord_key(v);
      atomicMax(&s->nmin, (unsigned long long)~k);
      atomicMax(&s->max, (unsigned long long)k);
    }
  }
}

// A group of `n` rows folded beforehand: `has_sum` when at least one had a
// value; nmin / max are 0 when none had a non-NaN value.
__device__ __forceinline__ void sslot_accum_n(GSlot* s, uint32_t n, bool has_sum, double sum, uint64_t nmin,
                                              uint64_t max) {
  atomicAdd(reinterpret_cast<unsigned int*>(&s->count), n);
  if (has_sum) atomicAdd(&s->sum, sum);
  if (nmin) atomicMax(&s->nmin, (unsigned long long)nmin);
  if (max) atomicMax(&s->max, (unsigned long long)max);
}

__device__ __forceinline__ void gslot_merge(GSlot* s, const GSlot& v) {
  atomicAdd(&s->count, v.count);
  atomicAdd(&s->sum, v.sum);
  atomicMax(&s->nmin, v.nmin);
  atomicMax(&s->max, v.max);
}

// Find or claim the slot of `skey` (nonzero) in a global table of mask+1
// slots.  A table that is too small (more groups than slots) fails fast: the
// probe is capped, the error word is set, and every later lookup sees the
// error word and gives up at once, so the kernel still ends promptly.
__device__ __forceinline__ GSlot* gtable_find(GSlot* table, uint64_t mask, uint64_t skey, int* err) {
  if (*reinterpret_cast<volatile int*>(err) != 0) return nullptr;
  uint64_t h = mix64(skey) & mask;
  const uint64_t limit = umin64(mask + 1, kGlobalProbeLimit);
  for (uint64_t probe = 0; probe < limit; ++probe) {
    GSlot* s = table + h;
    const uint64_t cur = *reinterpret_cast<volatile uint64_t*>(&s->key);
    if (cur == skey) return s;
    if (cur == 0) {
      const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(&s->key), 0ull,
                                      (unsigned long long)skey);
      if (prev == 0 || prev == skey) return s;
    }
    h = (h + 1) & mask;
  }
  atomicExch(err, kErrCapacity);
  return nullptr;
}

// gtable_find for a caller that has already loaded `cur`, the key word of the
// key's home slot h = mix64(skey) & mask (so that several lookups can have
// their first load in flight together).
__device__ __forceinline__ GSlot* gtable_find_from(GSlot* table, uint64_t mask, uint64_t skey, uint64_t h,
                                                   uint64_t cur, int* err) {
  const uint64_t limit = umin64(mask + 1, kGlobalProbeLimit);
  for (uint64_t probe = 0; probe < limit; ++probe) {
    GSlot* s = table + h;
    if (probe) cur = *reinterpret_cast<volatile uint64_t*>(&s->key);
    if (cur == skey) return s;
    if (cur == 0) {
      const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(&s->key), 0ull,
                                      (unsigned long long)skey);
      if (prev == 0 || prev == skey) return s;
    }
    h = (h + 1) & mask;
  }
  atomicExch(err, kErrCapacity);
  return nullptr;
}

// The CTA's shared-memory slot of `skey`, claiming one if free within
// kSmemProbe probes; nullptr when the key has no room there.
__device__ __forceinline__ GSlot* smem_table_slot(GSlot* tab, uint64_t skey) {
  uint32_t h = (uint32_t)mix64(skey) & (kSmemSlots - 1);
  for (uint32_t probe = 0; probe < kSmemProbe; ++probe) {
    GSlot* s = tab + h;
    const uint64_t cur = *reinterpret_cast<volatile uint64_t*>(&s->key);
    if (cur == skey) return s;
    if (cur == 0) {
      const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(&s->key), 0ull,
                                      (unsigned long long)skey);
      if (prev == 0 || prev == skey) return s;
    }
    h = (h + 1) & (kSmemSlots - 1);
  }
  return nullptr;
}

// The output row of a live slot (key given as stored, XOR 2^63).
__device__ __forceinline__ fdb_group_i64 gslot_group(uint64_t skey, const GSlot& s) {
  fdb_group_i64 g;
  g.key = (int64_t)(skey ^ (1ull << 63));
  g.count = (int64_t)s.count;
  g.sum = s.sum;
  g.min = s.nmin ? f64_from_ord_key(~s.nmin) : __longlong_as_double(0x7ff8000000000000ll);
  g.max = s.max ? f64_from_ord_key(s.max) : __longlong_as_double(0x7ff8000000000000ll);
  return g;
}

}  // namespace fdb
