// Device-side building blocks shared by every kernel of the engine:
//   * order-preserving key transforms used by ORDER BY / MIN / MAX,
//   * the predicate program evaluator (postfix WHERE terms),
//   * mbarrier + cp.async.bulk (TMA bulk copy) wrappers with bounded waits,
//   * warp reductions.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/falcondb_b200.h"

namespace fdb {

constexpr uint32_t kNullCode = 0xFFFFFFFFu;            // Utf8Column NULL code
constexpr int kWarp = 32;

// Device-side error word codes (written to Ctx::d_err, read by fdb_synchronize);
// the same values as kDevErrTimeout / kDevErrCapacity of the host engine.
constexpr int kErrTimeout = 1;
constexpr int kErrCapacity = 2;

// Iteration cap of every spin on an mbarrier or flag. A try_wait may suspend the
// thread for a hardware-defined slice, so this bounds one wait to well under a
// few seconds; a healthy wait for a 16 KB tile ends within microseconds.
constexpr uint32_t kSpinLimit = 1u << 22;

// ---------------------------------------------------------------------------
// Order keys (sort.rs:451-454 f64_ord_key; sort.rs:243-268 for signed ints).
// Ascending order of the key equals the SQL ascending order of the value;
// NaN (positive sign) sorts above +inf.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t f64_bits(double v) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(v);
#else
  uint64_t b;
  __builtin_memcpy(&b, &v, 8);
  return b;
#endif
}
__host__ __device__ __forceinline__ double f64_of_bits(uint64_t b) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double v;
  __builtin_memcpy(&v, &b, 8);
  return v;
#endif
}
__host__ __device__ __forceinline__ uint64_t f64_ord_key(double v) {
  const uint64_t b = f64_bits(v);
  return (b >> 63) == 0 ? (b ^ (1ull << 63)) : ~b;
}
__host__ __device__ __forceinline__ double f64_from_ord_key(uint64_t k) {
  return f64_of_bits((k >> 63) ? (k ^ (1ull << 63)) : ~k);
}
__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ uint64_t i64_ord_key(int64_t v) {
  return (uint64_t)v ^ (1ull << 63);
}

// MurmurHash3's fmix64 finaliser.  FalconDB mixes join keys with its first
// three steps (int_key_hash / bucket_with, join.rs:1368-1374, 1423-1429); the
// choice of hash is not observable in any result.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t h) {
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdull;
  h ^= h >> 33;
  h *= 0xc4ceb9fe1a85ec53ull;
  h ^= h >> 33;
  return h;
}

// ---------------------------------------------------------------------------
// Column access
// ---------------------------------------------------------------------------
struct DevCol {
  int32_t dtype;
  const void* values;
  const uint64_t* validity;
  uint64_t voff;
};

__device__ __forceinline__ bool col_valid(const DevCol& c, uint64_t row) {
  if (c.validity == nullptr) return true;
  uint64_t b = c.voff + row;
  return (c.validity[b >> 6] >> (b & 63)) & 1ull;
}

// ---------------------------------------------------------------------------
// Predicate program: postfix terms, evaluated with a bit stack in a register.
// Semantics follow expr.rs:635-1175: NULL fails every comparison; an Int64
// column against a Float64 literal is widened to f64 (expr.rs:1122-1132); a
// Float64 column against an Int64 literal compares against (double)lit.
// ---------------------------------------------------------------------------
struct PredProg {
  int32_t n;
  int32_t _pad;
  fdb_pred_term t[FDB_MAX_TERMS];
};

template <typename T>
__device__ __forceinline__ bool cmp_op(int op, T a, T b) {
  switch (op) {
    case FDB_EQ: return a == b;
    case FDB_NE: return a != b;
    case FDB_LT: return a < b;
    case FDB_LE: return a <= b;
    case FDB_GT: return a > b;
    default:     return a >= b;
  }
}

// Evaluate one leaf term for a row whose column values are provided by `get`.
// `get(col, &i64, &f64, &code, &valid)` loads column `col` of the row.
template <class Get>
__device__ __forceinline__ bool eval_leaf(const fdb_pred_term& t, const Get& get) {
  int64_t iv = 0; double fv = 0.0; uint32_t code = 0; bool valid = true;
  int dt = get(t.col, iv, fv, code, valid);
  // A Utf8 cell is NULL through its validity bit or the NULL code.
  const bool is_null = !valid || (dt == FDB_UTF8 && code == kNullCode);
  switch (t.kind) {
    case FDB_TERM_IS_NULL: return is_null;
    case FDB_TERM_IS_NOT_NULL: return !is_null;
    case FDB_TERM_CODE_SET:
      // lit_i holds the dictionary length: codes outside it never pass.
      if (is_null || (int64_t)code >= t.lit_i) return false;
      return (t.code_set[code >> 6] >> (code & 63)) & 1ull;
    default: break;
  }
  if (!valid) return false;
  if (dt == FDB_FLOAT64) {
    double lit = t.lit_type == FDB_FLOAT64 ? t.lit_f : (double)t.lit_i;
    return cmp_op<double>(t.op, fv, lit);
  }
  if (dt == FDB_INT64) {
    if (t.lit_type == FDB_FLOAT64) return cmp_op<double>(t.op, (double)iv, t.lit_f);
    return cmp_op<int64_t>(t.op, iv, t.lit_i);
  }
  // FDB_UTF8 with CMP: compare codes (host maps string literals to CODE_SET;
  // this form is only produced for code equality on shared dictionaries).
  if (code == kNullCode) return false;
  return cmp_op<int64_t>(t.op, (int64_t)code, t.lit_i);
}

template <class Get>
__device__ __forceinline__ bool eval_prog(const PredProg& p, const Get& get) {
  if (p.n == 0) return true;
  uint32_t stack = 0;   // bit 0 = top of stack
  for (int i = 0; i < p.n; ++i) {
    const fdb_pred_term& t = p.t[i];
    if (t.kind == FDB_TERM_AND || t.kind == FDB_TERM_OR) {
      uint32_t a = stack & 1u, b = (stack >> 1) & 1u;
      stack >>= 2;
      uint32_t r = t.kind == FDB_TERM_AND ? (a & b) : (a | b);
      stack = (stack << 1) | r;
    } else {
      stack = (stack << 1) | (eval_leaf(t, get) ? 1u : 0u);
    }
  }
  return stack & 1u;
}

// ---------------------------------------------------------------------------
// mbarrier / bulk-copy (TMA) wrappers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: true when the phase completed, false (and the error word set)
// when the spin limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, uint32_t limit = kSpinLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, kErrTimeout);
  return false;
}
// Bounded wait with back-off, for the single producer lane of a streaming
// kernel: between polls the lane sleeps `ns` nanoseconds, so that while the
// ring is full it does not take issue slots from the consumer warps of its
// SM sub-partition.  Same limit and error reporting as mbar_wait (the bound is
// kSpinLimit polls, i.e. at most kSpinLimit * ns of sleep plus the polls).
__device__ __forceinline__ bool mbar_wait_backoff(uint64_t* bar, uint32_t parity, int* err, unsigned ns) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    __nanosleep(ns);
  }
  if (err) atomicExch(err, kErrTimeout);
  return false;
}
// L2 policy for data that is streamed once: evict it first, so that it does
// not push out what is reused (hash tables probed at random, partials).
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// L2 policy for data that is reused at random (hash tables): evict it last.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// 1-D bulk copy global -> shared through the TMA unit, completing on `bar`,
// with an L2 cache-hint policy.  dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                         uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
      "%4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}
__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

}  // namespace fdb
