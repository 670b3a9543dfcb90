// Hash join on one int64 key: build and probe, with INNER / LEFT / SEMI / ANTI.
//
// Replaces (FalconDB src/query/join.rs):
//   build_hash_table + IntHashTable (chained, 2 buckets/row) ..... 607-645, 1054-1351
//   probe_in_place / probe_one / collect_matches ................... 297-375, 657-723
//   execute_hash_semi_anti_join (keep-mask over left rows) .......... 49-132
//   BuildFilter (Bloom) — not needed: a miss costs one L2 sector here.
//
// Build side layout (all in HBM, L2-resident at the configs' 1M build rows):
//   * slots[cap+1]: {key ^ 2^63, SUM(payload)} per DISTINCT key, open addressing
//     with linear probing over a power of two (an all-zero slot is empty, so the
//     table is cleared with cudaMemset).  Slot `cap` holds the key INT64_MIN,
//     whose stored pattern would be the empty one.
//   * cnt[cap+1]  build rows per key; pcnt[cap+1] rows with a non-NULL payload;
//   * off[cap+2] + rows[n]: the build row numbers of each key (CSR), for pairs.
// Duplicate build keys therefore cost O(1) to insert and to probe: an
// aggregate probe reads one 16-byte slot (plus cnt when keys repeat), where the
// reference walks a chain of every duplicate (join.rs:1319-1350).
// NULL keys never match (join.rs:637, 693-697): NULL build keys are not
// inserted; NULL probe keys find nothing (LEFT / ANTI still keep the row).
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "join_table.cuh"
#include "stream.cuh"

namespace fdb {

struct HashTable {
  Ctx* ctx = nullptr;
  DevBuf slots, cnt, pcnt, off, rows;
  uint64_t cap = 0;
  uint64_t nbuild = 0;
  bool unique = true;        // every key occurs once (cnt is 1 wherever set)
  bool payload_nulls = false;
  bool dense = false;        // key k lives in slot k - dmin (join_table.cuh)
  int64_t dmin = 0;          // the smallest build key
  uint64_t span = 0;         // kmax - kmin + 1 (0: no range); probe keys outside read nothing
  // Dense tables whose key range fits a CTA's shared memory as bits: bit
  // k - dmin is set when key k has a build row.  SEMI / ANTI probes test it
  // in shared memory and read nothing else.
  DevBuf bits;
};

// The widest key range whose presence bits a probe CTA keeps in shared
// memory (192 KB), next to its tile ring.
constexpr uint64_t kProbeBitsMaxSpan = 192ull * 1024 * 8;

// bits[w] = presence of slots 64w .. 64w+63 (one 32-bit half per warp ballot).
__global__ void join_bits_kernel(const unsigned int* __restrict__ cnt, uint64_t span, uint32_t* bits32) {
  const uint64_t n32 = (span + 63) / 64 * 64;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n32; i += (uint64_t)gridDim.x * blockDim.x) {
    const bool b = i < span && cnt[i] != 0u;
    const unsigned m = __ballot_sync(0xffffffffu, b);
    if ((threadIdx.x & 31) == 0) bits32[i >> 5] = m;
  }
}

// Order keys of the smallest and largest valid build key (INT64_MIN, the
// NULL group, excluded): out[0] = ~ord(min), out[1] = ord(max), both from a
// zero identity (0 = no key).
__global__ void join_key_range_kernel(const int64_t* __restrict__ keys, const uint64_t* kvalid, uint64_t kvoff,
                                      uint64_t n, unsigned long long* out) {
  unsigned long long mn = 0, mx = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (kvalid) {
      const uint64_t b = kvoff + i;
      if (!((kvalid[b >> 6] >> (b & 63)) & 1ull)) continue;
    }
    const int64_t k = keys[i];
    if (k == INT64_MIN) continue;
    const unsigned long long o = i64_ord_key(k);
    mn = ~o > mn ? ~o : mn;
    mx = o > mx ? o : mx;
  }
  mn = warp_max_u64(mn);
  mx = warp_max_u64(mx);
  if ((threadIdx.x & 31) == 0 && mx) {
    atomicMax(&out[0], mn);
    atomicMax(&out[1], mx);
  }
}

// ---------------------------------------------------------------------------
// Build
// ---------------------------------------------------------------------------
__global__ void join_insert_kernel(const int64_t* __restrict__ keys, const uint64_t* kvalid, uint64_t kvoff,
                                   const int64_t* __restrict__ payload, const uint64_t* pvalid, uint64_t pvoff,
                                   uint64_t n, JSlot* slots, unsigned int* cnt, unsigned int* pcnt, uint64_t cap,
                                   JoinMode mode, uint32_t* row_slot, unsigned int* dup, int* err) {
  const uint64_t mask = cap - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (kvalid) {
      const uint64_t b = kvoff + i;
      if (!((kvalid[b >> 6] >> (b & 63)) & 1ull)) {
        row_slot[i] = kNoSlot;
        continue;
      }
    }
    const int64_t k = keys[i];
    uint64_t s = kNoSlot;
    if (k == INT64_MIN) {
      s = cap;
    } else {
      const unsigned long long sk = (unsigned long long)k ^ (1ull << 63);
      uint64_t h = join_home(mode, k, sk);  // a build key lies in the range: h < cap
      if (h > mask) {  // cannot happen: the range was taken over these keys
        atomicExch(err, kErrCapacity);
        row_slot[i] = kNoSlot;
        continue;
      }
      for (uint64_t probe = 0; probe <= mask; ++probe) {  // cap > distinct keys: always ends
        const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&slots[h].key);
        if (cur == sk) { s = h; break; }
        if (cur == 0ull) {
          const unsigned long long prev = atomicCAS(&slots[h].key, 0ull, sk);
          if (prev == 0ull || prev == sk) { s = h; break; }
        }
        h = (h + 1) & mask;
      }
      if (s == kNoSlot) {
        atomicExch(err, kErrCapacity);
        row_slot[i] = kNoSlot;
        continue;
      }
    }
    if (atomicAdd(&cnt[s], 1u) != 0u) *dup = 1u;
    bool pv = payload != nullptr;
    if (pv && pvalid) {
      const uint64_t b = pvoff + i;
      pv = (pvalid[b >> 6] >> (b & 63)) & 1ull;
    }
    if (pv) {
      atomicAdd(&slots[s].psum, (unsigned long long)payload[i]);
      atomicAdd(&pcnt[s], 1u);
    }
    row_slot[i] = (uint32_t)s;
  }
}

// Exclusive scan of uint32 counts (cap+1 of them) into off[0..cap+1].
constexpr int kScanThreads = 1024, kScanPer = 4, kScanBlock = kScanThreads * kScanPer;

__device__ uint32_t block_scan_u32(uint32_t v, uint32_t* sm, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nw ? sm[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) sm[lane] = s;
  }
  __syncthreads();
  const uint32_t base = warp ? sm[warp - 1] : 0u;
  if (total) *total = sm[nw - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void scan_blocks_kernel(const unsigned int* in, uint64_t n, uint32_t* block_sums) {
  __shared__ uint32_t sm[32];
  const uint64_t i0 = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j)
    if (i0 + j < n) s += in[i0 + j];
  uint32_t tot;
  block_scan_u32(s, sm, &tot);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void scan_top_kernel(uint32_t* block_sums, uint64_t nblocks) {
  __shared__ uint32_t sm[32];
  const uint64_t per = (nblocks + blockDim.x - 1) / blockDim.x;
  const uint64_t b0 = threadIdx.x * per;
  uint32_t local = 0;
  for (uint64_t i = b0; i < b0 + per && i < nblocks; ++i) local += block_sums[i];
  uint32_t base = block_scan_u32(local, sm, nullptr);
  for (uint64_t i = b0; i < b0 + per && i < nblocks; ++i) {
    const uint32_t v = block_sums[i];
    block_sums[i] = base;
    base += v;
  }
}

__global__ void scan_apply_kernel(const unsigned int* in, uint64_t n, const uint32_t* block_sums, uint32_t* out) {
  __shared__ uint32_t sm[32];
  const uint64_t i0 = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
  uint32_t v[kScanPer];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    v[j] = (i0 + j < n) ? in[i0 + j] : 0u;
    s += v[j];
  }
  uint32_t run = block_sums[blockIdx.x] + block_scan_u32(s, sm, nullptr);
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    if (i0 + j < n) out[i0 + j] = run;
    run += v[j];
    if (i0 + j == n - 1) out[n] = run;  // total after the last element
  }
}

__global__ void join_scatter_kernel(const uint32_t* __restrict__ row_slot, uint64_t n, const uint32_t* off,
                                    unsigned int* fill, uint32_t* rows) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = row_slot[i];
    if (s == kNoSlot) continue;
    rows[off[s] + atomicAdd(&fill[s], 1u)] = (uint32_t)i;
  }
}

static JoinMode join_mode(const HashTable& h) {
  JoinMode m;
  m.dmin = h.dmin;
  m.dense = h.dense ? 1 : 0;
  m.span = h.span;
  int b = 0;
  while ((1ull << b) < h.cap) ++b;
  m.shift = 64 - b;  // join_shift(cap)
  return m;
}

HashTable* op_join_build(Ctx& c, const fdb_dev_column& key, const fdb_dev_column& payload, uint64_t n,
                         double load_factor) {
  if (key.dtype != FDB_INT64) fail(FDB_E_TYPE, "join keys must be INT64");
  if (payload.values && payload.dtype != FDB_INT64) fail(FDB_E_TYPE, "join payload must be INT64");
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "build side addresses rows as uint32");
  if (load_factor <= 0.0 || load_factor >= 1.0) load_factor = 0.5;
  uint64_t cap = 1024;
  while ((double)cap * load_factor < (double)n || cap <= n) cap <<= 1;
  std::unique_ptr<HashTable> h(new HashTable());
  h->ctx = &c;
  h->cap = cap;
  h->nbuild = n;
  h->payload_nulls = payload.values != nullptr && payload.validity != nullptr;
  h->slots = c.alloc_buf((cap + 1) * sizeof(JSlot));
  h->cnt = c.alloc_buf((cap + 1) * sizeof(uint32_t));
  h->pcnt = c.alloc_buf((cap + 1) * sizeof(uint32_t));
  h->off = c.alloc_buf((cap + 2) * sizeof(uint32_t));
  h->rows = c.alloc_buf(std::max<uint64_t>(n, 1) * sizeof(uint32_t));
  const uint64_t ns = cap + 1;
  const uint64_t nblocks = (ns + kScanBlock - 1) / kScanBlock;
  c.ensure_scratch(c.scratch_top + n * 4 + ns * 4 + nblocks * 4 + (1u << 20));
  uint32_t* row_slot = static_cast<uint32_t*>(c.scratch_take(std::max<uint64_t>(n, 1) * 4));
  unsigned int* fill = static_cast<unsigned int*>(c.scratch_take(ns * 4));
  uint32_t* bsums = static_cast<uint32_t*>(c.scratch_take(nblocks * 4));
  unsigned int* dup = static_cast<unsigned int*>(c.scratch_take(4));
  FDB_CUDA(cudaMemsetAsync(h->slots.ptr, 0, ns * sizeof(JSlot), c.stream));
  FDB_CUDA(cudaMemsetAsync(h->cnt.ptr, 0, ns * 4, c.stream));
  FDB_CUDA(cudaMemsetAsync(h->pcnt.ptr, 0, ns * 4, c.stream));
  FDB_CUDA(cudaMemsetAsync(fill, 0, ns * 4, c.stream));
  FDB_CUDA(cudaMemsetAsync(dup, 0, 4, c.stream));
  // Dense or hashed: the build keys' range decides (one 16-byte read back).
  bool dense = false;
  int64_t dmin = 0;
  uint64_t span = 0;
  if (n > 0) {
    unsigned long long* range = static_cast<unsigned long long*>(c.scratch_take(16));
    FDB_CUDA(cudaMemsetAsync(range, 0, 16, c.stream));
    const unsigned blocks = (unsigned)umin64((n + 255) / 256, (uint64_t)c.sm_count * 8);
    join_key_range_kernel<<<blocks, 256, 0, c.stream>>>(static_cast<const int64_t*>(key.values), key.validity,
                                                         key.validity_offset, n, range);
    FDB_CUDA(cudaGetLastError());
    unsigned long long hr[2] = {0, 0};
    FDB_CUDA(cudaMemcpyAsync(hr, range, 16, cudaMemcpyDeviceToHost, c.stream));
    FDB_CUDA(cudaStreamSynchronize(c.stream));
    if (hr[1] != 0) {
      const uint64_t kmin = ~hr[0] ^ (1ull << 63), kmax = hr[1] ^ (1ull << 63);  // two's complement bits
      // Both kinds keep the range: a hashed table uses it as a min/max filter
      // on probe keys (span 0 when the keys cover all 2^64 values).
      dmin = (int64_t)kmin;
      span = kmax - kmin + 1;
      dense = kmax - kmin < cap;
    }
  }
  h->dense = dense;
  h->dmin = dmin;
  h->span = span;
  const JoinMode mode = join_mode(*h);
  if (n > 0) {
    const unsigned blocks = (unsigned)umin64((n + 255) / 256, (uint64_t)c.sm_count * 16);
    join_insert_kernel<<<blocks, 256, 0, c.stream>>>(
        static_cast<const int64_t*>(key.values), key.validity, key.validity_offset,
        static_cast<const int64_t*>(payload.values), payload.validity, payload.validity_offset, n,
        static_cast<JSlot*>(h->slots.ptr), static_cast<unsigned int*>(h->cnt.ptr),
        static_cast<unsigned int*>(h->pcnt.ptr), cap, mode, row_slot, dup, c.d_err);
  }
  scan_blocks_kernel<<<(unsigned)nblocks, kScanThreads, 0, c.stream>>>(static_cast<const unsigned int*>(h->cnt.ptr),
                                                                        ns, bsums);
  scan_top_kernel<<<1, 1024, 0, c.stream>>>(bsums, nblocks);
  scan_apply_kernel<<<(unsigned)nblocks, kScanThreads, 0, c.stream>>>(
      static_cast<const unsigned int*>(h->cnt.ptr), ns, bsums, static_cast<uint32_t*>(h->off.ptr));
  if (n > 0) {
    const unsigned blocks = (unsigned)umin64((n + 255) / 256, (uint64_t)c.sm_count * 16);
    join_scatter_kernel<<<blocks, 256, 0, c.stream>>>(row_slot, n, static_cast<const uint32_t*>(h->off.ptr), fill,
                                                       static_cast<uint32_t*>(h->rows.ptr));
  }
  if (dense && span <= kProbeBitsMaxSpan) {
    const uint64_t words = (span + 63) / 64;
    h->bits = c.alloc_buf(words * 8);
    const unsigned blocks = (unsigned)umin64((words * 64 + 255) / 256, (uint64_t)c.sm_count * 8);
    join_bits_kernel<<<blocks, 256, 0, c.stream>>>(static_cast<const unsigned int*>(h->cnt.ptr), span,
                                                    static_cast<uint32_t*>(h->bits.ptr));
  }
  FDB_CUDA(cudaGetLastError());
  unsigned int hdup = 0;
  FDB_CUDA(cudaMemcpyAsync(&hdup, dup, 4, cudaMemcpyDeviceToHost, c.stream));
  const int e = c.check_device_error();  // synchronises the stream
  if (e) {
    join_free(h.release());
    fail(e, "join build failed on the device");
  }
  h->unique = hdup == 0;
  return h.release();
}

void join_free(HashTable* h) {
  if (!h) return;
  Ctx* c = h->ctx;
  c->free_buf(h->slots);
  c->free_buf(h->cnt);
  c->free_buf(h->pcnt);
  c->free_buf(h->off);
  c->free_buf(h->rows);
  c->free_buf(h->bits);
  delete h;
}
uint64_t join_capacity(const HashTable* h) { return h ? h->cap : 0; }

JoinView join_view(const HashTable* h) {
  JoinView v;
  v.slots = h->slots.ptr;
  v.cnt = static_cast<const unsigned int*>(h->cnt.ptr);
  v.cap = h->cap;
  v.unique = h->unique ? 1 : 0;
  v.dense = h->dense ? 1 : 0;
  v.dmin = h->dmin;
  v.span = h->span;
  return v;
}

// ---------------------------------------------------------------------------
// Probe with fused aggregation, over the TMA streamer (cols: key [, value]).
// ---------------------------------------------------------------------------
struct JoinAggAcc {
  unsigned long long count;
  long long psum;        // exact payload sum (two's complement wrap beyond int64)
  unsigned long long prows;
  double vsum;
};

struct ProbeParams {
  DevCol key;
  DevCol value;          // values == nullptr when absent
  const JSlot* slots;
  const unsigned int* cnt;
  const unsigned int* pcnt;
  uint64_t cap;
  JoinMode mode;
  int32_t unique;
  int32_t payload_nulls;
  int32_t has_value;
  int32_t _pad;
  JoinAggAcc* partials;   // [grid]
  unsigned int* ticket;
  fdb_join_agg* out;
  const unsigned long long* bits;  // presence bits of a dense table's key range (ProbeBitsOp)
  uint64_t span;
};

// Probe launch shape: ring stages, tile rows (one column), and resident CTAs
// per SM the register budget is sized for.
#ifndef FDB_PROBE_STAGES
#define FDB_PROBE_STAGES 2
#endif
#ifndef FDB_PROBE_TR
#define FDB_PROBE_TR 2048
#endif
#ifndef FDB_PROBE_MINB
#define FDB_PROBE_MINB 5
#endif

// JT: the join type (FDB_JOIN_*), fixed per instantiation.
// DENSE: the table is direct-addressed (JoinMode), so a row is one 16-byte
// slot read; FDB_PROBE_DENSE_ROWS rows per thread have their reads in flight
// together.  The probe is bound by resident warps more than by reads per
// thread: measured INNER / LEFT at 100M rows, 1 row per thread with no
// minimum CTAs per SM (ptxas keeps it at 40 registers: 5 CTAs per SM) 0.305 /
// 0.320 ms; 2 rows at 4 CTAs per SM 0.359 / 0.377 ms; 1 row at 5 or 6 CTAs
// per SM 0.338 / 0.378 ms; 4 rows at 3 CTAs 0.341 / 0.355 ms.
#ifndef FDB_PROBE_DENSE_ROWS
#define FDB_PROBE_DENSE_ROWS 1
#endif
#ifndef FDB_PROBE_DENSE_MINB
#define FDB_PROBE_DENSE_MINB 0
#endif
template <int JT, bool DENSE = false>
struct ProbeOp {
  using Params = ProbeParams;
  struct Local {
    JoinAggAcc a;
  };
  static constexpr size_t kSmem = 32 * sizeof(JoinAggAcc) + 16;

  static __device__ void init(Local& st, const Params&, unsigned char*, int, int) {
    st.a.count = 0;
    st.a.psum = 0;
    st.a.prows = 0;
    st.a.vsum = 0.0;
  }

  // Both slots of an aligned pair (32 bytes, one L2 sector) in one 256-bit load.
  static __device__ __forceinline__ void load_pair(const JSlot* pair, uint64_t pol, JSlot& a, JSlot& b) {
    asm volatile("ld.global.L2::cache_hint.v4.u64 {%0, %1, %2, %3}, [%4], %5;"
                 : "=l"(a.key), "=l"(a.psum), "=l"(b.key), "=l"(b.psum)
                 : "l"(pair), "l"(pol));
  }

  // One row per thread per pass.  Each probe round reads the aligned pair of
  // slots around the current position and resolves both in probe order
  // without branches: the first slot counts only when the position is even;
  // the walk ends at the key or at the first empty slot.
  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char*, const Acc& acc, uint32_t rows,
                              int ctid, int nct) {
    if constexpr (DENSE) {
      step_dense(st, p, acc, rows, ctid, nct);
      return;
    }
    const uint64_t mask = p.cap - 1;
    const uint64_t pol = l2_evict_last_policy();  // keep the table resident against the streamed keys
    for (uint32_t i = ctid; i < rows; i += nct) {
      uint32_t at = kNoSlot;
      uint64_t ps = 0;
      if (!p.key.validity || col_valid(p.key, acc.row(i))) {  // a NULL key matches nothing
        const int64_t k = acc.template get<int64_t>(0, i);
        if (k == INT64_MIN) {
          if (p.cnt[p.cap] != 0u) {
            at = (uint32_t)p.cap;
            ps = p.slots[p.cap].psum;
          }
        } else {
          const uint64_t sk = (uint64_t)k ^ (1ull << 63);
          uint64_t h = join_home(p.mode, k, sk);
          // A dense table holds key k only in slot k - min, so its walk ends in
          // the first round; a key outside its range reads nothing.
          for (uint64_t round = 0; h <= mask && round <= mask; ++round) {
            const uint64_t base = h & ~1ull;
            JSlot a, b;
            load_pair(p.slots + base, pol, a, b);
            const bool even = (h & 1ull) == 0;
            const bool hit0 = even && a.key == sk;
            const bool stop0 = even && (a.key == sk || a.key == 0ull);
            const bool hit1 = !stop0 && b.key == sk;
            if (hit0 || hit1) {
              at = (uint32_t)(base + (hit1 ? 1 : 0));
              ps = hit1 ? b.psum : a.psum;
              break;
            }
            if (stop0 || b.key == 0ull) break;
            h = (base + 2) & mask;
          }
        }
      }
      accumulate(st, p, acc, i, at, ps);
    }
  }

  // Row i matched slot `at` (kNoSlot: no build row) whose payload sum is ps.
  template <class Acc>
  static __device__ __forceinline__ void accumulate(Local& st, const Params& p, const Acc& acc, uint32_t i,
                                                    uint32_t at, uint64_t ps) {
    unsigned long long matches = 0, prows = 0;
    if (at != kNoSlot) {
      matches = p.unique ? 1ull : (unsigned long long)p.cnt[at];
      prows = p.payload_nulls ? (unsigned long long)p.pcnt[at] : matches;
    }
    if constexpr (JT == FDB_JOIN_INNER || JT == FDB_JOIN_LEFT) {
      st.a.count += (JT == FDB_JOIN_LEFT && matches == 0) ? 1ull : matches;
      st.a.psum += (long long)ps;
      st.a.prows += prows;
    } else {
      const bool keep = (JT == FDB_JOIN_SEMI) ? (matches != 0) : (matches == 0);
      if (keep) {
        st.a.count += 1;
        if (p.has_value && (!p.value.validity || col_valid(p.value, acc.row(i)))) {
          st.a.vsum += acc.template get<double>(1, i);
          st.a.prows += 1;
        }
      }
    }
  }

  // Direct-addressed table: every row's slot read is issued before any is used.
  template <class Acc>
  static __device__ void step_dense(Local& st, const Params& p, const Acc& acc, uint32_t rows, int ctid, int nct) {
    constexpr int R = FDB_PROBE_DENSE_ROWS;
    const uint64_t pol = l2_evict_last_policy();
    for (uint32_t i0 = ctid; i0 < rows; i0 += R * nct) {
      uint64_t sk[R], d[R];
      uint32_t at[R];
      uint64_t ps[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const uint32_t i = i0 + r * nct;
        sk[r] = 0;
        d[r] = p.cap;  // no read
        at[r] = kNoSlot;
        ps[r] = 0;
        if (i >= rows || (p.key.validity && !col_valid(p.key, acc.row(i)))) continue;  // a NULL key matches nothing
        const int64_t k = acc.template get<int64_t>(0, i);
        if (k == INT64_MIN) {
          if (p.cnt[p.cap] != 0u) {
            at[r] = (uint32_t)p.cap;
            ps[r] = p.slots[p.cap].psum;
          }
          continue;
        }
        sk[r] = (uint64_t)k ^ (1ull << 63);
        d[r] = join_home(p.mode, k, sk[r]);  // >= cap outside the build keys' span: no read
      }
      JSlot sl[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        sl[r].key = 0;
        sl[r].psum = 0;
        if (d[r] < p.cap)
          asm volatile("ld.global.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
                       : "=l"(sl[r].key), "=l"(sl[r].psum)
                       : "l"(p.slots + d[r]), "l"(pol));
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const uint32_t i = i0 + r * nct;
        if (i >= rows) continue;
        if (d[r] < p.cap && sl[r].key == sk[r]) {
          at[r] = (uint32_t)d[r];
          ps[r] = sl[r].psum;
        }
        accumulate(st, p, acc, i, at[r], ps[r]);
      }
    }
  }

  static __device__ JoinAggAcc warp_red(JoinAggAcc a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a.count += __shfl_xor_sync(0xffffffffu, a.count, o);
      a.psum += __shfl_xor_sync(0xffffffffu, a.psum, o);
      a.prows += __shfl_xor_sync(0xffffffffu, a.prows, o);
      a.vsum += __shfl_xor_sync(0xffffffffu, a.vsum, o);
    }
    return a;
  }

  static __device__ void block_red(Local& st, JoinAggAcc* sm, int ctid, int nct) {
    JoinAggAcc w = warp_red(st.a);
    if ((ctid & 31) == 0) sm[ctid >> 5] = w;
    consumer_bar(nct);
    if (ctid == 0) {
      JoinAggAcc t = sm[0];
      for (int i = 1; i < (nct >> 5); ++i) {
        t.count += sm[i].count;
        t.psum += sm[i].psum;
        t.prows += sm[i].prows;
        t.vsum += sm[i].vsum;
      }
      st.a = t;
    }
  }

  static __device__ void finish(Local& st, const Params& p, unsigned char* smr, int ctid, int nct) {
    JoinAggAcc* sm = reinterpret_cast<JoinAggAcc*>(smr);
    unsigned int* s_last = reinterpret_cast<unsigned int*>(smr + 32 * sizeof(JoinAggAcc));
    block_red(st, sm, ctid, nct);
    if (ctid == 0) {
      p.partials[blockIdx.x] = st.a;
      __threadfence();
      const unsigned int t = atomicAdd(p.ticket, 1u);
      *s_last = (t == gridDim.x - 1) ? 1u : 0u;
    }
    consumer_bar(nct);
    if (*s_last == 0) return;
    __threadfence();
    JoinAggAcc t;
    t.count = 0;
    t.psum = 0;
    t.prows = 0;
    t.vsum = 0.0;
    for (uint32_t b = ctid; b < gridDim.x; b += nct) {
      const JoinAggAcc* src = p.partials + b;
      t.count += __ldcg(&src->count);
      t.psum += __ldcg(&src->psum);
      t.prows += __ldcg(&src->prows);
      t.vsum += __ldcg(&src->vsum);
    }
    st.a = t;
    consumer_bar(nct);
    block_red(st, sm, ctid, nct);
    if (ctid == 0) {
      fdb_join_agg o;
      o.count = (int64_t)st.a.count;
      o.sum_payload = (int64_t)st.a.psum;
      o.sum_value = st.a.vsum;
      o.payload_rows = (int64_t)st.a.prows;
      *p.out = o;
      *p.ticket = 0u;
    }
  }
};

// SEMI / ANTI against a dense table whose key range fits shared memory as
// bits: every CTA copies the presence bits into shared memory once, and a row
// then costs one shared-memory bit test (no L2 access), so the probe streams
// its key (and value) columns at HBM speed.  Shared memory: ProbeOp's
// reduction area, then the bits.
template <int JT>
struct ProbeBitsOp : ProbeOp<JT, true> {
  static_assert(JT == FDB_JOIN_SEMI || JT == FDB_JOIN_ANTI, "presence alone answers SEMI / ANTI only");
  using Base = ProbeOp<JT, true>;
  using Params = ProbeParams;
  using Local = typename Base::Local;
  static constexpr size_t kBitsOff = (Base::kSmem + 127) / 128 * 128;

  static __device__ void init(Local& st, const Params& p, unsigned char* sm, int ctid, int nct) {
    Base::init(st, p, sm, ctid, nct);
    unsigned long long* bits = reinterpret_cast<unsigned long long*>(sm + kBitsOff);
    const uint64_t words = (p.span + 63) / 64;
    // 16-byte loads, eight in flight per thread (the bits buffer is a pool
    // allocation, 256-byte aligned; kBitsOff is a multiple of 128).
    const uint64_t pairs = words / 2;
    const uint4* src = reinterpret_cast<const uint4*>(p.bits);
    uint4* dst = reinterpret_cast<uint4*>(bits);
#pragma unroll 8
    for (uint64_t w = ctid; w < pairs; w += nct) dst[w] = __ldg(src + w);
    if ((words & 1) && ctid == 0) bits[words - 1] = __ldg(p.bits + words - 1);
  }

  template <class Acc>
  static __device__ void step(Local& st, const Params& p, unsigned char* sm, const Acc& acc, uint32_t rows,
                              int ctid, int nct) {
    const unsigned long long* bits = reinterpret_cast<const unsigned long long*>(sm + kBitsOff);
#pragma unroll 4
    for (uint32_t i = ctid; i < rows; i += nct) {
      bool match = false;
      if (!p.key.validity || col_valid(p.key, acc.row(i))) {  // a NULL key matches nothing
        const int64_t k = acc.template get<int64_t>(0, i);
        if (k == INT64_MIN) {
          match = p.cnt[p.cap] != 0u;
        } else {
          const uint64_t d = (uint64_t)k - (uint64_t)p.mode.dmin;
          match = d < p.span && ((bits[d >> 6] >> (d & 63)) & 1ull);
        }
      }
      if ((JT == FDB_JOIN_SEMI) == match) {
        st.a.count += 1;
        if (p.has_value && (!p.value.validity || col_valid(p.value, acc.row(i)))) {
          st.a.vsum += acc.template get<double>(1, i);
          st.a.prows += 1;
        }
      }
    }
  }
};

constexpr int kProbeMaxPerSm = 8;  // partials are sized for this many CTAs per SM

template <int NC, int JT, bool DENSE>
static void launch_probe_mode(Ctx& c, const fdb_dev_column* cols, uint64_t n, const ProbeParams& p) {
  constexpr int TR = NC == 1 ? FDB_PROBE_TR : FDB_PROBE_TR / 2, STAGES = FDB_PROBE_STAGES, NCW = 8;
  StreamSrc<NC> src;
  const void* bases[NC];
  for (int i = 0; i < NC; ++i) {
    src.base[i] = static_cast<const unsigned char*>(cols[i].values);
    src.esize[i] = 8;
    bases[i] = cols[i].values;
  }
  src.n = n;
  src.m_end = stream_m_end(bases, NC, n);
  const int op_off = (int)stream_smem_bytes<NC, TR, STAGES>();
  using Op = ProbeOp<JT, DENSE>;
  const size_t smem = op_off + Op::kSmem;
  auto kern = stream_kernel<Op, NC, TR, STAGES, NCW, 8, DENSE ? FDB_PROBE_DENSE_MINB : FDB_PROBE_MINB>;
  static PerDeviceOnce attr;  // per instantiation and device
  attr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)); });
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (NCW + 1) * 32, smem));
  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  const uint64_t want = ntiles ? ntiles : (n + NCW * 32 * 8 - 1) / (NCW * 32 * 8);
  const int grid = tuned_grid(c.tune.op[FDB_TUNE_PROBE], c.sm_count, per_sm, kProbeMaxPerSm, want, n);
  kern<<<grid, (NCW + 1) * 32, smem, c.stream>>>(src, p, c.d_err, op_off);
  FDB_CUDA(cudaGetLastError());
}

#ifndef FDB_PROBE_BITS_NCW
#define FDB_PROBE_BITS_NCW 16
#endif
// The presence-bit probe: one CTA per SM (the bits take most of its shared
// memory).  The tile ring gets what is left: the largest of 3 x 2 KB-row,
// 3 x 1 KB-row and 2 x 1 KB-row rings (per column) that fits, so that as many
// bytes as possible are in flight per SM.
template <int NC, int JT, int TR, int STAGES>
static void launch_probe_bits_shape(Ctx& c, const fdb_dev_column* cols, uint64_t n, const ProbeParams& p,
                                    size_t op_smem) {
  constexpr int NCW = FDB_PROBE_BITS_NCW;
  StreamSrc<NC> src;
  const void* bases[NC];
  for (int i = 0; i < NC; ++i) {
    src.base[i] = static_cast<const unsigned char*>(cols[i].values);
    src.esize[i] = 8;
    bases[i] = cols[i].values;
  }
  src.n = n;
  src.m_end = stream_m_end(bases, NC, n);
  const int op_off = (int)stream_smem_bytes<NC, TR, STAGES>();
  const size_t smem = op_off + op_smem;
  auto kern = stream_kernel<ProbeBitsOp<JT>, NC, TR, STAGES, NCW, 8, 1>;
  static PerDeviceOnce attr;  // per instantiation and device
  attr(c.device, [&] { FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)); });
  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  // One CTA per SM: the bits take most of its shared memory.
  const int grid = tuned_grid(c.tune.op[FDB_TUNE_PROBE], c.sm_count, 1, 1, ntiles, n);
  kern<<<grid, (NCW + 1) * 32, smem, c.stream>>>(src, p, c.d_err, op_off);
  FDB_CUDA(cudaGetLastError());
}

template <int NC, int JT>
static void launch_probe_bits(Ctx& c, const fdb_dev_column* cols, uint64_t n, const ProbeParams& p) {
  constexpr int TRB = NC == 1 ? 4096 : 2048, TRS = NC == 1 ? 2048 : 1024;
  constexpr size_t kMax = 227 * 1024;
  const size_t op_smem = ProbeBitsOp<JT>::kBitsOff + (p.span + 63) / 64 * 8;
  if (stream_smem_bytes<NC, TRB, 3>() + op_smem <= kMax)
    launch_probe_bits_shape<NC, JT, TRB, 3>(c, cols, n, p, op_smem);
  else if (stream_smem_bytes<NC, TRS, 3>() + op_smem <= kMax)
    launch_probe_bits_shape<NC, JT, TRS, 3>(c, cols, n, p, op_smem);
  else
    launch_probe_bits_shape<NC, JT, TRS, 2>(c, cols, n, p, op_smem);
}

template <int NC, int JT>
static void launch_probe(Ctx& c, const fdb_dev_column* cols, uint64_t n, const ProbeParams& p) {
  if constexpr (JT == FDB_JOIN_SEMI || JT == FDB_JOIN_ANTI) {
    if (p.bits) {
      launch_probe_bits<NC, JT>(c, cols, n, p);
      return;
    }
  }
  if (p.mode.dense)
    launch_probe_mode<NC, JT, true>(c, cols, n, p);
  else
    launch_probe_mode<NC, JT, false>(c, cols, n, p);
}

void op_join_probe_agg(Ctx& c, const HashTable& h, const fdb_dev_column& key, const fdb_dev_column* value,
                       uint64_t n, int join_type, fdb_join_agg* d_out) {
  if (key.dtype != FDB_INT64) fail(FDB_E_TYPE, "probe keys must be INT64");
  if (join_type < FDB_JOIN_INNER || join_type > FDB_JOIN_ANTI) fail(FDB_E_ARG, "bad join type");
  const bool has_value = value && value->values;
  if (has_value && value->dtype != FDB_FLOAT64) fail(FDB_E_TYPE, "probe value must be FLOAT64");
  ProbeParams p;
  std::memset(&p, 0, sizeof(p));
  p.key = DevCol{key.dtype, key.values, key.validity, key.validity_offset};
  if (has_value) p.value = DevCol{value->dtype, value->values, value->validity, value->validity_offset};
  p.slots = static_cast<const JSlot*>(h.slots.ptr);
  p.cnt = static_cast<const unsigned int*>(h.cnt.ptr);
  p.pcnt = static_cast<const unsigned int*>(h.pcnt.ptr);
  p.cap = h.cap;
  p.mode = join_mode(h);
  p.unique = h.unique ? 1 : 0;
  p.payload_nulls = h.payload_nulls ? 1 : 0;
  p.has_value = (has_value && (join_type == FDB_JOIN_SEMI || join_type == FDB_JOIN_ANTI)) ? 1 : 0;
  p.bits = static_cast<const unsigned long long*>(h.bits.ptr);
  p.span = h.bits.ptr ? h.span : 0;
  p.partials = static_cast<JoinAggAcc*>(c.scratch_take(sizeof(JoinAggAcc) * c.sm_count * kProbeMaxPerSm));
  p.ticket = c.d_ticket;
  p.out = d_out;
  if (n == 0) {
    FDB_CUDA(cudaMemsetAsync(d_out, 0, sizeof(fdb_join_agg), c.stream));
    return;
  }
  fdb_dev_column cols[2] = {key, has_value ? *value : key};
  switch (join_type) {
    case FDB_JOIN_INNER: launch_probe<1, FDB_JOIN_INNER>(c, cols, n, p); break;
    case FDB_JOIN_LEFT: launch_probe<1, FDB_JOIN_LEFT>(c, cols, n, p); break;
    case FDB_JOIN_SEMI:
      if (p.has_value) launch_probe<2, FDB_JOIN_SEMI>(c, cols, n, p);
      else launch_probe<1, FDB_JOIN_SEMI>(c, cols, n, p);
      break;
    default:
      if (p.has_value) launch_probe<2, FDB_JOIN_ANTI>(c, cols, n, p);
      else launch_probe<1, FDB_JOIN_ANTI>(c, cols, n, p);
  }
}

// ---------------------------------------------------------------------------
// Probe emitting row pairs (for SELECT of joined columns and multiset tests).
// ---------------------------------------------------------------------------
__global__ void join_pairs_kernel(const int64_t* __restrict__ keys, const uint64_t* kvalid, uint64_t kvoff,
                                  uint64_t n, const JSlot* __restrict__ slots, const unsigned int* cnt,
                                  const uint32_t* off, const uint32_t* brows, uint64_t cap, JoinMode mode,
                                  int join_type,
                                  uint32_t* out_l, uint32_t* out_r, uint64_t capacity,
                                  unsigned long long* counter, int* err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    bool valid = true;
    if (kvalid) {
      const uint64_t b = kvoff + i;
      valid = (kvalid[b >> 6] >> (b & 63)) & 1ull;
    }
    uint32_t at = kNoSlot;
    if (valid) {
      JSlot s;
      at = join_find(slots, cnt, cap, mode, keys[i], &s);
    }
    const uint32_t m = at == kNoSlot ? 0u : cnt[at];
    if (join_type == FDB_JOIN_INNER || join_type == FDB_JOIN_LEFT) {
      const uint32_t emit = m ? m : (join_type == FDB_JOIN_LEFT ? 1u : 0u);
      if (emit == 0) continue;
      const unsigned long long pos = atomicAdd(counter, (unsigned long long)emit);
      for (uint32_t j = 0; j < emit; ++j) {
        if (pos + j < capacity) {
          out_l[pos + j] = (uint32_t)i;
          out_r[pos + j] = m ? brows[off[at] + j] : FDB_NO_ROW;
        } else {
          atomicExch(err, kErrCapacity);
        }
      }
    } else {
      const bool keep = join_type == FDB_JOIN_SEMI ? m != 0 : m == 0;
      if (!keep) continue;
      const unsigned long long pos = atomicAdd(counter, 1ull);
      if (pos < capacity)
        out_l[pos] = (uint32_t)i;
      else
        atomicExch(err, kErrCapacity);
    }
  }
}

void op_join_probe_pairs(Ctx& c, const HashTable& h, const fdb_dev_column& key, uint64_t n, int join_type,
                         uint32_t* d_left, uint32_t* d_right, uint64_t capacity, uint64_t* d_count) {
  if (key.dtype != FDB_INT64) fail(FDB_E_TYPE, "probe keys must be INT64");
  if (join_type < FDB_JOIN_INNER || join_type > FDB_JOIN_ANTI) fail(FDB_E_ARG, "bad join type");
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "probe side addresses rows as uint32");
  if ((join_type == FDB_JOIN_INNER || join_type == FDB_JOIN_LEFT) && d_right == nullptr && capacity)
    fail(FDB_E_ARG, "INNER/LEFT pairs need a right-row buffer");
  unsigned long long* counter = static_cast<unsigned long long*>(c.scratch_take(8));
  FDB_CUDA(cudaMemsetAsync(counter, 0, 8, c.stream));
  if (n > 0) {
    const unsigned blocks = (unsigned)umin64((n + 255) / 256, (uint64_t)c.sm_count * 16);
    join_pairs_kernel<<<blocks, 256, 0, c.stream>>>(
        static_cast<const int64_t*>(key.values), key.validity, key.validity_offset, n,
        static_cast<const JSlot*>(h.slots.ptr), static_cast<const unsigned int*>(h.cnt.ptr),
        static_cast<const uint32_t*>(h.off.ptr), static_cast<const uint32_t*>(h.rows.ptr), h.cap, join_mode(h),
        join_type, d_left,
        d_right, capacity, counter, c.d_err);
    FDB_CUDA(cudaGetLastError());
  }
  FDB_CUDA(cudaMemcpyAsync(d_count, counter, 8, cudaMemcpyDeviceToDevice, c.stream));
}

}  // namespace fdb
