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
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "stream.cuh"

namespace fdb {

constexpr uint64_t kSampleStride = 256;
constexpr int kTopkR = 4;  // rows per consumer thread per sub-step

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
  static bool attr = false;
  if (!attr) {
    FDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    attr = true;
  }
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (NCW + 1) * 32, smem));
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 4) per_sm = 4;  // partials are sized for 4 CTAs per SM
  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  uint64_t want = ntiles ? ntiles : 1;
  const int grid = (int)umin64(want, (uint64_t)c.sm_count * per_sm);
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
  if (sample) {
    TopkParams ps = p;
    ps.row_stride = kSampleStride;
    ps.t0 = nullptr;
    ps.out_rows = nullptr;
    ps.out_count = nullptr;
    ps.out_t0 = t0;
    const uint32_t cap = topk_cap(k, 256);
    const size_t smem = topk_smem_bytes(cap);
    static bool attr = false;
    if (!attr) {
      FDB_CUDA(cudaFuncSetAttribute(topk_sample_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    200 * 1024));
      attr = true;
    }
    const int grid = (int)umin64((uint64_t)c.sm_count, (nsamples + 4095) / 4096);
    topk_sample_kernel<<<grid, 256, smem, c.stream>>>(ps, nsamples);
    FDB_CUDA(cudaGetLastError());
  }

  // 2. main pass
  uint32_t* keyed_rows = d_rows;
  uint64_t* keyed_count = d_count;
  const bool has_nulls = col.validity != nullptr;
  if (has_nulls) {
    keyed_rows = static_cast<uint32_t*>(c.scratch_take(sizeof(uint32_t) * k));
    keyed_count = static_cast<uint64_t*>(c.scratch_take(sizeof(uint64_t)));
  }
  p.row_stride = 1;
  p.t0 = sample ? t0 : nullptr;
  p.out_rows = keyed_rows;
  p.out_count = keyed_count;
  p.out_t0 = nullptr;
  launch_topk_main<NCW>(c, col, n, p);

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
