// Batched int64-key GROUP BY: many independent queries (each a GROUP BY key
// with COUNT(*), SUM, MIN, MAX of one value column over its own rows) run by
// one persistent kernel and one compaction kernel, captured once into a CUDA
// graph and replayed.
//
// Work list: the queries' rows cut into tiles of `tile_rows`, numbered query
// by query.  CTAs claim tile numbers from one atomic counter, so the grid
// walks the queries in order and a CTA's consecutive tiles usually belong to
// the same query.  Each CTA keeps the shared-memory table of the query it is
// working on (the frequent keys of that query) and flushes it into the
// query's global table when it moves to another query or runs out of tiles.
// The queries' tables (sized from each query's expected or estimated group
// count), their NULL slots, output counters and the claim counter live in one
// device arena, zeroed by one memset node at the head of the graph.
//
// Reference: GroupByExec fast_i64_gb (src/query/aggregate.rs:840-912), run
// once per query there.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "gtable.cuh"

namespace fdb {

constexpr int kBatchThreads = 512;
constexpr int kBatchMaxQueries = 1024;

struct BatchQuery {        // device descriptor of one query
  DevCol key;
  DevCol val;
  uint64_t n;
  uint64_t tile0;          // first tile number of this query
  GSlot* table;            // cap slots, then the NULL slot
  uint64_t mask;           // cap - 1
  uint64_t slot0;          // first slot number in the compaction's numbering
  fdb_group_i64* out;
  uint64_t out_cap;
  unsigned long long* counter;
  uint64_t* d_ngroups;
};

struct BatchArgs {
  const BatchQuery* q;
  int nq;
  uint32_t tile_rows;
  uint64_t total_tiles;
  uint64_t total_slots;
  unsigned int* claim;     // zero at launch
  int* err;
};

__device__ __forceinline__ int batch_find(const uint64_t* start, int nq, uint64_t t) {
  int lo = 0, hi = nq;     // start[lo] <= t < start[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (start[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ void batch_flush(GSlot* tab, const BatchQuery& q, int* err) {
  for (uint32_t i = threadIdx.x; i <= kSmemSlots; i += blockDim.x) {
    const GSlot s = tab[i];
    if (i == kSmemSlots) {
      if (s.count) gslot_merge(q.table + q.mask + 1, s);
    } else if (s.key != 0) {
      GSlot* g = gtable_find(q.table, q.mask, s.key, err);
      if (g) gslot_merge(g, s);
    }
    tab[i] = GSlot{0, 0, 0.0, 0, 0};
  }
}

__global__ void __launch_bounds__(kBatchThreads) gb_batch_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  GSlot* tab = reinterpret_cast<GSlot*>(smem);                          // kSmemSlots + NULL slot
  uint64_t* start = reinterpret_cast<uint64_t*>(tab + kSmemSlots + 1);  // [nq + 1]
  __shared__ unsigned int s_t;
  for (int i = threadIdx.x; i < a.nq; i += blockDim.x) start[i] = a.q[i].tile0;
  if (threadIdx.x == 0) start[a.nq] = a.total_tiles;
  for (uint32_t i = threadIdx.x; i < (kSmemSlots + 1) * sizeof(GSlot) / 8; i += blockDim.x)
    reinterpret_cast<uint64_t*>(tab)[i] = 0;
  __syncthreads();
  int cur = -1;
  uint64_t since_flush = 0;  // rows in the CTA table: its 32-bit row counts must not wrap
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(a.claim, 1u);
    __syncthreads();
    const uint64_t t = s_t;
    if (t >= a.total_tiles) break;
    const int qi = batch_find(start, a.nq, t);
    if (qi != cur || since_flush + a.tile_rows >= (1ull << 32)) {
      if (cur >= 0) batch_flush(tab, a.q[cur], a.err);
      __syncthreads();
      cur = qi;
      since_flush = 0;
    }
    since_flush += a.tile_rows;
    const BatchQuery& q = a.q[qi];
    const uint64_t r0 = (t - q.tile0) * a.tile_rows;
    const uint64_t r1 = umin64(r0 + a.tile_rows, q.n);
    const int64_t* keys = static_cast<const int64_t*>(q.key.values);
    for (uint64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const int64_t key = __ldcs(keys + r);
      const bool has_v = col_valid(q.val, r);
      double v = 0.0;
      if (has_v)
        v = q.val.dtype == FDB_FLOAT64 ? __ldcs(static_cast<const double*>(q.val.values) + r)
                                       : (double)__ldcs(static_cast<const int64_t*>(q.val.values) + r);
      if (!col_valid(q.key, r) || key == INT64_MIN) {  // NULL group
        sslot_accum(tab + kSmemSlots, v, has_v);
        continue;
      }
      const uint64_t skey = (uint64_t)key ^ (1ull << 63);
      GSlot* dst = smem_table_slot(tab, skey);
      if (dst) {
        sslot_accum(dst, v, has_v);
        continue;
      }
      dst = gtable_find(q.table, q.mask, skey, a.err);
      if (dst) gslot_accum(dst, v, has_v);
    }
    __syncthreads();  // the tile is done before s_t is rewritten or the table flushed
  }
  if (cur >= 0) batch_flush(tab, a.q[cur], a.err);
}

// Compaction of every query's table (slots numbered query by query, each
// query's NULL slot last): live slots are appended to their query's output.
__global__ void __launch_bounds__(256) gb_batch_compact_kernel(BatchArgs a) {
  __shared__ uint64_t start[kBatchMaxQueries + 1];
  for (int i = threadIdx.x; i < a.nq; i += blockDim.x) start[i] = a.q[i].slot0;
  if (threadIdx.x == 0) start[a.nq] = a.total_slots;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x; i0 < a.total_slots;
       i0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = i0 + threadIdx.x;
    int qi = -1;
    GSlot s;
    uint64_t skey = 0;
    bool live = false;
    if (i < a.total_slots) {
      qi = batch_find(start, a.nq, i);
      const BatchQuery& q = a.q[qi];
      const uint64_t local = i - q.slot0;
      s = q.table[local];
      if (local <= q.mask) {
        live = s.key != 0;
        skey = s.key;
      } else {
        live = s.count != 0;  // the NULL slot
        skey = 0;             // reads back as INT64_MIN
      }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, live ? qi : -1);
    if (live) {
      const BatchQuery& q = a.q[qi];
      const int leader = __ffs(peers) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(q.counter, (unsigned long long)__popc(peers));
      base = __shfl_sync(peers, base, leader);
      const uint64_t pos = base + __popc(peers & ((1u << lane) - 1u));
      if (pos < q.out_cap)
        q.out[pos] = gslot_group(skey, s);
      else
        atomicExch(a.err, kErrCapacity);
    }
  }
}

__global__ void gb_batch_counts_kernel(BatchArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nq; i += gridDim.x * blockDim.x)
    *a.q[i].d_ngroups = *a.q[i].counter;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct BatchPlan {
  Ctx* ctx = nullptr;
  DevBuf arena;            // tables, counters, claim
  DevBuf qdesc;            // BatchQuery[nq]
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nq = 0;
  uint64_t total_tiles = 0, total_slots = 0;
  size_t arena_bytes = 0;
  fdb_batch_tuning tuning{};
};

static void batch_free(BatchPlan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->ctx->free_buf(p->arena);
  p->ctx->free_buf(p->qdesc);
  delete p;
}

// Sizes, allocates and captures the plan.  expected[i] = groups to size query
// i's table for (already estimated), tuning fully specified.
static BatchPlan* batch_build(Ctx& c, const fdb_gb_query* qs, int nq, const std::vector<uint64_t>& expected,
                              const fdb_batch_tuning& t) {
  std::unique_ptr<BatchPlan, void (*)(BatchPlan*)> plan(new BatchPlan(), batch_free);
  plan->ctx = &c;
  plan->nq = nq;
  plan->tuning = t;
  std::vector<BatchQuery> dq(nq);
  std::vector<uint64_t> caps(nq);
  size_t bytes = 0;
  uint64_t tiles = 0, slots = 0;
  for (int i = 0; i < nq; ++i) {
    uint64_t cap = 1024;
    // Twice the estimate: a sketch may read a few percent low, and a table
    // that is too small fails the query rather than answering wrongly.
    const double want = 2.0 * (double)std::max<uint64_t>(expected[i], 1) / t.load_factor;
    while ((double)cap < want) cap <<= 1;
    caps[i] = cap;
    bytes += (cap + 1) * sizeof(GSlot);
    BatchQuery& d = dq[i];
    d.key = DevCol{qs[i].key.dtype, qs[i].key.values, qs[i].key.validity, qs[i].key.validity_offset};
    d.val = DevCol{qs[i].value.dtype, qs[i].value.values, qs[i].value.validity, qs[i].value.validity_offset};
    d.n = qs[i].nrows;
    d.tile0 = tiles;
    tiles += (qs[i].nrows + t.tile_rows - 1) / t.tile_rows;
    d.mask = cap - 1;
    d.slot0 = slots;
    slots += cap + 1;
    d.out = qs[i].d_groups;
    d.out_cap = qs[i].capacity;
    d.d_ngroups = qs[i].d_ngroups;
  }
  const size_t cnt_off = bytes;
  bytes += (size_t)nq * 8 + 8;
  plan->arena = c.alloc_buf(bytes);
  plan->arena_bytes = bytes;
  unsigned char* base = static_cast<unsigned char*>(plan->arena.ptr);
  size_t off = 0;
  for (int i = 0; i < nq; ++i) {
    dq[i].table = reinterpret_cast<GSlot*>(base + off);
    off += (caps[i] + 1) * sizeof(GSlot);
    dq[i].counter = reinterpret_cast<unsigned long long*>(base + cnt_off) + i;
  }
  plan->qdesc = c.alloc_buf(sizeof(BatchQuery) * nq);
  FDB_CUDA(cudaMemcpyAsync(plan->qdesc.ptr, dq.data(), sizeof(BatchQuery) * nq, cudaMemcpyHostToDevice, c.stream));
  plan->total_tiles = tiles;
  plan->total_slots = slots;

  BatchArgs a;
  a.q = static_cast<const BatchQuery*>(plan->qdesc.ptr);
  a.nq = nq;
  a.tile_rows = (uint32_t)t.tile_rows;
  a.total_tiles = tiles;
  a.total_slots = slots;
  a.claim = reinterpret_cast<unsigned int*>(base + cnt_off + (size_t)nq * 8);
  a.err = c.d_err;
  const size_t smem = (kSmemSlots + 1) * sizeof(GSlot) + (size_t)(nq + 1) * 8;
  FDB_CUDA(cudaFuncSetAttribute(gb_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  FDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb_batch_kernel, kBatchThreads, smem));
  const int ctas = std::max(1, std::min(per_sm, t.ctas_per_sm)) * c.sm_count;
  const unsigned cgrid = (unsigned)umin64((slots + 255) / 256, (uint64_t)c.sm_count * 8);

  FDB_CUDA(cudaStreamSynchronize(c.stream));  // the descriptor upload is not part of the graph
  FDB_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
  cudaMemsetAsync(base, 0, bytes, c.stream);
  gb_batch_kernel<<<ctas, kBatchThreads, smem, c.stream>>>(a);
  gb_batch_compact_kernel<<<cgrid, 256, 0, c.stream>>>(a);
  gb_batch_counts_kernel<<<1, 256, 0, c.stream>>>(a);
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(c.stream, &g);
  FDB_CUDA(ce);
  plan->graph = g;
  FDB_CUDA(cudaGraphInstantiate(&plan->exec, g, 0));
  return plan.release();
}

static fdb_batch_tuning batch_defaults(const fdb_batch_tuning* t) {
  fdb_batch_tuning d;
  d.load_factor = (t && t->load_factor > 0.0 && t->load_factor < 1.0) ? t->load_factor : 0.5;
  d.ctas_per_sm = (t && t->ctas_per_sm > 0) ? t->ctas_per_sm : 2;
  d.tile_rows = (t && t->tile_rows >= 256) ? t->tile_rows : 8192;
  return d;
}

static void batch_check(const fdb_gb_query* qs, int nq) {
  if (nq < 1 || nq > kBatchMaxQueries) fail(FDB_E_ARG, "between 1 and 1024 queries per batch");
  for (int i = 0; i < nq; ++i) {
    const fdb_gb_query& q = qs[i];
    if (q.key.dtype != FDB_INT64) fail(FDB_E_TYPE, "batched GROUP BY needs INT64 keys");
    if (q.value.dtype != FDB_FLOAT64 && q.value.dtype != FDB_INT64)
      fail(FDB_E_TYPE, "batched GROUP BY values must be FLOAT64 or INT64");
    if (q.nrows && (!q.key.values || !q.value.values)) fail(FDB_E_ARG, "column without values");
    if (!q.d_ngroups || (q.capacity && !q.d_groups)) fail(FDB_E_ARG, "query without outputs");
  }
}

static std::vector<uint64_t> batch_expected(Ctx& c, const fdb_gb_query* qs, int nq) {
  std::vector<uint64_t> e(nq);
  for (int i = 0; i < nq; ++i) e[i] = qs[i].expected_groups ? qs[i].expected_groups : estimate_distinct_i64(c, qs[i].key.values, qs[i].nrows);
  return e;
}

BatchPlan* op_gb_batch_prepare(Ctx& c, const fdb_gb_query* qs, int nq, const fdb_batch_tuning* t) {
  batch_check(qs, nq);
  const std::vector<uint64_t> e = batch_expected(c, qs, nq);
  return batch_build(c, qs, nq, e, batch_defaults(t));
}

void op_gb_batch_run(BatchPlan* p) {
  FDB_CUDA(cudaGraphLaunch(p->exec, p->ctx->stream));
}

void op_gb_batch_free(BatchPlan* p) { batch_free(p); }

// Times each candidate plan (one warm-up replay, then `reps` replays between
// CUDA events on the context stream) and returns the fastest tuning.
double op_gb_batch_autotune(Ctx& c, const fdb_gb_query* qs, int nq, int reps, fdb_batch_tuning* best) {
  batch_check(qs, nq);
  if (reps < 1) reps = 3;
  const std::vector<uint64_t> e = batch_expected(c, qs, nq);
  const double lfs[] = {0.35, 0.5, 0.7};
  const int fans[] = {1, 2, 3};
  const int tiles[] = {4096, 16384};
  double best_ms = -1.0;
  for (double lf : lfs)
    for (int fan : fans)
      for (int tr : tiles) {
        fdb_batch_tuning t{lf, fan, tr};
        BatchPlan* p = batch_build(c, qs, nq, e, t);
        op_gb_batch_run(p);
        FDB_CUDA(cudaEventRecord(c.ev0, c.stream));
        for (int r = 0; r < reps; ++r) op_gb_batch_run(p);
        FDB_CUDA(cudaEventRecord(c.ev1, c.stream));
        FDB_CUDA(cudaEventSynchronize(c.ev1));
        float ms = 0.f;
        FDB_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        batch_free(p);
        const int err = c.check_device_error();
        if (err) fail(err, "batched GROUP BY failed on the device while tuning");
        if (best_ms < 0 || ms / reps < best_ms) {
          best_ms = ms / reps;
          *best = t;
        }
      }
  return best_ms;
}

}  // namespace fdb
