// Persistent column streamer: the scan skeleton shared by the filter, aggregate,
// group-by, distinct, join-probe and top-k kernels.
//
// A CTA = NCW consumer warps + 1 producer warp.  The row range [0, m_end) of up
// to NC columns is cut into tiles of TR rows; tiles are dealt round-robin to the
// persistent CTAs.  The producer's elected lane stages each tile into a ring of
// STAGES shared-memory buffers with 1-D TMA bulk copies (cp.async.bulk, one per
// column, completing on the stage's `full` mbarrier); consumers wait on `full`,
// run Op::step over the tile, and release the stage on its `empty` mbarrier.
// Rows [m_end, n) — the ragged end that is not a multiple of 16 bytes, or every
// row when a column base is not 16-byte aligned — are read with plain loads in a
// grid-stride loop.  Every wait is bounded (kSpinLimit); on time-out the kernel
// records kErrTimeout in the context's error word and winds down.
#pragma once
#include "common.cuh"

namespace fdb {

// Test hook for the bounded waits (set through fdb_test_stall).  When
// withhold_tile1 = t + 1, the producer of the CTA that is to stage tile t
// stops before that tile's bulk copy, so its consumers' wait on the tile runs
// out (after spin_limit polls when nonzero, else kSpinLimit): the kernel
// records kErrTimeout and still ends.  Every copy issued before the stop has
// been waited for by then, so none is in flight when the CTA exits.  Each
// translation unit has its own zero (inactive) copy; only the one in
// k_scan.cu (the aggregate scans) is ever set.
struct StreamHook {
  uint64_t withhold_tile1;
  uint32_t spin_limit;
  uint32_t _pad;
};
static __device__ StreamHook g_stream_hook;

template <int NC>
struct StreamSrc {
  const unsigned char* base[NC];  // device pointers to row 0 of each column
  int esize[NC];                  // bytes per value (4 or 8)
  uint64_t n;                     // rows
  uint64_t m_end;                 // rows [0, m_end) are staged by TMA
  unsigned int* tile_ctr;         // dynamic tile order only: 0xFFFFFFFF on entry
};

// Rows staged in shared memory: column c of the current stage starts at
// stage + c * TR * CB (CB = bytes reserved per row per column, 8 or 4).
template <int TR, int CB = 8>
struct TileAcc {
  static constexpr bool kSmemTile = true;
  const unsigned char* stage;
  uint64_t row0;
  template <typename T>
  __device__ __forceinline__ const T* col_ptr(int c) const {
    return reinterpret_cast<const T*>(stage + (size_t)c * TR * CB);
  }
  template <typename T>
  __device__ __forceinline__ T get(int c, uint32_t i) const {
    return reinterpret_cast<const T*>(stage + (size_t)c * TR * CB)[i];
  }
  __device__ __forceinline__ uint64_t row(uint32_t i) const { return row0 + i; }
};

// Rows read straight from global memory.
template <int NC>
struct GlobAcc {
  static constexpr bool kSmemTile = false;
  template <typename T>
  __device__ __forceinline__ const T* col_ptr(int) const {
    return nullptr;
  }
  const unsigned char* base[NC];
  int esize[NC];
  uint64_t row0;
  template <typename T>
  __device__ __forceinline__ T get(int c, uint32_t i) const {
    const unsigned char* b = base[0];
#pragma unroll
    for (int k = 1; k < NC; ++k)
      if (c == k) b = base[k];
    return reinterpret_cast<const T*>(b)[row0 + i];
  }
  __device__ __forceinline__ uint64_t row(uint32_t i) const { return row0 + i; }
};

__device__ __forceinline__ void consumer_bar(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

constexpr int kBarBytes = 128;  // mbarrier block at the start of dynamic smem

template <int NC, int TR, int STAGES, int CB = 8>
constexpr size_t stream_smem_bytes() {
  return kBarBytes + (size_t)STAGES * NC * TR * CB;
}

// Host helper: the TMA-staged prefix of the row range.  Every column base must
// be 16-byte aligned; the staged prefix ends on a multiple of 4 rows so that
// every column's byte count is a multiple of 16.
inline uint64_t stream_m_end(const void* const* bases, int nc, uint64_t n) {
  for (int c = 0; c < nc; ++c)
    if (((uintptr_t)bases[c] & 15u) != 0) return 0;
  return n & ~uint64_t(3);
}

// Op interface:
//   struct Params; struct Local;
//   static __device__ void init(Local&, const Params&, unsigned char* op_smem, int ctid, int nct);
//   template <class Acc> static __device__ void step(Local&, const Params&, unsigned char* op_smem,
//        const Acc&, uint32_t rows, int ctid, int nct);   // rows [0,rows) of acc, cooperative
//   static __device__ void finish(Local&, const Params&, unsigned char* op_smem, int ctid, int nct);
// step() and finish() are executed by all consumer threads; block-wide syncs
// inside them must use consumer_bar(nct).
// MINB: resident CTAs per SM the register allocation must allow (0: none).
// DYN: tiles are handed out by an atomic counter (src.tile_ctr) instead of
// round-robin, so CTAs that run faster take more tiles and all finish
// together.  The tile order then varies run to run, so DYN is only for ops
// whose result does not depend on it (top-k, counts), and for ops whose step
// has no CTA-wide barrier: on a time-out a warp leaves the tile loop at once.
template <class Op, int NC, int TR, int STAGES, int NCW, int CB = 8, int MINB = 1, bool DYN = false>
__global__ void __launch_bounds__((NCW + 1) * 32, MINB)
    stream_kernel(StreamSrc<NC> src, typename Op::Params p, int* err, int op_smem_off) {
  static_assert((DYN ? 20 : 16) * STAGES <= kBarBytes, "mbarriers (and DYN tile ids) fit the barrier block");
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + STAGES;
  uint32_t* tile_id = reinterpret_cast<uint32_t*>(empty + STAGES);  // [STAGES], DYN only
  unsigned char* tiles = smem + kBarBytes;
  unsigned char* op_smem = smem + op_smem_off;
  constexpr int NCT = NCW * 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    fence_mbar_init();
  }
  __syncthreads();

  const uint64_t ntiles = (src.m_end + TR - 1) / TR;
  const StreamHook hook = g_stream_hook;
  const uint32_t spin_limit = hook.spin_limit ? hook.spin_limit : kSpinLimit;

  if (warp == NCW) {
    // ---------------- producer warp ----------------
    if (lane == 0) {
      const uint64_t policy = l2_evict_first_policy();  // columns are read once
      uint32_t it = 0;
      for (uint64_t t = blockIdx.x; t < ntiles || DYN; t += gridDim.x, ++it) {
        const int s = it % STAGES;
        const uint32_t ph = (it / STAGES) & 1u;
        if (it >= STAGES && !mbar_wait_backoff(&empty[s], ph ^ 1u, err, 64)) break;
        if constexpr (DYN) {
          // First tile: blockIdx.x; then gridDim.x + 0, 1, 2, ... in claim order
          // (the counter starts at 0xFFFFFFFF, so its first value wraps to 0).
          if (it > 0) t = (uint64_t)gridDim.x + (uint32_t)(atomicAdd(src.tile_ctr, 1u) + 1u);
          if (t >= ntiles) {
            tile_id[s] = 0xFFFFFFFFu;
            mbar_arrive(&full[s]);  // completes the phase with no bytes: the end mark
            break;
          }
          tile_id[s] = (uint32_t)t;
        }
        if (!DYN && hook.withhold_tile1 && t + 1 == hook.withhold_tile1) break;  // test hook only
        const uint64_t r0 = t * TR;
        const uint32_t rows = (uint32_t)umin64(TR, src.m_end - r0);
        uint32_t bytes = 0;
#pragma unroll
        for (int c = 0; c < NC; ++c) bytes += rows * src.esize[c];
        mbar_arrive_expect_tx(&full[s], bytes);
#pragma unroll
        for (int c = 0; c < NC; ++c)
          bulk_g2s(tiles + ((size_t)s * NC + c) * TR * CB, src.base[c] + r0 * src.esize[c],
                   rows * src.esize[c], &full[s], policy);
      }
    }
    return;  // consumers sync among themselves with named barrier 1
  }

  // ---------------- consumer warps ----------------
  const int ctid = threadIdx.x;  // consumers are warps 0..NCW-1
  typename Op::Local st;
  Op::init(st, p, op_smem, ctid, NCT);
  consumer_bar(NCT);

  // Every consumer thread runs every tile iteration, so the block-wide
  // barriers inside Op::step stay uniform.  A wait that runs out records the
  // error and the thread stops waiting from then on: the remaining tiles are
  // processed from whatever the buffers hold (indices stay in bounds; the
  // result is discarded by the host, which sees FDB_E_TIMEOUT), so the kernel
  // always ends.
  uint32_t it = 0;
  bool dead = false;
  for (uint64_t t = blockIdx.x; t < ntiles || DYN; t += gridDim.x, ++it) {
    const int s = it % STAGES;
    const uint32_t ph = (it / STAGES) & 1u;
    if constexpr (DYN) {
      // The wait's outcome is made warp-uniform so that the warp collectives
      // inside Op::step stay converged; a warp that timed out stops here.
      if (!__all_sync(0xffffffffu, mbar_wait(&full[s], ph, err, spin_limit))) break;
      const uint32_t tid = tile_id[s];
      if (tid == 0xFFFFFFFFu) break;
      t = tid;
    } else {
      if (!dead && !mbar_wait(&full[s], ph, err, spin_limit)) dead = true;
    }
    const uint64_t r0 = t * TR;
    const uint32_t rows = (uint32_t)umin64(TR, src.m_end - r0);
    TileAcc<TR, CB> acc{tiles + (size_t)s * NC * TR * CB, r0};
    Op::step(st, p, op_smem, acc, rows, ctid, NCT);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }

  // Plain-load region: rows [m_end, n), grid-stride in chunks of NCT*8 rows.
  const uint64_t plain_n = src.n - src.m_end;
  constexpr uint32_t CH = NCT * 8;
  for (uint64_t c0 = (uint64_t)blockIdx.x * CH; c0 < plain_n; c0 += (uint64_t)gridDim.x * CH) {
    GlobAcc<NC> acc;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      acc.base[c] = src.base[c];
      acc.esize[c] = src.esize[c];
    }
    acc.row0 = src.m_end + c0;
    const uint32_t rows = (uint32_t)umin64(CH, plain_n - c0);
    Op::step(st, p, op_smem, acc, rows, ctid, NCT);
  }

  Op::finish(st, p, op_smem, ctid, NCT);
}

}  // namespace fdb
