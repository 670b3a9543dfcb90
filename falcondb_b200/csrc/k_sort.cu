// Full ORDER BY on one FLOAT64 / INT64 column (execute_sort / sort_merged ->
// try_typed_sort, FalconDB src/query/sort.rs:118-133, 209-350): the rows of a
// column in the order of (order key, row), NULL rows first or last in row
// order (assemble, sort.rs:773-791).  Order keys are the ones the top-k uses
// (f64_ord_key, sort.rs:451-454; the sign flip for int64; bitwise NOT for
// DESC), so -0.0 sorts before +0.0 and NaN above +inf, as in the reference.
//
// A stable LSD radix sort of (order key, row) pairs with 8-bit digits:
//   * the key pass writes the pairs and ORs / ANDs every key, so a byte that
//     is the same in every key costs no pass;
//   * per pass, radix_hist_kernel counts the digits of each 4096-key tile
//     (histogram laid out digit-major, [digit][tile]); an exclusive scan of the
//     histogram gives every (digit, tile) its output offset;
//     radix_scatter_kernel stages each tile in shared memory (TMA bulk
//     copies, double-buffered), ranks its keys stably with warp votes, permutes
//     the tile into digit order in place and writes it out in runs, with the
//     next pass's digit of each key as a byte beside it, so every pass after
//     the first counts 1 byte per key (radix_hist_digits_kernel), not 8;
//   * the last pass writes the row numbers straight into the output.
// Every scatter position is checked against the key count (an error, never an
// out-of-bounds write).
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"
#include "topk_warp.cuh"

namespace fdb {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr uint32_t kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

// Keys of the selected rows (sel[i], or row i when sel is null) and their
// rows; vary[0] |= every key, vary[1] &= every key.  ORDER BY keys are order
// keys (wt_key; MODE 0 ascending, 1 descending, 2 / 3 the same for an INT64
// column taken as f64); DISTINCT keys (DISTINCT_KEY) only have to be equal exactly
// when the values are: FLOAT64 bits with every NaN made one NaN and -0.0 made
// +0.0 (norm_f64, select.rs:201-204), INT64 bits, UTF8 codes.
constexpr int DISTINCT_KEY = -1;
template <int DT, int MODE>
__device__ __forceinline__ uint64_t sort_key_of(const DevCol& col, uint32_t row) {
  if constexpr (MODE == DISTINCT_KEY) {
    if constexpr (DT == FDB_UTF8) {
      return static_cast<const uint32_t*>(col.values)[row];
    } else {
      uint64_t b = static_cast<const uint64_t*>(col.values)[row];
      if constexpr (DT == FDB_FLOAT64) {
        if ((b & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull) b = 0x7FF8000000000000ull;  // NaN
        if (b == 0x8000000000000000ull) b = 0;                                                 // -0.0
      }
      return b;
    }
  } else if constexpr (MODE >= 2) {
    // An INT64 key read as f64 first (ROW_NUMBER's eval_dense_f64, expr.rs:232).
    const double d = (double)static_cast<const int64_t*>(col.values)[row];
    return wt_key<FDB_FLOAT64, MODE == 3>((uint64_t)__double_as_longlong(d));
  } else {
    return wt_key<DT, MODE != 0>(static_cast<const uint64_t*>(col.values)[row]);
  }
}

template <int DT, int MODE>
__global__ void sort_key_kernel(DevCol col, const uint32_t* sel, uint32_t m, uint64_t* keys, uint32_t* vals,
                                unsigned long long* vary) {
  unsigned long long o = 0, a = ~0ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t row = sel ? sel[i] : i;
    const uint64_t k = sort_key_of<DT, MODE>(col, row);
    keys[i] = k;
    vals[i] = row;
    o |= k;
    a &= k;
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    o |= __shfl_xor_sync(0xffffffffu, o, s);
    a &= __shfl_xor_sync(0xffffffffu, a, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&vary[0], o);
    atomicAnd(&vary[1], a);
  }
}

// DISTINCT: the first row of every run of equal keys in the sorted pairs, and
// the first NULL row (nulls[0] when *nnull > 0), set in a row mask.
__global__ void distinct_heads_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ rows,
                                      uint32_t m, const uint32_t* nulls, const uint64_t* nnull,
                                      unsigned long long* mask) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (i == 0 || keys[i] != keys[i - 1]) {
      const uint32_t r = rows[i];
      atomicOr(&mask[r >> 6], 1ull << (r & 63));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && nnull && *nnull > 0) {
    const uint32_t r = nulls[0];
    atomicOr(&mask[r >> 6], 1ull << (r & 63));
  }
}

// Digit counts of one tile: hist[d * ntiles + tile].  Each thread counts a
// run of equal digits before it adds it to its warp's counters, so a byte that
// takes few values (the exponent bytes of a float column) costs few atomics.
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint64_t* __restrict__ keys, uint32_t m,
                                                                  int shift, uint32_t ntiles, uint32_t* hist) {
  __shared__ uint32_t cnt[kSortWarps][256];
  const int tid = threadIdx.x, warp = tid >> 5;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) cnt[w][tid] = 0;
  __syncthreads();
  const uint64_t t0 = (uint64_t)blockIdx.x * kSortTile;
  uint64_t k[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const uint64_t i = t0 + (uint64_t)r * kSortThreads + tid;
    k[r] = i < m ? keys[i] : 0ull;
  }
  uint32_t run_d = 0, run_c = 0;
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const uint64_t i = t0 + (uint64_t)r * kSortThreads + tid;
    if (i < m) {
      const uint32_t d = (uint32_t)(k[r] >> shift) & 255u;
      if (d != run_d && run_c) {
        atomicAdd(&cnt[warp][run_d], run_c);
        run_c = 0;
      }
      run_d = d;
      ++run_c;
    }
  }
  if (run_c) atomicAdd(&cnt[warp][run_d], run_c);
  __syncthreads();
  uint32_t t = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) t += cnt[w][tid];
  hist[(size_t)tid * ntiles + blockIdx.x] = t;
}

// The same counts from the digit bytes the previous pass's scatter wrote (one
// byte per key at the key's new position): one warp per tile, eight tiles per
// CTA, so each digit's counts of a CTA's tiles are one 32-byte store run.  A
// lane reads eight 16-byte chunks (128 consecutive keys in 16-key runs).
constexpr int kDigitHistWarps = 8;
constexpr uint32_t kDigitChunks = kSortTile / 16 / 32;  // 16-byte chunks per lane
static_assert(kSortTile % (16 * 32) == 0, "a tile is whole 16-byte chunks for every lane");

__global__ void __launch_bounds__(kDigitHistWarps * 32)
    radix_hist_digits_kernel(const uint8_t* __restrict__ dg, uint32_t m, uint32_t ntiles, uint32_t* hist) {
  __shared__ uint32_t cnt[kDigitHistWarps][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t tile = blockIdx.x * kDigitHistWarps + warp;
#pragma unroll
  for (int j = 0; j < 256; j += 32) cnt[warp][j + lane] = 0;
  __syncwarp();
  if (tile >= ntiles) return;
  const uint64_t t0 = (uint64_t)tile * kSortTile;
  const uint32_t n = (uint32_t)umin64(kSortTile, m - t0);
  uint32_t run_d = 0, run_c = 0;
  auto count = [&](uint32_t d) {
    if (d != run_d && run_c) {
      atomicAdd(&cnt[warp][run_d], run_c);
      run_c = 0;
    }
    run_d = d;
    ++run_c;
  };
  if (n == kSortTile) {
    uint4 v[kDigitChunks];
#pragma unroll
    for (uint32_t r = 0; r < kDigitChunks; ++r)
      v[r] = __ldcs(reinterpret_cast<const uint4*>(dg + t0) + r * 32 + lane);
#pragma unroll
    for (uint32_t r = 0; r < kDigitChunks; ++r) {
      const uint32_t w[4] = {v[r].x, v[r].y, v[r].z, v[r].w};
#pragma unroll
      for (int q = 0; q < 16; ++q) count((w[q >> 2] >> ((q & 3) * 8)) & 255u);
    }
  } else {  // the ragged last tile: byte loads below n
    for (uint32_t r = 0; r < kDigitChunks; ++r) {
      const uint32_t b0 = (r * 32 + lane) * 16;
      for (uint32_t q = 0; q < 16 && b0 + q < n; ++q) count(dg[t0 + b0 + q]);
    }
  }
  if (run_c) atomicAdd(&cnt[warp][run_d], run_c);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 256; j += 32) hist[(size_t)(j + lane) * ntiles + tile] = cnt[warp][j + lane];
}

// Exclusive scan of n uint32 in place: per-block sums, a scan of the sums,
// then each block's scan offset by its sum.
constexpr int kScanT = 1024, kScanPer = 4, kScanB = kScanT * kScanPer;

__device__ uint32_t sort_block_scan(uint32_t v, uint32_t* sm, uint32_t* total) {
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

__global__ void sort_scan_sums_kernel(const uint32_t* in, uint64_t n, uint32_t* bsum) {
  __shared__ uint32_t sm[32];
  const uint64_t i0 = (uint64_t)blockIdx.x * kScanB + threadIdx.x * kScanPer;
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j)
    if (i0 + j < n) s += in[i0 + j];
  uint32_t tot;
  sort_block_scan(s, sm, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void sort_scan_top_kernel(uint32_t* bsum, uint64_t nb) {
  __shared__ uint32_t sm[32];
  const uint64_t per = (nb + blockDim.x - 1) / blockDim.x;
  const uint64_t b0 = threadIdx.x * per;
  uint32_t local = 0;
  for (uint64_t i = b0; i < b0 + per && i < nb; ++i) local += bsum[i];
  uint32_t base = sort_block_scan(local, sm, nullptr);
  for (uint64_t i = b0; i < b0 + per && i < nb; ++i) {
    const uint32_t v = bsum[i];
    bsum[i] = base;
    base += v;
  }
}

__global__ void sort_scan_apply_kernel(uint32_t* data, uint64_t n, const uint32_t* bsum) {
  __shared__ uint32_t sm[32];
  const uint64_t i0 = (uint64_t)blockIdx.x * kScanB + threadIdx.x * kScanPer;
  uint32_t v[kScanPer];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    v[j] = i0 + j < n ? data[i0 + j] : 0u;
    s += v[j];
  }
  uint32_t run = bsum[blockIdx.x] + sort_block_scan(s, sm, nullptr);
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    if (i0 + j < n) data[i0 + j] = run;
    run += v[j];
  }
}

// Stable scatter of the tiles by digit.  Persistent CTAs take tiles
// round-robin; thread 0 stages each tile's keys and rows into one of two
// shared-memory buffers with TMA bulk copies, so the next tile arrives while
// this one is ranked (a ragged last tile, whose byte count is not a multiple
// of 16, is read with plain loads).  Warp w ranks the 512 keys
// [w*512, (w+1)*512) of the tile in index order (nine warp votes group a
// round's equal digits; a per-warp counter per digit carries the rank across
// rounds); one block-wide scan turns (digit, warp, rank) into the key's place
// in the tile sorted by digit; the tile is permuted into that order in place
// and written out in it, so neighbouring threads store neighbouring addresses
// of one digit's output range.  The last pass stores no keys.
constexpr int kScatterThreads = 256;
constexpr int kScatterWarps = kScatterThreads / 32;
constexpr int kSubTile = kSortTile / kScatterWarps;  // 512 keys per warp
constexpr int kSubRounds = kSubTile / 32;
constexpr int kScatterItems = kSortTile / kScatterThreads;
constexpr int kScatterCtasPerSm = 2;
struct ScatterSmem {
  uint64_t keys[2][kSortTile];
  uint32_t vals[2][kSortTile];
  uint16_t wc[kScatterWarps][256];  // per-warp digit counts, then tile offsets (< 4096)
  uint32_t gbase[256];
  uint32_t wsum[8];
  uint64_t full[2];
};

// The lanes of the warp whose d equals this lane's, d < 2^NB: one vote per bit.
template <int NB>
__device__ __forceinline__ unsigned warp_match_digit(uint32_t d) {
  unsigned peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const bool bit = (d >> b) & 1u;
    const unsigned vote = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? vote : ~vote;
  }
  return peers;
}

__device__ __forceinline__ bool sort_tile_ragged(uint64_t t, uint64_t ntiles, uint32_t m) {
  return t + 1 == ntiles && (m % kSortTile) % 4u != 0;
}

__device__ __forceinline__ void sort_stage_tile(ScatterSmem& S, int s, uint64_t t, uint32_t m,
                                                const uint64_t* kin, const uint32_t* vin, uint64_t policy) {
  const uint64_t t0 = t * kSortTile;
  const uint32_t n = (uint32_t)umin64(kSortTile, m - t0);
  mbar_arrive_expect_tx(&S.full[s], n * 12u);
  bulk_g2s(S.keys[s], kin + t0, n * 8u, &S.full[s], policy);
  bulk_g2s(S.vals[s], vin + t0, n * 4u, &S.full[s], policy);
}

__global__ void __launch_bounds__(kScatterThreads, kScatterCtasPerSm)
    radix_scatter_kernel(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t m, int shift,
                         const uint32_t* __restrict__ off, uint32_t ntiles, uint64_t* __restrict__ kout,
                         uint32_t* __restrict__ vout, bool write_keys, uint8_t* __restrict__ dg_out, int next_shift,
                         int* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  ScatterSmem& S = *reinterpret_cast<ScatterSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned below = (1u << lane) - 1u;
  uint64_t policy = 0;
  if (tid == 0) {
    mbar_init(&S.full[0], 1);
    mbar_init(&S.full[1], 1);
    fence_mbar_init();
    policy = l2_evict_first_policy();
  }
  __syncthreads();
  // Thread 0: per stage, a copy issued and not yet seen complete, and the
  // iteration it is for (its phase parity is (iteration / 2) & 1).
  uint32_t pending = 0;                // bit j: stage j
  uint32_t pend_it0 = 0, pend_it1 = 1;
  if (tid == 0) {
    for (int j = 0; j < 2; ++j) {
      const uint64_t t = blockIdx.x + (uint64_t)j * gridDim.x;
      if (t < ntiles && !sort_tile_ragged(t, ntiles, m)) {
        sort_stage_tile(S, j, t, m, kin, vin, policy);
        pending |= 1u << j;
      }
    }
  }
  bool dead = false;
  uint32_t it = 0;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int s = it & 1;
    const uint64_t t0 = t * kSortTile;
    const uint32_t tile_n = (uint32_t)umin64(kSortTile, m - t0);
    if (sort_tile_ragged(t, ntiles, m)) {
      for (uint32_t i = tid; i < tile_n; i += kScatterThreads) {
        S.keys[s][i] = kin[t0 + i];
        S.vals[s][i] = vin[t0 + i];
      }
      __syncthreads();
    } else {
      const bool ok = !dead && mbar_wait(&S.full[s], (it >> 1) & 1u, err);
      if (!ok) dead = true;  // the tile is processed from whatever the stage holds
      if (tid == 0 && ok) pending &= ~(1u << s);
    }

#pragma unroll
    for (int j = 0; j < 256; j += 32) S.wc[warp][j + lane] = 0;
    __syncwarp();
    const uint32_t w0 = (uint32_t)warp * kSubTile;
    const bool full_tile = tile_n == kSortTile;
    uint64_t k[kSubRounds];
    uint32_t rk[kSubRounds / 2];  // ranks (< 512) two to a register
#pragma unroll
    for (int r = 0; r < kSubRounds; ++r) {
      const uint32_t i = w0 + r * 32 + lane;
      k[r] = i < tile_n ? S.keys[s][i] : 0ull;
    }
#pragma unroll
    for (int r = 0; r < kSubRounds; ++r) {
      const uint32_t i = w0 + r * 32 + lane;
      const uint32_t d = i < tile_n ? (uint32_t)(k[r] >> shift) & 255u : 256u;
      const unsigned peers = full_tile ? warp_match_digit<8>(d) : warp_match_digit<9>(d);
      const int leader = __ffs(peers) - 1;
      uint32_t pre = 0;
      if (d < 256u && lane == leader) {
        pre = S.wc[warp][d];
        S.wc[warp][d] = (uint16_t)(pre + (uint32_t)__popc(peers));
      }
      pre = __shfl_sync(0xffffffffu, pre, leader);
      const uint32_t rank = pre + (uint32_t)__popc(peers & below);
      if (r & 1)
        rk[r >> 1] |= rank << 16;
      else
        rk[r >> 1] = rank;
      __syncwarp();
    }
    __syncthreads();

    // Threads 0..255 own digit tid: its count in this tile, where it starts
    // in the tile's digit order, and where each warp's keys of it start.
    uint32_t tot = 0, x = 0;
    if (tid < 256) {
#pragma unroll
      for (int w = 0; w < kScatterWarps; ++w) {
        const uint32_t c = S.wc[w][tid];
        S.wc[w][tid] = (uint16_t)tot;
        tot += c;
      }
      x = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) S.wsum[warp] = x;
    }
    __syncthreads();
    if (tid < 256) {
      uint32_t dstart = x - tot;
#pragma unroll
      for (int w = 0; w < 8; ++w)
        if (w < warp) dstart += S.wsum[w];
#pragma unroll
      for (int w = 0; w < kScatterWarps; ++w) S.wc[w][tid] = (uint16_t)(S.wc[w][tid] + dstart);
      S.gbase[tid] = off[(size_t)tid * ntiles + t] - dstart;
    }
    uint32_t v[kSubRounds];
#pragma unroll
    for (int r = 0; r < kSubRounds; ++r) {
      const uint32_t i = w0 + r * 32 + lane;
      v[r] = i < tile_n ? S.vals[s][i] : 0u;
    }
    __syncthreads();

    // Permute the tile in place into digit order.
#pragma unroll
    for (int r = 0; r < kSubRounds; ++r) {
      const uint32_t i = w0 + r * 32 + lane;
      if (i < tile_n) {
        const uint32_t d = (uint32_t)(k[r] >> shift) & 255u;
        const uint32_t lp = S.wc[warp][d] + ((rk[r >> 1] >> ((r & 1) * 16)) & 0xFFFFu);
        S.keys[s][lp] = k[r];
        S.vals[s][lp] = v[r];
      }
    }
    __syncthreads();

#pragma unroll 4
    for (int j = 0; j < kScatterItems; ++j) {
      const uint32_t i = (uint32_t)j * kScatterThreads + tid;
      if (i < tile_n) {
        const uint64_t kk = S.keys[s][i];
        const uint32_t pos = S.gbase[(uint32_t)(kk >> shift) & 255u] + i;
        if (pos < m) {
          if (write_keys) kout[pos] = kk;
          if (dg_out) dg_out[pos] = (uint8_t)(kk >> next_shift);
          vout[pos] = S.vals[s][i];
        } else {
          atomicExch(err, kErrCapacity);
        }
      }
    }
    fence_proxy_async_smem();  // this thread's stores to stage s come before the next bulk copy into it
    __syncthreads();           // stage s and the counters are free again
    if (tid == 0 && !dead) {  // after a time-out no further copies are started
      const uint64_t tn = t + 2ull * gridDim.x;
      if (tn < ntiles && !sort_tile_ragged(tn, ntiles, m)) {
        sort_stage_tile(S, s, tn, m, kin, vin, policy);
        pending |= 1u << s;
        if (s)
          pend_it1 = it + 2;
        else
          pend_it0 = it + 2;
      }
    }
  }
  // After a timed-out wait, let this CTA's own copies land before it exits.
  if (tid == 0) {
    if (pending & 1u) mbar_wait(&S.full[0], (pend_it0 >> 1) & 1u, nullptr);
    if (pending & 2u) mbar_wait(&S.full[1], (pend_it1 >> 1) & 1u, nullptr);
  }
}

// Validity bits of rows [0, n) re-aligned to row 0 (the column's bits start at
// bit voff), or their complement when `nulls` is set; bits past n are zero.
__global__ void sort_valid_mask_kernel(DevCol col, uint64_t n, bool nulls, uint64_t* mask) {
  const uint64_t words = (n + 63) / 64;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t rows = n - w * 64 < 64 ? n - w * 64 : 64;
    const uint64_t b = col.voff + w * 64;
    const int sh = (int)(b & 63);
    uint64_t x = col.validity[b >> 6] >> sh;
    if (sh != 0 && (uint64_t)(64 - sh) < rows) x |= col.validity[(b >> 6) + 1] << (64 - sh);
    if (nulls) x = ~x;
    if (rows < 64) x &= (1ull << rows) - 1;
    mask[w] = x;
  }
}

template <int DT, int MODE>
static void launch_sort_keys(Ctx& c, const DevCol& col, const uint32_t* sel, uint32_t m, uint64_t* keys,
                             uint32_t* vals, unsigned long long* vary) {
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((m + 255) / 256, (uint64_t)c.sm_count * 8));
  sort_key_kernel<DT, MODE><<<grid, 256, 0, c.stream>>>(col, sel, m, keys, vals, vary);
}

// Scratch a sort of up to n pairs takes: two (key, row) buffers, the
// histogram and its scan sums, and with the NULL split its mask and row lists.
static size_t sort_scratch_bytes(uint64_t n, bool nullable) {
  const uint64_t words = (n + 63) / 64;
  const uint64_t ntiles = (n + kSortTile - 1) / kSortTile;
  const uint64_t hn = 256ull * ntiles;
  const uint64_t nb = (hn + kScanB - 1) / kScanB;
  size_t need = 2 * n * 8 + 2 * n * 4 + n + hn * 4 + nb * 4 + 16;
  if (nullable) need += words * 8 + 2 * n * 4 + 16;
  return need + (2u << 20);  // + 256-byte rounding and the compaction's chunk counts
}

// The rows of a column split into non-NULL rows (`sel`, row order) and NULL
// rows (`nulls`, row order); both counts are also left on the device
// (d_counts[0], d_counts[1]).
struct NullSplit {
  const uint32_t* sel = nullptr;
  uint32_t* nulls = nullptr;
  uint64_t* d_counts = nullptr;
  uint64_t m = 0, nnull = 0;
};

static NullSplit split_nulls(Ctx& c, const DevCol& dc, uint64_t n) {
  NullSplit r;
  r.m = n;
  if (!dc.validity) return r;
  const uint64_t words = (n + 63) / 64;
  uint64_t* mask = static_cast<uint64_t*>(c.scratch_take(words * 8));
  uint32_t* vrows = static_cast<uint32_t*>(c.scratch_take(n * 4));
  r.nulls = static_cast<uint32_t*>(c.scratch_take(n * 4));
  r.d_counts = static_cast<uint64_t*>(c.scratch_take(16));
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((words + 255) / 256, (uint64_t)c.sm_count * 4));
  sort_valid_mask_kernel<<<g, 256, 0, c.stream>>>(dc, n, false, mask);
  op_compact_mask(c, mask, n, vrows, n, r.d_counts);
  sort_valid_mask_kernel<<<g, 256, 0, c.stream>>>(dc, n, true, mask);
  op_compact_mask(c, mask, n, r.nulls, n, r.d_counts + 1);
  uint64_t hc[2] = {0, 0};
  FDB_CUDA(cudaMemcpyAsync(hc, r.d_counts, 16, cudaMemcpyDeviceToHost, c.stream));
  FDB_CUDA(cudaStreamSynchronize(c.stream));
  if (hc[0] + hc[1] != n) fail(FDB_E_GENERIC, "sort: valid and NULL rows do not add up to the row count");
  r.m = hc[0];
  r.nnull = hc[1];
  r.sel = vrows;
  return r;
}

// Stable radix sort of the (key, row) pairs of `sel` (m rows): builds the
// pairs with key kernel `keys_fn`, then runs one pass per byte that varies.
// With `rows_out`, the last pass writes the rows there and no keys (and the
// result is in rows_out); otherwise the sorted keys and rows are returned in
// *keys_sorted / *rows_sorted (scratch).
template <class KeysFn>
static void radix_sort_pairs(Ctx& c, uint32_t m, KeysFn keys_fn, uint32_t* rows_out, const uint64_t** keys_sorted,
                             const uint32_t** rows_sorted) {
  uint64_t* ka = static_cast<uint64_t*>(c.scratch_take(m * 8));
  uint64_t* kb = static_cast<uint64_t*>(c.scratch_take(m * 8));
  uint32_t* va = static_cast<uint32_t*>(c.scratch_take(m * 4));
  uint32_t* vb = static_cast<uint32_t*>(c.scratch_take(m * 4));
  const uint32_t ntiles = (uint32_t)((m + kSortTile - 1) / kSortTile);
  const uint64_t hn = 256ull * ntiles;
  const uint64_t nb = (hn + kScanB - 1) / kScanB;
  uint32_t* hist = static_cast<uint32_t*>(c.scratch_take(hn * 4));
  uint32_t* bsum = static_cast<uint32_t*>(c.scratch_take(nb * 4));
  uint8_t* dg = static_cast<uint8_t*>(c.scratch_take(m));  // the next pass's digit of each key
  unsigned long long* vary = static_cast<unsigned long long*>(c.scratch_take(16));
  FDB_CUDA(cudaMemsetAsync(vary, 0, 8, c.stream));
  FDB_CUDA(cudaMemsetAsync(vary + 1, 0xFF, 8, c.stream));
  keys_fn(ka, va, vary);
  FDB_CUDA(cudaGetLastError());
  unsigned long long hv[2] = {0, 0};
  FDB_CUDA(cudaMemcpyAsync(hv, vary, 16, cudaMemcpyDeviceToHost, c.stream));
  FDB_CUDA(cudaStreamSynchronize(c.stream));
  const uint64_t varying = hv[0] ^ hv[1];  // bits that are not the same in every key
  int last_byte = -1;
  for (int byte = 0; byte < 8; ++byte)
    if ((varying >> (8 * byte)) & 0xFFull) last_byte = byte;
  int shifts[8], npass = 0;
  for (int byte = 0; byte <= last_byte; ++byte)
    if ((varying >> (8 * byte)) & 0xFFull) shifts[npass++] = 8 * byte;  // else one digit for every key
  const int grid = (int)std::min<uint64_t>(ntiles, (uint64_t)kScatterCtasPerSm * c.sm_count);
  for (int p = 0; p < npass; ++p) {
    const int shift = shifts[p];
    if (p == 0)
      radix_hist_kernel<<<ntiles, kSortThreads, 0, c.stream>>>(ka, m, shift, ntiles, hist);
    else  // the digits the last scatter wrote
      radix_hist_digits_kernel<<<(ntiles + kDigitHistWarps - 1) / kDigitHistWarps, kDigitHistWarps * 32, 0,
                                 c.stream>>>(dg, m, ntiles, hist);
    sort_scan_sums_kernel<<<(unsigned)nb, kScanT, 0, c.stream>>>(hist, hn, bsum);
    sort_scan_top_kernel<<<1, kScanT, 0, c.stream>>>(bsum, nb);
    sort_scan_apply_kernel<<<(unsigned)nb, kScanT, 0, c.stream>>>(hist, hn, bsum);
    const bool last = p + 1 == npass;
    const bool direct = rows_out && last;  // rows go straight to the output; keys are not needed
    radix_scatter_kernel<<<grid, kScatterThreads, sizeof(ScatterSmem), c.stream>>>(
        ka, va, m, shift, hist, ntiles, kb, direct ? rows_out : vb, !direct, last ? nullptr : dg,
        last ? 0 : shifts[p + 1], c.d_err);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  FDB_CUDA(cudaGetLastError());
  if (rows_out && last_byte < 0)  // every key equal: row order is the answer
    FDB_CUDA(cudaMemcpyAsync(rows_out, va, (size_t)m * 4, cudaMemcpyDeviceToDevice, c.stream));
  if (keys_sorted) *keys_sorted = ka;
  if (rows_sorted) *rows_sorted = va;
}

static void set_scatter_smem() {
  FDB_CUDA(cudaFuncSetAttribute(radix_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem)));
}

// Join row pairs as sort keys: (left << 32) | right (right = 0 without one).
__global__ void pair_key_kernel(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right, uint32_t n,
                                uint64_t* keys, uint32_t* vals, unsigned long long* vary) {
  unsigned long long o = 0, a = ~0ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ((uint64_t)left[i] << 32) | (right ? right[i] : 0u);
    keys[i] = k;
    vals[i] = i;
    o |= k;
    a &= k;
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    o |= __shfl_xor_sync(0xffffffffu, o, s);
    a &= __shfl_xor_sync(0xffffffffu, a, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&vary[0], o);
    atomicAnd(&vary[1], a);
  }
}

__global__ void pair_unpack_kernel(const uint64_t* __restrict__ keys, uint32_t n, uint32_t* left, uint32_t* right) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    left[i] = (uint32_t)(k >> 32);
    if (right) right[i] = (uint32_t)k;
  }
}

void op_sort_row_pairs(Ctx& c, uint32_t* d_left, uint32_t* d_right, uint64_t n) {
  if (n == 0) return;
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "a sort addresses rows as uint32");
  set_scatter_smem();
  c.ensure_scratch(c.scratch_top + sort_scratch_bytes(n, false));
  const uint32_t m = (uint32_t)n;
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)c.sm_count * 8));
  auto keys = [&](uint64_t* k, uint32_t* v, unsigned long long* vary) {
    pair_key_kernel<<<g, 256, 0, c.stream>>>(d_left, d_right, m, k, v, vary);
  };
  const uint64_t* sorted = nullptr;
  radix_sort_pairs(c, m, keys, nullptr, &sorted, nullptr);
  pair_unpack_kernel<<<g, 256, 0, c.stream>>>(sorted, m, d_left, d_right);
  FDB_CUDA(cudaGetLastError());
}

// rows[i] = position of row i in the order: ROW_NUMBER() OVER (ORDER BY ..)
// numbers the rows 1..n in sorted order (rank_dense, window.rs:259-300).
__global__ void row_number_kernel(const uint32_t* order, const uint32_t* list, uint32_t n, int64_t* rn) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t o = order ? order[j] : j;
    rn[list ? list[o] : o] = (int64_t)j + 1;
  }
}

void op_row_numbers(Ctx& c, const uint32_t* d_order, const uint32_t* d_list, uint64_t n, int64_t* d_rn) {
  if (n == 0) return;
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "ROW_NUMBER addresses rows as uint32");
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)c.sm_count * 8));
  row_number_kernel<<<g, 256, 0, c.stream>>>(d_order, d_list, (uint32_t)n, d_rn);
  FDB_CUDA(cudaGetLastError());
}

void op_sort(Ctx& c, const fdb_dev_column& col, uint64_t n, bool desc, bool nulls_last, uint32_t* d_rows) {
  op_sort_keyed(c, col, n, desc, nulls_last, false, d_rows);
}

void op_sort_keyed(Ctx& c, const fdb_dev_column& col, uint64_t n, bool desc, bool nulls_last, bool int_as_f64,
                   uint32_t* d_rows) {
  if (col.dtype != FDB_FLOAT64 && col.dtype != FDB_INT64) fail(FDB_E_TYPE, "ORDER BY needs a FLOAT64 or INT64 column");
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "a sort addresses rows as uint32");
  if (n == 0) return;
  if (!col.values) fail(FDB_E_ARG, "column without values");
  const DevCol dc{col.dtype, col.values, col.validity, col.validity_offset};
  set_scatter_smem();
  // Working memory comes from the context's scratch arena, which grows once
  // and stays resident.
  c.ensure_scratch(c.scratch_top + sort_scratch_bytes(n, col.validity != nullptr));

  // NULL rows leave the sort: the valid rows are sorted, the NULL rows keep
  // their row order before or after them.
  const NullSplit ns = split_nulls(c, dc, n);
  if (ns.m > 0) {
    const uint32_t m = (uint32_t)ns.m;
    auto keys = [&](uint64_t* k, uint32_t* v, unsigned long long* vary) {
      if (col.dtype == FDB_FLOAT64)
        desc ? launch_sort_keys<FDB_FLOAT64, 1>(c, dc, ns.sel, m, k, v, vary)
             : launch_sort_keys<FDB_FLOAT64, 0>(c, dc, ns.sel, m, k, v, vary);
      else if (int_as_f64)
        desc ? launch_sort_keys<FDB_INT64, 3>(c, dc, ns.sel, m, k, v, vary)
             : launch_sort_keys<FDB_INT64, 2>(c, dc, ns.sel, m, k, v, vary);
      else
        desc ? launch_sort_keys<FDB_INT64, 1>(c, dc, ns.sel, m, k, v, vary)
             : launch_sort_keys<FDB_INT64, 0>(c, dc, ns.sel, m, k, v, vary);
    };
    radix_sort_pairs(c, m, keys, d_rows + (nulls_last ? 0 : ns.nnull), nullptr, nullptr);
  }
  if (ns.nnull)
    FDB_CUDA(cudaMemcpyAsync(d_rows + (nulls_last ? ns.m : 0), ns.nulls, ns.nnull * 4, cudaMemcpyDeviceToDevice,
                             c.stream));
}

void op_distinct(Ctx& c, const fdb_dev_column& col, uint64_t n, uint32_t* d_rows, uint64_t* d_count) {
  if (col.dtype != FDB_FLOAT64 && col.dtype != FDB_INT64 && col.dtype != FDB_UTF8)
    fail(FDB_E_TYPE, "DISTINCT needs a FLOAT64, INT64 or UTF8 column");
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "DISTINCT addresses rows as uint32");
  if (n == 0) {
    FDB_CUDA(cudaMemsetAsync(d_count, 0, 8, c.stream));
    return;
  }
  if (!col.values) fail(FDB_E_ARG, "column without values");
  const DevCol dc{col.dtype, col.values, col.validity, col.validity_offset};
  set_scatter_smem();
  const uint64_t words = (n + 63) / 64;
  c.ensure_scratch(c.scratch_top + sort_scratch_bytes(n, col.validity != nullptr) + words * 8 + 256);
  unsigned long long* heads = static_cast<unsigned long long*>(c.scratch_take(words * 8));
  FDB_CUDA(cudaMemsetAsync(heads, 0, words * 8, c.stream));

  const NullSplit ns = split_nulls(c, dc, n);
  const uint64_t* skeys = nullptr;
  const uint32_t* srows = nullptr;
  if (ns.m > 0) {
    const uint32_t m = (uint32_t)ns.m;
    auto keys = [&](uint64_t* k, uint32_t* v, unsigned long long* vary) {
      if (col.dtype == FDB_FLOAT64)
        launch_sort_keys<FDB_FLOAT64, DISTINCT_KEY>(c, dc, ns.sel, m, k, v, vary);
      else if (col.dtype == FDB_INT64)
        launch_sort_keys<FDB_INT64, DISTINCT_KEY>(c, dc, ns.sel, m, k, v, vary);
      else
        launch_sort_keys<FDB_UTF8, DISTINCT_KEY>(c, dc, ns.sel, m, k, v, vary);
    };
    radix_sort_pairs(c, m, keys, nullptr, &skeys, &srows);
  }
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((ns.m + 255) / 256, (uint64_t)c.sm_count * 8));
  distinct_heads_kernel<<<g, 256, 0, c.stream>>>(skeys, srows, (uint32_t)ns.m, ns.nulls,
                                                 ns.nnull ? ns.d_counts + 1 : nullptr, heads);
  FDB_CUDA(cudaGetLastError());
  op_compact_mask(c, reinterpret_cast<const uint64_t*>(heads), n, d_rows, n, d_count);
}


// ---------------------------------------------------------------------------
// ORDER BY several keys, ORDER BY a text column, and DISTINCT over several
// columns (sort_merged over several SortExprs, sort.rs:118-165; the text
// column's dictionary ranked once and its rows sorted by rank, sort.rs:352-382;
// dedup_batches over whole rows, select.rs:238-269).
//
// Positions 0..n-1 of a row list (position p is row list[p], or row p) are put
// in order by a least-significant-key-first sequence of stable radix sorts:
// the last key first, then each earlier key over the order so far, so ties
// on every key keep position order, as the reference's (keys..., row)
// comparison does.  Each pass takes the key's NULL positions out (in the
// current order) and puts them first or last.
// ---------------------------------------------------------------------------
struct MKey {
  DevCol col;
  const uint32_t* rank;  // UTF8 ORDER BY: rank of each code in the sorted dictionary
  uint32_t rank_len;
  int32_t desc;
  int32_t distinct;      // DISTINCT keys (equal exactly when the values are) instead of order keys
};

__device__ __forceinline__ bool mkey_null(const MKey& k, uint32_t row) {
  if (k.col.validity && !col_valid(k.col, row)) return true;
  if (k.col.dtype == FDB_UTF8) {
    const uint32_t code = static_cast<const uint32_t*>(k.col.values)[row];
    return code == kNullCode || (k.rank && code >= k.rank_len);
  }
  return false;
}

__device__ __forceinline__ uint64_t mkey_of(const MKey& k, uint32_t row) {
  uint64_t key;
  if (k.col.dtype == FDB_UTF8) {
    const uint32_t code = static_cast<const uint32_t*>(k.col.values)[row];
    key = k.rank ? k.rank[code] : code;
  } else {
    uint64_t b = static_cast<const uint64_t*>(k.col.values)[row];
    if (k.distinct) {
      if (k.col.dtype == FDB_FLOAT64) {
        if ((b & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull) b = 0x7FF8000000000000ull;  // NaN
        if (b == 0x8000000000000000ull) b = 0;                                                 // -0.0
      }
      return b;
    }
    key = k.col.dtype == FDB_FLOAT64 ? f64_ord_key(__longlong_as_double((long long)b)) : (b ^ (1ull << 63));
  }
  return k.desc ? ~key : key;
}

__device__ __forceinline__ uint32_t list_row(const uint32_t* list, uint32_t pos) { return list ? list[pos] : pos; }

__global__ void iota_u32_kernel(uint32_t* out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)i;
}

__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx, uint64_t n,
                                  uint32_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = src[idx[i]];
}

// Bit i of the mask: the key at position order[i] is NULL (nulls) / is not.
// Bits past n are zero.  One 32-bit half word per warp (a ballot).
__global__ void mkey_null_mask_kernel(MKey k, const uint32_t* list, const uint32_t* order, uint64_t n, bool nulls,
                                      uint32_t* mask32) {
  const uint64_t n32 = (n + 63) / 64 * 64;  // whole 64-bit words
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n32; i += (uint64_t)gridDim.x * blockDim.x) {
    bool bit = false;
    if (i < n) bit = mkey_null(k, list_row(list, order[i])) == nulls;
    const unsigned b = __ballot_sync(0xffffffffu, bit);
    if ((threadIdx.x & 31) == 0) mask32[i >> 5] = b;
  }
}

__global__ void mkey_sort_key_kernel(MKey k, const uint32_t* list, const uint32_t* sel, uint32_t m, uint64_t* keys,
                                     uint32_t* vals, unsigned long long* vary) {
  unsigned long long o = 0, a = ~0ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t pos = sel[i];
    const uint64_t key = mkey_of(k, list_row(list, pos));
    keys[i] = key;
    vals[i] = pos;
    o |= key;
    a &= key;
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    o |= __shfl_xor_sync(0xffffffffu, o, s);
    a &= __shfl_xor_sync(0xffffffffu, a, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&vary[0], o);
    atomicAnd(&vary[1], a);
  }
}

constexpr int kMaxMultiKeys = 8;
struct MKeys {
  MKey k[kMaxMultiKeys];
  int32_t n;
};

// DISTINCT over several columns: position order[i] heads a run when i == 0 or
// any column's NULL-ness or DISTINCT key differs from position order[i-1]'s;
// its bit is set in the position mask.
__global__ void multi_heads_kernel(MKeys ks, const uint32_t* list, const uint32_t* order, uint64_t n,
                                   unsigned long long* mask) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = order[i];
    bool head = i == 0;
    if (!head) {
      const uint32_t r = list_row(list, p), q = list_row(list, order[i - 1]);
      for (int j = 0; j < ks.n && !head; ++j) {
        const bool nr = mkey_null(ks.k[j], r), nq = mkey_null(ks.k[j], q);
        head = nr != nq || (!nr && mkey_of(ks.k[j], r) != mkey_of(ks.k[j], q));
      }
    }
    if (head) atomicOr(&mask[p >> 6], 1ull << (p & 63));
  }
}

static MKey to_mkey(const SortKey& k) {
  MKey m;
  m.col = DevCol{k.col.dtype, k.col.values, k.col.validity, k.col.validity_offset};
  m.rank = k.rank;
  m.rank_len = k.rank_len;
  m.desc = k.desc ? 1 : 0;
  m.distinct = k.distinct ? 1 : 0;
  return m;
}

size_t sort_multi_scratch(uint64_t n) {
  const uint64_t words = (n + 63) / 64;
  return sort_scratch_bytes(n, true) + words * 8 + 4 * n * 4 + 16 + 4096;
}

void op_sort_multi(Ctx& c, const SortKey* keys, int nkeys, const uint32_t* d_list, uint64_t n, uint32_t* d_pos) {
  if (nkeys < 1 || nkeys > kMaxMultiKeys) fail(FDB_E_ARG, "between 1 and 8 sort keys");
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "a sort addresses rows as uint32");
  if (n == 0) return;
  for (int j = 0; j < nkeys; ++j) {
    const SortKey& k = keys[j];
    if (k.col.dtype != FDB_FLOAT64 && k.col.dtype != FDB_INT64 && k.col.dtype != FDB_UTF8)
      fail(FDB_E_TYPE, "sort keys are FLOAT64, INT64 or UTF8 columns");
    if (!k.col.values) fail(FDB_E_ARG, "column without values");
    if (k.col.dtype == FDB_UTF8 && !k.distinct && !k.rank) fail(FDB_E_ARG, "text ORDER BY key without ranks");
  }
  set_scatter_smem();
  c.ensure_scratch(c.scratch_top + sort_multi_scratch(n));
  const uint32_t m = (uint32_t)n;
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)c.sm_count * 8));
  iota_u32_kernel<<<g, 256, 0, c.stream>>>(d_pos, n);
  FDB_CUDA(cudaGetLastError());
  const uint64_t words = (n + 63) / 64;
  for (int j = nkeys - 1; j >= 0; --j) {
    const size_t mark = c.scratch_top;
    const SortKey& K = keys[j];
    const MKey mk = to_mkey(K);
    const bool nullable = K.col.validity != nullptr || K.col.dtype == FDB_UTF8;
    const uint32_t* vsel = d_pos;
    uint32_t* nsel = nullptr;
    uint64_t mv = n, mnull = 0;
    if (nullable) {
      // Indices i (into the current order) of the non-NULL and the NULL keys,
      // in order; both counts are read back before either list is used.
      uint64_t* mask = static_cast<uint64_t*>(c.scratch_take(words * 8));
      uint32_t* vidx = static_cast<uint32_t*>(c.scratch_take(n * 4));
      uint32_t* nidx = static_cast<uint32_t*>(c.scratch_take(n * 4));
      uint32_t* vs = static_cast<uint32_t*>(c.scratch_take(n * 4));
      nsel = static_cast<uint32_t*>(c.scratch_take(n * 4));
      uint64_t* cnt = static_cast<uint64_t*>(c.scratch_take(16));
      const unsigned gw = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((words * 64 + 255) / 256,
                                                                             (uint64_t)c.sm_count * 8));
      mkey_null_mask_kernel<<<gw, 256, 0, c.stream>>>(mk, d_list, d_pos, n, false, reinterpret_cast<uint32_t*>(mask));
      op_compact_mask(c, mask, n, vidx, n, cnt);
      mkey_null_mask_kernel<<<gw, 256, 0, c.stream>>>(mk, d_list, d_pos, n, true, reinterpret_cast<uint32_t*>(mask));
      op_compact_mask(c, mask, n, nidx, n, cnt + 1);
      uint64_t hc[2] = {0, 0};
      FDB_CUDA(cudaMemcpyAsync(hc, cnt, 16, cudaMemcpyDeviceToHost, c.stream));
      FDB_CUDA(cudaStreamSynchronize(c.stream));
      if (hc[0] + hc[1] != n) fail(FDB_E_GENERIC, "sort: valid and NULL positions do not add up");
      mv = hc[0];
      mnull = hc[1];
      if (mv) gather_u32_kernel<<<g, 256, 0, c.stream>>>(d_pos, vidx, mv, vs);
      if (mnull) gather_u32_kernel<<<g, 256, 0, c.stream>>>(d_pos, nidx, mnull, nsel);
      vsel = vs;
    }
    if (mv > 0) {
      auto kf = [&](uint64_t* k, uint32_t* v, unsigned long long* vary) {
        const unsigned gk = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((mv + 255) / 256,
                                                                               (uint64_t)c.sm_count * 8));
        mkey_sort_key_kernel<<<gk, 256, 0, c.stream>>>(mk, d_list, vsel, (uint32_t)mv, k, v, vary);
      };
      radix_sort_pairs(c, (uint32_t)mv, kf, d_pos + (K.nulls_last ? 0 : mnull), nullptr, nullptr);
    }
    if (mnull)
      FDB_CUDA(cudaMemcpyAsync(d_pos + (K.nulls_last ? mv : 0), nsel, mnull * 4, cudaMemcpyDeviceToDevice, c.stream));
    FDB_CUDA(cudaGetLastError());
    c.scratch_top = mark;
  }
  (void)m;
}

void op_distinct_multi(Ctx& c, const fdb_dev_column* cols, const uint32_t* const* ranks, const uint32_t* rank_lens,
                       int ncols, const uint32_t* d_list, uint64_t n, uint32_t* d_pos, uint64_t* d_count) {
  if (ncols < 1 || ncols > kMaxMultiKeys) fail(FDB_E_ARG, "DISTINCT over between 1 and 8 columns");
  if (n >= 0xFFFFFFFFull) fail(FDB_E_ARG, "DISTINCT addresses rows as uint32");
  if (n == 0) {
    FDB_CUDA(cudaMemsetAsync(d_count, 0, 8, c.stream));
    return;
  }
  const uint64_t words = (n + 63) / 64;
  c.ensure_scratch(c.scratch_top + sort_multi_scratch(n) + n * 4 + words * 8 + 512);
  uint32_t* order = static_cast<uint32_t*>(c.scratch_take(n * 4));
  unsigned long long* heads = static_cast<unsigned long long*>(c.scratch_take(words * 8));
  SortKey ks[kMaxMultiKeys];
  MKeys mk;
  mk.n = ncols;
  for (int j = 0; j < ncols; ++j) {
    ks[j] = SortKey{};
    ks[j].col = cols[j];
    ks[j].distinct = true;
    if (ranks && ranks[j]) {
      ks[j].rank = ranks[j];
      ks[j].rank_len = rank_lens[j];
    }
    mk.k[j] = to_mkey(ks[j]);
  }
  op_sort_multi(c, ks, ncols, d_list, n, order);
  FDB_CUDA(cudaMemsetAsync(heads, 0, words * 8, c.stream));
  const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)c.sm_count * 8));
  multi_heads_kernel<<<g, 256, 0, c.stream>>>(mk, d_list, order, n, heads);
  FDB_CUDA(cudaGetLastError());
  op_compact_mask(c, reinterpret_cast<const uint64_t*>(heads), n, d_pos, n, d_count);
}

}  // namespace fdb
