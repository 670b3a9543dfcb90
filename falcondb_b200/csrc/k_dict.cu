// Text column codes from per-chunk dictionaries (the Parquet loader's GPU
// dictionary, read_parquet / Utf8 batches, FalconDB
// src/storage/parquet_io.rs:290-500, column.rs:1320-1346).
//
// A Parquet text column arrives as chunks (row groups), each with its own
// dictionary and per-row indices into it.  The host merges the chunk
// dictionaries, which hold distinct strings, not rows, into one dictionary
// and a remap table per chunk; this kernel then turns every row's local index
// into its merged code, so no per-row work is done on the host.
#include <algorithm>

#include "common.cuh"
#include "engine.h"

namespace fdb {

constexpr uint32_t kDictRows = 8192;  // rows per CTA block (one chunk search per block)

__global__ void __launch_bounds__(256)
    dict_remap_kernel(const int32_t* __restrict__ idx, uint64_t n, const uint64_t* __restrict__ chunk_start,
                      uint32_t nchunks, const uint32_t* __restrict__ remap, const uint64_t* __restrict__ remap_off,
                      uint64_t remap_len, uint32_t* __restrict__ codes, int* err) {
  for (uint64_t b0 = (uint64_t)blockIdx.x * kDictRows; b0 < n; b0 += (uint64_t)gridDim.x * kDictRows) {
    // The chunk holding row b0: the last c with chunk_start[c] <= b0.
    uint32_t lo = 0, hi = nchunks;  // chunk_start[0] = 0 <= b0 < chunk_start[nchunks] = n
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (chunk_start[mid] <= b0) lo = mid; else hi = mid;
    }
    uint32_t c = lo;
    const uint64_t end = umin64(n, b0 + kDictRows);
    for (uint64_t i = b0 + threadIdx.x; i < end; i += blockDim.x) {
      while (c + 1 < nchunks && i >= chunk_start[c + 1]) ++c;  // rows only move forward
      const int32_t k = idx[i];
      uint32_t code = kNullCode;
      if (k >= 0) {
        const uint64_t at = remap_off[c] + (uint64_t)k;
        if (at < remap_len && (c + 1 == nchunks || at < remap_off[c + 1])) {
          code = remap[at];
        } else {
          atomicExch(err, kErrCapacity);  // an index past its chunk's dictionary
        }
      }
      codes[i] = code;
    }
  }
}

void op_dict_remap(Ctx& c, const int32_t* d_idx, uint64_t n, const uint64_t* d_chunk_start, uint32_t nchunks,
                   const uint32_t* d_remap, const uint64_t* d_remap_off, uint64_t remap_len, uint32_t* d_codes) {
  if (n == 0) return;
  if (nchunks == 0) fail(FDB_E_ARG, "fdb_dict_remap: no chunks");
  if (!d_idx || !d_chunk_start || !d_remap_off || !d_codes || (remap_len && !d_remap))
    fail(FDB_E_ARG, "fdb_dict_remap: null buffer");
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + kDictRows - 1) / kDictRows,
                                                                           (uint64_t)c.sm_count * 8));
  dict_remap_kernel<<<grid, 256, 0, c.stream>>>(d_idx, n, d_chunk_start, nchunks, d_remap, d_remap_off, remap_len,
                                                d_codes, c.d_err);
  FDB_CUDA(cudaGetLastError());
}

}  // namespace fdb
