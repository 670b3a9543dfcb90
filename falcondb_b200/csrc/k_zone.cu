// Zone maps: the bounds and NULL count of every 65,536-row batch of a column
// (BatchStats::compute / column_stats, src/storage/stats.rs:46-52, 148-260),
// computed once when a table is loaded.  One CTA per batch reads the batch's
// values once (coalesced, eight loads in flight per thread) and reduces them.
#include <cstdint>

#include "common.cuh"
#include "engine.h"

namespace fdb {
namespace {

constexpr int kZoneThreads = 256;
constexpr int kZoneUnroll = 8;

// Per-thread partial of one batch.  INT64 and UTF8 bounds are kept in lo/hi
// as int64; FLOAT64 bounds in flo/fhi (NaN skipped, as f64::min / max do).
struct ZonePart {
  int64_t lo, hi;
  double flo, fhi;
  uint64_t nulls;
  uint32_t flags;
};

__device__ __forceinline__ void part_init(ZonePart& z) {
  z.lo = INT64_MAX;
  z.hi = INT64_MIN;
  z.flo = __longlong_as_double(0x7ff0000000000000ll);   // +inf
  z.fhi = __longlong_as_double((long long)0xfff0000000000000ull);  // -inf
  z.nulls = 0;
  z.flags = 0;
}

__device__ __forceinline__ void part_merge(ZonePart& a, const ZonePart& b) {
  a.lo = min(a.lo, b.lo);
  a.hi = max(a.hi, b.hi);
  a.flo = fmin(a.flo, b.flo);
  a.fhi = fmax(a.fhi, b.fhi);
  a.nulls += b.nulls;
  a.flags |= b.flags;
}

__device__ __forceinline__ ZonePart part_shfl_down(const ZonePart& z, int o) {
  ZonePart r;
  r.lo = __shfl_down_sync(0xffffffffu, z.lo, o);
  r.hi = __shfl_down_sync(0xffffffffu, z.hi, o);
  r.flo = __shfl_down_sync(0xffffffffu, z.flo, o);
  r.fhi = __shfl_down_sync(0xffffffffu, z.fhi, o);
  r.nulls = __shfl_down_sync(0xffffffffu, z.nulls, o);
  r.flags = __shfl_down_sync(0xffffffffu, z.flags, o);
  return r;
}

template <int DT>
__device__ __forceinline__ void part_add(ZonePart& z, const void* values, uint64_t row, bool valid) {
  if (DT == FDB_UTF8) {
    const uint32_t code = static_cast<const uint32_t*>(values)[row];
    if (!valid || code == kNullCode) {
      ++z.nulls;
      return;
    }
    z.lo = min(z.lo, (int64_t)code);
    z.hi = max(z.hi, (int64_t)code);
    z.flags |= FDB_ZONE_VALUES;
  } else if (DT == FDB_INT64) {
    const int64_t v = static_cast<const int64_t*>(values)[row];
    if (!valid) {
      ++z.nulls;
      return;
    }
    z.lo = min(z.lo, v);
    z.hi = max(z.hi, v);
    z.flags |= FDB_ZONE_VALUES;
  } else {
    const double v = static_cast<const double*>(values)[row];
    if (!valid) {
      ++z.nulls;
      return;
    }
    if (isnan(v)) {
      z.flags |= FDB_ZONE_NAN;
      return;
    }
    z.flo = fmin(z.flo, v);
    z.fhi = fmax(z.fhi, v);
    z.flags |= FDB_ZONE_VALUES;
  }
}

template <int DT>
__global__ void __launch_bounds__(kZoneThreads)
    zone_map_kernel(const void* __restrict__ values, const uint64_t* __restrict__ validity, uint64_t n,
                    fdb_zone* __restrict__ out) {
  const uint64_t b = blockIdx.x;
  const uint64_t start = b * kZoneRows;
  const uint64_t end = min(n, start + kZoneRows);
  ZonePart z;
  part_init(z);
  // Row start + threadIdx.x + k * kZoneThreads: a warp reads consecutive rows.
  for (uint64_t r0 = start; r0 < end; r0 += (uint64_t)kZoneThreads * kZoneUnroll) {
#pragma unroll
    for (int u = 0; u < kZoneUnroll; ++u) {
      const uint64_t row = r0 + (uint64_t)u * kZoneThreads + threadIdx.x;
      if (row < end) {
        const bool valid = validity ? ((validity[row >> 6] >> (row & 63)) & 1ull) != 0 : true;
        part_add<DT>(z, values, row, valid);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part_merge(z, part_shfl_down(z, o));
  __shared__ ZonePart warp_part[kZoneThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_part[warp] = z;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kZoneThreads / 32; ++w) part_merge(z, warp_part[w]);
    fdb_zone e;
    e.min_i = (z.flags & FDB_ZONE_VALUES) && DT != FDB_FLOAT64 ? z.lo : 0;
    e.max_i = (z.flags & FDB_ZONE_VALUES) && DT != FDB_FLOAT64 ? z.hi : 0;
    e.min_f = (z.flags & FDB_ZONE_VALUES) && DT == FDB_FLOAT64 ? z.flo : 0.0;
    e.max_f = (z.flags & FDB_ZONE_VALUES) && DT == FDB_FLOAT64 ? z.fhi : 0.0;
    e.null_count = z.nulls;
    e.rows = (uint32_t)(end - start);
    e.flags = z.flags;
    out[b] = e;
  }
}

}  // namespace

void op_zone_map(cudaStream_t s, const Column& col, uint64_t nrows, fdb_zone* d_out) {
  const uint64_t nb = zone_batches(nrows);
  if (nb == 0) return;
  if (nb > 0x7fffffffull) fail(FDB_E_ARG, "zone map: too many batches");
  const uint64_t* validity = static_cast<const uint64_t*>(col.validity.ptr);
  switch (col.dtype) {
    case FDB_INT64:
      zone_map_kernel<FDB_INT64><<<(unsigned)nb, kZoneThreads, 0, s>>>(col.values.ptr, validity, nrows, d_out);
      break;
    case FDB_FLOAT64:
      zone_map_kernel<FDB_FLOAT64><<<(unsigned)nb, kZoneThreads, 0, s>>>(col.values.ptr, validity, nrows, d_out);
      break;
    case FDB_UTF8:
      zone_map_kernel<FDB_UTF8><<<(unsigned)nb, kZoneThreads, 0, s>>>(col.values.ptr, validity, nrows, d_out);
      break;
    default: fail(FDB_E_TYPE, "zone map: unsupported column type");
  }
  FDB_CUDA(cudaGetLastError());
}

}  // namespace fdb
