// Distinct-count estimate of an INT64 key column, for sizing hash tables: a
// HyperLogLog sketch (Flajolet, Fusy, Gandouet, Meunier, "HyperLogLog: the
// analysis of a near-optimal cardinality estimation algorithm", 2007) over all
// keys with 2^12 registers (standard error about 1.6 %).  One pass over the
// keys plus a 16 KB device-to-host copy; synchronises the context stream.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace fdb {

constexpr int kHllBits = 12;
constexpr int kHllRegs = 1 << kHllBits;

__global__ void __launch_bounds__(256) hll_kernel(const int64_t* __restrict__ keys, uint64_t n, unsigned int* regs) {
  __shared__ unsigned int r[kHllRegs];
  for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x) r[i] = 0;
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t h = mix64((uint64_t)__ldcs(keys + i) ^ (1ull << 63));
    const uint32_t idx = (uint32_t)(h >> (64 - kHllBits));
    const uint64_t w = (h << kHllBits) | (1ull << (kHllBits - 1));  // bounds the run of zeros
    atomicMax(&r[idx], (unsigned int)__clzll((long long)w) + 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x)
    if (r[i]) atomicMax(&regs[i], r[i]);
}

uint64_t estimate_distinct_i64(Ctx& c, const void* keys, uint64_t n) {
  if (n <= 4096) return n ? n : 1;
  unsigned int* regs = static_cast<unsigned int*>(c.scratch_take(kHllRegs * 4));
  FDB_CUDA(cudaMemsetAsync(regs, 0, kHllRegs * 4, c.stream));
  const unsigned grid = (unsigned)umin64((n + 255) / 256, (uint64_t)c.sm_count * 4);
  hll_kernel<<<grid, 256, 0, c.stream>>>(static_cast<const int64_t*>(keys), n, regs);
  FDB_CUDA(cudaGetLastError());
  std::vector<unsigned int> h(kHllRegs);
  FDB_CUDA(cudaMemcpyAsync(h.data(), regs, kHllRegs * 4, cudaMemcpyDeviceToHost, c.stream));
  FDB_CUDA(cudaStreamSynchronize(c.stream));
  double z = 0.0;
  int zeros = 0;
  for (unsigned int v : h) {
    z += std::ldexp(1.0, -(int)v);
    zeros += v == 0;
  }
  const double m = kHllRegs, alpha = 0.7213 / (1.0 + 1.079 / m);
  double e = alpha * m * m / z;
  if (e <= 2.5 * m && zeros > 0) e = m * std::log(m / zeros);  // small-range correction
  return std::min<uint64_t>(n, (uint64_t)std::ceil(e));
}

}  // namespace fdb
