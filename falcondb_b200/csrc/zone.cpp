// Zone maps on the host side: building them when a column is loaded, their
// host copy, and finding the column a device view belongs to.
#include <cstring>

#include "engine.h"

namespace fdb {

void build_zone_map(Ctx& c, Column& col, uint64_t nrows) {
  const uint64_t nb = zone_batches(nrows);
  col.zhost.clear();
  col.zhost_valid = false;
  if (!col.zones_ready) FDB_CUDA(cudaEventCreateWithFlags(&col.zones_ready, cudaEventDisableTiming));
  if (col.zones.bytes < nb * sizeof(fdb_zone)) {
    c.free_buf(col.zones);
    col.zones = c.alloc_buf(nb * sizeof(fdb_zone));
  }
  col.nzones = nb;
  // After the buffer's allocation (ordered on the context stream) and the
  // upload (col.ready), on a stream of its own so that the next column's copy
  // is not held up behind it.
  FDB_CUDA(cudaEventRecord(col.zones_ready, c.stream));
  FDB_CUDA(cudaStreamWaitEvent(c.zstream, col.zones_ready, 0));
  FDB_CUDA(cudaStreamWaitEvent(c.zstream, col.ready, 0));
  op_zone_map(c.zstream, col, nrows, static_cast<fdb_zone*>(col.zones.ptr));
  FDB_CUDA(cudaEventRecord(col.zones_ready, c.zstream));
}

void free_column(Ctx& c, Column& col) {
  // The buffers go back to the pool in the context stream's order, after the
  // zone map kernel that reads them.
  if (col.zones_ready) cudaStreamWaitEvent(c.stream, col.zones_ready, 0);
  c.free_buf(col.values);
  c.free_buf(col.validity);
  c.free_buf(col.zones);
  if (col.ready) cudaEventDestroy(col.ready);
  if (col.zones_ready) cudaEventDestroy(col.zones_ready);
  col.ready = nullptr;
  col.zones_ready = nullptr;
  col.zhost.clear();
  col.zhost_valid = false;
  col.nzones = 0;
}

const std::vector<fdb_zone>& column_zones(Ctx& c, Column& col) {
  if (!col.zhost_valid) {
    const size_t nb = col.zones.ptr ? col.nzones : 0;
    col.zhost.assign(nb, fdb_zone{});
    if (nb) {
      FDB_CUDA(cudaEventSynchronize(col.zones_ready));
      FDB_CUDA(cudaMemcpy(col.zhost.data(), col.zones.ptr, nb * sizeof(fdb_zone), cudaMemcpyDeviceToHost));
    }
    col.zhost_valid = true;
  }
  return col.zhost;
}

Column* column_by_values(Ctx& c, const void* values, uint64_t* table_rows, uint64_t* first_row) {
  if (!values) return nullptr;
  const uintptr_t p = reinterpret_cast<uintptr_t>(values);
  for (auto& kv : c.tables)
    for (Column& col : kv.second->cols) {
      const uintptr_t base = reinterpret_cast<uintptr_t>(col.values.ptr);
      const uint64_t width = (uint64_t)dtype_size(col.dtype);
      const uint64_t rows = kv.second->nrows;
      if (!base || p < base || p >= base + rows * width || (p - base) % width) continue;
      *table_rows = rows;
      *first_row = (p - base) / width;
      return &col;
    }
  return nullptr;
}

}  // namespace fdb
