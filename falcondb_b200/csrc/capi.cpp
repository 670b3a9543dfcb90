// The C ABI (include/falcondb_b200.h): context lifecycle, resident tables,
// result accessors and the operator layer.  Every entry point catches engine
// errors, stores the message in a thread-local string and returns a code, in
// the manner of FalconDB's c_ffi.rs (src/api/c_ffi.rs:27-144).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <sstream>

#include "../../include/falcondb_b200.h"
#include "engine.h"
#include "result.h"

struct fdb_db {
  fdb::Ctx ctx;
};
struct fdb_hash {
  fdb::HashTable* h = nullptr;
  fdb_db* db = nullptr;
};
struct fdb_server {
  fdb::Server* s = nullptr;
  fdb_db* db = nullptr;
};
struct fdb_batch {
  fdb::BatchPlan* plan = nullptr;
  fdb_db* db = nullptr;
};

namespace fdb {
HashTable* hash_of(const fdb_hash* h) {
  if (!h || !h->h) fail(FDB_E_ARG, "null join table");
  return h->h;
}

static thread_local std::string g_last_error;

void fail(int code, const std::string& msg) { throw Error(code, msg); }

void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  const int code = (e == cudaErrorMemoryAllocation) ? FDB_E_OOM : FDB_E_CUDA;
  throw Error(code, std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
                        ") in " + what);
}

int dtype_size(int32_t dtype) { return dtype == FDB_UTF8 ? 4 : 8; }

int Table::find(const std::string& n) const {
  for (size_t i = 0; i < cols.size(); ++i)
    if (cols[i].name == n) return (int)i;
  return -1;
}

Ctx::~Ctx() {
  tables.clear();
  if (scratch.ptr) cudaFree(scratch.ptr);
  if (d_err) cudaFree(d_err);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (stream) cudaStreamDestroy(stream);
  if (upload) cudaStreamDestroy(upload);
  if (zstream) cudaStreamDestroy(zstream);
}

// Device memory comes from the device's stream-ordered pool (cudaMallocAsync on
// the context stream, release threshold raised at open): allocating and freeing
// per query costs no device synchronisation and reuses cached blocks.
void* Ctx::dev_alloc(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (in_use.load() + bytes > budget)
    fail(FDB_E_OOM, "device memory budget exceeded: " + std::to_string(in_use.load() + bytes) + " > " +
                        std::to_string(budget) + " bytes");
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(FDB_E_OOM, std::string("cudaMallocAsync failed: ") + cudaGetErrorString(e));
  }
  in_use += bytes;
  return p;
}
void Ctx::dev_free(void* p, size_t bytes) {
  if (!p) return;
  cudaFreeAsync(p, stream);  // ordered after every operator already queued
  in_use -= bytes ? bytes : 16;
}
DevBuf Ctx::alloc_buf(size_t bytes) {
  DevBuf b;
  b.ptr = dev_alloc(bytes);
  b.bytes = bytes ? bytes : 16;
  return b;
}
void Ctx::free_buf(DevBuf& b) {
  dev_free(b.ptr, b.bytes);
  b.ptr = nullptr;
  b.bytes = 0;
}

void Ctx::ensure_scratch(size_t bytes) {
  if (scratch.bytes >= bytes) return;
  // The old arena is released in stream order (after the work that uses it).
  size_t want = std::max(bytes, scratch.bytes * 2);
  want = (want + (1u << 20) - 1) & ~size_t((1u << 20) - 1);
  if (scratch.ptr) free_buf(scratch);
  scratch = alloc_buf(want);
}

void* Ctx::scratch_take(size_t bytes) {
  const size_t aligned = (bytes + 255) & ~size_t(255);
  if (scratch_top + aligned > scratch.bytes)
    fail(FDB_E_OOM, "operator scratch exceeds the reserved arena (" + std::to_string(scratch.bytes) +
                        " bytes); reserve more before the call");
  void* p = static_cast<char*>(scratch.ptr) + scratch_top;
  scratch_top += aligned;
  return p;
}

int Ctx::check_device_error() {
  FDB_CUDA(cudaStreamSynchronize(stream));
  int e = 0;
  FDB_CUDA(cudaMemcpy(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    // Clear the error word and the ticket so the context stays usable.
    FDB_CUDA(cudaMemset(d_err, 0, kTicketBytes));
    return e == kDevErrTimeout ? FDB_E_TIMEOUT : FDB_E_CAPACITY;
  }
  return 0;
}

}  // namespace fdb

using namespace fdb;

namespace {

int set_error(int code, const std::string& msg) {
  fdb::g_last_error = msg;
  return code;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    fdb::g_last_error.clear();
    return FDB_OK;
  } catch (const Error& e) {
    return set_error(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return set_error(FDB_E_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_error(FDB_E_GENERIC, e.what());
  } catch (...) {
    return set_error(FDB_E_GENERIC, "unknown error");
  }
}

// Lock, make the context's device current, and reserve scratch for one call.
struct CallScope {
  std::lock_guard<std::recursive_mutex> lk;
  Ctx& c;
  CallScope(fdb_db* db, size_t scratch_bytes) : lk(db->ctx.mu), c(db->ctx) {
    FDB_CUDA(cudaSetDevice(c.device));
    c.scratch_reset();
    c.ensure_scratch(scratch_bytes);
  }
};

size_t default_scratch(Ctx&) { return (size_t)64 << 20; }

void need(bool ok, const char* msg) {
  if (!ok) fail(FDB_E_ARG, msg);
}

}  // namespace

extern "C" {

const char* fdb_version(void) { return "falcondb_b200 0.1.0 (sm_100a)"; }

const char* fdb_last_error(void) { return fdb::g_last_error.c_str(); }

int fdb_open(int device, uint64_t mem_budget_bytes, fdb_db** out) {
  if (!out) return set_error(FDB_E_ARG, "fdb_open: out is NULL");
  *out = nullptr;
  std::unique_ptr<fdb_db> db(new fdb_db());
  const int rc = guarded([&] {
    Ctx& c = db->ctx;
    int ndev = 0;
    FDB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) fail(FDB_E_ARG, "fdb_open: no such CUDA device");
    c.device = device;
    FDB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    FDB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) fail(FDB_E_CUDA, "fdb_open: this build targets sm_100a (B200)");
    c.sm_count = prop.multiProcessorCount;
    c.device_name = prop.name;
    size_t free_b = 0, total_b = 0;
    FDB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    c.budget = mem_budget_bytes ? (size_t)mem_budget_bytes : (size_t)(free_b * 0.9);
    FDB_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    FDB_CUDA(cudaStreamCreateWithFlags(&c.upload, cudaStreamNonBlocking));
    FDB_CUDA(cudaStreamCreateWithFlags(&c.zstream, cudaStreamNonBlocking));
    // Keep freed pool blocks cached in this process (the pool belongs to this
    // process's context; nothing outlives it).
    cudaMemPool_t pool;
    FDB_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t threshold = UINT64_MAX;
    FDB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    FDB_CUDA(cudaEventCreate(&c.ev0));
    FDB_CUDA(cudaEventCreate(&c.ev1));
    c.d_err = static_cast<int*>(c.dev_alloc(Ctx::kTicketBytes));
    FDB_CUDA(cudaMemsetAsync(c.d_err, 0, Ctx::kTicketBytes, c.stream));
    FDB_CUDA(cudaStreamSynchronize(c.stream));
    c.d_ticket = reinterpret_cast<unsigned int*>(reinterpret_cast<char*>(c.d_err) + 64);
    c.ensure_scratch(default_scratch(c));
  });
  if (rc == FDB_OK) *out = db.release();
  return rc;
}

void fdb_close(fdb_db* db) {
  if (!db) return;
  cudaSetDevice(db->ctx.device);
  cudaStreamSynchronize(db->ctx.stream);
  cudaStreamSynchronize(db->ctx.upload);
  cudaStreamSynchronize(db->ctx.zstream);
  {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    for (auto& kv : db->ctx.tables)
      for (auto& col : kv.second->cols) free_column(db->ctx, col);
    db->ctx.tables.clear();
  }
  delete db;
}

int64_t fdb_table_from_columns(fdb_db* db, const char* name, const fdb_column* cols, int32_t ncols,
                               uint64_t nrows) {
  if (!db || !name || (!cols && ncols > 0) || ncols < 0)
    return set_error(FDB_E_ARG, "fdb_table_from_columns: bad arguments");
  int rc = guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    Ctx& c = db->ctx;
    FDB_CUDA(cudaSetDevice(c.device));
    // Same name, row count and column layout as a resident table: overwrite its
    // device buffers in place (no free/allocate), once every operator already
    // queued on the context stream has read them.
    {
      auto it = c.tables.find(name);
      bool same = it != c.tables.end() && it->second->nrows == nrows && (int)it->second->cols.size() == ncols;
      for (int i = 0; same && i < ncols; ++i) {
        const Column& old = it->second->cols[i];
        same = cols[i].name && old.name == cols[i].name && old.dtype == cols[i].dtype &&
               (old.validity.ptr != nullptr) == (cols[i].validity != nullptr) &&
               (nrows == 0 || cols[i].values != nullptr);
      }
      if (same) {
        cudaEvent_t done;
        FDB_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        FDB_CUDA(cudaEventRecord(done, c.stream));
        FDB_CUDA(cudaStreamWaitEvent(c.upload, done, 0));
        FDB_CUDA(cudaEventDestroy(done));
        for (int i = 0; i < ncols; ++i) {
          Column& col = it->second->cols[i];
          const fdb_column& hc = cols[i];
          const size_t vbytes = nrows * dtype_size(hc.dtype);
          if (vbytes)
            FDB_CUDA(cudaMemcpyAsync(col.values.ptr, hc.values, vbytes, cudaMemcpyDefault, c.upload));
          if (hc.validity && nrows)
            FDB_CUDA(cudaMemcpyAsync(col.validity.ptr, hc.validity, ((nrows + 63) / 64) * 8,
                                     cudaMemcpyDefault, c.upload));
          if (hc.dtype == FDB_UTF8) {
            col.dict.clear();
            for (uint32_t d = 0; d < hc.dict_len; ++d) col.dict.emplace_back(hc.dict[d] ? hc.dict[d] : "");
          }
          FDB_CUDA(cudaEventRecord(col.ready, c.upload));
          build_zone_map(c, col, nrows);
        }
        return;
      }
    }
    auto t = std::make_shared<Table>();
    t->name = name;
    t->nrows = nrows;
    try {
      for (int i = 0; i < ncols; ++i) {
        const fdb_column& hc = cols[i];
        need(hc.name != nullptr, "column without a name");
        need(hc.dtype == FDB_INT64 || hc.dtype == FDB_FLOAT64 || hc.dtype == FDB_UTF8,
             "unsupported column type");
        need(nrows == 0 || hc.values != nullptr, "column without values");
        for (auto& prev : t->cols)
          if (prev.name == hc.name) fail(FDB_E_ARG, std::string("duplicate column ") + hc.name);
        Column col;
        col.name = hc.name;
        col.dtype = hc.dtype;
        const size_t vbytes = nrows * dtype_size(hc.dtype);
        const size_t wbytes = ((nrows + 63) / 64) * 8;
        col.values = c.alloc_buf(vbytes);
        if (hc.validity) col.validity = c.alloc_buf(wbytes);
        // The buffers come from the pool in the context stream's order; the
        // upload stream waits for that before copying into them.
        FDB_CUDA(cudaEventCreateWithFlags(&col.ready, cudaEventDisableTiming));
        FDB_CUDA(cudaEventRecord(col.ready, c.stream));
        FDB_CUDA(cudaStreamWaitEvent(c.upload, col.ready, 0));
        if (vbytes) FDB_CUDA(cudaMemcpyAsync(col.values.ptr, hc.values, vbytes, cudaMemcpyDefault, c.upload));
        if (hc.validity && wbytes)
          FDB_CUDA(cudaMemcpyAsync(col.validity.ptr, hc.validity, wbytes, cudaMemcpyDefault, c.upload));
        if (hc.dtype == FDB_UTF8) {
          need(hc.dict != nullptr || hc.dict_len == 0, "Utf8 column without a dictionary");
          for (uint32_t d = 0; d < hc.dict_len; ++d) col.dict.emplace_back(hc.dict[d] ? hc.dict[d] : "");
        }
        FDB_CUDA(cudaEventRecord(col.ready, c.upload));
        t->cols.push_back(std::move(col));
        build_zone_map(c, t->cols.back(), nrows);
      }
    } catch (...) {
      for (auto& col : t->cols) free_column(c, col);
      throw;
    }
    auto it = c.tables.find(name);
    if (it != c.tables.end()) {
      FDB_CUDA(cudaStreamSynchronize(c.stream));
      for (auto& col : it->second->cols) free_column(c, col);
      c.tables.erase(it);
    }
    c.tables[name] = t;
  });
  return rc == FDB_OK ? (int64_t)nrows : (int64_t)rc;
}

uint64_t fdb_table_row_count(const fdb_db* db, const char* name) {
  if (!db || !name) return 0;
  auto& c = const_cast<fdb_db*>(db)->ctx;
  std::lock_guard<std::recursive_mutex> lk(c.mu);
  auto it = c.tables.find(name);
  return it == c.tables.end() ? 0 : it->second->nrows;
}

int fdb_table_drop(fdb_db* db, const char* name) {
  if (!db || !name) return set_error(FDB_E_ARG, "fdb_table_drop: bad arguments");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    Ctx& c = db->ctx;
    auto it = c.tables.find(name);
    if (it == c.tables.end()) fail(FDB_E_NOTFOUND, std::string("no table ") + name);
    FDB_CUDA(cudaSetDevice(c.device));
    FDB_CUDA(cudaStreamSynchronize(c.stream));
    for (auto& col : it->second->cols) free_column(c, col);
    c.tables.erase(it);
  });
}

int fdb_table_column(const fdb_db* db, const char* table, const char* column, fdb_dev_column* out,
                     uint64_t* nrows) {
  if (!db || !table || !column || !out) return set_error(FDB_E_ARG, "fdb_table_column: bad arguments");
  fdb_db* d = const_cast<fdb_db*>(db);
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(d->ctx.mu);
    auto it = d->ctx.tables.find(table);
    if (it == d->ctx.tables.end()) fail(FDB_E_NOTFOUND, std::string("no table ") + table);
    const int ci = it->second->find(column);
    if (ci < 0) fail(FDB_E_NOTFOUND, std::string("no column ") + column);
    const Column& col = it->second->cols[ci];
    // Later operators on the context stream see the uploaded values.
    FDB_CUDA(cudaSetDevice(d->ctx.device));
    FDB_CUDA(cudaStreamWaitEvent(d->ctx.stream, col.ready, 0));
    out->dtype = col.dtype;
    out->_pad = 0;
    out->values = col.values.ptr;
    out->validity = static_cast<const uint64_t*>(col.validity.ptr);
    out->validity_offset = 0;
    if (nrows) *nrows = it->second->nrows;
  });
}

int fdb_table_zone_map(fdb_db* db, const char* table, const char* column, fdb_zone* out, uint64_t cap,
                       uint64_t* nbatches) {
  if (!db || !table || !column || (cap && !out)) return set_error(FDB_E_ARG, "fdb_table_zone_map: bad arguments");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    Ctx& c = db->ctx;
    FDB_CUDA(cudaSetDevice(c.device));
    auto it = c.tables.find(table);
    if (it == c.tables.end()) fail(FDB_E_NOTFOUND, std::string("no table ") + table);
    const int ci = it->second->find(column);
    if (ci < 0) fail(FDB_E_NOTFOUND, std::string("no column ") + column);
    const std::vector<fdb_zone>& z = column_zones(c, it->second->cols[ci]);
    if (nbatches) *nbatches = z.size();
    const uint64_t m = std::min<uint64_t>(cap, z.size());
    if (m) std::memcpy(out, z.data(), m * sizeof(fdb_zone));
  });
}

int fdb_zone_skip(fdb_db* db, const char* table, const char* const* cols, int32_t ncols, const fdb_pred_term* prog,
                  int32_t nterms, uint64_t* skip, uint64_t words, uint64_t* nbatches) {
  if (!db || !table || ncols < 0 || (ncols && !cols) || nterms < 0 || (nterms && !prog) || (words && !skip))
    return set_error(FDB_E_ARG, "fdb_zone_skip: bad arguments");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    Ctx& c = db->ctx;
    FDB_CUDA(cudaSetDevice(c.device));
    auto it = c.tables.find(table);
    if (it == c.tables.end()) fail(FDB_E_NOTFOUND, std::string("no table ") + table);
    Table& t = *it->second;
    std::vector<const std::vector<fdb_zone>*> zones;
    std::vector<int32_t> dtypes;
    for (int i = 0; i < ncols; ++i) {
      const int ci = cols[i] ? t.find(cols[i]) : -1;
      if (ci < 0) fail(FDB_E_NOTFOUND, std::string("no column ") + (cols[i] ? cols[i] : "(null)"));
      zones.push_back(&column_zones(c, t.cols[ci]));
      dtypes.push_back(t.cols[ci].dtype);
    }
    // Host copies of the CODE_SET bitmaps.
    std::vector<std::vector<uint64_t>> sets((size_t)nterms);
    for (int i = 0; i < nterms; ++i)
      if (prog[i].kind == FDB_TERM_CODE_SET && prog[i].code_set && prog[i].lit_i > 0) {
        sets[(size_t)i].resize(((uint64_t)prog[i].lit_i + 63) / 64);
        FDB_CUDA(cudaMemcpyAsync(sets[(size_t)i].data(), prog[i].code_set, sets[(size_t)i].size() * 8,
                                 cudaMemcpyDeviceToHost, c.stream));
      }
    FDB_CUDA(cudaStreamSynchronize(c.stream));
    const uint64_t nb = zone_batches(t.nrows);
    if (nbatches) *nbatches = nb;
    const std::vector<uint8_t> out = zone_rule_out(zones, dtypes, prog, nterms, sets, nb);
    if (words) std::memset(skip, 0, words * 8);
    for (uint64_t b = 0; b < nb && (b >> 6) < words; ++b)
      if (out[b]) skip[b >> 6] |= 1ull << (b & 63);
  });
}

int fdb_set_option(fdb_db* db, const char* name, int64_t value) {
  if (!db || !name) return set_error(FDB_E_ARG, "fdb_set_option: bad arguments");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    if (std::strcmp(name, "zone_maps") == 0) {
      db->ctx.zone_maps = value != 0;
      return;
    }
    fail(FDB_E_ARG, std::string("unknown option ") + name);
  });
}

int fdb_sql(fdb_db* db, const char* sql, fdb_result** out) {
  if (out) *out = nullptr;
  if (!db || !sql || !out) return set_error(FDB_E_ARG, "fdb_sql: bad arguments");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    FDB_CUDA(cudaSetDevice(db->ctx.device));
    *out = fdb::run_sql(db->ctx, sql);
  });
}

uint64_t fdb_result_row_count(const fdb_result* r) { return r ? r->rows : 0; }
int32_t fdb_result_num_columns(const fdb_result* r) { return r ? (int32_t)r->cols.size() : 0; }
const char* fdb_result_column_name(const fdb_result* r, int32_t col) {
  if (!r || col < 0 || col >= (int32_t)r->cols.size()) return nullptr;
  return r->cols[col].name.c_str();
}
int32_t fdb_result_column_dtype(const fdb_result* r, int32_t col) {
  if (!r || col < 0 || col >= (int32_t)r->cols.size()) return 0;
  return r->cols[col].dtype;
}
const void* fdb_result_column_values(const fdb_result* r, int32_t col) {
  if (!r || col < 0 || col >= (int32_t)r->cols.size()) return nullptr;
  const auto& c = r->cols[col];
  if (c.dtype == FDB_INT64) return c.i64.data();
  if (c.dtype == FDB_FLOAT64) return c.f64.data();
  return c.str_ptrs.data();
}
const uint8_t* fdb_result_column_nulls(const fdb_result* r, int32_t col) {
  if (!r || col < 0 || col >= (int32_t)r->cols.size()) return nullptr;
  const auto& c = r->cols[col];
  return c.has_nulls() ? c.nulls.data() : nullptr;
}
const char* fdb_result_display(fdb_result* r) { return r ? r->display_text().c_str() : nullptr; }
void fdb_result_free(fdb_result* r) { delete r; }

double fdb_last_kernel_ms(const fdb_db* db) { return db ? db->ctx.last_kernel_ms : 0.0; }
uint64_t fdb_last_scan_rows(const fdb_db* db) { return db ? db->ctx.last_scan_rows : 0; }

int fdb_memory_stats(fdb_db* db, fdb_mem_stats* out) {
  if (!db || !out) return set_error(FDB_E_ARG, "fdb_memory_stats: bad arguments");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    Ctx& c = db->ctx;
    FDB_CUDA(cudaSetDevice(c.device));
    out->in_use = c.in_use.load();
    out->budget = c.budget;
    out->scratch = c.scratch.bytes;
    cudaMemPool_t pool;
    FDB_CUDA(cudaDeviceGetDefaultMemPool(&pool, c.device));
    unsigned long long v = 0;  // the attribute value type (cuuint64_t)
    FDB_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v));
    out->pool_reserved = v;
    FDB_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &v));
    out->pool_used = v;
  });
}

void* fdb_stream(fdb_db* db) { return db ? (void*)db->ctx.stream : nullptr; }

int fdb_synchronize(fdb_db* db) {
  if (!db) return set_error(FDB_E_ARG, "fdb_synchronize: db is NULL");
  int dev_err = 0;
  const int rc = guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    FDB_CUDA(cudaSetDevice(db->ctx.device));
    FDB_CUDA(cudaStreamSynchronize(db->ctx.upload));
    dev_err = db->ctx.check_device_error();
  });
  if (rc != FDB_OK) return rc;
  if (dev_err) return set_error(dev_err, dev_err == FDB_E_TIMEOUT ? "a device-side wait timed out"
                                                                  : "an output buffer was too small");
  return FDB_OK;
}

// ----------------------------- operator layer ------------------------------

int fdb_filter_mask(fdb_db* db, const fdb_dev_column* cols, int32_t ncols, uint64_t nrows,
                    const fdb_pred_term* prog, int32_t nterms, uint64_t* d_mask) {
  if (!db || !cols || !d_mask || (nterms && !prog)) return set_error(FDB_E_ARG, "fdb_filter_mask: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_filter_mask(s.c, cols, ncols, nrows, prog, nterms, d_mask);
  });
}

int fdb_filter_count(fdb_db* db, const fdb_dev_column* cols, int32_t ncols, uint64_t nrows,
                     const fdb_pred_term* prog, int32_t nterms, uint64_t* d_count) {
  if (!db || !cols || !d_count || (nterms && !prog)) return set_error(FDB_E_ARG, "fdb_filter_count: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_filter_count(s.c, cols, ncols, nrows, prog, nterms, d_count);
  });
}

int fdb_compact_mask(fdb_db* db, const uint64_t* d_mask, uint64_t nrows, uint32_t* d_rows, uint64_t capacity,
                     uint64_t* d_count) {
  if (!db || (!d_mask && nrows) || !d_count || (!d_rows && capacity))
    return set_error(FDB_E_ARG, "fdb_compact_mask: bad arguments");
  if (nrows >= 0xFFFFFFFFull) return set_error(FDB_E_ARG, "fdb_compact_mask: rows are uint32");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_compact_mask(s.c, d_mask, nrows, d_rows, capacity, d_count);
  });
}

int fdb_gather(fdb_db* db, const fdb_dev_column* col, const uint32_t* d_rows, uint64_t n, void* d_out_values,
               uint64_t* d_out_validity) {
  if (!db || !col || (n && (!d_rows || !d_out_values))) return set_error(FDB_E_ARG, "fdb_gather: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_gather(s.c, *col, d_rows, n, d_out_values, d_out_validity);
  });
}

int fdb_aggregate(fdb_db* db, const fdb_dev_column* cols, int32_t ncols, uint64_t nrows,
                  const fdb_pred_term* prog, int32_t nterms, const fdb_agg_spec* aggs, int32_t naggs,
                  fdb_agg_value* d_out) {
  if (!db || !cols || !aggs || !d_out || (nterms && !prog)) return set_error(FDB_E_ARG, "fdb_aggregate: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_aggregate(s.c, cols, ncols, nrows, prog, nterms, aggs, naggs, d_out);
  });
}

int fdb_aggregate_noalloc(fdb_db* db, const fdb_dev_column* cols, int32_t ncols, uint64_t nrows,
                          const fdb_pred_term* prog, int32_t nterms, const fdb_agg_spec* aggs, int32_t naggs,
                          fdb_agg_value* d_out) {
  if (!db || !cols || !aggs || !d_out || (nterms && !prog))
    return set_error(FDB_E_ARG, "fdb_aggregate_noalloc: bad arguments");
  return guarded([&] {
    // No CallScope: it resets and may grow the scratch arena.
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    FDB_CUDA(cudaSetDevice(db->ctx.device));
    op_aggregate_noalloc(db->ctx, cols, ncols, nrows, prog, nterms, aggs, naggs, d_out);
  });
}

int fdb_dict_remap(fdb_db* db, const int32_t* d_idx, uint64_t nrows, const uint64_t* d_chunk_start,
                   uint32_t nchunks, const uint32_t* d_remap, const uint64_t* d_remap_off, uint64_t remap_len,
                   uint32_t* d_codes) {
  if (!db) return set_error(FDB_E_ARG, "fdb_dict_remap: db is NULL");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_dict_remap(s.c, d_idx, nrows, d_chunk_start, nchunks, d_remap, d_remap_off, remap_len, d_codes);
  });
}

int fdb_test_stall(fdb_db* db, uint64_t tile, uint32_t spin_limit) {
  if (!db) return set_error(FDB_E_ARG, "fdb_test_stall: db is NULL");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    FDB_CUDA(cudaSetDevice(db->ctx.device));
    stream_test_stall(db->ctx, tile, spin_limit);
  });
}

int fdb_distinct_codes(fdb_db* db, const fdb_dev_column* cols, int32_t ncols, uint64_t nrows,
                       const fdb_pred_term* prog, int32_t nterms, int32_t code_col, uint32_t dict_len,
                       uint64_t* d_bitmap) {
  if (!db || !cols || (!d_bitmap && dict_len) || (nterms && !prog))
    return set_error(FDB_E_ARG, "fdb_distinct_codes: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_distinct_codes(s.c, cols, ncols, nrows, prog, nterms, code_col, dict_len, d_bitmap);
  });
}

int fdb_group_by_codes(fdb_db* db, const fdb_dev_column* cols, int32_t ncols, uint64_t nrows,
                       const fdb_pred_term* prog, int32_t nterms, int32_t key_col, uint32_t dict_len,
                       const fdb_agg_spec* aggs, int32_t naggs, fdb_agg_value* d_out, int64_t* d_group_rows) {
  if (!db || !cols || !aggs || !d_out || !d_group_rows || (nterms && !prog))
    return set_error(FDB_E_ARG, "fdb_group_by_codes: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_group_by_codes(s.c, cols, ncols, nrows, prog, nterms, key_col, dict_len, aggs, naggs, d_out,
                      d_group_rows);
  });
}

int fdb_group_by_i64(fdb_db* db, const fdb_dev_column* key, const fdb_dev_column* value, uint64_t nrows,
                     const fdb_pred_term* prog, int32_t nterms, const fdb_dev_column* pred_cols,
                     int32_t npred_cols, uint64_t expected_groups, double load_factor, fdb_group_i64* d_groups,
                     uint64_t capacity, uint64_t* d_ngroups) {
  if (!db || !key || !value || !d_ngroups || (!d_groups && capacity) || (nterms && !prog) ||
      (npred_cols && !pred_cols))
    return set_error(FDB_E_ARG, "fdb_group_by_i64: bad arguments");
  return guarded([&] {
    Ctx& c = db->ctx;
    double lf = (load_factor > 0.0 && load_factor < 1.0) ? load_factor : 0.5;
    CallScope s(db, default_scratch(c));
    const GbSizing sz = group_by_i64_sizing(s.c, *key, nrows, expected_groups);
    s.c.scratch_reset();
    s.c.ensure_scratch(group_by_i64_scratch(sz, lf) + (16u << 20));
    op_group_by_i64(s.c, *key, *value, nrows, prog, nterms, pred_cols, npred_cols, sz, lf, d_groups, capacity,
                    d_ngroups);
  });
}

int fdb_join_build(fdb_db* db, const fdb_dev_column* key, const fdb_dev_column* payload, uint64_t nrows,
                   double load_factor, fdb_hash** out) {
  if (out) *out = nullptr;
  if (!db || !key || !out) return set_error(FDB_E_ARG, "fdb_join_build: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    fdb_dev_column none;
    std::memset(&none, 0, sizeof(none));
    HashTable* h = op_join_build(s.c, *key, payload ? *payload : none, nrows, load_factor);
    fdb_hash* fh = new fdb_hash();
    fh->h = h;
    fh->db = db;
    *out = fh;
  });
}

void fdb_join_free(fdb_hash* h) {
  if (!h) return;
  {
    std::lock_guard<std::recursive_mutex> lk(h->db->ctx.mu);
    cudaSetDevice(h->db->ctx.device);
    cudaStreamSynchronize(h->db->ctx.stream);
    join_free(h->h);
  }
  delete h;
}

uint64_t fdb_join_capacity(const fdb_hash* h) { return h ? join_capacity(h->h) : 0; }
int fdb_join_dense(const fdb_hash* h) { return h ? join_view(h->h).dense : 0; }

int fdb_join_probe_agg(fdb_db* db, const fdb_hash* h, const fdb_dev_column* probe_key, const fdb_dev_column* value,
                       uint64_t nrows, int32_t join_type, fdb_join_agg* d_out) {
  if (!db || !h || !probe_key || !d_out) return set_error(FDB_E_ARG, "fdb_join_probe_agg: bad arguments");
  if (h->db != db) return set_error(FDB_E_ARG, "fdb_join_probe_agg: hash table belongs to another context");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_join_probe_agg(s.c, *h->h, *probe_key, value, nrows, join_type, d_out);
  });
}

int fdb_join_probe_pairs(fdb_db* db, const fdb_hash* h, const fdb_dev_column* probe_key, uint64_t nrows,
                         int32_t join_type, uint32_t* d_left, uint32_t* d_right, uint64_t capacity,
                         uint64_t* d_count) {
  if (!db || !h || !probe_key || !d_count || (capacity && !d_left))
    return set_error(FDB_E_ARG, "fdb_join_probe_pairs: bad arguments");
  if (h->db != db) return set_error(FDB_E_ARG, "fdb_join_probe_pairs: hash table belongs to another context");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_join_probe_pairs(s.c, *h->h, *probe_key, nrows, join_type, d_left, d_right, capacity, d_count);
  });
}

int fdb_topk(fdb_db* db, const fdb_dev_column* col, uint64_t nrows, uint32_t k, int32_t desc, int32_t nulls_last,
             uint32_t* d_rows, uint64_t* d_count) {
  if (!db || !col || !d_rows || !d_count) return set_error(FDB_E_ARG, "fdb_topk: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_topk(s.c, *col, nrows, k, desc != 0, nulls_last != 0, d_rows, d_count);
  });
}

int fdb_sort(fdb_db* db, const fdb_dev_column* col, uint64_t nrows, int32_t desc, int32_t nulls_last,
             uint32_t* d_rows) {
  if (!db || !col || (!d_rows && nrows)) return set_error(FDB_E_ARG, "fdb_sort: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_sort(s.c, *col, nrows, desc != 0, nulls_last != 0, d_rows);
  });
}

int fdb_distinct(fdb_db* db, const fdb_dev_column* col, uint64_t nrows, uint32_t* d_rows, uint64_t* d_count) {
  if (!db || !col || !d_count || (!d_rows && nrows)) return set_error(FDB_E_ARG, "fdb_distinct: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_distinct(s.c, *col, nrows, d_rows, d_count);
  });
}

int fdb_gb_batch_prepare(fdb_db* db, const fdb_gb_query* queries, int32_t nqueries, const fdb_batch_tuning* tuning,
                         fdb_batch** out) {
  if (out) *out = nullptr;
  if (!db || !queries || !out) return set_error(FDB_E_ARG, "fdb_gb_batch_prepare: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    std::unique_ptr<fdb_batch> b(new fdb_batch());
    b->db = db;
    b->plan = op_gb_batch_prepare(s.c, queries, nqueries, tuning ? tuning : &s.c.tune.batch);
    *out = b.release();
  });
}

int fdb_gb_batch_run(fdb_batch* b) {
  if (!b || !b->plan) return set_error(FDB_E_ARG, "fdb_gb_batch_run: bad batch");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(b->db->ctx.mu);
    FDB_CUDA(cudaSetDevice(b->db->ctx.device));
    op_gb_batch_run(b->plan);
  });
}

void fdb_gb_batch_free(fdb_batch* b) {
  if (!b) return;
  guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(b->db->ctx.mu);
    FDB_CUDA(cudaSetDevice(b->db->ctx.device));
    op_gb_batch_free(b->plan);
  });
  delete b;
}

int fdb_gb_batch_autotune(fdb_db* db, const fdb_gb_query* queries, int32_t nqueries, int32_t reps,
                          fdb_batch_tuning* best, double* best_ms) {
  if (!db || !queries || !best) return set_error(FDB_E_ARG, "fdb_gb_batch_autotune: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    const double ms = op_gb_batch_autotune(s.c, queries, nqueries, reps, best);
    s.c.tune.batch = *best;
    if (best_ms) *best_ms = ms;
  });
}

int fdb_get_tuning(fdb_db* db, int32_t kind, fdb_op_tuning* out) {
  if (!db || !out || kind < 0 || kind >= FDB_TUNE_KINDS) return set_error(FDB_E_ARG, "fdb_get_tuning: bad arguments");
  std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
  const OpTuning& t = db->ctx.tune.op[kind];
  out->ctas_per_sm = t.ctas_per_sm;
  out->_pad = 0;
  out->min_rows_per_cta = t.min_rows_per_cta;
  return FDB_OK;
}

int fdb_set_tuning(fdb_db* db, int32_t kind, const fdb_op_tuning* in) {
  if (!db || !in || kind < 0 || kind >= FDB_TUNE_KINDS || in->ctas_per_sm < 0 || in->ctas_per_sm > 64)
    return set_error(FDB_E_ARG, "fdb_set_tuning: bad arguments");
  std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
  db->ctx.tune.op[kind].ctas_per_sm = in->ctas_per_sm;
  db->ctx.tune.op[kind].min_rows_per_cta = in->min_rows_per_cta;
  return FDB_OK;
}

int fdb_autotune_ops(fdb_db* db, uint64_t rows, int32_t reps, fdb_op_tuning* best, double* ms_per_call) {
  if (!db) return set_error(FDB_E_ARG, "fdb_autotune_ops: bad arguments");
  return guarded([&] {
    CallScope s(db, default_scratch(db->ctx));
    op_autotune(s.c, rows, reps, best, ms_per_call);
  });
}

int fdb_tuning_save(fdb_db* db, const char* path) {
  if (!db || !path) return set_error(FDB_E_ARG, "fdb_tuning_save: bad arguments");
  return guarded([&] {
    std::string text;
    {
      std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
      text = tuning_to_json(db->ctx.tune, db->ctx.device_name, db->ctx.sm_count);
    }
    std::FILE* f = std::fopen(path, "wb");
    if (!f) fail(FDB_E_ARG, std::string("cannot write ") + path);
    const size_t w = std::fwrite(text.data(), 1, text.size(), f);
    const int closed = std::fclose(f);
    if (w != text.size() || closed != 0) fail(FDB_E_GENERIC, std::string("short write to ") + path);
  });
}

int fdb_tuning_load(fdb_db* db, const char* path) {
  if (!db || !path) return set_error(FDB_E_ARG, "fdb_tuning_load: bad arguments");
  return guarded([&] {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) fail(FDB_E_NOTFOUND, std::string("cannot read ") + path);
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0 && text.size() < (1u << 20)) text.append(buf, got);
    std::fclose(f);
    TuningSet t;
    std::string device;
    int sms = 0;
    const std::string err = tuning_from_json(text, &t, &device, &sms);
    if (!err.empty()) fail(FDB_E_ARG, std::string(path) + ": " + err);
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    if (device != db->ctx.device_name || sms != db->ctx.sm_count)
      fail(FDB_E_ARG, std::string(path) + " was tuned on " + device + " (" + std::to_string(sms) + " SMs), not " +
                          db->ctx.device_name + " (" + std::to_string(db->ctx.sm_count) + " SMs)");
    db->ctx.tune = t;
  });
}

int fdb_server_start(fdb_db* db, const fdb_serve_config* cfg, fdb_server** out) {
  if (out) *out = nullptr;
  if (!db || !out) return set_error(FDB_E_ARG, "fdb_server_start: bad arguments");
  return guarded([&] {
    std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
    FDB_CUDA(cudaSetDevice(db->ctx.device));
    std::unique_ptr<fdb_server> h(new fdb_server());
    h->db = db;
    h->s = server_start(db, db->ctx, cfg);
    *out = h.release();
  });
}

int fdb_server_submit(fdb_server* s, const fdb_serve_query* q, uint64_t* ticket) {
  if (!s || !q || !ticket) return set_error(FDB_E_ARG, "fdb_server_submit: bad arguments");
  return guarded([&] { *ticket = server_submit(*s->s, *q, -1.0); });
}

int fdb_server_wait(fdb_server* s, uint64_t ticket, int64_t timeout_ns, fdb_serve_result* out) {
  if (!s) return set_error(FDB_E_ARG, "fdb_server_wait: bad arguments");
  bool ok = false;
  const int rc = guarded([&] { ok = server_wait(*s->s, ticket, timeout_ns, out); });
  if (rc < 0) return rc;
  return ok ? FDB_OK : set_error(FDB_E_TIMEOUT, "fdb_server_wait: not answered yet");
}

int fdb_server_stop(fdb_server* s, fdb_serve_stats* stats) {
  if (!s) return set_error(FDB_E_ARG, "fdb_server_stop: bad arguments");
  const int rc = guarded([&] { server_stop(s->s, stats); });
  delete s;
  return rc;
}

int fdb_serve_trace(fdb_db* db, const fdb_serve_query* queries, int32_t nqueries, const fdb_serve_config* cfg,
                    fdb_serve_result* out, fdb_serve_stats* stats) {
  if (!db || (nqueries && !queries)) return set_error(FDB_E_ARG, "fdb_serve_trace: bad arguments");
  return guarded([&] {
    {
      std::lock_guard<std::recursive_mutex> lk(db->ctx.mu);
      FDB_CUDA(cudaSetDevice(db->ctx.device));
      FDB_CUDA(cudaStreamSynchronize(db->ctx.stream));  // tables and hash tables are built
    }
    serve_trace(db, db->ctx, queries, nqueries, cfg, out, stats);
  });
}

}  // extern "C"
