// Host-side internals of the engine: the execution context (device, stream,
// scratch arena, deferred device errors), resident tables, and the operator
// launchers that the C ABI and the SQL planner call.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/falcondb_b200.h"
#include "once.h"
#include "tuning.h"
#include "zone.h"

namespace fdb {

// Codes a kernel writes to the context's device error word (read back by
// fdb_synchronize and turned into FDB_E_TIMEOUT / FDB_E_CAPACITY).
constexpr int kDevErrTimeout = 1;
constexpr int kDevErrCapacity = 2;

// Error carried from the engine to the C ABI, which turns it into a return code
// plus the thread-local message.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void fail(int code, const std::string& msg);
void cuda_check(cudaError_t e, const char* what);
#define FDB_CUDA(x) ::fdb::cuda_check((x), #x)

// One device allocation accounted against the context's budget.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

struct Ctx;

// A resident column: dense values in HBM, optional validity words, and for
// FDB_UTF8 the host dictionary (codes are indices into it).
struct Column {
  std::string name;
  int32_t dtype = 0;
  DevBuf values;
  DevBuf validity;              // empty when the column has no NULLs
  std::vector<std::string> dict;
  cudaEvent_t ready = nullptr;  // recorded on the upload stream after the copy
  // Zone map: one fdb_zone per 65,536-row batch, computed on the zone stream
  // once the upload is done; the host copy is fetched on first use.
  DevBuf zones;
  uint64_t nzones = 0;
  cudaEvent_t zones_ready = nullptr;
  std::vector<fdb_zone> zhost;
  bool zhost_valid = false;
};

struct Table {
  std::string name;
  uint64_t nrows = 0;
  std::vector<Column> cols;
  int find(const std::string& n) const;
};

// Per-kernel launch configuration chosen by the autotuner (or its defaults).
struct LaunchCfg {
  int grid = 0;        // CTAs (persistent grid)
  int threads = 0;     // threads per CTA
};

struct Ctx {
  int device = 0;
  int sm_count = 0;
  size_t budget = 0;
  std::atomic<size_t> in_use{0};
  cudaStream_t stream = nullptr;         // operator stream
  cudaStream_t upload = nullptr;         // host->device copies
  cudaStream_t zstream = nullptr;        // zone maps of freshly loaded columns
  bool zone_maps = true;                 // option "zone_maps"
  std::string device_name;               // cudaDeviceProp::name
  TuningSet tune;                        // launch tuning (fdb_set_tuning / autotune / cache)
  std::recursive_mutex mu;               // serialises calls on this context

  // Scratch arena: a device buffer carved per operator call.  The first
  // kTicketBytes hold zeroed counters that kernels reset before they exit.
  static constexpr size_t kTicketBytes = 256;
  DevBuf scratch;
  size_t scratch_top = kTicketBytes;
  int* d_err = nullptr;                  // deferred device error word (in scratch head)
  unsigned int* d_ticket = nullptr;      // last-CTA ticket (in scratch head)

  std::map<std::string, std::shared_ptr<Table>> tables;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_kernel_ms = 0.0;
  uint64_t last_scan_rows = 0;           // rows of the table the last fdb_sql scanned

  ~Ctx();
  void* dev_alloc(size_t bytes);                 // budgeted cudaMalloc
  void dev_free(void* p, size_t bytes);
  DevBuf alloc_buf(size_t bytes);
  void free_buf(DevBuf& b);
  // Scratch for the current operator call (16-byte aligned, grows on demand by
  // synchronising the stream first).  Reset with scratch_reset().
  void* scratch_take(size_t bytes);
  void scratch_reset() { scratch_top = kTicketBytes; }
  void ensure_scratch(size_t bytes);
  int check_device_error();                      // reads and clears d_err (syncs)
};

// Converts the C view to the kernel view.
struct DevColV {
  int32_t dtype;
  const void* values;
  const uint64_t* validity;
  uint64_t voff;
};
inline DevColV to_v(const fdb_dev_column& c) {
  return DevColV{c.dtype, c.values, c.validity, c.validity_offset};
}
int dtype_size(int32_t dtype);

// ---------------------------------------------------------------------------
// Operator launchers (asynchronous on ctx.stream). Implemented in the .cu files.
// ---------------------------------------------------------------------------
void op_filter_mask(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                    const fdb_pred_term* prog, int nterms, uint64_t* d_mask);
void op_filter_count(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                     const fdb_pred_term* prog, int nterms, uint64_t* d_count);
void op_compact_mask(Ctx& c, const uint64_t* d_mask, uint64_t n, uint32_t* d_rows,
                     uint64_t capacity, uint64_t* d_count);
void op_gather(Ctx& c, const fdb_dev_column& col, const uint32_t* d_rows, uint64_t n,
               void* d_out, uint64_t* d_out_validity);
// Gather where a row number of FDB_NO_ROW yields NULL (the right side of an
// unmatched LEFT JOIN row); always writes validity words.
void op_gather_opt(Ctx& c, const fdb_dev_column& col, const uint32_t* d_rows, uint64_t n,
                   void* d_out, uint64_t* d_out_validity);
void op_aggregate(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                  const fdb_pred_term* prog, int nterms, const fdb_agg_spec* aggs, int naggs,
                  fdb_agg_value* d_out);
// op_aggregate's interpreted scan with its partials and ticket in a fixed
// device array instead of the scratch arena: allocates nothing.
void op_aggregate_noalloc(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                          const fdb_pred_term* prog, int nterms, const fdb_agg_spec* aggs, int naggs,
                          fdb_agg_value* d_out);
// Merged text codes of n rows from per-chunk dictionary indices (k_dict.cu):
// chunk c holds rows [chunk_start[c], chunk_start[c+1]) (chunk_start has
// nchunks + 1 entries, the first 0, the last n); row i's index k >= 0 maps to
// remap[remap_off[c] + k], k < 0 to the NULL code.
void op_dict_remap(Ctx& c, const int32_t* d_idx, uint64_t n, const uint64_t* d_chunk_start, uint32_t nchunks,
                   const uint32_t* d_remap, const uint64_t* d_remap_off, uint64_t remap_len, uint32_t* d_codes);
// Test hook of the bounded waits (stream.cuh StreamHook) for the streamed
// scans of k_scan.cu on the current device; tile = ~0 clears it.
void stream_test_stall(Ctx& c, uint64_t tile, uint32_t spin_limit);
void op_distinct_codes(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                       const fdb_pred_term* prog, int nterms, int code_col, uint32_t dict_len,
                       uint64_t* d_bitmap);
void op_group_by_codes(Ctx& c, const fdb_dev_column* cols, int ncols, uint64_t n,
                       const fdb_pred_term* prog, int nterms, int key_col, uint32_t dict_len,
                       const fdb_agg_spec* aggs, int naggs, fdb_agg_value* d_out,
                       int64_t* d_group_rows);
// How an int64-key GROUP BY sizes its table: the groups to expect and, when
// known, the range of the non-NULL keys.  A range that is dense enough makes
// the table direct-addressed (one slot per key value, no hashing or probing).
struct GbSizing {
  uint64_t groups = 0;
  bool has_range = false;
  int64_t kmin = 0, kmax = 0;
};
// `expected_groups` when nonzero (no pass over the keys, no range), else the
// sizing pass over the key column: estimate plus headroom, and the key range
// (synchronises).
GbSizing group_by_i64_sizing(Ctx& c, const fdb_dev_column& key, uint64_t n, uint64_t expected_groups);
// Scratch bytes op_group_by_i64 takes for `s` at `load_factor`.
size_t group_by_i64_scratch(const GbSizing& s, double load_factor);
void op_group_by_i64(Ctx& c, const fdb_dev_column& key, const fdb_dev_column& value, uint64_t n,
                     const fdb_pred_term* prog, int nterms, const fdb_dev_column* pred_cols,
                     int npred, const GbSizing& s, double load_factor,
                     fdb_group_i64* d_groups, uint64_t capacity, uint64_t* d_ngroups);
struct HashTable;  // join build side (k_join.cu)
// Device pointers of a join build table for kernels outside k_join.cu.
struct JoinView {
  const void* slots;         // JSlot[cap + 1]
  const unsigned int* cnt;   // build rows per slot
  uint64_t cap;
  int32_t unique;
  int32_t dense;             // key k lives in slot k - dmin (see join_table.cuh)
  int64_t dmin;              // the smallest build key
  uint64_t span;             // keys outside [dmin, dmin + span) have no slot (0: no range)
};
JoinView join_view(const HashTable* h);

HashTable* hash_of(const fdb_hash* h);  // the build side behind a C handle

// Serving loop (serve.cu).
struct Server;
Server* server_start(fdb_db* db, Ctx& c, const fdb_serve_config* cfg);
uint64_t server_submit(Server& s, const fdb_serve_query& q, double arrival_s);  // arrival_s < 0: now
bool server_wait(Server& s, uint64_t ticket, int64_t timeout_ns, fdb_serve_result* out);  // false: timed out
void server_stop(Server* s, fdb_serve_stats* st);
void serve_trace(fdb_db* db, Ctx& c, const fdb_serve_query* qs, int nq, const fdb_serve_config* cfg,
                 fdb_serve_result* out, fdb_serve_stats* st);

// One sizing pass over an INT64 key column (hll.cu): a HyperLogLog estimate of
// its distinct keys and the range of its non-NULL keys (NULL: a clear validity
// bit, or INT64_MIN).  Synchronises the context stream.
struct KeyStats {
  uint64_t distinct = 0;
  bool has_range = false;  // false when every key is NULL (or there are none)
  int64_t kmin = 0, kmax = 0;
};
KeyStats key_stats_i64(Ctx& c, const fdb_dev_column& key, uint64_t n);

// Zone maps (k_zone.cu, zone.cpp; pruning in zone_prune.cpp).
// Fills d_out[0 .. zone_batches(nrows)) on stream s.
void op_zone_map(cudaStream_t s, const Column& col, uint64_t nrows, fdb_zone* d_out);
// (Re)computes col's zone map on the zone stream after its upload.
void build_zone_map(Ctx& c, Column& col, uint64_t nrows);
void free_column(Ctx& c, Column& col);
// The host copy of col's zone map (waits for it once).
const std::vector<fdb_zone>& column_zones(Ctx& c, Column& col);
// The resident column whose values hold `values` (a view starting at row
// *first_row of it), or nullptr.
Column* column_by_values(Ctx& c, const void* values, uint64_t* table_rows, uint64_t* first_row);
// The estimate alone, over a column without NULLs.
uint64_t estimate_distinct_i64(Ctx& c, const void* keys, uint64_t n);

struct BatchPlan;
BatchPlan* op_gb_batch_prepare(Ctx& c, const fdb_gb_query* qs, int nq, const fdb_batch_tuning* t);
void op_gb_batch_run(BatchPlan* p);
// Launch-shape autotuner of the streamed operators (k_tune.cu): fills
// c.tune.op and best[FDB_TUNE_KINDS]; ms_at_rows may be null.
void op_autotune(Ctx& c, uint64_t rows, int reps, fdb_op_tuning* best, double* ms_at_rows);
void op_gb_batch_free(BatchPlan* p);
double op_gb_batch_autotune(Ctx& c, const fdb_gb_query* qs, int nq, int reps, fdb_batch_tuning* best);
void op_topk(Ctx& c, const fdb_dev_column& col, uint64_t n, uint32_t k, bool desc,
             bool nulls_last, uint32_t* d_rows, uint64_t* d_count);
// Every row of one FLOAT64 / INT64 column in ORDER BY order (k_sort.cu):
// d_rows receives n row numbers.
void op_sort(Ctx& c, const fdb_dev_column& col, uint64_t n, bool desc, bool nulls_last,
             uint32_t* d_rows);
// SELECT DISTINCT over one FLOAT64 / INT64 / UTF8 column (k_sort.cu): the
// positions of each value's first occurrence, ascending; *d_count = how many.
void op_distinct(Ctx& c, const fdb_dev_column& col, uint64_t n, uint32_t* d_rows, uint64_t* d_count);
// op_sort with, when int_as_f64, an INT64 column ordered by its f64 value.
void op_sort_keyed(Ctx& c, const fdb_dev_column& col, uint64_t n, bool desc, bool nulls_last, bool int_as_f64,
                   uint32_t* d_rows);
// One key of a multi-key sort (op_sort_multi).  ORDER BY keys order FLOAT64 /
// INT64 values as the single-key sort does and a UTF8 column by `rank` (the
// rank of each dictionary code in the sorted dictionary, equal strings equal
// ranks; codes at or past rank_len read as NULL); DISTINCT keys only group
// equal values together (a UTF8 DISTINCT key compares ranks when given, else
// codes).
struct SortKey {
  fdb_dev_column col{};
  bool desc = false, nulls_last = false;
  bool distinct = false;
  const uint32_t* rank = nullptr;  // device, rank_len entries
  uint32_t rank_len = 0;
};
// Positions 0..n-1 of a row list (position p is row d_list[p], or row p when
// d_list is null) in the order of keys[0], then keys[1], ..., then position:
// d_pos receives n positions.  Up to 8 keys.
void op_sort_multi(Ctx& c, const SortKey* keys, int nkeys, const uint32_t* d_list, uint64_t n, uint32_t* d_pos);
// Scratch bytes op_sort_multi takes beyond the caller's.
size_t sort_multi_scratch(uint64_t n);
// SELECT DISTINCT over several columns: the positions (ascending) of the first
// occurrence of each distinct row of `cols` over the row list; *d_count = how
// many.  NULLs are one value per column; FLOAT64 compares with every NaN one
// value and -0.0 equal to +0.0; UTF8 compares ranks[j] (rank_lens[j]
// entries) when given, else codes.  ranks may be null.
void op_distinct_multi(Ctx& c, const fdb_dev_column* cols, const uint32_t* const* ranks, const uint32_t* rank_lens,
                       int ncols, const uint32_t* d_list, uint64_t n, uint32_t* d_pos, uint64_t* d_count);
// Join row pairs (d_left[i], d_right[i]) put in (left, right) order in place;
// d_right may be null (left rows only).
void op_sort_row_pairs(Ctx& c, uint32_t* d_left, uint32_t* d_right, uint64_t n);
// d_rn[list[order[j]]] = j + 1 for j < n (order / list null = identity).
void op_row_numbers(Ctx& c, const uint32_t* d_order, const uint32_t* d_list, uint64_t n, int64_t* d_rn);

struct HashTable;  // join build side (k_join.cu)
HashTable* op_join_build(Ctx& c, const fdb_dev_column& key, const fdb_dev_column& payload,
                         uint64_t n, double load_factor);
void join_free(HashTable* h);
uint64_t join_capacity(const HashTable* h);
void op_join_probe_agg(Ctx& c, const HashTable& h, const fdb_dev_column& key,
                       const fdb_dev_column* value, uint64_t n, int join_type,
                       fdb_join_agg* d_out);
void op_join_probe_pairs(Ctx& c, const HashTable& h, const fdb_dev_column& key, uint64_t n,
                         int join_type, uint32_t* d_left, uint32_t* d_right, uint64_t capacity,
                         uint64_t* d_count);

}  // namespace fdb
