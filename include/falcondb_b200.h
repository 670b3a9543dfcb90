/*
 * falcondb_b200.h — C ABI of the B200 execution engine for FalconDB's relational
 * hot path: scan, filter, aggregate, GROUP BY, hash join, ORDER BY (top-k and
 * full sort) and SELECT DISTINCT.
 *
 * Two layers, both plain C (opaque handles, pointers and sizes; no C++ or torch
 * types cross this boundary):
 *
 *  1. Database layer — mirrors FalconDB's C FFI (src/api/c_ffi.rs:27-144) and its
 *     `Database::sql` entry point (src/db.rs:242).  Tables are copied from host
 *     columns into HBM once and stay resident; `fdb_sql` plans and runs a query on
 *     the GPU and returns a host-side result owned by the library.
 *
 *  2. Operator layer — one entry point per CPU physical operator routine that
 *     FalconDB's planner calls (src/db.rs:1439-1717), taking DEVICE pointers and
 *     writing DEVICE results on the context's CUDA stream without a host sync, so
 *     a GPU operator is a drop-in for the matching CPU plan node.
 *
 * Conventions (kept from c_ffi.rs): 0 = success; a negative FDB_E* code on error
 * (-1 is the generic error, as in c_ffi.rs); a thread-local message is returned by
 * fdb_last_error().  Results are owned by the library until *_free.  No C++
 * exception crosses the ABI.  A context (fdb_db) owns one CUDA stream and its
 * scratch memory; calls on one context are serialised by the library, so several
 * host threads may share it, and independent contexts run concurrently.
 *
 * Row numbers on the operator layer are uint32 (as FalconDB's typed paths use
 * u32 row ids, src/query/join.rs:1394-1415, sort.rs:209-215); a single call
 * covers fewer than 2^32 rows.
 */
#ifndef FALCONDB_B200_H
#define FALCONDB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Error codes                                                                */
/* ------------------------------------------------------------------------- */
#define FDB_OK            0
#define FDB_E_GENERIC    -1   /* c_ffi.rs returns -1 / NULL on every error     */
#define FDB_E_ARG        -2   /* invalid argument (NULL handle, bad enum, ...) */
#define FDB_E_CUDA       -3   /* CUDA runtime error                           */
#define FDB_E_OOM        -4   /* device memory budget or allocation exceeded  */
#define FDB_E_SQL        -5   /* SQL text outside the supported shapes        */
#define FDB_E_NOTFOUND   -6   /* unknown table / column                       */
#define FDB_E_TYPE       -7   /* type mismatch (e.g. join keys of two types)  */
#define FDB_E_TIMEOUT    -8   /* a bounded device-side wait gave up           */
#define FDB_E_CAPACITY   -9   /* an output buffer was too small               */

/* Column physical types (src/storage/column.rs:8-21).  FDB_UTF8 columns are
 * dictionary encoded: uint32 codes per row, a host dictionary of strings, and
 * code 0xFFFFFFFF meaning NULL (column.rs:1257-1277). */
#define FDB_INT64    1
#define FDB_FLOAT64  2
#define FDB_UTF8     3

/* Comparison operators of `col op literal` (src/query/expr.rs:1076-1175).
 * Floating comparisons are IEEE ordered (NaN fails) except NE, which is
 * unordered (NaN passes), as cmp_f64_avx2 (expr.rs:894-899) does. */
#define FDB_EQ 0
#define FDB_NE 1
#define FDB_LT 2
#define FDB_LE 3
#define FDB_GT 4
#define FDB_GE 5

/* Aggregate functions (src/query/aggregate.rs:33-47). Result types follow
 * build_agg_col (aggregate.rs:3390-3420): COUNT* -> int64, others -> float64. */
#define FDB_AGG_COUNT_STAR      0   /* COUNT(*): rows that pass the filter     */
#define FDB_AGG_COUNT           1   /* COUNT(col): non-NULL values             */
#define FDB_AGG_SUM             2
#define FDB_AGG_AVG             3
#define FDB_AGG_MIN             4   /* NaN ignored, as f64::min does            */
#define FDB_AGG_MAX             5
#define FDB_AGG_COUNT_DISTINCT  6   /* FDB_UTF8 columns on the operator layer   */

/* Join types (src/query/join.rs:29-41). SEMI/ANTI return left columns only
 * (join.rs:45-48). */
#define FDB_JOIN_INNER 0
#define FDB_JOIN_LEFT  1
#define FDB_JOIN_SEMI  2
#define FDB_JOIN_ANTI  3

/* "No matching build row" marker in emitted join pairs (join.rs NO_ROW). */
#define FDB_NO_ROW 0xFFFFFFFFu

/* ------------------------------------------------------------------------- */
/* Opaque handles                                                             */
/* ------------------------------------------------------------------------- */
typedef struct fdb_db     fdb_db;      /* context: device, stream, scratch, catalog */
typedef struct fdb_result fdb_result;  /* host-side query result                    */
typedef struct fdb_hash   fdb_hash;    /* resident join build side (IntHashTable)   */

/* Host column handed to fdb_table_from_columns (copied into HBM). */
typedef struct fdb_column {
    const char*        name;
    int32_t            dtype;      /* FDB_INT64 | FDB_FLOAT64 | FDB_UTF8            */
    const void*        values;     /* int64[n] | double[n] | uint32 codes[n]        */
    const uint64_t*    validity;   /* LSB-first bit per row, 1 = valid; may be NULL */
    const char* const* dict;       /* FDB_UTF8 only: dict_len strings               */
    uint32_t           dict_len;
} fdb_column;

/* Device column view used by the operator layer.  `values` points at row 0 of
 * the view; validity bit i of the view is bit (validity_offset + i). */
typedef struct fdb_dev_column {
    int32_t         dtype;
    int32_t         _pad;
    const void*     values;            /* device pointer                          */
    const uint64_t* validity;          /* device pointer or NULL                  */
    uint64_t        validity_offset;
} fdb_dev_column;

/* One term of a WHERE predicate, in postfix order (expr.rs:635-808).
 * A program of CMP/IS_NULL/IS_NOT_NULL/CODE_SET leaves and AND/OR nodes; an
 * empty program selects every row. NULL values fail every leaf except IS_NULL. */
#define FDB_TERM_CMP          0  /* cols[col] op literal                           */
#define FDB_TERM_IS_NULL      1  /* validity bit clear, or the Utf8 NULL code       */
#define FDB_TERM_IS_NOT_NULL  2
#define FDB_TERM_CODE_SET     3  /* FDB_UTF8: code < lit_i (the dictionary length)
                                    and bit `code` of code_set (device) is set;
                                    how Utf8 comparisons, IN and LIKE are decided
                                    once per dictionary entry (expr.rs:1143-1171) */
#define FDB_TERM_AND          4
#define FDB_TERM_OR           5
#define FDB_MAX_TERMS        16

typedef struct fdb_pred_term {
    int32_t         kind;
    int32_t         col;
    int32_t         op;        /* FDB_EQ..FDB_GE for FDB_TERM_CMP                 */
    int32_t         lit_type;  /* FDB_INT64 | FDB_FLOAT64                         */
    int64_t         lit_i;
    double          lit_f;
    const uint64_t* code_set;  /* device bitmap over dictionary codes             */
} fdb_pred_term;

typedef struct fdb_agg_spec {
    int32_t func;              /* FDB_AGG_*                                       */
    int32_t col;               /* input column index; ignored for COUNT(*)        */
} fdb_agg_spec;

/* One aggregate result, written to device memory by the operator layer.
 * int64 results (COUNT*) are in `i`; float64 results in `f`; `valid` = 0 means
 * SQL NULL (SUM/AVG/MIN/MAX over no non-NULL rows, aggregate.rs:420-440). */
typedef struct fdb_agg_value {
    double  f;
    int64_t i;
    int64_t n;                 /* rows that contributed                            */
    int32_t is_int;            /* 1: result is int64 (`i`), 0: float64 (`f`)       */
    int32_t valid;
} fdb_agg_value;

/* Join aggregate result (device): COUNT(*) and SUM(payload) for INNER/LEFT;
 * COUNT(*) and SUM(value) of the kept left rows for SEMI/ANTI. */
typedef struct fdb_join_agg {
    int64_t count;
    int64_t sum_payload;       /* exact int64 sum of matched non-NULL payloads     */
    double  sum_value;         /* FP64 sum of the left `value` column (SEMI/ANTI)  */
    int64_t payload_rows;      /* non-NULL payloads summed (SUM NULL when 0)        */
} fdb_join_agg;

/* One output group of the int64-key hash GROUP BY (aggregate.rs:840-912). */
typedef struct fdb_group_i64 {
    int64_t key;
    int64_t count;
    double  sum;
    double  min;
    double  max;
} fdb_group_i64;

/* ------------------------------------------------------------------------- */
/* 1. Database layer  (c_ffi.rs:27-144, db.rs:242)                            */
/* ------------------------------------------------------------------------- */

/* Open a context on CUDA device `device`.  mem_budget_bytes caps the device
 * memory the context may hold (tables, hash tables, scratch); 0 = 90% of free.
 * Replaces falcondb_open (c_ffi.rs:27-30). */
int  fdb_open(int device, uint64_t mem_budget_bytes, fdb_db** out);

/* Replaces falcondb_close (c_ffi.rs:32-37). Frees every device allocation. */
void fdb_close(fdb_db* db);

/* Thread-local message of the last failed call on this thread ("" if none).
 * c_ffi.rs exports no message; this adds one without changing return codes. */
const char* fdb_last_error(void);

/* Create (or replace) table `name` from host columns; the values are copied to
 * HBM (asynchronously on an upload stream when `host` buffers are pinned) and the
 * library owns the device copy.  A values or validity pointer may also be device
 * memory on the context's device (e.g. fdb_dict_remap's output), copied device
 * to device after the work already queued on the context's stream.  Replaces the loaders falcondb_load_csv /
 * falcondb_load_fdb (c_ffi.rs:41-79) and Database::create_table_from_batches
 * (db.rs:180-204) for in-memory columns. Returns rows loaded or a negative code. */
int64_t fdb_table_from_columns(fdb_db* db, const char* name, const fdb_column* cols,
                               int32_t ncols, uint64_t nrows);

/* Rows of table `name`, or 0 if absent (falcondb_table_row_count, c_ffi.rs:131-144). */
uint64_t fdb_table_row_count(const fdb_db* db, const char* name);

/* Drop table `name` and free its device memory. */
int  fdb_table_drop(fdb_db* db, const char* name);

/* Device view of a resident column, for the operator layer. */
int  fdb_table_column(const fdb_db* db, const char* table, const char* column,
                      fdb_dev_column* out, uint64_t* nrows);

/* Zone maps (src/storage/stats.rs:22-52): the bounds and NULL count of every
 * 65,536-row batch of a column (Table::DEFAULT_BATCH_SIZE, table.rs:339),
 * computed on the GPU when the table is loaded, as Table::append_batch and
 * append_batches compute BatchStats (table.rs:373, 391-404).
 *   FDB_INT64  : min_i / max_i, exact (the reference goes through f64).
 *   FDB_FLOAT64: min_f / max_f over the non-NaN values (f64::min / max skip
 *                NaN); FDB_ZONE_NAN when the batch holds a NaN.
 *   FDB_UTF8   : min_i / max_i = the smallest and largest dictionary code.
 * FDB_ZONE_VALUES is set when the batch holds a non-NULL (for FLOAT64 a
 * non-NULL, non-NaN) value; the bounds are meaningful only then. */
#define FDB_ZONE_BATCH_ROWS 65536
#define FDB_ZONE_VALUES     1
#define FDB_ZONE_NAN        2
typedef struct fdb_zone {
    int64_t  min_i, max_i;
    double   min_f, max_f;
    uint64_t null_count;
    uint32_t rows;
    uint32_t flags;
} fdb_zone;

/* Copy the zone map of table.column into out[0 .. min(cap, batches)); the
 * batch count goes to *nbatches.  out may be NULL with cap 0. */
int  fdb_table_zone_map(fdb_db* db, const char* table, const char* column, fdb_zone* out,
                        uint64_t cap, uint64_t* nbatches);

/* The batches of `table` that a WHERE program cannot select, from the zone
 * maps alone (BatchStats::can_skip, stats.rs:57-113): bit b of skip (LSB
 * first, ceil(batches / 64) words) is set when no row of batch b can pass.
 * cols[i] names the table column that the program's column i refers to;
 * CODE_SET bitmaps are device pointers, as for the operators.  Pruning is
 * conservative and never changes a result: a CMP leaf rules a batch out when
 * its bounds exclude the literal (compared exactly for INT64 against an INT64
 * literal, in float64 otherwise, as the filter compares), IS NULL when the
 * batch has no NULL, IS NOT NULL when it is all NULL, CODE_SET when no code in
 * the batch's code range is in the set; AND rules out when either side does,
 * OR when both do.  NE on FLOAT64 never rules out a batch holding a NaN
 * (NaN != x is true), which the reference's rule (stats.rs:110) misses. */
int  fdb_zone_skip(fdb_db* db, const char* table, const char* const* cols, int32_t ncols,
                   const fdb_pred_term* prog, int32_t nterms, uint64_t* skip, uint64_t words,
                   uint64_t* nbatches);

/* Context options.  "zone_maps" (default 1): fdb_sql scans only the batches
 * from the first to the last one that zone maps cannot rule out, and an
 * int64-key GROUP BY over a resident column takes its key range from the
 * column's zone maps instead of a pass over the keys.  0 turns both off. */
int  fdb_set_option(fdb_db* db, const char* name, int64_t value);

/* Execute SQL (falcondb_sql, c_ffi.rs:86-99 -> Database::sql, db.rs:242-316).
 * *out is NULL on error.  Supported shapes (others fail with FDB_E_SQL):
 *   SELECT [DISTINCT] items FROM t [[INNER] | LEFT [OUTER] JOIN u ON t.k = u.k] [WHERE pred]
 *          [GROUP BY col] [ORDER BY col|alias|n [ASC|DESC] [NULLS FIRST|LAST], ...] [LIMIT n]
 *   items: *, col, COUNT(*), COUNT(col), COUNT(DISTINCT col), SUM/AVG/MIN/MAX(col),
 *          ROW_NUMBER() OVER ([ORDER BY col [ASC|DESC]]) [AS a]
 *   pred : col op literal, IS [NOT] NULL, [NOT] IN (...), [NOT] LIKE (Utf8), AND, OR,
 *          parentheses, and [NOT] EXISTS (SELECT ... FROM u WHERE u.k = t.k).
 * ORDER BY runs on the GPU: one FLOAT64 / INT64 key through fdb_topk (LIMIT <= 4096)
 * or fdb_sort; several keys, or a UTF8 key (by the rank of its string), through one
 * stable radix pass per key, last key first.  DISTINCT compares whole rows on the GPU
 * and runs after ORDER BY and LIMIT, as the reference does (db.rs:1699-1729).  With a
 * WHERE on one table, only the batches from the first to the last one that the zone
 * maps cannot rule out are scanned (execute_select, select.rs:105-160). */
int  fdb_sql(fdb_db* db, const char* sql, fdb_result** out);

/* Result accessors (c_ffi.rs:103-127). */
uint64_t    fdb_result_row_count(const fdb_result* r);
int32_t     fdb_result_num_columns(const fdb_result* r);
const char* fdb_result_column_name(const fdb_result* r, int32_t col);
int32_t     fdb_result_column_dtype(const fdb_result* r, int32_t col);
/* int64[rows] / double[rows] / const char*[rows] (FDB_UTF8); valid until free. */
const void* fdb_result_column_values(const fdb_result* r, int32_t col);
/* uint8 per row, 1 = NULL; NULL pointer when the column has no NULLs. */
const uint8_t* fdb_result_column_nulls(const fdb_result* r, int32_t col);
/* Pretty-printed table, valid until the result is freed (c_ffi.rs:108-121). */
const char* fdb_result_display(fdb_result* r);
void        fdb_result_free(fdb_result* r);

/* Device time of the kernels of the last fdb_sql on this context, in ms. */
double      fdb_last_kernel_ms(const fdb_db* db);
/* Rows of its table that the last single-table fdb_sql scanned, after zone-map
 * pruning (the table's row count when nothing was pruned). */
uint64_t    fdb_last_scan_rows(const fdb_db* db);

/* Device memory the context holds, for monitoring (no counterpart in the
 * reference, whose memory is the host heap).  in_use: bytes counted against
 * the context's budget (resident tables, join tables, the operator scratch
 * arena); budget: that cap; scratch: the arena's current size; pool_reserved /
 * pool_used: cudaMemPoolAttrReservedMemCurrent / UsedMemCurrent of the
 * device's default pool, which the context allocates from and which other
 * users of that pool in the process share. */
typedef struct fdb_mem_stats {
    uint64_t in_use;
    uint64_t budget;
    uint64_t scratch;
    uint64_t pool_reserved;
    uint64_t pool_used;
} fdb_mem_stats;
int         fdb_memory_stats(fdb_db* db, fdb_mem_stats* out);

/* ------------------------------------------------------------------------- */
/* 2. Operator layer (device pointers; asynchronous on the context's stream) */
/* ------------------------------------------------------------------------- */

/* The context's CUDA stream (a cudaStream_t), for events and synchronisation. */
void* fdb_stream(fdb_db* db);
/* Block until every operator queued on the context has finished; returns the
 * first deferred device-side error (e.g. FDB_E_TIMEOUT) if one was recorded. */
int   fdb_synchronize(fdb_db* db);

/* WHERE mask: packed uint64 words, bit i of word i/64 = row i passes; bits past
 * nrows are zero.  Replaces Expr::eval_mask_bits / fast_cmp_mask
 * (expr.rs:635-652, 1076-1175) and clear_null_bits / mask_off_padding
 * (expr.rs:961-986). d_mask holds ceil(nrows/64) words. */
int fdb_filter_mask(fdb_db* db, const fdb_dev_column* cols, int32_t ncols,
                    uint64_t nrows, const fdb_pred_term* prog, int32_t nterms,
                    uint64_t* d_mask);

/* COUNT(*) WHERE pred without materialising the mask: replaces the popcount fast
 * path of execute_plan (db.rs:1439-1476). */
int fdb_filter_count(fdb_db* db, const fdb_dev_column* cols, int32_t ncols,
                     uint64_t nrows, const fdb_pred_term* prog, int32_t nterms,
                     uint64_t* d_count);

/* Stable selection compaction: the row numbers of the set bits of d_mask in
 * ascending order, and their count.  Replaces gather_by_bitmask's row walk
 * (column.rs:1077-1123, table.rs:148-189). d_rows holds `capacity` entries;
 * FDB_E_CAPACITY (deferred to fdb_synchronize) if more rows pass. */
int fdb_compact_mask(fdb_db* db, const uint64_t* d_mask, uint64_t nrows,
                     uint32_t* d_rows, uint64_t capacity, uint64_t* d_count);

/* Gather rows `d_rows[0..n)` of a column (values and validity) into a dense
 * device column (Column::gather_u32, column.rs:1502-1520). d_out_validity may be
 * NULL when the input has no validity. */
int fdb_gather(fdb_db* db, const fdb_dev_column* col, const uint32_t* d_rows,
               uint64_t n, void* d_out_values, uint64_t* d_out_validity);

/* No-key aggregates over the rows that pass `prog` (execute_agg_only +
 * accumulate_typed, aggregate.rs:1394-1528, 3121-3386).  FLOAT64 SUM/AVG are
 * FP64 with a fixed reduction tree (deterministic for a given device); INT64 SUM
 * is exact.  COUNT_DISTINCT is answered by fdb_distinct_codes. */
int fdb_aggregate(fdb_db* db, const fdb_dev_column* cols, int32_t ncols,
                  uint64_t nrows, const fdb_pred_term* prog, int32_t nterms,
                  const fdb_agg_spec* aggs, int32_t naggs, fdb_agg_value* d_out);

/* fdb_aggregate for callers that must not allocate device memory.  No
 * counterpart in the reference: FalconDB's CPU aggregates allocate freely.
 * Same arguments, semantics and results as fdb_aggregate (always through its
 * general interpreted kernel), but the per-CTA partials and the completion
 * ticket live in a fixed 128 KB module-scope device array rather than in the
 * context's scratch arena, and the call makes no cudaMalloc / cudaFree /
 * pool allocation.  Returns FDB_E_CAPACITY if the device's SM count needs
 * more partials than the array holds.  The first call on each device looks the
 * array's address up (cudaGetSymbolAddress); make that first call before any
 * stream capture.  Every call on one device uses the same array: calls whose
 * kernels can overlap in time (other streams, other contexts on the device,
 * other threads) race and must be serialised by the caller. */
int fdb_aggregate_noalloc(fdb_db* db, const fdb_dev_column* cols, int32_t ncols,
                          uint64_t nrows, const fdb_pred_term* prog, int32_t nterms,
                          const fdb_agg_spec* aggs, int32_t naggs, fdb_agg_value* d_out);

/* Merged dictionary codes of a text column read in chunks (a Parquet file's
 * row groups, each with its own dictionary; read_parquet, parquet_io.rs:290-500,
 * with per-batch dictionaries, column.rs:1320-1346).  Device pointers:
 * d_idx[nrows] holds each row's index into its chunk's dictionary (negative =
 * NULL); chunk c covers rows [d_chunk_start[c], d_chunk_start[c+1])
 * (nchunks + 1 entries, 0 first, nrows last); d_remap[d_remap_off[c] + k] is the
 * merged code of entry k of chunk c's dictionary (remap_len entries in all).
 * Writes d_codes[nrows] (NULL rows: 0xFFFFFFFF), ready to be the values of an
 * FDB_UTF8 column (fdb_table_from_columns accepts device buffers).  An index
 * past its chunk's dictionary is reported as FDB_E_CAPACITY at the next
 * fdb_synchronize.  Asynchronous on the context's stream. */
int fdb_dict_remap(fdb_db* db, const int32_t* d_idx, uint64_t nrows, const uint64_t* d_chunk_start,
                   uint32_t nchunks, const uint32_t* d_remap, const uint64_t* d_remap_off, uint64_t remap_len,
                   uint32_t* d_codes);

/* Test hook for the device-side bounded waits (no counterpart in the
 * reference, which has no device).  After this call, the streamed scans of
 * fdb_aggregate / fdb_filter_count / fdb_aggregate_noalloc on this context's
 * device stop staging input before tile `tile` (a tile is a few thousand rows),
 * so the CTA that processes it finds its wait for the tile unanswered; the wait
 * gives up after `spin_limit` polls (0 = the normal bound), the kernel records
 * a time-out and ends, and the next fdb_synchronize returns FDB_E_TIMEOUT.
 * Results of calls made while the hook is set are meaningless.  tile =
 * UINT64_MAX clears the hook; the context stays usable throughout. */
int fdb_test_stall(fdb_db* db, uint64_t tile, uint32_t spin_limit);

/* Presence bitmap of the dictionary codes that occur among rows passing `prog`
 * (present_codes, aggregate.rs:3167-3200): d_bitmap holds ceil(dict_len/64)
 * words.  COUNT(DISTINCT) is the number of distinct strings whose code is set. */
int fdb_distinct_codes(fdb_db* db, const fdb_dev_column* cols, int32_t ncols,
                       uint64_t nrows, const fdb_pred_term* prog, int32_t nterms,
                       int32_t code_col, uint32_t dict_len, uint64_t* d_bitmap);

/* Dictionary-code GROUP BY (fast_utf8_gb, aggregate.rs:619-836), with value
 * semantics: group g is dictionary code g, group dict_len is the NULL key.
 * d_out[g*naggs + a] is aggregate a of group g; d_group_rows[g] counts the rows
 * of group g that passed the filter (0 = group absent).  Both arrays hold
 * (dict_len+1) groups.  Requires (dict_len+1) * slots <= 2048, where an
 * aggregate takes 2 slots for AVG and 1 otherwise, plus 1 for the row count. */
int fdb_group_by_codes(fdb_db* db, const fdb_dev_column* cols, int32_t ncols,
                       uint64_t nrows, const fdb_pred_term* prog, int32_t nterms,
                       int32_t key_col, uint32_t dict_len,
                       const fdb_agg_spec* aggs, int32_t naggs,
                       fdb_agg_value* d_out, int64_t* d_group_rows);

/* int64-key hash GROUP BY with COUNT(*), SUM, MIN and MAX of one float64 or
 * int64 value column (fast_i64_gb, aggregate.rs:840-912).  NULL keys (and
 * i64::MIN, which fast_i64_gb reads as NULL, aggregate.rs:867) form one group
 * reported with key INT64_MIN.  Groups are written to d_groups (order
 * unspecified) and their number to d_ngroups; `capacity` bounds d_groups
 * (FDB_E_CAPACITY, deferred, if exceeded).  expected_groups sizes the table
 * (0 = nrows); load_factor in (0,1) (0 = autotuned). */
int fdb_group_by_i64(fdb_db* db, const fdb_dev_column* key, const fdb_dev_column* value,
                     uint64_t nrows, const fdb_pred_term* prog, int32_t nterms,
                     const fdb_dev_column* pred_cols, int32_t npred_cols,
                     uint64_t expected_groups, double load_factor,
                     fdb_group_i64* d_groups, uint64_t capacity, uint64_t* d_ngroups);

/* Build side of an int64 equi-join (build_hash_table + IntHashTable,
 * join.rs:607-645, 1054-1351): open addressing with linear probing over
 * next_pow2(rows / load_factor) slots (load_factor 0 = autotuned).  NULL keys
 * are never inserted (they match nothing, join.rs:637).  The table keeps
 * device pointers to `payload`, which must stay alive while it is used. */
int fdb_join_build(fdb_db* db, const fdb_dev_column* key, const fdb_dev_column* payload,
                   uint64_t nrows, double load_factor, fdb_hash** out);
void fdb_join_free(fdb_hash* h);
uint64_t fdb_join_capacity(const fdb_hash* h);
/* 1 when the table is direct-addressed: its build keys span fewer values than
 * it has slots, so key k lives in slot k - min(key) and a probe reads one slot;
 * 0 when keys are hashed with linear probing.  No counterpart in the reference
 * (its IntHashTable always hashes, join.rs:1368-1429); results are the same. */
int fdb_join_dense(const fdb_hash* h);

/* Probe with aggregation fused in (probe_in_place / probe_one + execute_agg_only,
 * join.rs:297-375, 657-723; execute_hash_semi_anti_join, join.rs:49-132):
 *   INNER: count = matched pairs, sum_payload = SUM(payload) over them;
 *   LEFT : count = matched pairs + unmatched left rows, sum_payload as INNER;
 *   SEMI : count = left rows with a match, sum_value = SUM(value) over them;
 *   ANTI : count = left rows without a match (NULL keys included),
 *          sum_value = SUM(value) over them.
 * `value` may be NULL (sum_value is then 0). */
int fdb_join_probe_agg(fdb_db* db, const fdb_hash* h, const fdb_dev_column* probe_key,
                       const fdb_dev_column* value, uint64_t nrows, int32_t join_type,
                       fdb_join_agg* d_out);

/* Probe emitting the joined row pairs (left row, build row); build row is
 * FDB_NO_ROW for LEFT's unmatched rows; SEMI/ANTI emit left rows only
 * (d_right untouched).  Pair order is unspecified. */
int fdb_join_probe_pairs(fdb_db* db, const fdb_hash* h, const fdb_dev_column* probe_key,
                         uint64_t nrows, int32_t join_type, uint32_t* d_left,
                         uint32_t* d_right, uint64_t capacity, uint64_t* d_count);

/* ORDER BY col [DESC] LIMIT k over one FLOAT64 / INT64 column
 * (execute_sort_limit + top_k_ascending + assemble, sort.rs:59-115, 564-620,
 * 773-791): the k best row numbers, in order, ties broken by row ascending;
 * NULL rows first or last as `nulls_last` says.  1 <= k <= 4096.  d_rows holds
 * k entries; d_count receives min(k, nrows). */
int fdb_topk(fdb_db* db, const fdb_dev_column* col, uint64_t nrows, uint32_t k,
             int32_t desc, int32_t nulls_last, uint32_t* d_rows, uint64_t* d_count);

/* ORDER BY col [DESC] over one FLOAT64 / INT64 column, no LIMIT
 * (execute_sort -> sort_merged -> try_typed_sort -> assemble, sort.rs:118-133,
 * 209-350, 773-791): all nrows row numbers in order.  Keys are the reference's
 * order keys (f64_ord_key, sort.rs:451-454; sign flip for INT64; every bit
 * flipped for DESC), so -0.0 sorts before +0.0 and NaN after +inf; ties keep
 * row order; NULL rows come first or last, in row order, as `nulls_last` says.
 * d_rows holds nrows entries (device); nrows < 2^32 - 1. */
int fdb_sort(fdb_db* db, const fdb_dev_column* col, uint64_t nrows, int32_t desc,
             int32_t nulls_last, uint32_t* d_rows);

/* SELECT DISTINCT col over one FLOAT64 / INT64 / UTF8 column (dedup_batches ->
 * dedup_single_primitive and the row_hash / row_eq path, select.rs:171-457):
 * the row numbers of each value's first occurrence, in row order.  FLOAT64
 * values are compared with every NaN equal and -0.0 equal to +0.0 (norm_f64,
 * select.rs:201-204); UTF8 compares codes (a code names one string); all NULL
 * rows are one value, kept at its first row.  d_rows holds nrows entries
 * (device); d_count receives how many were written. */
int fdb_distinct(fdb_db* db, const fdb_dev_column* col, uint64_t nrows, uint32_t* d_rows,
                 uint64_t* d_count);

/* ---- Batched GROUP BY -------------------------------------------------------
 * Many independent `GROUP BY key` queries (COUNT(*), SUM, MIN, MAX of one
 * value column, each over its own rows, e.g. slices of one table) run as one
 * persistent kernel plus one compaction kernel, captured into a CUDA graph at
 * prepare time and replayed by each run.  The reference answers each query
 * with its own GroupByExec::execute (fast_i64_gb, aggregate.rs:840-912); each
 * query's result equals fdb_group_by_i64 on its rows (groups unordered). */
typedef struct fdb_gb_query {
    fdb_dev_column key;        /* FDB_INT64; values point at the query's first row */
    fdb_dev_column value;      /* FDB_FLOAT64 or FDB_INT64, same rows              */
    uint64_t       nrows;
    uint64_t       expected_groups;  /* 0: estimated by a HyperLogLog pass      */
    fdb_group_i64* d_groups;   /* output groups (device), `capacity` entries     */
    uint64_t       capacity;
    uint64_t*      d_ngroups;  /* output group count (device)                     */
} fdb_gb_query;

/* Launch shape and table sizing of a batch; zero fields take defaults
 * (load factor 0.5, 2 CTAs per SM, 8192-row tiles). */
typedef struct fdb_batch_tuning {
    double  load_factor;       /* table slots = 2 x expected groups / load_factor, pow2 */
    int32_t ctas_per_sm;       /* persistent CTAs per SM (capped by occupancy)    */
    int32_t tile_rows;         /* rows per claimed work unit (>= 256)             */
} fdb_batch_tuning;

typedef struct fdb_batch fdb_batch;

/* Size the queries' tables (one device arena), upload their descriptors and
 * capture the batch into a CUDA graph.  Inputs and outputs must stay valid
 * while the batch exists.  tuning NULL: the context's (the last autotune's or
 * a loaded cache's; the defaults otherwise). */
int fdb_gb_batch_prepare(fdb_db* db, const fdb_gb_query* queries, int32_t nqueries,
                         const fdb_batch_tuning* tuning, fdb_batch** out);
/* Replay the batch on the context stream (asynchronous). */
int fdb_gb_batch_run(fdb_batch* b);
void fdb_gb_batch_free(fdb_batch* b);
/* Autotuner (replaces the reference's fixed parallel cut-offs, tuning.rs:39-53):
 * times every (load factor, CTAs per SM, tile rows) candidate on these queries
 * and returns the fastest in *best and its time per run in *best_ms.  The
 * context keeps it: fdb_gb_batch_prepare with tuning NULL uses it, and
 * fdb_tuning_save stores it. */
int fdb_gb_batch_autotune(fdb_db* db, const fdb_gb_query* queries, int32_t nqueries, int32_t reps,
                          fdb_batch_tuning* best, double* best_ms);

/* ---- Launch tuning of the streamed operators ----------------------------------
 * The reference sizes its parallel regions with fixed cut-offs, "rows per
 * thread x threads" (par_min_rows / par_min_rows_per_batch_fanout,
 * tuning.rs:39-53).  Here each kind of streamed operator has two knobs: the
 * resident CTAs per SM of its persistent grid (0 = as many as fit, up to the
 * kernel's own cap) and the rows each CTA must have before another CTA is
 * launched (0 = one CTA per tile, up to the grid).  The autotuner times
 * candidates on synthetic columns in device memory; the choices (and the
 * batched GROUP BY's) persist in a JSON cache file. */
#define FDB_TUNE_SCAN       0   /* filter mask / count, aggregates, COUNT(DISTINCT) */
#define FDB_TUNE_GROUP      1   /* dictionary GROUP BY                              */
#define FDB_TUNE_GROUP_I64  2   /* int64-key GROUP BY                               */
#define FDB_TUNE_PROBE      3   /* join probes                                      */
#define FDB_TUNE_TOPK       4   /* top-k                                            */
#define FDB_TUNE_KINDS      5

typedef struct fdb_op_tuning {
    int32_t  ctas_per_sm;       /* 0 = occupancy limit                          */
    int32_t  _pad;
    uint64_t min_rows_per_cta;  /* 0 = no row minimum                           */
} fdb_op_tuning;

int fdb_get_tuning(fdb_db* db, int32_t kind, fdb_op_tuning* out);
int fdb_set_tuning(fdb_db* db, int32_t kind, const fdb_op_tuning* in);
/* Times, for each kind, CTAs per SM in {1, 2, 3, 4, occupancy} on `rows`
 * synthetic rows and rows per CTA in {0, 2^15, 2^17, 2^19} on rows / 64, each
 * candidate `reps` times (median), keeps the fastest in the context and
 * returns them in best[FDB_TUNE_KINDS] (ms_per_call[FDB_TUNE_KINDS] at `rows`
 * may be NULL).  The synthetic columns (about 40 B per row) are freed before
 * it returns. */
int fdb_autotune_ops(fdb_db* db, uint64_t rows, int32_t reps, fdb_op_tuning* best, double* ms_per_call);
/* The context's tuning (every kind, and the batched GROUP BY's defaults) as a
 * JSON file keyed by the device's name and SM count; loading a file written
 * for another device fails with FDB_E_ARG and changes nothing. */
int fdb_tuning_save(fdb_db* db, const char* path);
int fdb_tuning_load(fdb_db* db, const char* path);

/* ---- Serving loop ------------------------------------------------------------
 * A request loop over device-resident tables with continuous batching: queries
 * are admitted under a device-memory budget as they arrive, and whatever has
 * been admitted when a launch slot frees up goes to the GPU as one batch, run
 * by one persistent kernel (plus a top-k finish kernel) replayed from a CUDA
 * graph; batches on different slots overlap on the device.  No counterpart in
 * the reference, whose server (src/bin/server.rs:151-169) runs each request
 * through Database::sql on its own.
 *
 * Templates (over rows [0, nrows) of the given columns, literal x):
 *   FDB_SERVE_COUNT   SELECT COUNT(*) WHERE c0 > x                 (c0 FLOAT64)
 *   FDB_SERVE_GROUP   SELECT c1, COUNT(*), SUM(c0), SUM(c2) WHERE c0 > x GROUP BY c1
 *                     (c0 FLOAT64, c1 dictionary codes < dict_len <= 16, c2 INT64;
 *                      AVG(c2) = SUM / COUNT)
 *   FDB_SERVE_JOIN    SELECT COUNT(*), SUM(payload) FROM probe JOIN build ON c0 = key
 *                     WHERE c1 < x / 100                           (c0 INT64 keys,
 *                      c1 FLOAT64, `table` the resident build side)
 *   FDB_SERVE_TOPK    SELECT row WHERE c0 < x ORDER BY c0 DESC LIMIT k   (k <= 32;
 *                      ties by row ascending)
 * Columns hold no NULLs. */
#define FDB_SERVE_COUNT 0
#define FDB_SERVE_GROUP 1
#define FDB_SERVE_JOIN  2
#define FDB_SERVE_TOPK  3
#define FDB_SERVE_MAX_GROUPS 16
#define FDB_SERVE_MAX_K 32

typedef struct fdb_serve_query {
    int32_t     kind;          /* FDB_SERVE_*                                    */
    int32_t     k;             /* TOPK: LIMIT                                    */
    uint64_t    nrows;
    double      threshold;     /* the literal x                                  */
    const void* c0;
    const void* c1;
    const void* c2;
    uint32_t    dict_len;      /* GROUP                                          */
    uint32_t    _pad;
    fdb_hash*   table;         /* JOIN                                           */
    double      arrival_s;     /* fdb_serve_trace: seconds after the trace starts */
} fdb_serve_query;

typedef struct fdb_serve_result {
    int64_t  count;            /* COUNT rows / JOIN rows / TOPK rows returned    */
    int64_t  sum_payload;      /* JOIN                                           */
    int64_t  group_count[FDB_SERVE_MAX_GROUPS];
    double   group_sum0[FDB_SERVE_MAX_GROUPS];
    int64_t  group_sum2[FDB_SERVE_MAX_GROUPS];
    uint32_t rows[FDB_SERVE_MAX_K];
    double   arrival_s, start_s, done_s;   /* admitted at start_s, result on host at done_s */
    int32_t  batch_size;       /* queries in the launch that answered it         */
    int32_t  status;           /* FDB_OK or an error code                         */
} fdb_serve_result;

typedef struct fdb_serve_config {
    int32_t  max_batch;        /* queries per launch (1 = one query at a time)    */
    int32_t  slots;            /* launches in flight; slot 0 runs any batch, the
                                  others only batches of short scans            */
    uint64_t mem_budget;       /* bytes resident tables + admitted queries may hold; 0 = the context's budget */
} fdb_serve_config;

typedef struct fdb_serve_stats {
    double   wall_s;           /* first arrival to last result                    */
    double   qps;
    double   p50_ms, p99_ms, max_ms;   /* latency = done_s - arrival_s              */
    double   mean_batch;
    int64_t  batches;
    uint64_t peak_reserved;    /* peak bytes held by admitted queries             */
    uint64_t resident_bytes;   /* device bytes of the context when serving started */
} fdb_serve_stats;

typedef struct fdb_server fdb_server;

/* Start the scheduler thread (it owns `slots` streams and launch graphs). */
int fdb_server_start(fdb_db* db, const fdb_serve_config* cfg, fdb_server** out);
/* Queue a query; *ticket identifies it.  Returns at once. */
int fdb_server_submit(fdb_server* s, const fdb_serve_query* q, uint64_t* ticket);
/* Wait up to timeout_ns for a ticket's result (FDB_E_TIMEOUT if not ready). */
int fdb_server_wait(fdb_server* s, uint64_t ticket, int64_t timeout_ns, fdb_serve_result* out);
/* Drain, stop the thread, free the slots; *stats summarises every answered query. */
int fdb_server_stop(fdb_server* s, fdb_serve_stats* stats);
/* Replay an arrival trace: each query is submitted at its arrival_s (in
 * order), results land in out[i]; returns when all are answered. */
int fdb_serve_trace(fdb_db* db, const fdb_serve_query* queries, int32_t nqueries,
                    const fdb_serve_config* cfg, fdb_serve_result* out, fdb_serve_stats* stats);

/* Library version string. */
const char* fdb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FALCONDB_B200_H */
