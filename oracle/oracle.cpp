// ORACLE — test infrastructure only.  A serial CPU restatement of FalconDB's
// relational operators (FalconTechDev/falcondb, Rust; the crate cannot be built
// here: no cargo/rustc), used by tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg as the checker.  Nothing in the product links or calls it.
//
// Parity is pinned by the known-answer tests of the reference's own test suites
// (restated in tests/test_oracle_golden.py with their file:line), not by running
// the reference.  Each function names the reference routine it follows.
//
// Value semantics: GROUP BY over a Utf8 column groups by string value (the
// reference's fast_utf8_gb takes batch 0's dictionary order for every batch,
// src/query/aggregate.rs:655-658 — a multi-batch hazard recorded, not copied).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <utility>
#include <vector>

extern "C" {

// ---------------------------------------------------------------------------
// Filter: `col op literal` -> packed u64 mask (expr.rs:1076-1175).
// op: 0 EQ 1 NE 2 LT 3 LE 4 GT 5 GE.  dtype 1 = Int64, 2 = Float64.
// lit_type 1 = Int64 literal, 2 = Float64 literal.
// Float64 col vs Int64 literal: literal widened (`*v as f64`, expr.rs:1117).
// Int64 col vs Float64 literal: column widened to f64 (expr.rs:1122-1132).
// Float compares are IEEE ordered except NE (_CMP_NEQ_UQ, expr.rs:894-899).
// NULL rows cleared (clear_null_bits, expr.rs:961-973); padding bits zero
// (mask_off_padding, expr.rs:979-986).
// ---------------------------------------------------------------------------
static bool cmp_d(int op, double a, double b) {
  switch (op) {
    case 0: return a == b;
    case 1: return a != b;
    case 2: return a < b;
    case 3: return a <= b;
    case 4: return a > b;
    default: return a >= b;
  }
}
static bool cmp_i(int op, int64_t a, int64_t b) {
  switch (op) {
    case 0: return a == b;
    case 1: return a != b;
    case 2: return a < b;
    case 3: return a <= b;
    case 4: return a > b;
    default: return a >= b;
  }
}
static bool valid_at(const uint64_t* validity, uint64_t i) {
  return validity == nullptr || ((validity[i >> 6] >> (i & 63)) & 1ull);
}

void orc_cmp_mask(int dtype, const void* values, const uint64_t* validity, uint64_t n, int op,
                  int lit_type, int64_t lit_i, double lit_f, uint64_t* out) {
  const uint64_t words = (n + 63) / 64;
  std::memset(out, 0, words * 8);
  for (uint64_t i = 0; i < n; ++i) {
    bool hit;
    if (dtype == 2) {
      const double v = static_cast<const double*>(values)[i];
      hit = cmp_d(op, v, lit_type == 2 ? lit_f : (double)lit_i);
    } else {
      const int64_t v = static_cast<const int64_t*>(values)[i];
      hit = lit_type == 2 ? cmp_d(op, (double)v, lit_f) : cmp_i(op, v, lit_i);
    }
    if (hit && valid_at(validity, i)) out[i >> 6] |= 1ull << (i & 63);
  }
}

// Utf8 arm: decide once per dictionary entry, then read codes; the NULL code
// (u32::MAX) fails (expr.rs:1143-1171).  pass[d] != 0 means entry d passes.
void orc_code_mask(const uint32_t* codes, const uint64_t* validity, uint64_t n, const uint8_t* pass,
                   uint32_t dict_len, uint64_t* out) {
  const uint64_t words = (n + 63) / 64;
  std::memset(out, 0, words * 8);
  for (uint64_t i = 0; i < n; ++i) {
    const uint32_t c = codes[i];
    if (c == 0xFFFFFFFFu || c >= dict_len || !pass[c] || !valid_at(validity, i)) continue;
    out[i >> 6] |= 1ull << (i & 63);
  }
}

// COUNT(*) + WHERE: population count of the mask words (db.rs:1453-1458).
uint64_t orc_popcount(const uint64_t* words, uint64_t nwords) {
  uint64_t c = 0;
  for (uint64_t i = 0; i < nwords; ++i) c += (uint64_t)__builtin_popcountll(words[i]);
  return c;
}

// Selection: row numbers of set bits in order (gather_by_bitmask's tzcnt walk,
// column.rs:1077-1123).
uint64_t orc_mask_rows(const uint64_t* words, uint64_t n, uint32_t* out) {
  uint64_t k = 0;
  for (uint64_t w = 0; w < (n + 63) / 64; ++w) {
    uint64_t x = words[w];
    while (x) {
      const int b = __builtin_ctzll(x);
      x &= x - 1;
      const uint64_t r = w * 64 + b;
      if (r < n) out[k++] = (uint32_t)r;
    }
  }
  return k;
}

// ---------------------------------------------------------------------------
// Sums (aggregate.rs:1557-1590 sum_lanes; 3039-3104 sum_i64 / checked_sum_i64).
// ---------------------------------------------------------------------------
// Eight independent f64 lanes, then the lane total, then the remainder.
double orc_sum_lanes_f64(const double* v, uint64_t n) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const uint64_t full = n / 8 * 8;
  for (uint64_t i = 0; i < full; i += 8)
    for (int l = 0; l < 8; ++l) acc[l] += v[i + l];
  double t = 0.0;
  for (int l = 0; l < 8; ++l) t += acc[l];
  for (uint64_t i = full; i < n; ++i) t += v[i];
  return t;
}
// Plain left-to-right FP64 sum: the serial oracle every GPU FP64 sum is held to.
double orc_sum_serial_f64(const double* v, uint64_t n) {
  double t = 0.0;
  for (uint64_t i = 0; i < n; ++i) t += v[i];
  return t;
}
// Four checked i64 lanes; returns 1 and the total when no lane overflowed,
// else 0 (the reference then falls back to sum_lanes in f64).
int orc_checked_sum_i64(const int64_t* v, uint64_t n, int64_t* out) {
  int64_t acc[4] = {0, 0, 0, 0};
  const uint64_t full = n / 4 * 4;
  for (uint64_t i = 0; i < full; i += 4)
    for (int l = 0; l < 4; ++l)
      if (__builtin_add_overflow(acc[l], v[i + l], &acc[l])) return 0;
  int64_t t = 0;
  for (int l = 0; l < 4; ++l)
    if (__builtin_add_overflow(t, acc[l], &t)) return 0;
  for (uint64_t i = full; i < n; ++i)
    if (__builtin_add_overflow(t, v[i], &t)) return 0;
  *out = t;
  return 1;
}

// ---------------------------------------------------------------------------
// No-key aggregates over the rows selected by `mask` (NULL = all rows)
// (execute_agg_only + accumulate_typed, aggregate.rs:1394-1528, 3121-3386;
// Accumulator semantics 237-481).  out[0] = count of contributing values,
// out[1] = value (SUM serial f64; AVG = sum/count; MIN/MAX via f64::min/max,
// which skip NaN).  func: 1 COUNT 2 SUM 3 AVG 4 MIN 5 MAX.  Returns validity.
// ---------------------------------------------------------------------------
int orc_agg(int func, int dtype, const void* values, const uint64_t* validity, const uint64_t* mask,
            uint64_t n, double* out_value, int64_t* out_count) {
  double acc = 0.0;
  int64_t cnt = 0;
  bool any = false;
  double best = func == 4 ? INFINITY : -INFINITY;
  for (uint64_t i = 0; i < n; ++i) {
    if (mask && !((mask[i >> 6] >> (i & 63)) & 1ull)) continue;
    if (!valid_at(validity, i)) continue;
    const double v = dtype == 2 ? static_cast<const double*>(values)[i]
                                : (double)static_cast<const int64_t*>(values)[i];
    if (func == 4 || func == 5) {
      if (std::isnan(v)) continue;
      best = func == 4 ? std::fmin(best, v) : std::fmax(best, v);
      any = true;
      ++cnt;
      continue;
    }
    acc += v;
    ++cnt;
  }
  *out_count = cnt;
  if (func == 1) {
    *out_value = (double)cnt;
    return 1;
  }
  if (func == 4 || func == 5) {
    *out_value = any ? best : 0.0;
    return any ? 1 : 0;
  }
  if (cnt == 0) {
    *out_value = 0.0;
    return 0;
  }
  *out_value = func == 3 ? acc / (double)cnt : acc;
  return 1;
}

// Exact SUM over Int64 (sum_i64): exact i64 total when no overflow.
int orc_sum_i64_masked(const int64_t* v, const uint64_t* validity, const uint64_t* mask, uint64_t n,
                       int64_t* out) {
  int64_t t = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (mask && !((mask[i >> 6] >> (i & 63)) & 1ull)) continue;
    if (!valid_at(validity, i)) continue;
    if (__builtin_add_overflow(t, v[i], &t)) return 0;
  }
  *out = t;
  return 1;
}

// Presence of dictionary codes among selected rows (present_codes,
// aggregate.rs:3167-3200).  out[d] = 1 if code d occurs.
void orc_present_codes(const uint32_t* codes, const uint64_t* validity, const uint64_t* mask, uint64_t n,
                       uint32_t dict_len, uint8_t* out) {
  std::memset(out, 0, dict_len);
  for (uint64_t i = 0; i < n; ++i) {
    if (mask && !((mask[i >> 6] >> (i & 63)) & 1ull)) continue;
    if (!valid_at(validity, i)) continue;
    const uint32_t c = codes[i];
    if (c != 0xFFFFFFFFu && c < dict_len) out[c] = 1;
  }
}

// ---------------------------------------------------------------------------
// GROUP BY dictionary code (value semantics) — accumulate_batch
// (aggregate.rs:916-1169): COUNT(*) per group, SUM of a Float64 column in row
// order, SUM of an Int64 column added as f64 per row (1020-1036), and the
// non-NULL count of each.  Group dict_len is the NULL key.  Arrays hold
// dict_len+1 entries; any value pointer may be NULL.
// ---------------------------------------------------------------------------
void orc_group_codes(const uint32_t* codes, const uint64_t* kvalid, const uint64_t* mask, uint64_t n,
                     uint32_t dict_len, const double* fvals, const uint64_t* fvalid, const int64_t* ivals,
                     const uint64_t* ivalid, int64_t* rows, double* fsum, int64_t* fcnt, double* isum,
                     int64_t* icnt, double* fmin_, double* fmax_) {
  const uint32_t ng = dict_len + 1;
  for (uint32_t g = 0; g < ng; ++g) {
    rows[g] = 0;
    fsum[g] = 0.0;
    fcnt[g] = 0;
    isum[g] = 0.0;
    icnt[g] = 0;
    fmin_[g] = INFINITY;
    fmax_[g] = -INFINITY;
  }
  for (uint64_t i = 0; i < n; ++i) {
    if (mask && !((mask[i >> 6] >> (i & 63)) & 1ull)) continue;
    uint32_t c = codes[i];
    const uint32_t g = (!valid_at(kvalid, i) || c == 0xFFFFFFFFu || c >= dict_len) ? dict_len : c;
    rows[g]++;
    if (fvals && valid_at(fvalid, i)) {
      fsum[g] += fvals[i];
      fcnt[g]++;
      if (!std::isnan(fvals[i])) {
        fmin_[g] = std::fmin(fmin_[g], fvals[i]);
        fmax_[g] = std::fmax(fmax_[g], fvals[i]);
      }
    }
    if (ivals && valid_at(ivalid, i)) {
      isum[g] += (double)ivals[i];
      icnt[g]++;
    }
  }
}

// ---------------------------------------------------------------------------
// GROUP BY int64 key (fast_i64_gb, aggregate.rs:840-912): COUNT(*), SUM (f64
// in row order), MIN, MAX of a Float64 value.  i64::MIN keys read as NULL
// (aggregate.rs:867, 1207) and form one group reported with key INT64_MIN.
// Output sorted by key; returns the number of groups.  out arrays hold n+1.
// ---------------------------------------------------------------------------
uint64_t orc_group_i64(const int64_t* keys, const uint64_t* kvalid, const double* vals, const uint64_t* mask,
                       uint64_t n, int64_t* out_key, int64_t* out_count, double* out_sum, double* out_min,
                       double* out_max) {
  struct Acc {
    int64_t count = 0;
    double sum = 0.0;
    double mn = INFINITY, mx = -INFINITY;
  };
  std::unordered_map<int64_t, Acc> m;
  m.reserve(n / 4 + 16);
  for (uint64_t i = 0; i < n; ++i) {
    if (mask && !((mask[i >> 6] >> (i & 63)) & 1ull)) continue;
    int64_t k = keys[i];
    if (!valid_at(kvalid, i)) k = INT64_MIN;
    Acc& a = m[k];
    a.count++;
    a.sum += vals[i];
    if (!std::isnan(vals[i])) {
      a.mn = std::fmin(a.mn, vals[i]);
      a.mx = std::fmax(a.mx, vals[i]);
    }
  }
  std::vector<int64_t> ks;
  ks.reserve(m.size());
  for (auto& kv : m) ks.push_back(kv.first);
  std::sort(ks.begin(), ks.end());
  uint64_t o = 0;
  for (int64_t k : ks) {
    const Acc& a = m[k];
    out_key[o] = k;
    out_count[o] = a.count;
    out_sum[o] = a.sum;
    out_min[o] = a.mn;
    out_max[o] = a.mx;
    ++o;
  }
  return o;
}

// ---------------------------------------------------------------------------
// Hash join on one Int64 key (join.rs): IntHashTable with 2 buckets per build
// row rounded to a power of two, LIFO chains through `next`, bucket_with's
// mix (join.rs:1054-1351, 1423-1429); NULL keys never match (637, 693-697).
// Probe left rows in order (probe_one, 657-723); SEMI/ANTI as a keep-mask
// (49-132).  Results: count, exact SUM(payload) over matched non-NULL
// payloads, their number, and the serial FP64 SUM(value) over kept left rows
// (SEMI/ANTI).  join_type 0 INNER 1 LEFT 2 SEMI 3 ANTI.
// ---------------------------------------------------------------------------
struct OrcHash {
  std::vector<uint32_t> head, next;
  uint64_t mask = 0;
};
static uint64_t bucket_with(uint64_t mask, int64_t key) {
  uint64_t h = (uint64_t)key;
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdull;
  h ^= h >> 33;
  return h & mask;
}
static OrcHash orc_build(const int64_t* bkeys, const uint64_t* bvalid, uint64_t nb) {
  OrcHash t;
  uint64_t buckets = 1;
  while (buckets < std::max<uint64_t>(nb * 2, 1)) buckets <<= 1;
  t.mask = buckets - 1;
  t.head.assign(buckets, 0xFFFFFFFFu);
  t.next.assign(nb, 0xFFFFFFFFu);
  for (uint64_t r = 0; r < nb; ++r) {
    if (!valid_at(bvalid, r)) continue;  // NULL keys are never inserted
    const uint64_t b = bucket_with(t.mask, bkeys[r]);
    t.next[r] = t.head[b];
    t.head[b] = (uint32_t)r;
  }
  return t;
}

void orc_join_agg(const int64_t* bkeys, const uint64_t* bvalid, const int64_t* bpay, const uint64_t* bpvalid,
                  uint64_t nb, const int64_t* pkeys, const uint64_t* pvalid, const double* pval,
                  const uint64_t* pvvalid, uint64_t np, int join_type, int64_t* out_count, int64_t* out_psum,
                  int64_t* out_prows, double* out_vsum) {
  const OrcHash t = orc_build(bkeys, bvalid, nb);
  int64_t count = 0, psum = 0, prows = 0;
  double vsum = 0.0;
  for (uint64_t i = 0; i < np; ++i) {
    int64_t matches = 0, ps = 0, pr = 0;
    if (valid_at(pvalid, i)) {
      const int64_t k = pkeys[i];
      for (uint32_t r = t.head[bucket_with(t.mask, k)]; r != 0xFFFFFFFFu; r = t.next[r]) {
        if (bkeys[r] != k) continue;
        ++matches;
        if (bpay && valid_at(bpvalid, r)) {
          ps += bpay[r];
          ++pr;
        }
      }
    }
    if (join_type == 0 || join_type == 1) {
      count += join_type == 1 && matches == 0 ? 1 : matches;
      psum += ps;
      prows += pr;
    } else {
      const bool keep = join_type == 2 ? matches != 0 : matches == 0;
      if (keep) {
        ++count;
        if (pval && valid_at(pvvalid, i)) {
          vsum += pval[i];
          ++prows;
        }
      }
    }
  }
  *out_count = count;
  *out_psum = psum;
  *out_prows = prows;
  *out_vsum = vsum;
}

// Joined row pairs in the reference's emission order: left rows ascending,
// each left row's matches in chain order (LIFO, i.e. descending build row);
// LEFT's unmatched rows carry 0xFFFFFFFF; SEMI/ANTI fill `left` only.
uint64_t orc_join_pairs(const int64_t* bkeys, const uint64_t* bvalid, uint64_t nb, const int64_t* pkeys,
                        const uint64_t* pvalid, uint64_t np, int join_type, uint32_t* left, uint32_t* right,
                        uint64_t cap) {
  const OrcHash t = orc_build(bkeys, bvalid, nb);
  uint64_t o = 0;
  for (uint64_t i = 0; i < np; ++i) {
    uint64_t matches = 0;
    const bool kv = valid_at(pvalid, i);
    if (kv) {
      const int64_t k = pkeys[i];
      for (uint32_t r = t.head[bucket_with(t.mask, k)]; r != 0xFFFFFFFFu; r = t.next[r]) {
        if (bkeys[r] != k) continue;
        ++matches;
        if (join_type <= 1) {
          if (o < cap) {
            left[o] = (uint32_t)i;
            right[o] = r;
          }
          ++o;
        }
      }
    }
    if (join_type == 1 && matches == 0) {
      if (o < cap) {
        left[o] = (uint32_t)i;
        right[o] = 0xFFFFFFFFu;
      }
      ++o;
    } else if ((join_type == 2 && matches) || (join_type == 3 && !matches)) {
      if (o < cap) left[o] = (uint32_t)i;
      ++o;
    }
  }
  return o;
}

// ---------------------------------------------------------------------------
// ORDER BY col [DESC] LIMIT k (sort.rs): order keys (f64_ord_key 451-454; sign
// flip for i64 243-268; NOT for DESC), bounded buffer of max(2k,1024) pairs
// with select-nth when full (top_k_ascending, 564-599), pairs sorted as
// (key,row) tuples, NULL rows before or after (assemble, 773-791).
// Writes min(k, n) row numbers; returns that count.
// ---------------------------------------------------------------------------
static uint64_t ord_f64(double v) {
  uint64_t b;
  std::memcpy(&b, &v, 8);
  return (b >> 63) == 0 ? (b ^ (1ull << 63)) : ~b;
}

uint64_t orc_topk(int dtype, const void* values, const uint64_t* validity, uint64_t n, uint32_t k, int desc,
                  int nulls_last, uint32_t* out) {
  if (k == 0) return 0;
  typedef std::pair<uint64_t, uint32_t> P;
  const size_t cap = std::max<size_t>(2 * (size_t)k, 1024);
  std::vector<P> buf;
  buf.reserve(cap);
  bool have_worst = false;
  P worst{0, 0};
  std::vector<uint32_t> nulls;
  for (uint64_t i = 0; i < n; ++i) {
    if (!valid_at(validity, i)) {
      if (nulls.size() < k) nulls.push_back((uint32_t)i);
      continue;
    }
    uint64_t key = dtype == 2 ? ord_f64(static_cast<const double*>(values)[i])
                              : ((uint64_t)static_cast<const int64_t*>(values)[i] ^ (1ull << 63));
    if (desc) key = ~key;
    const P pr{key, (uint32_t)i};
    if (have_worst && pr.first > worst.first) continue;
    buf.push_back(pr);
    if (buf.size() == cap) {
      std::nth_element(buf.begin(), buf.begin() + (k - 1), buf.end());
      worst = buf[k - 1];
      have_worst = true;
      buf.resize(k);
    }
  }
  std::sort(buf.begin(), buf.end());
  if (buf.size() > k) buf.resize(k);
  uint64_t o = 0;
  if (!nulls_last)
    for (uint32_t r : nulls)
      if (o < k) out[o++] = r;
  for (const P& p : buf)
    if (o < k) out[o++] = p.second;
  if (nulls_last)
    for (uint32_t r : nulls)
      if (o < k) out[o++] = r;
  return o;
}

// ---------------------------------------------------------------------------
// ORDER BY col [DESC] without LIMIT (sort_merged -> try_typed_sort, sort.rs:
// 118-133, 209-350): (order key, row) pairs of the non-NULL rows sorted as
// tuples (sort_pairs_ord, 692-698; the INT64 arm's sort_pairs, 749-760,
// compares keys only and leaves ties unordered -- row order is one of its
// outcomes), NULL rows before or after in row order (assemble, 773-791).
// Writes n row numbers.
// ---------------------------------------------------------------------------
void orc_sort(int dtype, const void* values, const uint64_t* validity, uint64_t n, int desc, int nulls_last,
              uint32_t* out) {
  typedef std::pair<uint64_t, uint32_t> P;
  std::vector<P> pairs;
  pairs.reserve(n);
  std::vector<uint32_t> nulls;
  for (uint64_t i = 0; i < n; ++i) {
    if (!valid_at(validity, i)) {
      nulls.push_back((uint32_t)i);
      continue;
    }
    uint64_t key = dtype == 2 ? ord_f64(static_cast<const double*>(values)[i])
                              : ((uint64_t)static_cast<const int64_t*>(values)[i] ^ (1ull << 63));
    if (desc) key = ~key;
    pairs.push_back(P{key, (uint32_t)i});
  }
  std::sort(pairs.begin(), pairs.end());
  uint64_t o = 0;
  if (!nulls_last)
    for (uint32_t r : nulls) out[o++] = r;
  for (const P& p : pairs) out[o++] = p.second;
  if (nulls_last)
    for (uint32_t r : nulls) out[o++] = r;
}

// ---------------------------------------------------------------------------
// SELECT DISTINCT col (dedup_batches, select.rs:238-269, and its one-column
// fast path dedup_single_primitive, 311-457): first occurrence wins, output in
// row order.  Values compare as row_eq does (select.rs:210-236): FLOAT64 with
// every NaN one value and -0.0 == +0.0 (norm_f64, 201-204), INT64 exactly,
// UTF8 by code (dtype 3, uint32 codes); all NULL rows are one value.
// Writes the kept row numbers; returns their count.
// ---------------------------------------------------------------------------
uint64_t orc_distinct(int dtype, const void* values, const uint64_t* validity, uint64_t n, uint32_t* out) {
  std::unordered_map<uint64_t, char> seen;
  bool null_seen = false;
  uint64_t o = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (!valid_at(validity, i)) {
      if (!null_seen) out[o++] = (uint32_t)i;
      null_seen = true;
      continue;
    }
    uint64_t k;
    if (dtype == 3) {
      k = static_cast<const uint32_t*>(values)[i];
    } else {
      std::memcpy(&k, static_cast<const char*>(values) + i * 8, 8);
      if (dtype == 2) {
        double d;
        std::memcpy(&d, &k, 8);
        if (std::isnan(d)) k = 0x7FF8000000000000ull;
        else if (d == 0.0) k = 0;
      }
    }
    if (seen.emplace(k, 1).second) out[o++] = (uint32_t)i;
  }
  return o;
}

}  // extern "C"
