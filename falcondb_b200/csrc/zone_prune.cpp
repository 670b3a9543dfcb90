// Zone-map pruning: which batches a WHERE program cannot select, from the
// batches' bounds alone (BatchStats::can_skip, src/storage/stats.rs:57-113),
// and GROUP BY key ranges from zone maps.
#include "zone.h"

#include <algorithm>
#include <cmath>

namespace fdb {

namespace {

// Can no row of batch z pass `col op lit`?  The filter's arithmetic
// (eval_leaf): INT64 (or UTF8 code) against an INT64 literal exactly, INT64
// against a FLOAT64 literal as (double)value, FLOAT64 against either as
// double.  NULL rows fail every comparison; NaN rows pass NE only.
bool cmp_rules_out(const fdb_zone& z, int32_t dtype, const fdb_pred_term& t) {
  const bool values = (z.flags & FDB_ZONE_VALUES) != 0;
  const bool nan = (z.flags & FDB_ZONE_NAN) != 0;
  if (dtype == FDB_FLOAT64 || (dtype == FDB_INT64 && t.lit_type == FDB_FLOAT64)) {
    double lo, hi;
    const double lit = t.lit_type == FDB_FLOAT64 ? t.lit_f : (double)t.lit_i;
    if (dtype == FDB_FLOAT64) {
      lo = z.min_f;
      hi = z.max_f;
    } else {
      // (double) is monotone, so every (double)v lies in [(double)min, (double)max].
      lo = (double)z.min_i;
      hi = (double)z.max_i;
    }
    if (t.op == FDB_NE) {
      if (nan) return false;          // NaN != lit passes
      if (!values) return true;       // every row NULL
      if (std::isnan(lit)) return false;
      return lo == hi && lo == lit;   // every value equals lit
    }
    if (!values || std::isnan(lit)) return true;  // ordered compares: NULL and NaN fail
    switch (t.op) {
      case FDB_EQ: return lit < lo || lit > hi;
      case FDB_LT: return lo >= lit;
      case FDB_LE: return lo > lit;
      case FDB_GT: return hi <= lit;
      default:     return hi < lit;   // FDB_GE
    }
  }
  if (!values) return true;
  const int64_t lo = z.min_i, hi = z.max_i, lit = t.lit_i;
  switch (t.op) {
    case FDB_EQ: return lit < lo || lit > hi;
    case FDB_NE: return lo == hi && lo == lit;
    case FDB_LT: return lo >= lit;
    case FDB_LE: return lo > lit;
    case FDB_GT: return hi <= lit;
    default:     return hi < lit;
  }
}

// Set bits of a code bitmap below each word, for counting the codes of a
// range that are in the set in constant time.
struct CodeRank {
  const std::vector<uint64_t>* set = nullptr;
  std::vector<uint64_t> below;  // set bits in words [0, w)
  void build(const std::vector<uint64_t>& s) {
    set = &s;
    below.assign(s.size() + 1, 0);
    for (size_t w = 0; w < s.size(); ++w) below[w + 1] = below[w] + (uint64_t)__builtin_popcountll(s[w]);
  }
  // Set bits among codes [0, x).
  uint64_t rank(uint64_t x) const {
    const uint64_t w = x >> 6;
    if (w >= set->size()) return below.back();
    const uint64_t part = x & 63 ? (*set)[w] & ((1ull << (x & 63)) - 1) : 0;
    return below[w] + (uint64_t)__builtin_popcountll(part);
  }
};

bool leaf_rules_out(const fdb_zone& z, int32_t dtype, const fdb_pred_term& t, const CodeRank* rank) {
  switch (t.kind) {
    case FDB_TERM_IS_NULL: return z.null_count == 0;
    case FDB_TERM_IS_NOT_NULL: return z.null_count == z.rows;
    case FDB_TERM_CODE_SET: {
      if (dtype != FDB_UTF8 || !rank) return false;
      if (!(z.flags & FDB_ZONE_VALUES)) return true;  // every row NULL
      const int64_t lo = std::max<int64_t>(z.min_i, 0);
      const int64_t hi = std::min<int64_t>(z.max_i, t.lit_i - 1);  // codes >= lit_i never pass
      if (hi < lo) return true;
      return rank->rank((uint64_t)hi + 1) == rank->rank((uint64_t)lo);
    }
    case FDB_TERM_CMP: return cmp_rules_out(z, dtype, t);
    default: return false;
  }
}

}  // namespace

std::vector<uint8_t> zone_rule_out(const std::vector<const std::vector<fdb_zone>*>& zones,
                                   const std::vector<int32_t>& dtypes, const fdb_pred_term* prog, int nterms,
                                   const std::vector<std::vector<uint64_t>>& code_sets, uint64_t nbatches) {
  std::vector<uint8_t> out(nbatches, 0);
  if (nterms <= 0) return out;
  std::vector<uint8_t> stack;
  stack.reserve((size_t)nterms);
  std::vector<CodeRank> ranks((size_t)nterms);
  for (int i = 0; i < nterms; ++i)
    if (prog[i].kind == FDB_TERM_CODE_SET && (size_t)i < code_sets.size()) ranks[(size_t)i].build(code_sets[(size_t)i]);
  for (uint64_t b = 0; b < nbatches; ++b) {
    stack.clear();
    for (int i = 0; i < nterms; ++i) {
      const fdb_pred_term& t = prog[i];
      if (t.kind == FDB_TERM_AND || t.kind == FDB_TERM_OR) {
        if (stack.size() < 2) fail(FDB_E_ARG, "malformed predicate program");
        const uint8_t a = stack.back();
        stack.pop_back();
        const uint8_t c = stack.back();
        stack.pop_back();
        // AND is impossible when either side is; OR only when both are.
        stack.push_back(t.kind == FDB_TERM_AND ? (a | c) : (a & c));
        continue;
      }
      if (t.col < 0 || (size_t)t.col >= zones.size()) fail(FDB_E_ARG, "predicate column out of range");
      const std::vector<fdb_zone>* z = zones[(size_t)t.col];
      uint8_t r = 0;
      if (z && b < z->size())
        r = leaf_rules_out((*z)[b], dtypes[(size_t)t.col], t, ranks[(size_t)i].set ? &ranks[(size_t)i] : nullptr);
      stack.push_back(r);
    }
    if (stack.size() != 1) fail(FDB_E_ARG, "malformed predicate program");
    out[b] = stack.back();
  }
  return out;
}

bool zone_key_range(const std::vector<fdb_zone>& z, uint64_t first_row, uint64_t n, int64_t* kmin, int64_t* kmax) {
  if (n == 0) return false;
  const uint64_t b0 = first_row / kZoneRows, b1 = zone_batches(first_row + n);
  if (b1 > z.size()) return false;
  bool any = false;
  int64_t lo = INT64_MAX, hi = INT64_MIN;
  for (uint64_t b = b0; b < b1; ++b) {
    if (!(z[b].flags & FDB_ZONE_VALUES)) continue;
    any = true;
    lo = std::min(lo, z[b].min_i);
    hi = std::max(hi, z[b].max_i);
  }
  // INT64_MIN reads as a NULL key in GROUP BY; the exact pass excludes it.
  if (!any || lo == INT64_MIN) return false;
  *kmin = lo;
  *kmax = hi;
  return true;
}

}  // namespace fdb
