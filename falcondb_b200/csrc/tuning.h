// Launch tuning of the streamed operators and its JSON cache: host logic
// only, no CUDA (the grid arithmetic and the file format).
#pragma once
#include <cstdint>
#include <string>

#include "../../include/falcondb_b200.h"

namespace fdb {

struct OpTuning {
  int ctas_per_sm = 0;            // 0: occupancy limit
  uint64_t min_rows_per_cta = 0;  // 0: no row minimum
};

struct TuningSet {
  OpTuning op[FDB_TUNE_KINDS];
  fdb_batch_tuning batch{};       // zero fields: the batch defaults
};

// Grid of a persistent streamed kernel: `want` CTAs at most (the kernel's own
// choice, e.g. one per tile), `occ` resident per SM by occupancy, at most
// `cap` per SM (the kernel's partials), then the tuning's cap and row minimum
// over n rows.  Always at least 1.
inline int tuned_grid(const OpTuning& t, int sm_count, int occ, int cap, uint64_t want, uint64_t n) {
  int per_sm = occ < 1 ? 1 : occ;
  if (per_sm > cap) per_sm = cap;
  if (t.ctas_per_sm > 0 && t.ctas_per_sm < per_sm) per_sm = t.ctas_per_sm;
  if (want < 1) want = 1;
  if (t.min_rows_per_cta > 0) {
    const uint64_t by_rows = (n + t.min_rows_per_cta - 1) / t.min_rows_per_cta;
    if (by_rows < want) want = by_rows < 1 ? 1 : by_rows;
  }
  const uint64_t most = (uint64_t)sm_count * (uint64_t)per_sm;
  return (int)(want < most ? want : most);
}

const char* tune_kind_name(int kind);
// JSON text of a tuning set for device `device` (name, SM count).
std::string tuning_to_json(const TuningSet& t, const std::string& device, int sm_count);
// Parses tuning_to_json's format (keys in any order, unknown keys ignored).
// Returns "" and fills *out, *device, *sm_count, or an error message.
std::string tuning_from_json(const std::string& text, TuningSet* out, std::string* device, int* sm_count);

}  // namespace fdb
