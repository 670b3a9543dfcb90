// Zone-map pruning (BatchStats::can_skip, src/storage/stats.rs:57-113) and
// key ranges from zone maps: host logic only, no CUDA.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/falcondb_b200.h"

namespace fdb {

[[noreturn]] void fail(int code, const std::string& msg);

constexpr uint64_t kZoneRows = FDB_ZONE_BATCH_ROWS;
inline uint64_t zone_batches(uint64_t nrows) { return (nrows + kZoneRows - 1) / kZoneRows; }

// Per batch, 1 when the postfix program cannot pass any row of it.  zones[i]
// is the zone map of the program's column i (nullptr: unknown, never rules
// out) and dtypes[i] its type; code_sets[i] is the host copy of term i's
// CODE_SET bitmap.
std::vector<uint8_t> zone_rule_out(const std::vector<const std::vector<fdb_zone>*>& zones,
                                   const std::vector<int32_t>& dtypes, const fdb_pred_term* prog, int nterms,
                                   const std::vector<std::vector<uint64_t>>& code_sets, uint64_t nbatches);

// A key range covering rows [first_row, first_row + n) of an INT64 column,
// from the zone map of the batches that hold them; false when they hold no
// value or a key is INT64_MIN (a NULL key to GROUP BY, which only the exact
// pass leaves out).
bool zone_key_range(const std::vector<fdb_zone>& z, uint64_t first_row, uint64_t n, int64_t* kmin, int64_t* kmax);

}  // namespace fdb
