// Host-side query result (the C ABI's fdb_result) and the SQL entry point.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

struct fdb_result {
  struct Col {
    std::string name;
    int32_t dtype = 0;
    std::vector<int64_t> i64;
    std::vector<double> f64;
    std::vector<std::string> str;
    std::vector<const char*> str_ptrs;
    std::vector<uint8_t> nulls;  // empty when the column has no NULLs
    bool has_nulls() const {
      for (uint8_t b : nulls)
        if (b) return true;
      return false;
    }
  };
  std::vector<Col> cols;
  uint64_t rows = 0;
  void finalize();                    // fills str_ptrs
  const std::string& display_text();  // the table as text, built on first use (QueryResult::display, db.rs:63-64)

 private:
  std::string display_;
  bool display_built_ = false;
};

namespace fdb {
// Database::sql (FalconDB src/db.rs:242-316 -> run_select 989-1007 ->
// execute_plan 1226-1743) for the query shapes of the hot path.
fdb_result* run_sql(Ctx& c, const std::string& sql);
}  // namespace fdb
