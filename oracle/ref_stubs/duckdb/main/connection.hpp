// Minimal stand-in for duckdb::Connection so that the reference's
// include/db/table.hpp (pulled in through include/batch.hpp) compiles; the
// kernels never talk to DuckDB.
#pragma once
#include <memory>
#include <string>
namespace duckdb {
struct QueryResult {
  bool HasError() const { return false; }
  std::string GetError() const { return std::string(); }
};
struct Connection {
  std::unique_ptr<QueryResult> Query(const std::string&) { return std::make_unique<QueryResult>(); }
};
}  // namespace duckdb
