// Minimal stand-in for duckdb::LogicalType, enough for the reference's
// include/enums/data_type_utils.hpp to compile (getDataTypeFromDuck is unused
// by the kernels).
#pragma once
namespace duckdb {
struct LogicalType {
  int id = 0;
  bool IsIntegral() const { return false; }
  bool IsNumeric() const { return false; }
  bool IsTemporal() const { return false; }
  bool operator==(const LogicalType& o) const { return id == o.id; }
  static const LogicalType INTERVAL;
};
inline const LogicalType LogicalType::INTERVAL = LogicalType{27};
}  // namespace duckdb
