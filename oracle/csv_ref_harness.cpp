// Test infrastructure: the reference's own CSV path, for pinning the oracle
// and the device CSV scan. Compiled by oracle/Makefile (target csvref) against
// the reference's vendored csv-parser header where it lies
// ($(REF)/vendor/csv-parser/csv.hpp); nothing of it is copied here.
//
// ref_csv_scan replays GetOperator::next's per-row loop
// (src/engine/operators/get_operator.cpp:56-101): csv::CSVReader(path) with the
// default format (get_operator.cpp:26), read_row, each projected field taken
// as a std::string and converted by std::stoi / std::stof / strptime+timegm
// (include/enums/data_type_utils.hpp:24-44) / a NUL-padded copy of at most
// width-1 bytes (include/kernels/string_kernel.hpp:16-31); an empty field is
// NULL with the sentinels of get_operator.cpp:80-86. Where the reference would
// throw (and exit), the harness writes 0 into the cell and counts it.
#include "csv.hpp"

#include <climits>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <ctime>
#include <stdexcept>
#include <string>

namespace {

int64_t date_time(const std::string& s) {
  std::tm t = {};
  if (strptime(s.c_str(), "%Y-%m-%d %H:%M:%S", &t) == nullptr) return 0;
  return static_cast<int64_t>(timegm(&t));
}

}  // namespace

extern "C" {

// field_type[f]: -1 skipped, 0 INT, 1 FLOAT, 2 DATETIME, 3 STRING (slot of field_width[f] bytes).
// guess != 0: the reference's own call, CSVReader(path) with the default
// format, which guesses the delimiter and header row from the first rows;
// guess == 0: the format that guess settles on for a comma-separated file with
// its header on the first line (',' delimiter, '"' quote, header row 0), for
// inputs whose early rows would mislead the guess.
// Returns 0, -1 when the header's field count differs from nfields, -2 when
// more rows than `capacity` were read.
int ref_csv_scan(const char* path, int guess, int nfields, const int* field_type, const int* field_width,
                 void** out_data, unsigned char** out_nulls, uint64_t capacity, uint64_t* rows, uint64_t* bad_cells,
                 int64_t* first_bad_row, int* first_bad_field, int* first_bad_kind) {
  csv::CSVFormat fixed;
  fixed.delimiter(',').quote('"').header_row(0);
  csv::CSVReader reader(path, guess ? csv::CSVFormat::guess_csv() : fixed);
  if ((int)reader.get_col_names().size() != nfields) return -1;
  csv::CSVRow row;
  uint64_t r = 0;
  *bad_cells = 0;
  *first_bad_row = -1;
  *first_bad_field = -1;
  *first_bad_kind = 0;
  while (reader.read_row(row)) {
    if (r >= capacity) return -2;
    for (int f = 0; f < nfields; ++f) {
      const int ty = field_type[f];
      if (ty < 0) continue;
      const std::string v = row[f].get<std::string>();
      out_nulls[f][r] = v.empty() ? 1 : 0;
      int kind = 0;
      if (ty == 0) {
        int x = INT_MIN;
        if (!v.empty()) {
          try { x = std::stoi(v); } catch (const std::invalid_argument&) { x = 0; kind = 1; }
          catch (const std::out_of_range&) { x = 0; kind = 2; }
        }
        static_cast<int32_t*>(out_data[f])[r] = x;
      } else if (ty == 1) {
        float x = FLT_MIN;
        if (!v.empty()) {
          try { x = std::stof(v); } catch (const std::invalid_argument&) { x = 0; kind = 1; }
          catch (const std::out_of_range&) { x = 0; kind = 2; }
        }
        static_cast<float*>(out_data[f])[r] = x;
      } else if (ty == 2) {
        static_cast<int64_t*>(out_data[f])[r] = v.empty() ? 0 : date_time(v);
      } else {
        char* slot = static_cast<char*>(out_data[f]) + r * (uint64_t)field_width[f];
        std::memset(slot, 0, field_width[f]);
        const char* src = v.c_str();
        for (int i = 0; i < field_width[f] - 1 && src[i]; ++i) slot[i] = src[i];
      }
      if (kind) {
        if (*bad_cells == 0) { *first_bad_row = (int64_t)r; *first_bad_field = f; *first_bad_kind = kind; }
        ++*bad_cells;
      }
    }
    ++r;
  }
  *rows = r;
  return 0;
}

}  // extern "C"
