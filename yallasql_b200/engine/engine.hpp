// C++ operator layer over the yq kernels: the reference's pull-based
// physical operators re-expressed on top of include/yq_ops.h.
//
//   reference                                         here
//   Batch (include/batch.hpp:21-145)                  yq::engine::Batch
//   NullBitSet (include/null_bit_set.hpp:5-32)        Batch::nulls (one byte per row)
//   CacheManager (include/engine/cache_manager.hpp)   yq::engine::CacheManager (64-bit budget)
//   Operator::init / next (operator.hpp:45-47)        yq::engine::Operator
//   GetOperator (get_operator.cpp:56-148)             ScanOperator (host columns -> pinned,
//                                                     double-buffered H2D on a copy stream)
//   FilterOperator (filter_operator.hpp:31-98)        FilterOperator -> yq_filter_project
//   ProjectionOperator (projection_operator.hpp)      ProjectionOperator -> yq_filter_project
//   AggregateOperator (aggregate_operator.hpp)        AggregateOperator -> yq_filter_aggregate
//                                                     (absorbs a child FilterOperator's predicate)
//   OrderOperator (order_operator.hpp/.cpp)           OrderOperator -> yq_sort_segments + yq_gather
//                                                     + yq_merge_pass per level
//   JoinOperator (join_operator.hpp)                  JoinOperator -> yq_join_project
//   CrossProductOperator (cross_product_operator.hpp) CrossProductOperator -> yq_join_project (no condition)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <future>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/yq_engine.h"
#include "../../include/yq_ops.h"

namespace yq::engine {

using BatchID = uint64_t;

// Where a batch's columns live: the device, pinned host memory, or a file in
// the plan's cache directory (the reference's Device::GPU / CPU / FS,
// include/enums/device.hpp).
enum class Device : uint8_t { CPU, GPU, FS };

struct Column {
  int32_t type;
  int32_t width;
};
using ColumnPtr = std::shared_ptr<Column>;

class Error : public std::runtime_error {
 public:
  int status;
  Error(int st, const std::string& where)
      : std::runtime_error(where + ": " + yq_status_string(st)), status(st) {}
};

inline void check(int st, const char* where) {
  if (st != YQ_OK) throw Error(st, where);
}
inline void check_cuda(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw Error(YQ_ERR_CUDA, std::string(where) + " (" + cudaGetErrorString(e) + ")");
}

// Columnar batch: per column a buffer of rows * width bytes and an optional
// null-byte array; on the device (stream-ordered allocations on `stream`), in
// pinned host memory after a spill, or in a file after a second spill (the
// null bytes travel with the data on every tier).
class Batch {
 public:
  std::vector<ColumnPtr> columns;
  std::vector<void*> data;
  std::vector<uint8_t*> nulls;
  uint64_t rows = 0;
  Device location = Device::GPU;
  cudaStream_t stream = nullptr;

  Batch(std::vector<ColumnPtr> cols, uint64_t rows, cudaStream_t s, bool with_nulls);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  uint64_t bytes() const;
  bool nullable(size_t c) const { return nulls[c] != nullptr || (c < null_flag_.size() && null_flag_[c]); }
  // Move between tiers. To FS: the file `path` is written by a background
  // task that then frees the host buffers (Batch::moveCpuToFs with
  // serializeBatchAsync, src/batch.cu:75-95); any later move or the
  // destructor waits for that task first. From FS: the file is read back
  // into pinned memory and removed.
  void moveTo(Device target, const std::string& path = std::string());
  yq_batch view(std::vector<yq_column>& storage) const;
  yq_column column(size_t c) const;

 private:
  void gpuToCpu();
  void cpuToGpu();
  void cpuToFs(const std::string& path);
  void fsToCpu();
  void waitWrite();
  std::string file_;
  std::future<bool> write_;
  std::vector<uint8_t> null_flag_;  // per column: nullable, while the null bytes are in the file
  bool write_failed_ = false;
};

// BatchID -> Batch with a device budget and a host budget; when the device
// budget is exceeded the oldest device batches move to pinned host memory, and
// when the host budget is exceeded the oldest host batches move to files in
// `cache_dir` (CacheManager::handleOverflow,
// include/engine/cache_manager.hpp:67-88; accounting here is 64-bit). A host
// budget of 0, or no cache directory, keeps every spilled batch in host memory.
class CacheManager {
 public:
  explicit CacheManager(uint64_t gpu_budget, uint64_t host_budget = 0, std::string cache_dir = std::string())
      : budget_(gpu_budget), host_budget_(host_budget), dir_(std::move(cache_dir)) {}
  BatchID putBatch(std::unique_ptr<Batch> b);
  std::unique_ptr<Batch> getBatch(BatchID id);  // ownership back to the caller, on the device
  Batch& refBatch(BatchID id);
  uint64_t spilled() const { return spilled_; }
  uint64_t spilledToDisk() const { return disk_; }

 private:
  void handleOverflow();
  std::string filePath(BatchID id) const;
  std::map<BatchID, std::unique_ptr<Batch>> batches_;
  BatchID next_ = 1;
  uint64_t budget_;
  uint64_t host_budget_;
  std::string dir_;
  uint64_t gpu_bytes_ = 0;
  uint64_t host_bytes_ = 0;
  uint64_t spilled_ = 0;
  uint64_t disk_ = 0;
};

struct ExecContext {
  cudaStream_t compute = nullptr;
  cudaStream_t copy = nullptr;
  yq_plan_stats stats{};
};

class Operator {
 public:
  std::vector<ColumnPtr> columns;  // schema of the batches next() returns
  bool isFinished = false;
  virtual ~Operator() = default;
  virtual void init() = 0;
  virtual BatchID next(CacheManager& cache) = 0;  // 0 = no more batches
  void setContext(ExecContext* ctx) {
    ctx_ = ctx;
    for (auto& c : children_) c->setContext(ctx);
  }
  Operator* child(size_t i) { return children_[i].get(); }
  std::vector<std::unique_ptr<Operator>>& children() { return children_; }
  virtual const char* kind() const = 0;

 protected:
  std::vector<std::unique_ptr<Operator>> children_;
  ExecContext* ctx_ = nullptr;
  bool isInitialized_ = false;
};

// Compiled expression programs kept alive with their constants.
struct ProgramHolder {
  std::vector<yq_insn> code;
  yq_program prog() const { return yq_program{code.empty() ? nullptr : code.data(), (int32_t)code.size()}; }
};
struct ConstantsHolder {
  std::vector<int64_t> values;
  std::vector<char> text;
  int32_t text_count = 0, text_width = 0;
  void assign(const yq_constants* k);
  yq_constants get() const {
    return yq_constants{values.empty() ? nullptr : values.data(), (int32_t)values.size(),
                        text.empty() ? nullptr : text.data(), text_count, text_width};
  }
};

}  // namespace yq::engine
