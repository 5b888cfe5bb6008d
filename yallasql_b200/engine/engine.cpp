// C++ operator layer over the yq kernels (see engine.hpp for the mapping to
// the reference's classes) and its C entry points (include/yq_engine.h).
#include "engine.hpp"

#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <numeric>

namespace yq::engine {

static int32_t width_of(int32_t type, int32_t text_width = 16) {
  switch (type) {
    case YQ_INT32:
    case YQ_FLOAT32: return 4;
    case YQ_INT64:
    case YQ_DATETIME:
    case YQ_FLOAT64: return 8;
    case YQ_BOOL: return 1;
    default: return text_width;
  }
}

// ------------------------------------------------------------------ Batch
Batch::Batch(std::vector<ColumnPtr> cols, uint64_t n, cudaStream_t s, bool with_nulls)
    : columns(std::move(cols)), rows(n), location(Device::GPU), stream(s) {
  data.resize(columns.size(), nullptr);
  nulls.resize(columns.size(), nullptr);
  for (size_t c = 0; c < columns.size(); ++c) {
    const size_t b = std::max<uint64_t>(1, n) * columns[c]->width;
    check_cuda(cudaMallocAsync(&data[c], b, s), "Batch alloc");
    if (with_nulls) check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&nulls[c]), std::max<uint64_t>(1, n), s),
                               "Batch nulls alloc");
  }
}

Batch::~Batch() {
  waitWrite();
  for (size_t c = 0; c < columns.size(); ++c) {
    if (location == Device::GPU) {
      if (data[c]) cudaFreeAsync(data[c], stream);
      if (nulls[c]) cudaFreeAsync(nulls[c], stream);
    } else if (location == Device::CPU) {
      if (data[c]) cudaFreeHost(data[c]);
      if (nulls[c]) cudaFreeHost(nulls[c]);
    }
  }
  if (location == Device::FS && !file_.empty()) std::remove(file_.c_str());
}

uint64_t Batch::bytes() const {
  uint64_t b = 0;
  for (size_t c = 0; c < columns.size(); ++c) b += rows * columns[c]->width + (nullable(c) ? rows : 0);
  return b;
}

// GPU <-> pinned host (Batch::moveGpuToCpu / moveCpuToGpu, src/batch.cu:28-73),
// pinned host <-> file (moveCpuToFs / moveFsToCpu, src/batch.cu:75-110).
void Batch::moveTo(Device target, const std::string& path) {
  if (target == location) return;
  if (location == Device::FS) fsToCpu();
  if (location == Device::GPU && target != Device::GPU) gpuToCpu();
  if (target == Device::GPU && location == Device::CPU) cpuToGpu();
  if (target == Device::FS && location == Device::CPU) cpuToFs(path);
}

void Batch::gpuToCpu() {
  for (size_t c = 0; c < columns.size(); ++c) {
    const size_t b = std::max<uint64_t>(1, rows) * columns[c]->width;
    const size_t nb = std::max<uint64_t>(1, rows);
    void* p = nullptr;
    void* q = nullptr;
    check_cuda(cudaMallocHost(&p, b), "spill alloc");
    check_cuda(cudaMemcpyAsync(p, data[c], b, cudaMemcpyDeviceToHost, stream), "spill copy");
    if (nulls[c]) {
      check_cuda(cudaMallocHost(&q, nb), "spill alloc");
      check_cuda(cudaMemcpyAsync(q, nulls[c], nb, cudaMemcpyDeviceToHost, stream), "spill copy");
    }
    check_cuda(cudaStreamSynchronize(stream), "spill sync");
    cudaFreeAsync(data[c], stream);
    if (nulls[c]) cudaFreeAsync(nulls[c], stream);
    data[c] = p;
    nulls[c] = static_cast<uint8_t*>(q);
  }
  location = Device::CPU;
}

void Batch::cpuToGpu() {
  for (size_t c = 0; c < columns.size(); ++c) {
    const size_t b = std::max<uint64_t>(1, rows) * columns[c]->width;
    const size_t nb = std::max<uint64_t>(1, rows);
    void* p = nullptr;
    void* q = nullptr;
    check_cuda(cudaMallocAsync(&p, b, stream), "reload alloc");
    check_cuda(cudaMemcpyAsync(p, data[c], b, cudaMemcpyHostToDevice, stream), "reload copy");
    if (nulls[c]) {
      check_cuda(cudaMallocAsync(&q, nb, stream), "reload alloc");
      check_cuda(cudaMemcpyAsync(q, nulls[c], nb, cudaMemcpyHostToDevice, stream), "reload copy");
    }
    check_cuda(cudaStreamSynchronize(stream), "reload sync");
    cudaFreeHost(data[c]);
    if (nulls[c]) cudaFreeHost(nulls[c]);
    data[c] = p;
    nulls[c] = static_cast<uint8_t*>(q);
  }
  location = Device::GPU;
}

// File layout: a header (magic, rows, column count, then per column type,
// width and a null flag) followed, per column, by rows * width data bytes and,
// for a nullable column, rows null bytes. The reference writes the data only
// and so loses the null bytes on this tier.
namespace {
constexpr uint64_t kBatchFileMagic = 0x3148435441425159ull;  // "YQBATCH1"
}

void Batch::cpuToFs(const std::string& path) {
  if (path.empty()) throw Error(YQ_ERR_INVALID_ARG, "spill to disk: no cache directory");
  file_ = path;
  std::vector<void*> d = data;
  std::vector<uint8_t*> nl = nulls;
  std::vector<std::pair<int32_t, int32_t>> meta;
  for (auto& c : columns) meta.emplace_back(c->type, c->width);
  const uint64_t n = rows;
  null_flag_.assign(columns.size(), 0);
  // The host buffers now belong to the write task: it frees them once the
  // file is complete (or failed), and the batch forgets them.
  for (size_t c = 0; c < columns.size(); ++c) {
    data[c] = nullptr;
    null_flag_[c] = nulls[c] != nullptr;
    nulls[c] = nullptr;
  }
  location = Device::FS;
  int dev = 0;
  cudaGetDevice(&dev);  // the task frees the host buffers with the caller's device current
  write_ = std::async(std::launch::async, [path, d, nl, meta, n, dev]() -> bool {
    cudaSetDevice(dev);
    bool ok = false;
    if (FILE* f = std::fopen(path.c_str(), "wb")) {
      const uint64_t head[3] = {kBatchFileMagic, n, (uint64_t)meta.size()};
      ok = std::fwrite(head, sizeof(head), 1, f) == 1;
      for (size_t c = 0; ok && c < meta.size(); ++c) {
        const int32_t m[3] = {meta[c].first, meta[c].second, nl[c] != nullptr};
        ok = std::fwrite(m, sizeof(m), 1, f) == 1;
      }
      for (size_t c = 0; ok && c < meta.size(); ++c) {
        const size_t b = std::max<uint64_t>(1, n) * meta[c].second;
        ok = std::fwrite(d[c], 1, b, f) == b;
        if (ok && nl[c]) ok = std::fwrite(nl[c], 1, std::max<uint64_t>(1, n), f) == std::max<uint64_t>(1, n);
      }
      ok = (std::fclose(f) == 0) && ok;
    }
    for (size_t c = 0; c < d.size(); ++c) {
      if (d[c]) cudaFreeHost(d[c]);
      if (nl[c]) cudaFreeHost(nl[c]);
    }
    return ok;
  });
}

void Batch::waitWrite() {
  if (!write_.valid()) return;
  const bool ok = write_.get();
  if (!ok && location == Device::FS) write_failed_ = true;
}

void Batch::fsToCpu() {
  waitWrite();
  if (write_failed_) throw Error(YQ_ERR_CUDA, "spill to disk: writing " + file_ + " failed");
  FILE* f = std::fopen(file_.c_str(), "rb");
  if (!f) throw Error(YQ_ERR_INVALID_ARG, "reload from disk: cannot open " + file_);
  bool ok = true;
  uint64_t head[3] = {0, 0, 0};
  ok = std::fread(head, sizeof(head), 1, f) == 1 && head[0] == kBatchFileMagic && head[1] == rows &&
       head[2] == columns.size();
  std::vector<int32_t> has(columns.size(), 0);
  for (size_t c = 0; ok && c < columns.size(); ++c) {
    int32_t m[3];
    ok = std::fread(m, sizeof(m), 1, f) == 1 && m[0] == columns[c]->type && m[1] == columns[c]->width;
    has[c] = m[2];
  }
  for (size_t c = 0; ok && c < columns.size(); ++c) {
    const size_t b = std::max<uint64_t>(1, rows) * columns[c]->width;
    const size_t nb = std::max<uint64_t>(1, rows);
    void* p = nullptr;
    check_cuda(cudaMallocHost(&p, b), "reload alloc");
    data[c] = p;
    ok = std::fread(p, 1, b, f) == b;
    if (ok && has[c]) {
      void* q = nullptr;
      check_cuda(cudaMallocHost(&q, nb), "reload alloc");
      nulls[c] = static_cast<uint8_t*>(q);
      ok = std::fread(q, 1, nb, f) == nb;
    }
  }
  std::fclose(f);
  location = Device::CPU;  // buffers read so far are freed as host memory by the destructor
  null_flag_.clear();
  const std::string name = file_;
  std::remove(file_.c_str());
  file_.clear();
  if (!ok) throw Error(YQ_ERR_INVALID_ARG, "reload from disk: " + name + " is truncated or not this batch");
}

yq_column Batch::column(size_t c) const {
  return yq_column{data[c], nulls[c], columns[c]->type, columns[c]->width};
}

yq_batch Batch::view(std::vector<yq_column>& storage) const {
  storage.clear();
  for (size_t c = 0; c < columns.size(); ++c) storage.push_back(column(c));
  return yq_batch{storage.data(), (int32_t)storage.size(), (uint32_t)rows};
}

// ----------------------------------------------------------- CacheManager
BatchID CacheManager::putBatch(std::unique_ptr<Batch> b) {
  const BatchID id = next_++;
  if (b->location == Device::GPU) gpu_bytes_ += b->bytes();
  else if (b->location == Device::CPU) host_bytes_ += b->bytes();
  batches_[id] = std::move(b);
  handleOverflow();
  return id;
}

std::unique_ptr<Batch> CacheManager::getBatch(BatchID id) {
  auto it = batches_.find(id);
  if (it == batches_.end()) throw Error(YQ_ERR_INVALID_ARG, "getBatch: unknown batch");
  std::unique_ptr<Batch> b = std::move(it->second);
  batches_.erase(it);
  const uint64_t bytes = b->bytes();
  if (b->location == Device::GPU) gpu_bytes_ -= std::min(gpu_bytes_, bytes);
  else if (b->location == Device::CPU) host_bytes_ -= std::min(host_bytes_, bytes);
  b->moveTo(Device::GPU);
  return b;
}

Batch& CacheManager::refBatch(BatchID id) { return *batches_.at(id); }

std::string CacheManager::filePath(BatchID id) const {
  static std::atomic<uint64_t> seq{0};
  return dir_ + "/yq_batch_" + std::to_string((unsigned long)getpid()) + "_" +
         std::to_string((unsigned long long)seq.fetch_add(1)) + "_" + std::to_string((unsigned long long)id) + ".bin";
}

void CacheManager::handleOverflow() {
  // Oldest device batches (lowest id) move to pinned host memory first ...
  for (auto& kv : batches_) {
    if (gpu_bytes_ <= budget_) break;
    Batch& b = *kv.second;
    if (b.location != Device::GPU) continue;
    const uint64_t bytes = b.bytes();
    b.moveTo(Device::CPU);
    gpu_bytes_ -= std::min(gpu_bytes_, bytes);
    host_bytes_ += bytes;
    ++spilled_;
  }
  // ... and the oldest host batches to files when host memory is over its budget.
  if (host_budget_ == 0 || dir_.empty()) return;
  for (auto& kv : batches_) {
    if (host_bytes_ <= host_budget_) break;
    Batch& b = *kv.second;
    if (b.location != Device::CPU) continue;
    const uint64_t bytes = b.bytes();
    b.moveTo(Device::FS, filePath(kv.first));
    host_bytes_ -= std::min(host_bytes_, bytes);
    ++disk_;
  }
}

void ConstantsHolder::assign(const yq_constants* k) {
  values.clear();
  text.clear();
  text_count = text_width = 0;
  if (!k) return;
  if (k->count > 0) values.assign(k->values, k->values + k->count);
  if (k->text_count > 0) {
    text.assign(k->text, k->text + (size_t)k->text_count * k->text_width);
    text_count = k->text_count;
    text_width = k->text_width;
  }
}

static ProgramHolder hold(const yq_program* p) {
  ProgramHolder h;
  if (p && p->len > 0) h.code.assign(p->code, p->code + p->len);
  return h;
}

// ------------------------------------------------------------ ScanOperator
// Streams host columns to the device in batches. Pageable host memory is
// first copied into one of two pinned staging sets; the H2D copy runs on the
// copy stream and the compute stream waits on an event, so the copy of the
// next batch overlaps the kernels of the current one.
class ScanOperator final : public Operator {
 public:
  ScanOperator(const yq_host_column* cols, int ncols, uint64_t rows, uint32_t batch_rows)
      : host_(cols, cols + ncols), rows_(rows) {
    uint64_t row_bytes = 0;
    for (auto& c : host_) {
      columns.push_back(std::make_shared<Column>(Column{c.type, c.width}));
      row_bytes += c.width;
    }
    if (batch_rows) {
      batch_rows_ = batch_rows;
    } else {  // calculateOptimalBatchSize (include/config.hpp:28-36)
      const uint64_t per = (4ull << 20) / std::max<uint64_t>(1, row_bytes);
      batch_rows_ = std::max<uint64_t>(256, per / 256 * 256);
    }
    pinned_ = true;
    for (auto& c : host_) {
      cudaPointerAttributes a{};
      if (cudaPointerGetAttributes(&a, c.data) != cudaSuccess || a.type != cudaMemoryTypeHost) pinned_ = false;
      if (c.nulls && (cudaPointerGetAttributes(&a, c.nulls) != cudaSuccess || a.type != cudaMemoryTypeHost))
        pinned_ = false;
    }
    cudaGetLastError();
  }
  ~ScanOperator() override {
    for (int s = 0; s < 2; ++s) {
      for (auto* p : stage_[s]) cudaFreeHost(p);
      if (done_[s]) cudaEventDestroy(done_[s]);
    }
  }
  const char* kind() const override { return "scan"; }
  void init() override {
    if (isInitialized_) return;
    for (int s = 0; s < 2; ++s) {
      check_cuda(cudaEventCreateWithFlags(&done_[s], cudaEventDisableTiming), "scan event");
      if (!pinned_) {
        for (size_t c = 0; c < host_.size(); ++c) {
          void* p = nullptr;
          check_cuda(cudaMallocHost(&p, batch_rows_ * host_[c].width + (host_[c].nulls ? batch_rows_ : 0)), "stage");
          stage_[s].push_back(static_cast<char*>(p));
        }
      }
    }
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (issued_ == 0) {
      issue();
      issue();
    }
    if (taken_ == issued_) {
      isFinished = true;
      return 0;
    }
    const int slot = taken_ % 2;
    std::unique_ptr<Batch> b = std::move(pending_[slot]);
    check_cuda(cudaStreamWaitEvent(ctx_->compute, done_[slot], 0), "scan wait");
    b->stream = ctx_->compute;
    ++taken_;
    ++ctx_->stats.batches;
    const BatchID id = cache.putBatch(std::move(b));
    issue();  // refill the freed slot: its copy overlaps the consumer's kernels
    return id;
  }

 private:
  void issue() {
    if (pos_ >= rows_) return;
    const int slot = issued_ % 2;
    const uint64_t n = std::min<uint64_t>(batch_rows_, rows_ - pos_);
    bool any_nulls = false;
    for (auto& c : host_) any_nulls |= c.nulls != nullptr;
    auto b = std::make_unique<Batch>(columns, n, ctx_->copy, any_nulls);
    if (!pinned_) check_cuda(cudaEventSynchronize(done_[slot]), "stage reuse");  // staging set free again
    for (size_t c = 0; c < host_.size(); ++c) {
      const size_t w = host_[c].width;
      const char* src = static_cast<const char*>(host_[c].data) + pos_ * w;
      const uint8_t* nsrc = host_[c].nulls ? host_[c].nulls + pos_ : nullptr;
      if (!pinned_) {
        memcpy(stage_[slot][c], src, n * w);
        if (nsrc) memcpy(stage_[slot][c] + batch_rows_ * w, nsrc, n);
        src = stage_[slot][c];
        if (nsrc) nsrc = reinterpret_cast<uint8_t*>(stage_[slot][c] + batch_rows_ * w);
      }
      check_cuda(cudaMemcpyAsync(b->data[c], src, n * w, cudaMemcpyHostToDevice, ctx_->copy), "scan H2D");
      ctx_->stats.h2d_bytes += n * w;
      if (b->nulls[c]) {
        if (nsrc) {
          check_cuda(cudaMemcpyAsync(b->nulls[c], nsrc, n, cudaMemcpyHostToDevice, ctx_->copy), "scan H2D");
          ctx_->stats.h2d_bytes += n;
        } else {
          check_cuda(cudaMemsetAsync(b->nulls[c], 0, n, ctx_->copy), "scan nulls");
        }
      }
    }
    check_cuda(cudaEventRecord(done_[slot], ctx_->copy), "scan record");
    pending_[slot] = std::move(b);
    pos_ += n;
    ++issued_;
  }

  std::vector<yq_host_column> host_;
  uint64_t rows_, batch_rows_ = 0, pos_ = 0;
  bool pinned_ = false;
  std::vector<char*> stage_[2];
  cudaEvent_t done_[2] = {nullptr, nullptr};
  std::unique_ptr<Batch> pending_[2];
  uint64_t issued_ = 0, taken_ = 0;
};

// --------------------------------------------------------- CsvScanOperator
// GetOperator (src/engine/operators/get_operator.cpp:17-109) over CSV text:
// the file's body (header line removed) goes to the device once, one record
// index splits it (yq_csv_index), and each next() converts the next batch of
// records into a Batch (yq_csv_parse) instead of the reference's host
// csv-parser loop and per-column synchronous copies. Batch rows follow
// calculateOptimalBatchSize over the projected columns (include/config.hpp:28-36).
// A cell that std::stoi / std::stof would reject raises YQ_ERR_INVALID_ARG
// (the reference's process exits there).
class CsvScanOperator final : public Operator {
 public:
  CsvScanOperator(const uint8_t* text, uint64_t nbytes, const int32_t* types, int nfields, const int32_t* project,
                  int nproj, int32_t text_width, uint32_t batch_rows)
      : host_(text), nbytes_(nbytes), types_(types, types + nfields), project_(project, project + nproj) {
    uint64_t row_bytes = 0;
    field_col_.assign(nfields, -1);
    for (int i = 0; i < nproj; ++i) {
      const int f = project_[i];
      if (f < 0 || f >= nfields || field_col_[f] >= 0) throw Error(YQ_ERR_INVALID_ARG, "csv projection");
      field_col_[f] = i;
      const int32_t w = width_of(types_[f], text_width);
      columns.push_back(std::make_shared<Column>(Column{types_[f], w}));
      row_bytes += w;
    }
    if (batch_rows) {
      batch_rows_ = batch_rows;
    } else {
      const uint64_t per = (4ull << 20) / std::max<uint64_t>(1, row_bytes);
      batch_rows_ = std::max<uint64_t>(256, per / 256 * 256);
    }
  }
  ~CsvScanOperator() override {
    if (text_) cudaFree(text_);
    if (starts_) cudaFree(starts_);
  }
  const char* kind() const override { return "csv_scan"; }
  void init() override {
    if (isInitialized_) return;
    if (nbytes_) {
      check_cuda(cudaMalloc(&text_, nbytes_), "csv text");
      check_cuda(cudaMemcpyAsync(text_, host_, nbytes_, cudaMemcpyHostToDevice, ctx_->compute), "csv H2D");
      ctx_->stats.h2d_bytes += nbytes_;
      uint64_t n = 0;
      int st = yq_csv_index(text_, nbytes_, nullptr, 0, &n, nullptr, 0, ctx_->compute);
      if (st != YQ_OK && st != YQ_ERR_CAPACITY) check(st, "yq_csv_index");
      records_ = n;
      check_cuda(cudaMalloc(&starts_, std::max<uint64_t>(1, n) * sizeof(uint32_t)), "csv record starts");
      check(yq_csv_index(text_, nbytes_, starts_, n, &n, nullptr, 0, ctx_->compute), "yq_csv_index");
    }
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (isFinished || pos_ >= records_) {
      isFinished = true;
      return 0;
    }
    const uint64_t n = std::min<uint64_t>(batch_rows_, records_ - pos_);
    // records [pos_, pos_+n) end where the next one starts (or at the end of the text)
    uint64_t end = nbytes_;
    if (pos_ + n < records_) {
      uint32_t e = 0;
      check_cuda(cudaMemcpyAsync(&e, starts_ + pos_ + n, sizeof(e), cudaMemcpyDeviceToHost, ctx_->compute), "csv end");
      check_cuda(cudaStreamSynchronize(ctx_->compute), "csv end");
      end = e;
    }
    auto b = std::make_unique<Batch>(columns, n, ctx_->compute, true);
    std::vector<yq_column> out(columns.size());
    for (size_t c = 0; c < columns.size(); ++c) out[c] = b->column(c);
    uint32_t rows = 0;
    yq_csv_error err{};
    const int st = yq_csv_parse(text_, end, starts_ + pos_, (uint32_t)n, field_col_.data(), (int32_t)types_.size(),
                                out.data(), (int32_t)out.size(), &rows, &err, nullptr, 0, ctx_->compute);
    if (st != YQ_OK) {
      if (st == YQ_ERR_INVALID_ARG && err.bad_cells)
        throw Error(st, "csv scan: a field std::stoi/std::stof rejects, batch row " + std::to_string(err.first_row) +
                            ", field " + std::to_string(err.first_field));
      check(st, "yq_csv_parse");
    }
    b->rows = rows;  // rows with another field count are dropped (csv-parser IGNORE_ROW)
    pos_ += n;
    ++ctx_->stats.batches;
    return cache.putBatch(std::move(b));
  }

 private:
  const uint8_t* host_;
  uint64_t nbytes_;
  std::vector<int32_t> types_, project_, field_col_;
  uint64_t batch_rows_ = 0, records_ = 0, pos_ = 0;
  uint8_t* text_ = nullptr;
  uint32_t* starts_ = nullptr;
};

static bool has_nulls(const Batch& b) {
  for (auto* n : b.nulls)
    if (n) return true;
  return false;
}

// ---------------------------------------------------------- FilterOperator
class FilterOperator final : public Operator {
 public:
  FilterOperator(std::unique_ptr<Operator> child, const yq_program* pred, const yq_constants* k) : pred_(hold(pred)) {
    children_.push_back(std::move(child));
    consts_.assign(k);
  }
  const char* kind() const override { return "filter"; }
  void init() override {
    if (isInitialized_) return;
    children_[0]->init();
    columns = children_[0]->columns;
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (isFinished) return 0;
    const BatchID id = children_[0]->next(cache);
    if (!id) {
      isFinished = true;
      return 0;
    }
    auto in = cache.getBatch(id);
    if (pred_.code.empty()) return cache.putBatch(std::move(in));
    std::vector<yq_column> iv;
    const yq_batch v = in->view(iv);
    auto out = std::make_unique<Batch>(columns, in->rows, ctx_->compute, has_nulls(*in));
    std::vector<yq_projection> proj(columns.size());
    std::vector<yq_column> ov(columns.size());
    for (size_t c = 0; c < columns.size(); ++c) {
      proj[c].column = (int32_t)c;
      ov[c] = out->column(c);
    }
    const yq_program p = pred_.prog();
    const yq_constants k = consts_.get();
    uint32_t count = 0;
    check(yq_filter_project(&v, &p, &k, proj.data(), (int32_t)proj.size(), ov.data(), (uint32_t)in->rows, nullptr,
                            &count, nullptr, 0, ctx_->compute),
          "FilterOperator");
    out->rows = count;
    return cache.putBatch(std::move(out));
  }
  // AggregateOperator absorbs this node: its predicate is evaluated inside the
  // aggregate kernel on the child's batches instead of compacting them first.
  const ProgramHolder& predicate() const { return pred_; }
  const ConstantsHolder& constants() const { return consts_; }

 private:
  ProgramHolder pred_;
  ConstantsHolder consts_;
};

// ------------------------------------------------------ ProjectionOperator
class ProjectionOperator final : public Operator {
 public:
  ProjectionOperator(std::unique_ptr<Operator> child, const yq_projection* proj, int nproj, const yq_constants* k) {
    children_.push_back(std::move(child));
    consts_.assign(k);
    for (int i = 0; i < nproj; ++i) {
      proj_.push_back(proj[i]);
      progs_.push_back(hold(&proj[i].program));
    }
  }
  const char* kind() const override { return "projection"; }
  void init() override {
    if (isInitialized_) return;
    children_[0]->init();
    for (auto& p : proj_) {
      if (p.column >= 0) columns.push_back(children_[0]->columns.at(p.column));
      else columns.push_back(std::make_shared<Column>(Column{p.out_type, width_of(p.out_type)}));
    }
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (isFinished) return 0;
    const BatchID id = children_[0]->next(cache);
    if (!id) {
      isFinished = true;
      return 0;
    }
    auto in = cache.getBatch(id);
    std::vector<yq_column> iv;
    const yq_batch v = in->view(iv);
    auto out = std::make_unique<Batch>(columns, in->rows, ctx_->compute, true);
    std::vector<yq_projection> proj = proj_;
    for (size_t i = 0; i < proj.size(); ++i) proj[i].program = progs_[i].prog();
    std::vector<yq_column> ov;
    for (size_t c = 0; c < columns.size(); ++c) ov.push_back(out->column(c));
    const yq_program none{nullptr, 0};
    const yq_constants k = consts_.get();
    uint32_t count = 0;
    check(yq_filter_project(&v, &none, &k, proj.data(), (int32_t)proj.size(), ov.data(), (uint32_t)in->rows, nullptr,
                            &count, nullptr, 0, ctx_->compute),
          "ProjectionOperator");
    out->rows = count;
    return cache.putBatch(std::move(out));
  }

 private:
  std::vector<yq_projection> proj_;
  std::vector<ProgramHolder> progs_;
  ConstantsHolder consts_;
};

// ------------------------------------------------------- AggregateOperator
class AggregateOperator final : public Operator {
 public:
  AggregateOperator(std::unique_ptr<Operator> child, const yq_agg_spec* aggs, int nagg, const yq_constants* k) {
    children_.push_back(std::move(child));
    consts_.assign(k);
    for (int i = 0; i < nagg; ++i) {
      aggs_.push_back(aggs[i]);
      progs_.push_back(hold(&aggs[i].input));
    }
  }
  const char* kind() const override { return "aggregate"; }
  void init() override {
    if (isInitialized_) return;
    Operator* c = children_[0].get();
    c->init();
    source_ = c;
    if (auto* f = dynamic_cast<FilterOperator*>(c)) {
      // Fuse WHERE into the aggregate: merge the filter's constants in front
      // of ours and shift our constant indices.
      pred_ = f->predicate();
      ConstantsHolder merged = f->constants();
      const int shift = (int)merged.values.size();
      const int tshift = merged.text_count;
      if (!consts_.text.empty() && !merged.text.empty() && consts_.text_width != merged.text_width)
        throw Error(YQ_ERR_UNSUPPORTED, "AggregateOperator: text constant widths differ");
      merged.values.insert(merged.values.end(), consts_.values.begin(), consts_.values.end());
      merged.text.insert(merged.text.end(), consts_.text.begin(), consts_.text.end());
      merged.text_count += consts_.text_count;
      if (!merged.text_width) merged.text_width = consts_.text_width;
      for (auto& p : progs_)
        for (auto& I : p.code) {
          const bool num = I.op == YQ_OP_CONST || I.op == YQ_OP_ARITH_CONST ||
                           ((I.op == YQ_OP_CMP_COL_CONST || I.op == YQ_OP_AND_CMP_COL_CONST) && I.type != YQ_TEXT);
          const bool txt = (I.op == YQ_OP_CMP_COL_CONST || I.op == YQ_OP_AND_CMP_COL_CONST) && I.type == YQ_TEXT;
          if (num) I.imm += shift;
          if (txt) I.imm += tshift;
        }
      consts_ = merged;
      source_ = f->child(0);
    }
    for (auto& a : aggs_) {
      int32_t t;
      switch (a.kind) {
        case YQ_AGG_COUNT_STAR:
        case YQ_AGG_COUNT: t = YQ_INT64; break;
        case YQ_AGG_AVG: t = YQ_FLOAT64; break;
        case YQ_AGG_SUM: t = (a.input_type == YQ_FLOAT32 || a.input_type == YQ_FLOAT64) ? YQ_FLOAT64 : YQ_INT64; break;
        default: t = a.input_type;
      }
      columns.push_back(std::make_shared<Column>(Column{t, width_of(t)}));
    }
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (isFinished) return 0;
    isFinished = true;
    const int nagg = (int)aggs_.size();
    std::vector<yq_agg_spec> specs = aggs_;
    for (int i = 0; i < nagg; ++i) specs[i].input = progs_[i].prog();
    void* state = nullptr;
    check_cuda(cudaMallocAsync(&state, std::max<size_t>(256, yq_agg_state_bytes(nagg)), ctx_->compute), "agg state");
    check(yq_agg_state_init(state, specs.data(), nagg, ctx_->compute), "yq_agg_state_init");
    const yq_program p = pred_.prog();
    const yq_constants k = consts_.get();
    for (BatchID id = source_->next(cache); id; id = source_->next(cache)) {
      auto in = cache.getBatch(id);
      std::vector<yq_column> iv;
      const yq_batch v = in->view(iv);
      check(yq_filter_aggregate(&v, &p, &k, specs.data(), nagg, state, nullptr, 0, ctx_->compute),
            "AggregateOperator");
    }
    std::vector<yq_agg_result> res(nagg);
    check(yq_agg_state_read(state, specs.data(), nagg, res.data(), ctx_->compute), "yq_agg_state_read");
    cudaFreeAsync(state, ctx_->compute);
    // One result row (SQL semantics over an empty input: counts 0, others NULL).
    auto out = std::make_unique<Batch>(columns, 1, ctx_->compute, true);
    for (int i = 0; i < nagg; ++i) {
      unsigned char cell[8] = {0};
      const int32_t t = columns[i]->type;
      const yq_agg_result& r = res[i];
      switch (t) {
        case YQ_INT32: { int32_t v = (int32_t)r.i; memcpy(cell, &v, 4); break; }
        case YQ_FLOAT32: { float v = (float)r.f; memcpy(cell, &v, 4); break; }
        case YQ_FLOAT64: { double v = r.f; memcpy(cell, &v, 8); break; }
        default: { int64_t v = r.i; memcpy(cell, &v, 8); break; }
      }
      uint8_t nul = (uint8_t)r.is_null;
      check_cuda(cudaMemcpyAsync(out->data[i], cell, columns[i]->width, cudaMemcpyHostToDevice, ctx_->compute),
                 "agg result");
      check_cuda(cudaMemcpyAsync(out->nulls[i], &nul, 1, cudaMemcpyHostToDevice, ctx_->compute), "agg result");
      check_cuda(cudaStreamSynchronize(ctx_->compute), "agg result");
    }
    return cache.putBatch(std::move(out));
  }

 private:
  std::vector<yq_agg_spec> aggs_;
  std::vector<ProgramHolder> progs_;
  ProgramHolder pred_;
  ConstantsHolder consts_;
  Operator* source_ = nullptr;
};

// Every batch of `child` back to back in one device batch (the merge path and
// the sort-based GROUP BY read contiguous rows); run r of the result is rows
// [offs[r], offs[r+1]) and holds child batch r.
static std::unique_ptr<Batch> collect_runs(Operator* child, CacheManager& cache, const std::vector<ColumnPtr>& columns,
                                           cudaStream_t s, std::vector<uint32_t>& offs) {
  std::vector<std::unique_ptr<Batch>> runs;
  uint64_t total = 0;
  bool nullable = false;
  for (BatchID id = child->next(cache); id; id = child->next(cache)) {
    auto b = cache.getBatch(id);
    if (b->rows == 0) continue;
    total += b->rows;
    nullable |= has_nulls(*b);
    runs.push_back(std::move(b));
  }
  offs.assign(1, 0u);
  if (runs.empty()) return nullptr;
  if (total > 0xffffffffull) throw Error(YQ_ERR_UNSUPPORTED, "more than 2^32 rows in one sorted table");
  auto all = std::make_unique<Batch>(columns, total, s, nullable);
  for (auto& r : runs) {
    const uint64_t o = offs.back();
    for (size_t c = 0; c < columns.size(); ++c) {
      const size_t w = columns[c]->width;
      check_cuda(cudaMemcpyAsync((char*)all->data[c] + o * w, r->data[c], r->rows * w, cudaMemcpyDeviceToDevice, s),
                 "concat");
      if (all->nulls[c]) {
        if (r->nulls[c])
          check_cuda(cudaMemcpyAsync(all->nulls[c] + o, r->nulls[c], r->rows, cudaMemcpyDeviceToDevice, s), "concat");
        else
          check_cuda(cudaMemsetAsync(all->nulls[c] + o, 0, r->rows, s), "concat");
      }
    }
    offs.push_back((uint32_t)(o + r->rows));
  }
  return all;
}

// ----------------------------------------------------------- OrderOperator
// Every child batch becomes a run; yq_order_by sorts the runs (segmented radix
// sort), merges them pairwise by merge path until one remains and gathers the
// rows (OrderOperator::firstPass / merge_all_sorted, order_operator.hpp:89-193).
// The reference sorts by its first ORDER BY key only (`orders[0]`,
// order_operator.hpp:277); here every key counts: with more than one key (or a
// text key longer than the merge path's 32-byte key) the concatenated runs are
// sorted at once by all keys (stable LSD over the keys, yq_sort_indices_multi)
// and gathered.
class OrderOperator final : public Operator {
 public:
  OrderOperator(std::unique_ptr<Operator> child, std::vector<int32_t> keys, std::vector<int32_t> desc,
                std::vector<int32_t> nulls_first)
      : keys_(std::move(keys)), desc_(std::move(desc)), nulls_first_(std::move(nulls_first)) {
    children_.push_back(std::move(child));
  }
  const char* kind() const override { return "order"; }
  void init() override {
    if (isInitialized_) return;
    children_[0]->init();
    columns = children_[0]->columns;
    if (keys_.empty() || keys_.size() > YQ_MAX_BATCH_COLUMNS) throw Error(YQ_ERR_INVALID_ARG, "OrderOperator keys");
    for (int k : keys_)
      if (k < 0 || k >= (int)columns.size()) throw Error(YQ_ERR_INVALID_ARG, "OrderOperator key");
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (isFinished) return 0;
    isFinished = true;
    cudaStream_t s = ctx_->compute;
    std::vector<uint32_t> offs;
    auto all = collect_runs(children_[0].get(), cache, columns, s, offs);
    if (!all) return 0;
    const uint64_t total = all->rows;
    const bool nullable = has_nulls(*all);
    std::vector<yq_column> av, rv;
    all->view(av);
    auto result = std::make_unique<Batch>(columns, total, s, nullable);
    result->view(rv);
    yq_batch ib{av.data(), (int32_t)av.size(), (uint32_t)total};
    yq_batch ob{rv.data(), (int32_t)rv.size(), (uint32_t)total};
    int st = YQ_ERR_UNSUPPORTED;
    if (keys_.size() == 1)  // sort every run, merge (key words, row id) level by level, gather once
      st = yq_order_by(&ib, keys_[0], desc_[0], nulls_first_[0], offs.data(), (int32_t)offs.size() - 1, &ob, nullptr,
                       0, s);
    if (st == YQ_ERR_UNSUPPORTED) {
      std::vector<yq_column> kc;
      for (int k : keys_) kc.push_back(av[k]);
      uint32_t* perm = nullptr;
      check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&perm), total * sizeof(uint32_t), s), "order perm");
      st = yq_sort_indices_multi(kc.data(), desc_.data(), nulls_first_.data(), (int32_t)kc.size(), (uint32_t)total,
                                 perm, nullptr, nullptr, 0, s);
      if (st == YQ_OK) st = yq_gather(av.data(), (int32_t)av.size(), perm, (uint32_t)total, rv.data(), s);
      cudaFreeAsync(perm, s);
    }
    check(st, "OrderOperator");
    return cache.putBatch(std::move(result));
  }

 private:
  std::vector<int32_t> keys_, desc_, nulls_first_;
};

// --------------------------------------------------------- GroupByOperator
// SELECT key, aggregates ... GROUP BY key. The reference's AggregateOperator
// ignores the groups and folds every row into one result
// (include/engine/operators/aggregate_operator.hpp:84-104); this operator
// returns one row per distinct key in ascending key order (NULL group last)
// with SQL aggregate semantics (yq_group_by): the child's batches are
// concatenated and grouped in one call.
class GroupByOperator final : public Operator {
 public:
  GroupByOperator(std::unique_ptr<Operator> child, int key, const yq_group_agg* aggs, int nagg)
      : key_(key), aggs_(aggs, aggs + nagg) {
    children_.push_back(std::move(child));
  }
  const char* kind() const override { return "group_by"; }
  void init() override {
    if (isInitialized_) return;
    children_[0]->init();
    const auto& in = children_[0]->columns;
    if (key_ < 0 || key_ >= (int)in.size() || aggs_.size() > YQ_MAX_AGGREGATES)
      throw Error(YQ_ERR_INVALID_ARG, "GroupByOperator");
    columns.push_back(in[key_]);
    for (const auto& a : aggs_) {
      if (a.kind != YQ_AGG_COUNT_STAR && (a.column < 0 || a.column >= (int)in.size()))
        throw Error(YQ_ERR_INVALID_ARG, "GroupByOperator aggregate column");
      const int32_t it = a.kind == YQ_AGG_COUNT_STAR ? YQ_INT64 : in[a.column]->type;
      int32_t t;
      switch (a.kind) {
        case YQ_AGG_COUNT_STAR:
        case YQ_AGG_COUNT: t = YQ_INT64; break;
        case YQ_AGG_AVG: t = YQ_FLOAT64; break;
        case YQ_AGG_SUM: t = (it == YQ_FLOAT32 || it == YQ_FLOAT64) ? YQ_FLOAT64 : YQ_INT64; break;
        default: t = it;
      }
      columns.push_back(std::make_shared<Column>(Column{t, width_of(t)}));
    }
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (isFinished) return 0;
    isFinished = true;
    cudaStream_t s = ctx_->compute;
    std::vector<uint32_t> offs;
    auto all = collect_runs(children_[0].get(), cache, children_[0]->columns, s, offs);
    if (!all) return 0;
    const uint64_t total = all->rows;
    std::vector<yq_column> av, rv;
    all->view(av);
    // at most one group per row: outputs sized for every row, trimmed to the group count
    auto result = std::make_unique<Batch>(columns, total, s, true);
    result->view(rv);
    yq_batch ib{av.data(), (int32_t)av.size(), (uint32_t)total};
    uint32_t groups = 0;
    check(yq_group_by(&ib, key_, aggs_.data(), (int32_t)aggs_.size(), rv.data(), (uint32_t)total, &groups, nullptr, 0,
                      s),
          "GroupByOperator");
    result->rows = groups;
    return cache.putBatch(std::move(result));
  }

 private:
  int key_;
  std::vector<yq_group_agg> aggs_;
};

// ---------------------------------------- JoinOperator / CrossProductOperator
// All left batches are cached first; then every right batch meets every left
// batch (JoinOperator::next, join_operator.hpp:36-100). Each pair of batches
// yields one output batch with all left columns followed by all right columns.
class JoinOperator final : public Operator {
 public:
  JoinOperator(std::unique_ptr<Operator> l, std::unique_ptr<Operator> r, const yq_join_cond* conds, int ncond,
               const int32_t* disjunct = nullptr)
      : conds_(conds, conds + ncond) {
    if (disjunct) disjunct_.assign(disjunct, disjunct + ncond);
    children_.push_back(std::move(l));
    children_.push_back(std::move(r));
  }
  const char* kind() const override { return conds_.empty() ? "cross_product" : "join"; }
  void init() override {
    if (isInitialized_) return;
    children_[0]->init();
    children_[1]->init();
    columns = children_[0]->columns;
    columns.insert(columns.end(), children_[1]->columns.begin(), children_[1]->columns.end());
    isInitialized_ = true;
  }
  BatchID next(CacheManager& cache) override {
    if (!isInitialized_) init();
    if (isFinished) return 0;
    if (!cached_) {
      for (BatchID id = children_[0]->next(cache); id; id = children_[0]->next(cache)) left_.push_back(id);
      cached_ = true;
    }
    for (;;) {
      if (!right_ || li_ >= left_.size()) {
        if (right_) right_.reset();
        const BatchID rid = children_[1]->next(cache);
        if (!rid || left_.empty()) {
          isFinished = true;
          return 0;
        }
        right_ = cache.getBatch(rid);
        li_ = 0;
      }
      auto lb = cache.getBatch(left_[li_]);
      BatchID out = join_pair(*lb, *right_, cache);
      left_[li_] = cache.putBatch(std::move(lb));
      ++li_;
      if (out) return out;
    }
  }

 private:
  BatchID join_pair(const Batch& l, const Batch& r, CacheManager& cache) {
    std::vector<yq_column> lv, rv;
    const yq_batch L = l.view(lv), R = r.view(rv);
    std::vector<yq_join_output> outs;
    for (size_t c = 0; c < l.columns.size(); ++c) outs.push_back({0, (int32_t)c});
    for (size_t c = 0; c < r.columns.size(); ++c) outs.push_back({1, (int32_t)c});
    const bool nullable = has_nulls(l) || has_nulls(r);
    uint64_t cap = conds_.empty() ? l.rows * r.rows : std::max<uint64_t>(1, l.rows * 2);
    for (int attempt = 0; attempt < 2; ++attempt) {
      auto out = std::make_unique<Batch>(columns, cap, ctx_->compute, nullable);
      std::vector<yq_column> ov;
      out->view(ov);
      uint64_t count = 0;
      const int st =
          disjunct_.empty()
              ? yq_join_project(&L, &R, conds_.data(), (int32_t)conds_.size(), outs.data(), (int32_t)outs.size(),
                                ov.data(), cap, &count, nullptr, 0, ctx_->compute)
              : yq_join_project_or(&L, &R, conds_.data(), disjunct_.data(), (int32_t)conds_.size(), outs.data(),
                                   (int32_t)outs.size(), ov.data(), cap, &count, nullptr, 0, ctx_->compute);
      if (st == YQ_ERR_CAPACITY) {
        cap = count;
        continue;
      }
      check(st, "JoinOperator");
      if (count == 0) return 0;
      out->rows = count;
      return cache.putBatch(std::move(out));
    }
    throw Error(YQ_ERR_CAPACITY, "JoinOperator");
  }

  std::vector<yq_join_cond> conds_;
  std::vector<int32_t> disjunct_;  // empty: all conditions ANDed
  std::vector<BatchID> left_;
  bool cached_ = false;
  std::unique_ptr<Batch> right_;
  size_t li_ = 0;
};

}  // namespace yq::engine

// ================================================================== C API
using namespace yq::engine;

struct yq_plan {
  std::vector<std::unique_ptr<Operator>> owned;  // nodes not yet attached to a parent
  std::vector<Operator*> nodes;
  ExecContext ctx;
  uint64_t budget;
  uint64_t host_budget = 0;
  std::string cache_dir;
};

struct yq_result {
  uint64_t rows = 0;
  std::vector<yq_host_column> cols;
  std::vector<void*> bufs;
  ~yq_result() {
    for (void* p : bufs) cudaFreeHost(p);
  }
};

namespace {

template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const Error& e) {
    return -e.status;
  } catch (const std::exception&) {
    return -YQ_ERR_INVALID_ARG;
  }
}

std::unique_ptr<Operator> take(yq_plan* p, int id) {
  if (id < 0 || id >= (int)p->nodes.size()) throw Error(YQ_ERR_INVALID_ARG, "unknown node");
  for (auto& o : p->owned)
    if (o.get() == p->nodes[id]) {
      std::unique_ptr<Operator> r = std::move(o);
      p->owned.erase(std::remove(p->owned.begin(), p->owned.end(), nullptr), p->owned.end());
      return r;
    }
  throw Error(YQ_ERR_INVALID_ARG, "node already has a parent");
}

int add(yq_plan* p, std::unique_ptr<Operator> op) {
  p->nodes.push_back(op.get());
  p->owned.push_back(std::move(op));
  return (int)p->nodes.size() - 1;
}

}  // namespace

extern "C" {

yq_plan* yq_plan_create(uint64_t gpu_budget_bytes) {
  auto* p = new yq_plan();
  p->budget = gpu_budget_bytes ? gpu_budget_bytes : (1ull << 30);
  if (cudaStreamCreateWithFlags(&p->ctx.compute, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&p->ctx.copy, cudaStreamNonBlocking) != cudaSuccess) {
    delete p;
    return nullptr;
  }
  return p;
}

int yq_plan_set_spill(yq_plan* p, uint64_t host_budget_bytes, const char* cache_dir) {
  if (!p || (host_budget_bytes && (!cache_dir || !*cache_dir))) return YQ_ERR_INVALID_ARG;
  p->host_budget = host_budget_bytes;
  p->cache_dir = host_budget_bytes ? std::string(cache_dir) : std::string();
  return YQ_OK;
}

void yq_plan_destroy(yq_plan* p) {
  if (!p) return;
  cudaStreamSynchronize(p->ctx.compute);
  cudaStreamSynchronize(p->ctx.copy);
  p->owned.clear();
  cudaStreamDestroy(p->ctx.compute);
  cudaStreamDestroy(p->ctx.copy);
  delete p;
}

int yq_plan_scan(yq_plan* p, const yq_host_column* cols, int32_t ncols, uint64_t rows, uint32_t batch_rows) {
  if (!p || !cols || ncols <= 0 || ncols > YQ_MAX_BATCH_COLUMNS) return -YQ_ERR_INVALID_ARG;
  return guarded([&] { return add(p, std::make_unique<ScanOperator>(cols, ncols, rows, batch_rows)); });
}

int yq_plan_scan_csv(yq_plan* p, const uint8_t* text, uint64_t nbytes, const int32_t* field_types,
                     int32_t nfields, const int32_t* project, int32_t nproj, int32_t text_width,
                     uint32_t batch_rows) {
  if (!p || (nbytes && !text) || !field_types || nfields <= 0 || nfields > YQ_CSV_MAX_FIELDS || !project ||
      nproj <= 0 || nproj > YQ_MAX_BATCH_COLUMNS || text_width < 4 || text_width > YQ_MAX_TEXT_WIDTH ||
      text_width % 4 || nbytes >= (1ull << 32))
    return -YQ_ERR_INVALID_ARG;
  return guarded([&] {
    return add(p, std::make_unique<CsvScanOperator>(text, nbytes, field_types, nfields, project, nproj, text_width,
                                                    batch_rows));
  });
}

int yq_plan_filter(yq_plan* p, int32_t child, const yq_program* pred, const yq_constants* k) {
  if (!p) return -YQ_ERR_INVALID_ARG;
  return guarded([&] { return add(p, std::make_unique<FilterOperator>(take(p, child), pred, k)); });
}

int yq_plan_project(yq_plan* p, int32_t child, const yq_projection* proj, int32_t nproj, const yq_constants* k) {
  if (!p || !proj || nproj <= 0) return -YQ_ERR_INVALID_ARG;
  return guarded([&] { return add(p, std::make_unique<ProjectionOperator>(take(p, child), proj, nproj, k)); });
}

int yq_plan_aggregate(yq_plan* p, int32_t child, const yq_agg_spec* aggs, int32_t nagg, const yq_constants* k) {
  if (!p || !aggs || nagg <= 0 || nagg > YQ_MAX_AGGREGATES) return -YQ_ERR_INVALID_ARG;
  return guarded([&] { return add(p, std::make_unique<AggregateOperator>(take(p, child), aggs, nagg, k)); });
}

int yq_plan_order(yq_plan* p, int32_t child, int32_t key, int32_t desc, int32_t nulls_first) {
  if (!p) return -YQ_ERR_INVALID_ARG;
  return guarded([&] {
    return add(p, std::make_unique<OrderOperator>(take(p, child), std::vector<int32_t>{key},
                                                  std::vector<int32_t>{desc != 0}, std::vector<int32_t>{nulls_first != 0}));
  });
}

int yq_plan_order_multi(yq_plan* p, int32_t child, const int32_t* keys, const int32_t* descending,
                        const int32_t* nulls_first, int32_t nkeys) {
  if (!p || !keys || nkeys <= 0 || nkeys > YQ_MAX_BATCH_COLUMNS) return -YQ_ERR_INVALID_ARG;
  return guarded([&] {
    std::vector<int32_t> k(keys, keys + nkeys), d(nkeys, 0), nf(nkeys, 0);
    for (int i = 0; i < nkeys; ++i) {
      d[i] = descending ? descending[i] != 0 : 0;
      nf[i] = nulls_first ? nulls_first[i] != 0 : 0;
    }
    return add(p, std::make_unique<OrderOperator>(take(p, child), k, d, nf));
  });
}

int yq_plan_group_by(yq_plan* p, int32_t child, int32_t key_col, const yq_group_agg* aggs, int32_t nagg) {
  if (!p || nagg < 0 || nagg > YQ_MAX_AGGREGATES || (nagg && !aggs)) return -YQ_ERR_INVALID_ARG;
  return guarded([&] { return add(p, std::make_unique<GroupByOperator>(take(p, child), key_col, aggs, nagg)); });
}

int yq_plan_join(yq_plan* p, int32_t left, int32_t right, const yq_join_cond* conds, int32_t ncond) {
  if (!p || ncond <= 0 || !conds) return -YQ_ERR_INVALID_ARG;
  return guarded([&] {
    auto l = take(p, left);
    auto r = take(p, right);
    return add(p, std::make_unique<JoinOperator>(std::move(l), std::move(r), conds, ncond));
  });
}

int yq_plan_join_or(yq_plan* p, int32_t left, int32_t right, const yq_join_cond* conds, const int32_t* disjunct,
                    int32_t ncond) {
  if (!p || ncond <= 0 || !conds || !disjunct) return -YQ_ERR_INVALID_ARG;
  return guarded([&] {
    auto l = take(p, left);
    auto r = take(p, right);
    return add(p, std::make_unique<JoinOperator>(std::move(l), std::move(r), conds, ncond, disjunct));
  });
}

int yq_plan_cross(yq_plan* p, int32_t left, int32_t right) {
  if (!p) return -YQ_ERR_INVALID_ARG;
  return guarded([&] {
    auto l = take(p, left);
    auto r = take(p, right);
    return add(p, std::make_unique<JoinOperator>(std::move(l), std::move(r), nullptr, 0));
  });
}

int yq_plan_execute(yq_plan* p, int32_t root, yq_result** out) {
  if (!p || !out || root < 0 || root >= (int)p->nodes.size()) return YQ_ERR_INVALID_ARG;
  const int st = guarded([&]() -> int {
    Operator* op = p->nodes[root];
    p->ctx.stats = yq_plan_stats{};
    op->setContext(&p->ctx);
    CacheManager cache(p->budget, p->host_budget, p->cache_dir);
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    check_cuda(cudaEventRecord(e0, p->ctx.compute), "event");
    op->init();
    std::vector<std::unique_ptr<Batch>> batches;
    uint64_t rows = 0;
    for (BatchID id = op->next(cache); id; id = op->next(cache)) {
      auto b = cache.getBatch(id);
      rows += b->rows;
      batches.push_back(std::move(b));
    }
    auto res = std::make_unique<yq_result>();
    res->rows = rows;
    for (size_t c = 0; c < op->columns.size(); ++c) {
      const size_t w = op->columns[c]->width;
      void* buf = nullptr;
      void* nbuf = nullptr;
      check_cuda(cudaMallocHost(&buf, std::max<uint64_t>(1, rows) * w), "result");
      res->bufs.push_back(buf);
      bool nullable = false;
      for (auto& b : batches) nullable |= b->nulls[c] != nullptr;
      if (nullable) {
        check_cuda(cudaMallocHost(&nbuf, std::max<uint64_t>(1, rows)), "result");
        res->bufs.push_back(nbuf);
      }
      uint64_t o = 0;
      for (auto& b : batches) {
        check_cuda(cudaMemcpyAsync((char*)buf + o * w, b->data[c], b->rows * w, cudaMemcpyDeviceToHost, p->ctx.compute),
                   "result D2H");
        p->ctx.stats.d2h_bytes += b->rows * w;
        if (nbuf) {
          if (b->nulls[c])
            check_cuda(cudaMemcpyAsync((char*)nbuf + o, b->nulls[c], b->rows, cudaMemcpyDeviceToHost, p->ctx.compute),
                       "result D2H");
          else
            memset((char*)nbuf + o, 0, b->rows);  // host memory: no device work
        }
        o += b->rows;
      }
      res->cols.push_back(yq_host_column{buf, static_cast<uint8_t*>(nbuf), op->columns[c]->type, (int32_t)w});
    }
    check_cuda(cudaEventRecord(e1, p->ctx.compute), "event");
    check_cuda(cudaStreamSynchronize(p->ctx.compute), "execute");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    p->ctx.stats.compute_ms = ms;
    p->ctx.stats.spilled_batches = cache.spilled();
    p->ctx.stats.disk_batches = cache.spilledToDisk();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    batches.clear();
    *out = res.release();
    return YQ_OK;
  });
  return st < 0 ? -st : st;
}

uint64_t yq_result_rows(const yq_result* r) { return r ? r->rows : 0; }
int32_t yq_result_ncols(const yq_result* r) { return r ? (int32_t)r->cols.size() : 0; }
int yq_result_column(const yq_result* r, int32_t c, yq_host_column* out) {
  if (!r || !out || c < 0 || c >= (int32_t)r->cols.size()) return YQ_ERR_INVALID_ARG;
  *out = r->cols[c];
  return YQ_OK;
}
void yq_result_destroy(yq_result* r) { delete r; }

int yq_plan_stats_read(const yq_plan* p, yq_plan_stats* out) {
  if (!p || !out) return YQ_ERR_INVALID_ARG;
  *out = p->ctx.stats;
  return YQ_OK;
}

}  // extern "C"
