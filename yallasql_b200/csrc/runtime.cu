// Library runtime: error bookkeeping, launch accounting, device queries.
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#include <stdio.h>
#include <string.h>
#include "yq_common.cuh"

namespace yq {

static thread_local int g_last_cuda_error = 0;
static std::atomic<unsigned long long> g_launches{0};

void set_cuda_error(cudaError_t e) { g_last_cuda_error = (int)e; }
void count_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

// ------------------------------------------------------ small host uploads
// A copy from pageable host memory may make the host wait for the stream;
// small descriptor arrays (segment offsets, merge pairs) go through a ring of
// pinned slots instead, so the call that issues them does not block. A slot
// is reused only after the event recorded behind its previous copy fired.
namespace {
constexpr int kStageSlots = 16;
constexpr size_t kStageSlotBytes = 64 * 1024;
std::mutex g_stage_mu;
char* g_stage_host = nullptr;
cudaEvent_t g_stage_ev[kStageSlots] = {};
int g_stage_next = 0;
int g_stage_dev = -1;
}  // namespace

// Under stream capture a copy from a reused pinned slot would be replayed
// from whatever the slot holds then; the bytes go as kernel parameters
// instead, which the graph keeps with the node.
struct ParamChunk {
  uint32_t words[1024];
};

__global__ void k_param_copy(uint32_t* __restrict__ dst, const __grid_constant__ ParamChunk c, uint32_t nwords) {
  for (uint32_t i = threadIdx.x; i < nwords; i += blockDim.x) dst[i] = c.words[i];
}

// Uploads up to kParamPathBytes travel as kernel parameters rather than
// through a copy engine: an operator's small uploads then never queue behind a
// bulk transfer another stream has in flight on the same engine.
constexpr size_t kParamPathBytes = 16 * 1024;

int h2d_async(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return YQ_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  YQ_TRY_CUDA(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone || (bytes <= kParamPathBytes && !(bytes & 3u) &&
                                            !(reinterpret_cast<uintptr_t>(dst) & 3u))) {
    if ((bytes & 3u) || (reinterpret_cast<uintptr_t>(dst) & 3u)) return YQ_ERR_UNSUPPORTED;
    const uint32_t* w = static_cast<const uint32_t*>(src);
    const size_t nw = bytes / 4;
    for (size_t o = 0; o < nw; o += 1024) {
      ParamChunk c;
      const uint32_t n = (uint32_t)((nw - o) < 1024 ? (nw - o) : 1024);
      memcpy(c.words, w + o, (size_t)n * 4);
      k_param_copy<<<1, 256, 0, s>>>(static_cast<uint32_t*>(dst) + o, c, n);
      YQ_CHECK_LAUNCH();
    }
    return YQ_OK;
  }
  int dev = 0;
  YQ_TRY_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_stage_mu);
  if (bytes > kStageSlotBytes || (g_stage_dev >= 0 && g_stage_dev != dev)) {
    YQ_TRY_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return YQ_OK;
  }
  if (!g_stage_host) {
    void* h = nullptr;
    YQ_TRY_CUDA(cudaMallocHost(&h, kStageSlots * kStageSlotBytes));
    for (int i = 0; i < kStageSlots; ++i) YQ_TRY_CUDA(cudaEventCreateWithFlags(&g_stage_ev[i], cudaEventDisableTiming));
    g_stage_host = static_cast<char*>(h);
    g_stage_dev = dev;
  }
  const int slot = g_stage_next;
  g_stage_next = (g_stage_next + 1) % kStageSlots;
  YQ_TRY_CUDA(cudaEventSynchronize(g_stage_ev[slot]));  // the slot's previous copy has been read
  char* h = g_stage_host + (size_t)slot * kStageSlotBytes;
  memcpy(h, src, bytes);
  YQ_TRY_CUDA(cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, s));
  YQ_TRY_CUDA(cudaEventRecord(g_stage_ev[slot], s));
  return YQ_OK;
}

// -------------------------------------------------------- small read-backs
// A small device -> host read that the host needs now: a kernel copies the
// words into mapped pinned host memory (stores over the link, not a copy
// engine), the stream is synchronised, the bytes are copied out. Larger reads
// take cudaMemcpyAsync. Each call takes a mapped buffer from its device's free
// list (allocated on first need, never freed) and gives it back after the
// copy, so calls from several host threads wait on their own streams only.
namespace {
constexpr size_t kMappedBytes = 64 * 1024;
std::mutex g_mapped_mu;
std::vector<uint32_t*> g_mapped_free[64];
}  // namespace

__global__ void k_to_host(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, uint32_t nwords) {
  for (uint32_t i = threadIdx.x; i < nwords; i += blockDim.x) dst[i] = src[i];
  __threadfence_system();
}

int d2h_sync(void* host_dst, const void* dev_src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return YQ_OK;
  int dev = 0;
  YQ_TRY_CUDA(cudaGetDevice(&dev));
  const bool small = bytes <= kMappedBytes && dev >= 0 && dev < 64 && !(bytes & 3u) &&
                     !(reinterpret_cast<uintptr_t>(dev_src) & 3u);
  if (!small) {
    YQ_TRY_CUDA(cudaMemcpyAsync(host_dst, dev_src, bytes, cudaMemcpyDeviceToHost, s));
    YQ_TRY_CUDA(cudaStreamSynchronize(s));
    return YQ_OK;
  }
  uint32_t* buf = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mapped_mu);
    if (!g_mapped_free[dev].empty()) {
      buf = g_mapped_free[dev].back();
      g_mapped_free[dev].pop_back();
    }
  }
  if (!buf) {
    void* h = nullptr;
    YQ_TRY_CUDA(cudaHostAlloc(&h, kMappedBytes, cudaHostAllocMapped | cudaHostAllocPortable));
    buf = static_cast<uint32_t*>(h);
  }
  uint32_t* dptr = nullptr;
  cudaError_t e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&dptr), buf, 0);
  if (e == cudaSuccess) {
    k_to_host<<<1, 256, 0, s>>>(dptr, static_cast<const uint32_t*>(dev_src), (uint32_t)(bytes / 4));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) memcpy(host_dst, buf, bytes);
  {
    std::lock_guard<std::mutex> lk(g_mapped_mu);
    g_mapped_free[dev].push_back(buf);
  }
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return YQ_ERR_CUDA;
  }
  return YQ_OK;
}

// ---------------------------------------------------------------- profiler
namespace {
struct ProfRec {
  std::string tag;
  cudaEvent_t a, b;
  double units;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;            // open and closed records, in launch order
std::vector<size_t> g_prof_open;        // indices of records awaiting prof_end (nested scopes)
std::vector<cudaEvent_t> g_event_pool;

cudaEvent_t take_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

void prof_begin(const char* tag, cudaStream_t s, double units) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on) return;
  ProfRec r;
  r.tag = tag;
  r.units = units;
  r.a = take_event();
  r.b = take_event();
  cudaEventRecord(r.a, s);
  g_prof_open.push_back(g_prof.size());
  g_prof.push_back(r);
}

void prof_end(cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on || g_prof_open.empty()) return;
  ProfRec& r = g_prof[g_prof_open.back()];
  g_prof_open.pop_back();
  cudaEventRecord(r.b, s);
}

int sm_count() {
  static std::atomic<int> cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int v = cached[dev].load(std::memory_order_relaxed);
  if (!v) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cached[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

// ------------------------------------------------- per-device launch settings
// cudaFuncSetAttribute applies to the current device only, and host threads
// may launch concurrently: the shared-memory opt-in and the occupancy of each
// kernel are kept per (device, kernel[, block, smem]) under one lock.
namespace {
std::mutex g_kattr_mu;
std::map<std::pair<int, const void*>, size_t> g_kattr_smem;
std::map<std::tuple<int, const void*, int, size_t>, int> g_kattr_blocks;
}  // namespace

int kernel_allow_smem(const void* kernel, size_t smem) {
  if (smem <= 48 * 1024) return YQ_OK;
  int dev = 0;
  YQ_TRY_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_kattr_mu);
  size_t& cap = g_kattr_smem[{dev, kernel}];
  if (smem <= cap) return YQ_OK;  // the cap only rises: a smaller launch never lowers it
  YQ_TRY_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cap = smem;
  return YQ_OK;
}

int kernel_blocks_per_sm(const void* kernel, int block, size_t smem) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  if (kernel_allow_smem(kernel, smem) != YQ_OK) return 1;
  std::lock_guard<std::mutex> lk(g_kattr_mu);
  const auto key = std::make_tuple(dev, kernel, block, smem);
  auto it = g_kattr_blocks.find(key);
  if (it != g_kattr_blocks.end()) return it->second;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  g_kattr_blocks.emplace(key, per_sm);
  return per_sm;
}

}  // namespace yq

extern "C" {

const char* yq_status_string(int status) {
  switch (status) {
    case YQ_OK: return "ok";
    case YQ_ERR_INVALID_ARG: return "invalid argument";
    case YQ_ERR_UNSUPPORTED: return "unsupported";
    case YQ_ERR_CAPACITY: return "output capacity exceeded";
    case YQ_ERR_TIMEOUT: return "bounded device wait timed out";
    case YQ_ERR_CUDA: return "CUDA error";
    case YQ_ERR_ALLOC: return "device allocation failed";
    default: return "unknown status";
  }
}

int yq_last_cuda_error(void) { return yq::g_last_cuda_error; }
int yq_abi_version(void) { return YQ_ABI_VERSION; }
int yq_device_sm_count(void) { return yq::sm_count(); }
uint64_t yq_launch_count(void) { return yq::g_launches.load(std::memory_order_relaxed); }

int yq_profile_enable(int32_t on) {
  std::lock_guard<std::mutex> lk(yq::g_prof_mu);
  yq::g_prof_on = on != 0;
  return YQ_OK;
}

int yq_profile_read(char* out, size_t cap, int32_t reset) {
  // Synchronises on every recorded event, then reports per tag: launches,
  // total device milliseconds and total work units (as tagged by the caller).
  std::lock_guard<std::mutex> lk(yq::g_prof_mu);
  struct Agg { long n = 0; double ms = 0, units = 0; };
  std::map<std::string, Agg> agg;
  for (auto& r : yq::g_prof) {
    if (cudaEventSynchronize(r.b) != cudaSuccess) continue;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) continue;
    Agg& a = agg[r.tag];
    a.n += 1;
    a.ms += ms;
    a.units += r.units;
  }
  std::string js = "{";
  bool first = true;
  for (auto& kv : agg) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s\"%s\": {\"launches\": %ld, \"ms\": %.6f, \"units\": %.1f}", first ? "" : ", ",
             kv.first.c_str(), kv.second.n, kv.second.ms, kv.second.units);
    js += buf;
    first = false;
  }
  js += "}";
  if (reset) {
    for (auto& r : yq::g_prof) {
      yq::g_event_pool.push_back(r.a);
      yq::g_event_pool.push_back(r.b);
    }
    yq::g_prof.clear();
    yq::g_prof_open.clear();
  }
  if (out && cap > 0) {
    size_t n = js.size() < cap - 1 ? js.size() : cap - 1;
    memcpy(out, js.data(), n);
    out[n] = 0;
  }
  return (int)js.size();
}

}  // extern "C"
