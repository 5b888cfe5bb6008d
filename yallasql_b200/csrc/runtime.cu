// Library runtime: error bookkeeping, launch accounting, device queries.
#include <atomic>
#include "yq_common.cuh"

namespace yq {

static thread_local int g_last_cuda_error = 0;
static std::atomic<unsigned long long> g_launches{0};

void set_cuda_error(cudaError_t e) { g_last_cuda_error = (int)e; }
void count_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cached[dev] = v;
  }
  return cached[dev];
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

}  // extern "C"
