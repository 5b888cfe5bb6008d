// Shared device/host plumbing for the yq kernels (sm_100a).
#pragma once

#ifdef __CUDACC_RTC__
// Program-specialised kernels are compiled at run time (jit.cu) without the
// system headers: the fixed-width types and limits device code uses are here.
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
typedef unsigned long uintptr_t;
typedef decltype(sizeof(0)) size_t;
#define INT32_MIN (-2147483647 - 1)
#define INT32_MAX 2147483647
#define LLONG_MAX 9223372036854775807LL
#define LLONG_MIN (-LLONG_MAX - 1LL)
#else
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#endif

#include "../../include/yq_ops.h"

namespace yq {

#ifndef __CUDACC_RTC__

// ------------------------------------------------------------------ errors
void set_cuda_error(cudaError_t e);
void count_launch(int n = 1);

// Optional per-kernel device timing (yq_profile_enable): records a CUDA
// event pair on the launch stream around each tagged launch.
void prof_begin(const char* tag, cudaStream_t s, double units);
void prof_end(cudaStream_t s);
struct ProfScope {
  cudaStream_t s;
  ProfScope(const char* tag, cudaStream_t st, double units = 0.0) : s(st) { prof_begin(tag, st, units); }
  ~ProfScope() { prof_end(s); }
};

#define YQ_TRY_CUDA(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) {                                \
      ::yq::set_cuda_error(_e);                             \
      return YQ_ERR_CUDA;                                   \
    }                                                       \
  } while (0)

#define YQ_TRY(expr)                                        \
  do {                                                      \
    int _s = (expr);                                        \
    if (_s != YQ_OK) return _s;                             \
  } while (0)

// After a kernel launch: picks up launch-configuration errors.
#define YQ_CHECK_LAUNCH()                                   \
  do {                                                      \
    ::yq::count_launch();                                   \
    cudaError_t _e = cudaGetLastError();                    \
    if (_e != cudaSuccess) {                                \
      ::yq::set_cuda_error(_e);                             \
      return YQ_ERR_CUDA;                                   \
    }                                                       \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Host -> device copy of a small host array that returns without waiting for
// the stream (staged through pinned memory; runtime.cu).
int h2d_async(void* dst, const void* src, size_t bytes, cudaStream_t s);

// Device -> host read of `bytes` that the host waits for (synchronises `s`);
// small reads bypass the copy engines (runtime.cu).
int d2h_sync(void* host_dst, const void* dev_src, size_t bytes, cudaStream_t s);

int sm_count();

// Per-device, thread-safe launch settings (runtime.cu): raise `kernel`'s
// dynamic shared-memory limit on the current device to at least `smem`, and
// the number of `block`-thread blocks with `smem` bytes resident per SM (>= 1).
int kernel_allow_smem(const void* kernel, size_t smem);
int kernel_blocks_per_sm(const void* kernel, int block, size_t smem);

#endif  // !__CUDACC_RTC__

template <typename T>
__host__ __device__ inline T ceil_div(T a, T b) { return (a + b - 1) / b; }

#ifndef __CUDACC_RTC__

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Bump allocator over one workspace region. When the caller passes no
// workspace, `Workspace::acquire` allocates it stream-ordered and the
// destructor frees it stream-ordered (cudaFreeAsync), so a call never blocks
// on allocation and the memory returns to the pool after the work it backs.
struct Workspace {
  char* base = nullptr;
  size_t bytes = 0;
  size_t used = 0;
  bool owned = false;
  cudaStream_t stream = nullptr;

  int acquire(void* user, size_t user_bytes, size_t need, cudaStream_t s) {
    stream = s;
    if (user) {
      if (user_bytes < need) return YQ_ERR_INVALID_ARG;
      base = static_cast<char*>(user);
      bytes = user_bytes;
      return YQ_OK;
    }
    if (need == 0) return YQ_OK;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, need, s);
    if (e != cudaSuccess) {
      set_cuda_error(e);
      return YQ_ERR_ALLOC;
    }
    base = static_cast<char*>(p);
    bytes = need;
    owned = true;
    return YQ_OK;
  }
  template <typename T>
  T* take(size_t count) {
    size_t off = align_up(used, 256);
    used = off + count * sizeof(T);
    return reinterpret_cast<T*>(base + off);
  }
  ~Workspace() {
    if (owned && base) cudaFreeAsync(base, stream);
  }
};

// Size helper mirroring Workspace::take's alignment.
struct WsSize {
  size_t used = 0;
  template <typename T>
  void add(size_t count) { used = align_up(used, 256) + count * sizeof(T); }
  size_t total() const { return align_up(used, 256) + 256; }
};

#endif  // !__CUDACC_RTC__

// ---------------------------------------------------------- device helpers
// Bound on every spin wait: ~2^22 polls with a 64-256 ns back-off is well
// over a second, far beyond any legitimate wait on a predecessor tile.
constexpr uint32_t kSpinLimit = 1u << 22;

// Error word layout inside workspaces: bit 0 = a bounded wait ran out,
// bit 1 = a computed index fell outside its buffer (the access was skipped).
constexpr uint32_t kErrTimeout = 1u;
constexpr uint32_t kErrBounds = 2u;

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint4 ldg_nc_v4(const void* p) {
  uint4 v;
  asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// Block-wide exclusive sum over one value per thread (BLOCK threads).
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t x, uint32_t* s_warp, uint32_t& total) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += y;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < NW ? s_warp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
      if (lane >= d) wi += y;
    }
    if (lane < NW) s_warp[lane] = wi - w;  // exclusive warp offsets
    if (lane == NW - 1) s_warp[NW] = wi;   // block total
  }
  __syncthreads();
  uint32_t excl = s_warp[warp] + inc - x;
  total = s_warp[NW];
  __syncthreads();
  return excl;
}

// Block-wide exclusive sum of two 64-bit words per thread in one pass (each
// word holds independent fields that never carry into one another).
// `s_warp` holds 2 * (BLOCK / 32 + 1) words; a and b become the exclusive sums.
template <int BLOCK>
__device__ __forceinline__ void block_exclusive_sum2(unsigned long long& a, unsigned long long& b,
                                                     unsigned long long* s_warp, unsigned long long& ta,
                                                     unsigned long long& tb) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long ia = a, ib = b;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long ya = __shfl_up_sync(0xffffffffu, ia, d);
    const unsigned long long yb = __shfl_up_sync(0xffffffffu, ib, d);
    if (lane >= d) {
      ia += ya;
      ib += yb;
    }
  }
  if (lane == 31) {
    s_warp[2 * warp] = ia;
    s_warp[2 * warp + 1] = ib;
  }
  __syncthreads();
  if (warp == 0) {
    const unsigned long long wa = lane < NW ? s_warp[2 * lane] : 0ull;
    const unsigned long long wb = lane < NW ? s_warp[2 * lane + 1] : 0ull;
    unsigned long long sa = wa, sb = wb;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long ya = __shfl_up_sync(0xffffffffu, sa, d);
      const unsigned long long yb = __shfl_up_sync(0xffffffffu, sb, d);
      if (lane >= d) {
        sa += ya;
        sb += yb;
      }
    }
    if (lane < NW) {
      s_warp[2 * lane] = sa - wa;
      s_warp[2 * lane + 1] = sb - wb;
    }
    if (lane == NW - 1) {
      s_warp[2 * NW] = sa;
      s_warp[2 * NW + 1] = sb;
    }
  }
  __syncthreads();
  const unsigned long long ea = s_warp[2 * warp] + ia - a, eb = s_warp[2 * warp + 1] + ib - b;
  ta = s_warp[2 * NW];
  tb = s_warp[2 * NW + 1];
  __syncthreads();
  a = ea;
  b = eb;
}

// ---------------------------------------------- mbarrier + 1-D bulk copies
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// 1-D bulk copy global -> shared (both 16-byte aligned, bytes % 16 == 0).
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// L2 cache policies for bulk copies: keep a line for a later re-read of the
// same data (evict_last) or let it go first (evict_first, streaming data).
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// tma_load_1d with an L2 cache policy.
__device__ __forceinline__ void tma_load_1d_hint(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                                 uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// Bounded wait for phase `parity` of `bar`. When the bound runs out, thread 0
// sets kErrTimeout in *err and the copies still in flight get one more
// bounded wait before the caller goes on (its data is then not used as valid:
// the error word fails the call).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t* err) {
  uint32_t spins = 0;
  bool done = mbar_try_wait(bar, parity);
  while (!done && ++spins < kSpinLimit) done = mbar_try_wait(bar, parity);
  if (done) return true;
  if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
  for (uint32_t s2 = 0; s2 < kSpinLimit && !mbar_try_wait(bar, parity); ++s2) {
  }
  return false;
}

}  // namespace yq
