// Reference-compatible element kernels: one C entry per YallaSQL::Kernel::launch_*
// (include/kernels/*.hpp) with the reference's semantics, so its expression
// classes can forward unchanged. These are the adapter path; the fused
// operator kernels (k_filter.cu, k_sort.cu, k_merge.cu, k_join.cu) are the
// fast path.
//
// Every kernel reads and writes with 16-byte vector accesses where the
// buffers allow it and uses a grid sized to a multiple of the SM count.
#include <string.h>
#include <type_traits>
#include "yq_lookback.cuh"

namespace yq {

constexpr int kElemBlock = 256;

static int elem_grid(uint64_t n, int per_thread) {
  const uint64_t want = (n + (uint64_t)kElemBlock * per_thread - 1) / ((uint64_t)kElemBlock * per_thread);
  const uint64_t cap = (uint64_t)sm_count() * 16;
  return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

static bool fixed_width_ok(int type, int width) {
  switch (type) {
    case YQ_INT32:
    case YQ_FLOAT32: return width == 4;
    case YQ_INT64:
    case YQ_DATETIME:
    case YQ_FLOAT64: return width == 8;
    case YQ_BOOL: return width == 1;
    case YQ_TEXT: return width >= 4 && width <= YQ_MAX_TEXT_WIDTH && width % 4 == 0;
    default: return false;
  }
}

// ------------------------------------------------------------- compare
// String order of the reference: strcmp_device over unsigned bytes, stopping
// at the first NUL of the left operand (include/kernels/string_kernel.hpp:48-57).
__device__ __forceinline__ int str_cmp(const uint8_t* a, const uint8_t* b, int width) {
  for (int i = 0; i < width; ++i) {
    const uint8_t x = a[i], y = b[i];
    if (x == 0 || x != y) return (int)x - (int)y;
  }
  return 0;
}

template <typename T>
__device__ __forceinline__ bool cmp_op(T a, T b, int op) {
  switch (op) {
    case YQ_LT: return a < b;
    case YQ_LE: return a <= b;
    case YQ_GT: return a > b;
    case YQ_GE: return a >= b;
    case YQ_EQ: return a == b;
    default: return a != b;
  }
}

__device__ __forceinline__ bool sign_op(int s, int op) {
  switch (op) {
    case YQ_LT: return s < 0;
    case YQ_LE: return s <= 0;
    case YQ_GT: return s > 0;
    case YQ_GE: return s >= 0;
    case YQ_EQ: return s == 0;
    default: return s != 0;
  }
}

template <typename T>
__global__ void k_compare(const T* __restrict__ lhs, const T* __restrict__ rhs, int ls, int rs, int op, int neg,
                          uint8_t* __restrict__ out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool r = cmp_op<T>(lhs[ls ? 0 : i], rhs[rs ? 0 : i], op);
    out[i] = (uint8_t)(r != (neg != 0));
  }
}

__global__ void k_compare_text(const uint8_t* __restrict__ lhs, const uint8_t* __restrict__ rhs, int ls, int rs,
                               int width, int op, int neg, uint8_t* __restrict__ out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = str_cmp(lhs + (size_t)(ls ? 0 : i) * width, rhs + (size_t)(rs ? 0 : i) * width, width);
    out[i] = (uint8_t)(sign_op(s, op) != (neg != 0));
  }
}

__global__ void k_logic(const uint8_t* __restrict__ lhs, const uint8_t* __restrict__ rhs, int ls, int rs, int is_or,
                        uint8_t* __restrict__ out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool a = lhs[ls ? 0 : i] != 0, b = rhs[rs ? 0 : i] != 0;
    out[i] = (uint8_t)(is_or ? (a || b) : (a && b));
  }
}

// ------------------------------------------------------------ arithmetic
// DIV / MOD by zero give 0 (DivOperator / RemOperator, binary_operators_kernel.hpp:44-53).
template <typename T>
__device__ __forceinline__ T arith_ref(T a, T b, int op) {
  switch (op) {
    case YQ_ADD: return a + b;
    case YQ_SUB: return a - b;
    case YQ_MUL: return a * b;
    case YQ_DIV: return b != (T)0 ? a / b : (T)0;
    default: return b != (T)0 ? a % b : (T)0;
  }
}
template <>
__device__ __forceinline__ float arith_ref<float>(float a, float b, int op) {
  switch (op) {
    case YQ_ADD: return a + b;
    case YQ_SUB: return a - b;
    case YQ_MUL: return a * b;
    case YQ_DIV: return b != 0.f ? a / b : 0.f;
    default: return b != 0.f ? fmodf(a, b) : 0.f;
  }
}
template <>
__device__ __forceinline__ int32_t arith_ref<int32_t>(int32_t a, int32_t b, int op) {
  const uint32_t ua = (uint32_t)a, ub = (uint32_t)b;
  switch (op) {
    case YQ_ADD: return (int32_t)(ua + ub);
    case YQ_SUB: return (int32_t)(ua - ub);
    case YQ_MUL: return (int32_t)(ua * ub);
    case YQ_DIV: return b == 0 ? 0 : (b == -1 ? (int32_t)(0u - ua) : a / b);
    default: return (b == 0 || b == -1) ? 0 : a % b;
  }
}
template <>
__device__ __forceinline__ int64_t arith_ref<int64_t>(int64_t a, int64_t b, int op) {
  const uint64_t ua = (uint64_t)a, ub = (uint64_t)b;
  switch (op) {
    case YQ_ADD: return (int64_t)(ua + ub);
    case YQ_SUB: return (int64_t)(ua - ub);
    case YQ_MUL: return (int64_t)(ua * ub);
    case YQ_DIV: return b == 0 ? 0 : (b == -1 ? (int64_t)(0ull - ua) : a / b);
    default: return (b == 0 || b == -1) ? 0 : a % b;
  }
}

template <typename T>
__global__ void k_binary(const T* __restrict__ lhs, const T* __restrict__ rhs, int ls, int rs, int op,
                         T* __restrict__ out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = arith_ref<T>(lhs[ls ? 0 : i], rhs[rs ? 0 : i], op);
}

// ----------------------------------------------------------------- casts
// static_cast semantics (numerical_cast_kernel, cast_operators_kernel.cu:6-16).
template <typename S, typename D>
__global__ void k_cast(const S* __restrict__ src, D* __restrict__ dst, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = static_cast<D>(src[i]);
}

// --------------------------------------------------------- prefix sums
// Inclusive scan in tiles of kScanTile elements, one decoupled look-back per
// tile. Each thread scans kScanItems consecutive elements in registers
// (16-byte loads when the input is 16-byte aligned and the tile is full: two
// per thread for masks, eight for 32-bit values); the results go through shared
// memory so that each warp's stores cover 128 contiguous bytes.
constexpr int kScanItems = 32;
constexpr uint32_t kScanTile = kElemBlock * kScanItems;
constexpr int kScanPitch = kScanItems + 1;  // padded row of a thread's results in shared memory

template <typename T>
__device__ __forceinline__ void scan_load(const T* __restrict__ in, uint32_t i0, uint32_t n, bool vec,
                                          uint32_t (&v)[kScanItems]) {
  if (vec && i0 + kScanItems <= n) {
    if constexpr (sizeof(T) == 1) {
#pragma unroll
      for (int c = 0; c < kScanItems / 16; ++c) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(in + i0) + c);
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 16; ++k) v[16 * c + k] = (w[k >> 2] >> (8 * (k & 3))) & 0xffu;
      }
      return;
    } else {
#pragma unroll
      for (int c = 0; c < kScanItems / 4; ++c) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(in + i0) + c);
        v[4 * c] = q.x;
        v[4 * c + 1] = q.y;
        v[4 * c + 2] = q.z;
        v[4 * c + 3] = q.w;
      }
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) v[k] = (i0 + k < n) ? (uint32_t)in[i0 + k] : 0u;
}

template <typename T>
__global__ void __launch_bounds__(kElemBlock) k_scan(const T* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
                                                     uint32_t* tile_counter, unsigned long long* status,
                                                     uint32_t* err, int vec) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kElemBlock / 32 + 1];
  __shared__ unsigned long long s_prefix;
  __shared__ uint32_t s_out[kElemBlock * kScanPitch];
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t t0 = tile * kScanTile;
  const uint32_t i0 = t0 + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  scan_load<T>(in, i0, n, vec != 0, v);
#pragma unroll
  for (int k = 1; k < kScanItems; ++k) v[k] += v[k - 1];
  uint32_t total;
  const uint32_t excl = block_exclusive_sum<kElemBlock>(v[kScanItems - 1], s_warp, total);
  if (threadIdx.x < 32) {
    const unsigned long long p = tile_lookback(status, tile, total, err);
    if (threadIdx.x == 0) s_prefix = p;
  }
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s_out[threadIdx.x * kScanPitch + k] = excl + v[k];
  __syncthreads();
  const uint32_t base = (uint32_t)s_prefix;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint32_t e = (uint32_t)j * kElemBlock + threadIdx.x;  // element of the tile
    if (t0 + e < n) out[t0 + e] = base + s_out[(e / kScanItems) * kScanPitch + (e % kScanItems)];
  }
}

// ------------------------------------------------------------ row moves
__device__ __forceinline__ void copy_w(char* dst, const char* src, int w) {
  if (w == 4) *reinterpret_cast<uint32_t*>(dst) = *reinterpret_cast<const uint32_t*>(src);
  else if (w == 8) *reinterpret_cast<unsigned long long*>(dst) = *reinterpret_cast<const unsigned long long*>(src);
  else if (w == 1) *dst = *src;
  else
    for (int i = 0; i < w; i += 4) *reinterpret_cast<uint32_t*>(dst + i) = *reinterpret_cast<const uint32_t*>(src + i);
}

// out[map[i]-1] = src[i] where mask[i] and the cell is not NULL; NULL cells
// leave their slot untouched (move_rows_filter_kernel, move_rows_kernel.cu:33-49).
__global__ void k_move_filter(const char* __restrict__ src, const uint8_t* __restrict__ nulls, int w,
                              const uint32_t* __restrict__ map, const uint8_t* __restrict__ mask, uint32_t n,
                              char* __restrict__ dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (mask[i] && !(nulls && nulls[i]) && map[i] > 0) copy_w(dst + (size_t)(map[i] - 1) * w, src + (size_t)i * w, w);
}

__global__ void k_move_join(const char* __restrict__ src, const uint8_t* __restrict__ nulls, int w,
                            const uint32_t* __restrict__ pairs, uint32_t npairs, int side, char* __restrict__ dst,
                            uint8_t* __restrict__ dnulls) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < npairs; k += gridDim.x * blockDim.x) {
    const uint32_t r = pairs[2 * k + side];
    copy_w(dst + (size_t)k * w, src + (size_t)r * w, w);
    if (dnulls) dnulls[k] = nulls ? nulls[r] : 0;
  }
}

__global__ void k_move_merge(const char* __restrict__ a, const uint8_t* __restrict__ an, const char* __restrict__ b,
                             const uint8_t* __restrict__ bn, int w, const uint32_t* __restrict__ idx,
                             const uint8_t* __restrict__ from_a, int asc, uint32_t n, char* __restrict__ dst,
                             uint8_t* __restrict__ dnulls) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t d = asc ? i : n - 1 - i;
    const uint32_t s = idx[i];
    const bool fa = from_a[i] != 0;
    copy_w(dst + (size_t)d * w, (fa ? a : b) + (size_t)s * w, w);
    if (dnulls) {
      const uint8_t* nl = fa ? an : bn;
      dnulls[d] = nl ? nl[s] : 0;
    }
  }
}

__global__ void k_cross_col(const char* __restrict__ src, const uint8_t* __restrict__ nulls, int w, uint32_t L,
                            uint32_t R, int is_left, char* __restrict__ dst, uint8_t* __restrict__ dnulls) {
  const unsigned long long total = (unsigned long long)L * R;
  for (unsigned long long p = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; p < total;
       p += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t s = is_left ? (uint32_t)(p / R) : (uint32_t)(p % R);
    copy_w(dst + (size_t)p * w, src + (size_t)s * w, w);
    if (dnulls) dnulls[p] = nulls ? nulls[s] : 0;
  }
}

// ------------------------------------------------------------ reductions
// One atomic per block into *result (reduction_sum_wrap / reduction_count_notnull,
// src/kernels/reduction_kernel.cu:79-166): SUM of float accumulates in double.
__device__ __forceinline__ void atomic_min_f(float* addr, float v) {
  int* a = reinterpret_cast<int*>(addr);
  int old = *a, assumed;
  do {
    assumed = old;
    old = atomicCAS(a, assumed, __float_as_int(fminf(v, __int_as_float(assumed))));
  } while (assumed != old);
}
__device__ __forceinline__ void atomic_max_f(float* addr, float v) {
  int* a = reinterpret_cast<int*>(addr);
  int old = *a, assumed;
  do {
    assumed = old;
    old = atomicCAS(a, assumed, __float_as_int(fmaxf(v, __int_as_float(assumed))));
  } while (assumed != old);
}

template <typename T, typename R>
__global__ void __launch_bounds__(kElemBlock) k_reduce(const T* __restrict__ x, const uint8_t* __restrict__ nulls,
                                                       uint32_t n, int kind, R* result) {
  __shared__ R s_w[kElemBlock / 32];
  __shared__ int s_any[kElemBlock / 32];
  R acc = 0;
  bool any = false;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (nulls && nulls[i]) continue;
    const R v = (R)x[i];
    if (kind == YQ_AGG_SUM) acc += v;
    else if (!any) acc = v;
    else if (kind == YQ_AGG_MIN) acc = v < acc ? v : acc;
    else acc = v > acc ? v : acc;
    any = true;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const R o = __shfl_down_sync(0xffffffffu, acc, d);
    const int oa = __shfl_down_sync(0xffffffffu, (int)any, d);
    if (oa) {
      if (kind == YQ_AGG_SUM) acc += o;
      else if (!any) acc = o;
      else if (kind == YQ_AGG_MIN) acc = o < acc ? o : acc;
      else acc = o > acc ? o : acc;
      any = true;
    }
  }
  if (lane == 0) {
    s_w[warp] = acc;
    s_any[warp] = any;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    R t = 0;
    bool ta = false;
    for (int w = 0; w < kElemBlock / 32; ++w) {
      if (!s_any[w]) continue;
      if (kind == YQ_AGG_SUM) t += s_w[w];
      else if (!ta) t = s_w[w];
      else if (kind == YQ_AGG_MIN) t = s_w[w] < t ? s_w[w] : t;
      else t = s_w[w] > t ? s_w[w] : t;
      ta = true;
    }
    if (ta) {
      // only the (type, op) pairs the host dispatches are instantiated
      if constexpr (std::is_same<R, double>::value || std::is_same<R, unsigned long long>::value) {
        atomicAdd(result, t);
      } else if constexpr (std::is_same<R, long long>::value) {
        if (kind == YQ_AGG_MIN) atomicMin(result, t);
        else atomicMax(result, t);
      } else {
        if (kind == YQ_AGG_SUM) atomicAdd(result, t);
        else if (kind == YQ_AGG_MIN) atomicMin(result, t);
        else atomicMax(result, t);
      }
    }
  }
}

// float MIN/MAX need the CAS loop of the reference (reduction_kernel.cu:56-75).
template <>
__global__ void __launch_bounds__(kElemBlock) k_reduce<float, float>(const float* __restrict__ x,
                                                                     const uint8_t* __restrict__ nulls, uint32_t n,
                                                                     int kind, float* result) {
  __shared__ float s_w[kElemBlock / 32];
  __shared__ int s_any[kElemBlock / 32];
  float acc = 0.f;
  bool any = false;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (nulls && nulls[i]) continue;
    const float v = x[i];
    acc = !any ? v : (kind == YQ_AGG_MIN ? fminf(acc, v) : fmaxf(acc, v));
    any = true;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const float o = __shfl_down_sync(0xffffffffu, acc, d);
    const int oa = __shfl_down_sync(0xffffffffu, (int)any, d);
    if (oa) {
      acc = !any ? o : (kind == YQ_AGG_MIN ? fminf(acc, o) : fmaxf(acc, o));
      any = true;
    }
  }
  if (lane == 0) {
    s_w[warp] = acc;
    s_any[warp] = any;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    bool ta = false;
    for (int w = 0; w < kElemBlock / 32; ++w) {
      if (!s_any[w]) continue;
      t = !ta ? s_w[w] : (kind == YQ_AGG_MIN ? fminf(t, s_w[w]) : fmaxf(t, s_w[w]));
      ta = true;
    }
    if (ta) {
      if (kind == YQ_AGG_MIN) atomic_min_f(result, t);
      else atomic_max_f(result, t);
    }
  }
}

__global__ void __launch_bounds__(kElemBlock) k_count_notnull(const uint8_t* __restrict__ nulls, uint32_t n,
                                                              int* result) {
  __shared__ int s_w[kElemBlock / 32];
  int c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    c += nulls ? (nulls[i] == 0) : 1;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kElemBlock / 32; ++w) t += s_w[w];
    atomicAdd(result, t);
  }
}

// ---------------------------------------------------------- key transforms
// int_to_uint32 / float_to_uint32 and their inverses (radix_sort_utils.cu:4-37).
__global__ void k_key_transform(const uint32_t* __restrict__ src, int is_float, int inverse, uint32_t* __restrict__ dst,
                                uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t x = src[i];
    uint32_t r;
    if (!is_float) r = x ^ 0x80000000u;
    else if (!inverse) r = (x & 0x80000000u) ? ~x : (x ^ 0x80000000u);
    else r = (x & 0x80000000u) ? (x ^ 0x80000000u) : ~x;
    dst[i] = r;
  }
}

// 64-bit integers (INT64 / DATETIME read as uint64 by the reference's sort,
// radix_sort_kernel.cu:173): flipping the top bit maps signed order to
// unsigned order and back.
__global__ void k_key_transform64(const unsigned long long* __restrict__ src, unsigned long long* __restrict__ dst,
                                  uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = src[i] ^ 0x8000000000000000ull;
}

// -------------------------------------------------------------- merge path
// merge_sorted_array_kernel_v1 (merge_batchs.cu:33-77): compares raw values
// (AscSortMergeOp / DescSortMergeOp), ties take A; emits keys, source index,
// from-A flag for the first k outputs, and the co-rank of k in A.
template <typename T>
__device__ __forceinline__ bool le_ref(const T& a, const T& b, int desc) { return desc ? (a >= b) : (a <= b); }

__device__ __forceinline__ bool le_text(const uint8_t* a, const uint8_t* b, int w, int desc) {
  const int s = str_cmp(a, b, w);
  return desc ? s >= 0 : s <= 0;
}

template <typename T>
__device__ uint32_t corank_ref(const T* A, const T* B, uint32_t m, uint32_t n, uint32_t k, int desc) {
  uint32_t lo = k > n ? k - n : 0u, hi = k < m ? k : m;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (le_ref<T>(A[mid], B[k - mid - 1], desc)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

constexpr int kMpItems = 6;  // ELE_PER_TH of the reference

template <typename T>
__global__ void k_merge_ref(const T* __restrict__ A, const T* __restrict__ B, uint32_t m, uint32_t n, uint32_t kmax,
                            int desc, T* __restrict__ C, uint32_t* __restrict__ idx, uint8_t* __restrict__ from_a,
                            int32_t* last_a) {
  const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) * kMpItems;
  if (blockIdx.x == 0 && threadIdx.x == 0 && last_a) *last_a = (int32_t)corank_ref<T>(A, B, m, n, kmax, desc);
  if (k >= kmax || k >= m + n) return;
  uint32_t i = corank_ref<T>(A, B, m, n, k, desc), j = k - i;
  for (int d = 0; d < kMpItems && k + d < kmax && k + d < m + n; ++d) {
    const bool ta = j >= n || (i < m && le_ref<T>(A[i], B[j], desc));
    if (ta) {
      C[k + d] = A[i];
      from_a[k + d] = 1;
      idx[k + d] = i++;
    } else {
      C[k + d] = B[j];
      from_a[k + d] = 0;
      idx[k + d] = j++;
    }
  }
}

__global__ void k_merge_ref_text(const uint8_t* __restrict__ A, const uint8_t* __restrict__ B, int w, uint32_t m,
                                 uint32_t n, uint32_t kmax, int desc, uint8_t* __restrict__ C,
                                 uint32_t* __restrict__ idx, uint8_t* __restrict__ from_a, int32_t* last_a) {
  auto corank = [&](uint32_t k) {
    uint32_t lo = k > n ? k - n : 0u, hi = k < m ? k : m;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (le_text(A + (size_t)mid * w, B + (size_t)(k - mid - 1) * w, w, desc)) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  };
  const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) * kMpItems;
  if (blockIdx.x == 0 && threadIdx.x == 0 && last_a) *last_a = (int32_t)corank(kmax);
  if (k >= kmax || k >= m + n) return;
  uint32_t i = corank(k), j = k - i;
  for (int d = 0; d < kMpItems && k + d < kmax && k + d < m + n; ++d) {
    const bool ta = j >= n || (i < m && le_text(A + (size_t)i * w, B + (size_t)j * w, w, desc));
    const uint8_t* src = ta ? A + (size_t)i * w : B + (size_t)j * w;
    for (int b = 0; b < w; b += 4)
      *reinterpret_cast<uint32_t*>(C + (size_t)(k + d) * w + b) = *reinterpret_cast<const uint32_t*>(src + b);
    from_a[k + d] = ta;
    idx[k + d] = ta ? i++ : j++;
  }
}

template <typename T>
static int prefix_sum(const T* in, uint32_t* out, uint32_t n, void* workspace, size_t workspace_bytes,
                      cudaStream_t s) {
  if (!in || !out) return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  const uint32_t ntiles = ceil_div<uint32_t>(n, kScanTile);
  Workspace ws;
  WsSize w;
  w.add<unsigned long long>((size_t)ntiles + 1);
  w.add<uint32_t>(4);
  YQ_TRY(ws.acquire(workspace, workspace_bytes, w.total(), s));
  unsigned long long* status = ws.take<unsigned long long>((size_t)ntiles + 1);
  uint32_t* misc = ws.take<uint32_t>(4);
  YQ_TRY_CUDA(cudaMemsetAsync(status, 0, ((size_t)ntiles + 1) * sizeof(unsigned long long), s));
  YQ_TRY_CUDA(cudaMemsetAsync(misc, 0, 4 * sizeof(uint32_t), s));
  ProfScope ps("prefix_sum", s, (double)n * (sizeof(T) + 4.0));
  const int vec = (reinterpret_cast<uintptr_t>(in) & 15u) == 0u;
  k_scan<T><<<ntiles, kElemBlock, 0, s>>>(in, out, n, misc, status, misc + 1, vec);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

}  // namespace yq

using namespace yq;

extern "C" {

int yq_compare(yq_operand lhs, yq_operand rhs, int32_t cmp, int32_t negate, uint8_t* out_mask, uint32_t n,
               void* stream) {
  if (!lhs.data || !rhs.data || !out_mask || lhs.type != rhs.type || cmp < YQ_LT || cmp > YQ_NE)
    return YQ_ERR_INVALID_ARG;
  if (!fixed_width_ok(lhs.type, lhs.width) || lhs.width != rhs.width) return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  const int g = elem_grid(n, 4);
  ProfScope ps("elem_compare", s, (double)n * (2.0 * lhs.width + 1));
  switch (lhs.type) {
    case YQ_INT32:
      k_compare<int32_t><<<g, kElemBlock, 0, s>>>((const int32_t*)lhs.data, (const int32_t*)rhs.data, lhs.is_scalar,
                                                  rhs.is_scalar, cmp, negate, out_mask, n);
      break;
    case YQ_FLOAT32:
      k_compare<float><<<g, kElemBlock, 0, s>>>((const float*)lhs.data, (const float*)rhs.data, lhs.is_scalar,
                                                rhs.is_scalar, cmp, negate, out_mask, n);
      break;
    case YQ_INT64:
    case YQ_DATETIME:
      k_compare<int64_t><<<g, kElemBlock, 0, s>>>((const int64_t*)lhs.data, (const int64_t*)rhs.data, lhs.is_scalar,
                                                  rhs.is_scalar, cmp, negate, out_mask, n);
      break;
    case YQ_FLOAT64:
      k_compare<double><<<g, kElemBlock, 0, s>>>((const double*)lhs.data, (const double*)rhs.data, lhs.is_scalar,
                                                 rhs.is_scalar, cmp, negate, out_mask, n);
      break;
    case YQ_BOOL:
      k_compare<uint8_t><<<g, kElemBlock, 0, s>>>((const uint8_t*)lhs.data, (const uint8_t*)rhs.data, lhs.is_scalar,
                                                  rhs.is_scalar, cmp, negate, out_mask, n);
      break;
    default:
      k_compare_text<<<g, kElemBlock, 0, s>>>((const uint8_t*)lhs.data, (const uint8_t*)rhs.data, lhs.is_scalar,
                                              rhs.is_scalar, lhs.width, cmp, negate, out_mask, n);
  }
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_logic(yq_operand lhs, yq_operand rhs, int32_t is_or, uint8_t* out_mask, uint32_t n, void* stream) {
  if (!lhs.data || !rhs.data || !out_mask) return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  ProfScope ps("elem_logic", s, (double)n * 3.0);
  k_logic<<<elem_grid(n, 4), kElemBlock, 0, s>>>((const uint8_t*)lhs.data, (const uint8_t*)rhs.data, lhs.is_scalar,
                                                 rhs.is_scalar, is_or, out_mask, n);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_binary(yq_operand lhs, yq_operand rhs, int32_t arith, void* out, uint32_t n, void* stream) {
  if (!lhs.data || !rhs.data || !out || lhs.type != rhs.type || arith < YQ_ADD || arith > YQ_MOD)
    return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  const int g = elem_grid(n, 4);
  ProfScope ps("elem_binary", s, (double)n * 3.0 * lhs.width);
  switch (lhs.type) {
    case YQ_INT32:
      k_binary<int32_t><<<g, kElemBlock, 0, s>>>((const int32_t*)lhs.data, (const int32_t*)rhs.data, lhs.is_scalar,
                                                 rhs.is_scalar, arith, (int32_t*)out, n);
      break;
    case YQ_FLOAT32:
      k_binary<float><<<g, kElemBlock, 0, s>>>((const float*)lhs.data, (const float*)rhs.data, lhs.is_scalar,
                                               rhs.is_scalar, arith, (float*)out, n);
      break;
    case YQ_INT64:
    case YQ_DATETIME:
      k_binary<int64_t><<<g, kElemBlock, 0, s>>>((const int64_t*)lhs.data, (const int64_t*)rhs.data, lhs.is_scalar,
                                                 rhs.is_scalar, arith, (int64_t*)out, n);
      break;
    default: return YQ_ERR_INVALID_ARG;
  }
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_cast(const void* src, int32_t src_type, void* dst, int32_t dst_type, uint32_t n, void* stream) {
  if (!src || !dst) return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  const int g = elem_grid(n, 4);
  auto norm = [](int t) { return t == YQ_DATETIME ? YQ_INT64 : t; };
  const int a = norm(src_type), b = norm(dst_type);
  ProfScope ps("elem_cast", s, (double)n * 8.0);
#define YQ_CAST(S_, SE, D_, DE)                                                                         \
  if (a == SE && b == DE) {                                                                             \
    k_cast<S_, D_><<<g, kElemBlock, 0, s>>>((const S_*)src, (D_*)dst, n);                               \
    YQ_CHECK_LAUNCH();                                                                                  \
    return YQ_OK;                                                                                       \
  }
  YQ_CAST(int32_t, YQ_INT32, float, YQ_FLOAT32)
  YQ_CAST(int32_t, YQ_INT32, int64_t, YQ_INT64)
  YQ_CAST(float, YQ_FLOAT32, int32_t, YQ_INT32)
  YQ_CAST(float, YQ_FLOAT32, int64_t, YQ_INT64)
  YQ_CAST(int64_t, YQ_INT64, int32_t, YQ_INT32)
  YQ_CAST(int64_t, YQ_INT64, float, YQ_FLOAT32)
  YQ_CAST(uint8_t, YQ_BOOL, uint32_t, YQ_INT32)
  YQ_CAST(float, YQ_FLOAT32, double, YQ_FLOAT64)
  YQ_CAST(double, YQ_FLOAT64, float, YQ_FLOAT32)
#undef YQ_CAST
  return YQ_ERR_UNSUPPORTED;
}

size_t yq_prefix_sum_workspace_size(uint32_t n) {
  WsSize w;
  w.add<unsigned long long>((size_t)ceil_div<uint32_t>(n, kScanTile) + 1);
  w.add<uint32_t>(4);
  return w.total();
}

int yq_prefix_sum_mask(const uint8_t* mask, uint32_t* out, uint32_t n, void* workspace, size_t workspace_bytes,
                       void* stream) {
  return prefix_sum<uint8_t>(mask, out, n, workspace, workspace_bytes, as_stream(stream));
}

int yq_prefix_sum_u32(const uint32_t* in, uint32_t* out, uint32_t n, void* workspace, size_t workspace_bytes,
                      void* stream) {
  return prefix_sum<uint32_t>(in, out, n, workspace, workspace_bytes, as_stream(stream));
}
int yq_move_rows_filter(const yq_column* src, const uint32_t* map, const uint8_t* mask, uint32_t n, yq_column* out,
                        void* stream) {
  if (!src || !out || !map || !mask || !src->data || !out->data || src->width != out->width ||
      !fixed_width_ok(src->type, src->width))
    return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  ProfScope ps("elem_move_filter", s, (double)n * (src->width + 5.0));
  k_move_filter<<<elem_grid(n, 4), kElemBlock, 0, s>>>((const char*)src->data, src->nulls, src->width, map, mask, n,
                                                       (char*)out->data);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_move_rows_join(const yq_column* src, const uint32_t* pairs, uint32_t npairs, int32_t is_right, yq_column* out,
                      void* stream) {
  if (!src || !out || !pairs || !src->data || !out->data || src->width != out->width ||
      !fixed_width_ok(src->type, src->width))
    return YQ_ERR_INVALID_ARG;
  if (npairs == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  ProfScope ps("elem_move_join", s, (double)npairs * (2.0 * src->width + 4.0));
  k_move_join<<<elem_grid(npairs, 4), kElemBlock, 0, s>>>((const char*)src->data, src->nulls, src->width, pairs,
                                                          npairs, is_right ? 1 : 0, (char*)out->data,
                                                          const_cast<uint8_t*>(out->nulls));
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_move_rows_merge(const yq_column* a, const yq_column* b, const uint32_t* idx, const uint8_t* from_a,
                       int32_t ascending, uint32_t n, yq_column* out, void* stream) {
  if (!a || !b || !out || !idx || !from_a || !a->data || !b->data || !out->data || a->width != out->width ||
      b->width != out->width || !fixed_width_ok(a->type, a->width))
    return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  ProfScope ps("elem_move_merge", s, (double)n * (2.0 * a->width + 5.0));
  k_move_merge<<<elem_grid(n, 4), kElemBlock, 0, s>>>((const char*)a->data, a->nulls, (const char*)b->data, b->nulls,
                                                      a->width, idx, from_a, ascending, n, (char*)out->data,
                                                      const_cast<uint8_t*>(out->nulls));
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_reduce(const void* values, int32_t type, const uint8_t* nulls, uint32_t n, int32_t kind, void* result,
              void* stream) {
  if (!result || (n > 0 && !values && kind != YQ_AGG_COUNT)) return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  const int g = elem_grid(n, 4);
  ProfScope ps("elem_reduce", s, (double)n * 4.0);
  if (kind == YQ_AGG_COUNT) {
    k_count_notnull<<<g, kElemBlock, 0, s>>>(nulls, n, (int*)result);
    YQ_CHECK_LAUNCH();
    return YQ_OK;
  }
  if (kind != YQ_AGG_SUM && kind != YQ_AGG_MIN && kind != YQ_AGG_MAX) return YQ_ERR_INVALID_ARG;
  switch (type) {
    case YQ_INT32:
      k_reduce<int32_t, int32_t><<<g, kElemBlock, 0, s>>>((const int32_t*)values, nulls, n, kind, (int32_t*)result);
      break;
    case YQ_INT64:
    case YQ_DATETIME:
      if (kind == YQ_AGG_SUM)
        k_reduce<long long, unsigned long long><<<g, kElemBlock, 0, s>>>((const long long*)values, nulls, n, kind,
                                                                         (unsigned long long*)result);
      else
        k_reduce<long long, long long><<<g, kElemBlock, 0, s>>>((const long long*)values, nulls, n, kind,
                                                                (long long*)result);
      break;
    case YQ_FLOAT32:
      if (kind == YQ_AGG_SUM)
        k_reduce<float, double><<<g, kElemBlock, 0, s>>>((const float*)values, nulls, n, kind, (double*)result);
      else
        k_reduce<float, float><<<g, kElemBlock, 0, s>>>((const float*)values, nulls, n, kind, (float*)result);
      break;
    default: return YQ_ERR_UNSUPPORTED;
  }
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_key_transform(const void* src, int32_t type, uint32_t* dst, uint32_t n, int32_t inverse, void* stream) {
  if (!src || !dst || (type != YQ_INT32 && type != YQ_FLOAT32 && type != YQ_INT64 && type != YQ_DATETIME))
    return YQ_ERR_INVALID_ARG;
  if (n == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  if (type == YQ_INT64 || type == YQ_DATETIME) {
    ProfScope ps("elem_key_transform", s, (double)n * 16.0);
    k_key_transform64<<<elem_grid(n, 4), kElemBlock, 0, s>>>((const unsigned long long*)src,
                                                             reinterpret_cast<unsigned long long*>(dst), n);
    YQ_CHECK_LAUNCH();
    return YQ_OK;
  }
  ProfScope ps("elem_key_transform", s, (double)n * 8.0);
  k_key_transform<<<elem_grid(n, 4), kElemBlock, 0, s>>>((const uint32_t*)src, type == YQ_FLOAT32, inverse, dst, n);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_merge_path(const void* a, const void* b, int32_t type, int32_t width, int32_t descending, uint32_t m,
                  uint32_t n, uint32_t k, void* out_keys, uint32_t* out_idx, uint8_t* out_from_a, int32_t* last_a,
                  void* stream) {
  if ((m && !a) || (n && !b) || !out_keys || !out_idx || !out_from_a || k > m + n || !fixed_width_ok(type, width))
    return YQ_ERR_INVALID_ARG;
  cudaStream_t s = as_stream(stream);
  const int g = (int)ceil_div<uint32_t>(k > 0 ? k : 1, kElemBlock * kMpItems);
  ProfScope ps("elem_merge_path", s, (double)k * (2.0 * width + 5.0));
  switch (type) {
    case YQ_INT32:
      k_merge_ref<int32_t><<<g, kElemBlock, 0, s>>>((const int32_t*)a, (const int32_t*)b, m, n, k, descending,
                                                    (int32_t*)out_keys, out_idx, out_from_a, last_a);
      break;
    case YQ_FLOAT32:
      k_merge_ref<float><<<g, kElemBlock, 0, s>>>((const float*)a, (const float*)b, m, n, k, descending,
                                                  (float*)out_keys, out_idx, out_from_a, last_a);
      break;
    case YQ_INT64:
    case YQ_DATETIME:
      k_merge_ref<int64_t><<<g, kElemBlock, 0, s>>>((const int64_t*)a, (const int64_t*)b, m, n, k, descending,
                                                    (int64_t*)out_keys, out_idx, out_from_a, last_a);
      break;
    case YQ_TEXT:
      k_merge_ref_text<<<g, kElemBlock, 0, s>>>((const uint8_t*)a, (const uint8_t*)b, width, m, n, k, descending,
                                                (uint8_t*)out_keys, out_idx, out_from_a, last_a);
      break;
    default: return YQ_ERR_UNSUPPORTED;
  }
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_cross_product_col(const yq_column* col, uint32_t left_rows, uint32_t right_rows, int32_t is_left,
                         yq_column* out, void* stream) {
  if (!col || !out || !col->data || !out->data || col->width != out->width || !fixed_width_ok(col->type, col->width))
    return YQ_ERR_INVALID_ARG;
  const unsigned long long total = (unsigned long long)left_rows * right_rows;
  if (total == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  ProfScope ps("elem_cross_col", s, (double)total * (col->width + (out->nulls ? 1.0 : 0.0)));
  k_cross_col<<<elem_grid(total > 0xffffffffull ? 0xffffffffu : (uint32_t)total, 4), kElemBlock, 0, s>>>(
      (const char*)col->data, col->nulls, col->width, left_rows, right_rows, is_left, (char*)out->data,
      const_cast<uint8_t*>(out->nulls));
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

// --------------------------------------------------- bounded-wait test hook
// Runs the production look-back (tile_lookback, the single-pass scan under
// WHERE compaction, projection and the prefix sums) as tile 1 of a chain whose
// tile 0 never publishes its status word, with the poll bound lowered to
// `spin_limit`: the wait runs out, the error word gets kErrTimeout and the
// call returns YQ_ERR_TIMEOUT. Nothing waits without a bound, so the device
// stays usable afterwards.
}  // extern "C"

namespace {
__global__ void k_debug_lookback_stall(unsigned long long* status, uint32_t* err, uint32_t limit,
                                       unsigned long long* excl_out) {
  const unsigned long long excl = tile_lookback(status, 1u, 7ull, err, limit);
  if (threadIdx.x == 0) *excl_out = excl;
}
}  // namespace

extern "C" int yq_debug_lookback_stall(uint32_t spin_limit, void* workspace, size_t workspace_bytes, void* stream) {
  if (!workspace || workspace_bytes < 64 || spin_limit == 0 || spin_limit > kSpinLimit) return YQ_ERR_INVALID_ARG;
  cudaStream_t s = as_stream(stream);
  unsigned long long* status = static_cast<unsigned long long*>(workspace);  // [0] tile 0, [1] tile 1
  uint32_t* err = reinterpret_cast<uint32_t*>(status + 2);
  unsigned long long* excl = status + 3;
  YQ_TRY_CUDA(cudaMemsetAsync(workspace, 0, 64, s));
  k_debug_lookback_stall<<<1, 32, 0, s>>>(status, err, spin_limit, excl);
  YQ_CHECK_LAUNCH();
  uint32_t e = 0;
  YQ_TRY(d2h_sync(&e, err, sizeof(e), s));
  return (e & kErrTimeout) ? YQ_ERR_TIMEOUT : YQ_OK;
}

extern "C" {
}  // extern "C"
