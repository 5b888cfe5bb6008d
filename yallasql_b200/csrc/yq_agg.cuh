// Aggregate states and their block / grid reduction (sm_100a).
//
// Every thread keeps one count and one 64-bit running value per aggregate
// (yq_vm.cuh AggEmit). At the end of a kernel the block reduces them with
// warp shuffles and one pass over the warps, writes one partial per block,
// and the last block to finish folds the partials in block order into the
// caller's state (one ticket atomic per block), so the result does not
// depend on which block finished last.
#pragma once

#ifndef __CUDACC_RTC__
#include <limits.h>
#endif
#include "yq_vm.cuh"

namespace yq {

struct Acc {
  long long cnt;            // values absorbed (COUNT, and the divisor of AVG)
  unsigned long long bits;  // int64 or double bits of SUM / MIN / MAX
};

// State buffer of yq_agg_state_*: YQ_MAX_AGGREGATES states, then an error word.
constexpr size_t kAggStateBytes = 256;
static_assert(sizeof(Acc) * YQ_MAX_AGGREGATES + sizeof(uint32_t) <= kAggStateBytes, "aggregate state layout");

__host__ __device__ inline uint32_t* agg_state_err(Acc* state) {
  return reinterpret_cast<uint32_t*>(state + YQ_MAX_AGGREGATES);
}

__host__ __device__ inline unsigned long long acc_identity(int upd) {
  switch (upd) {
    case UPD_MIN_I: return (unsigned long long)LLONG_MAX;
    case UPD_MAX_I: return (unsigned long long)LLONG_MIN;
    case UPD_MIN_F: return 0x7ff0000000000000ull;  // +inf
    case UPD_MAX_F: return 0xfff0000000000000ull;  // -inf
    default: return 0ull;
  }
}

__device__ __forceinline__ unsigned long long acc_merge(int upd, unsigned long long a, unsigned long long b) {
  switch (upd) {
    case UPD_SUM_I: return (unsigned long long)((long long)a + (long long)b);
    case UPD_MIN_I: return (long long)b < (long long)a ? b : a;
    case UPD_MAX_I: return (long long)b > (long long)a ? b : a;
    case UPD_SUM_F: return from_f64(as_f64(a) + as_f64(b));
    case UPD_MIN_F: return as_f64(b) < as_f64(a) ? b : a;
    case UPD_MAX_F: return as_f64(b) > as_f64(a) ? b : a;
    default: return a;
  }
}

struct AggParams {
  int32_t nagg;
  uint8_t upd[YQ_MAX_AGGREGATES];
};

__device__ __forceinline__ void agg_thread_init(AggEmit& E, const AggParams& A) {
#pragma unroll
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) {
    E.cnt[a] = 0u;
    E.acc[a] = acc_identity(a < A.nagg ? A.upd[a] : UPD_COUNT);
  }
}

// Block reduction of every thread's accumulators into out[0, nagg) (one
// partial per block and step); ends with the block synchronised.
template <int BLOCK>
__device__ __forceinline__ void agg_block_partial(const AggEmit& E, uint32_t nsel, const AggParams& A, Acc* out) {
  __shared__ Acc s_part[BLOCK / 32][YQ_MAX_AGGREGATES];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) {
    if (a < A.nagg) {
      const int upd = A.upd[a];
      long long c = (upd == UPD_COUNT_STAR) ? (long long)nsel : (long long)E.cnt[a];
      unsigned long long v = E.acc[a];
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, d);
        v = acc_merge(upd, v, __shfl_down_sync(0xffffffffu, v, d));
      }
      if (lane == 0) s_part[warp][a] = Acc{c, v};
    }
  }
  __syncthreads();
  if (threadIdx.x < A.nagg) {
    const int a = threadIdx.x, upd = A.upd[a];
    Acc t = s_part[0][a];
    for (int w = 1; w < BLOCK / 32; ++w) {
      t.cnt += s_part[w][a].cnt;
      t.bits = acc_merge(upd, t.bits, s_part[w][a].bits);
    }
    out[a] = t;
  }
  __syncthreads();
}

// `nsel` = rows this thread selected (COUNT(*)).
template <int BLOCK>
__device__ __forceinline__ void agg_block_finish(const AggEmit& E, uint32_t nsel, const AggParams& A,
                                                 Acc* __restrict__ partials, uint32_t* ticket, Acc* state) {
  __shared__ Acc s_acc[BLOCK / 32][YQ_MAX_AGGREGATES];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) {
    if (a < A.nagg) {
      const int upd = A.upd[a];
      long long c = (upd == UPD_COUNT_STAR) ? (long long)nsel : (long long)E.cnt[a];
      unsigned long long v = E.acc[a];
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, d);
        v = acc_merge(upd, v, __shfl_down_sync(0xffffffffu, v, d));
      }
      if (lane == 0) s_acc[warp][a] = Acc{c, v};
    }
  }
  __syncthreads();
  if (threadIdx.x < A.nagg) {
    const int a = threadIdx.x, upd = A.upd[a];
    Acc t = s_acc[0][a];
    for (int w = 1; w < BLOCK / 32; ++w) {
      t.cnt += s_acc[w][a].cnt;
      t.bits = acc_merge(upd, t.bits, s_acc[w][a].bits);
    }
    partials[blockIdx.x * YQ_MAX_AGGREGATES + a] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // The last block folds the partials with every thread (blocks t, t + BLOCK,
  // ... per thread, then the warps, then across warps): independent loads
  // instead of one chain of gridDim.x dependent ones.
#pragma unroll
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) {
    if (a < A.nagg) {
      const int upd = A.upd[a];
      long long c = 0;
      unsigned long long v = acc_identity(upd);
      for (uint32_t b = threadIdx.x; b < gridDim.x; b += BLOCK) {
        const Acc* p = partials + b * YQ_MAX_AGGREGATES + a;
        c += __ldcg(&p->cnt);
        v = acc_merge(upd, v, __ldcg(&p->bits));
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, d);
        v = acc_merge(upd, v, __shfl_down_sync(0xffffffffu, v, d));
      }
      if (lane == 0) s_acc[warp][a] = Acc{c, v};
    }
  }
  __syncthreads();
  if (threadIdx.x < A.nagg) {
    const int a = threadIdx.x, upd = A.upd[a];
    Acc t = s_acc[0][a];
    for (int w = 1; w < BLOCK / 32; ++w) {
      t.cnt += s_acc[w][a].cnt;
      t.bits = acc_merge(upd, t.bits, s_acc[w][a].bits);
    }
    Acc s = state[a];
    s.cnt += t.cnt;
    s.bits = acc_merge(upd, s.bits, t.bits);
    state[a] = s;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

}  // namespace yq
