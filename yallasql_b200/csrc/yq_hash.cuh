// Cell access and equality hashing of join keys (sm_100a).
#pragma once

#include "yq_common.cuh"

namespace yq {

struct JCol {
  const char* data;
  const uint8_t* nulls;
  int32_t type;
  int32_t width;
};

// ----------------------------------------------------------- cell access
__device__ __forceinline__ uint64_t cell_u64(const JCol& c, uint32_t row) {
  switch (c.width) {
    case 4: {
      const uint32_t v = __ldg(reinterpret_cast<const uint32_t*>(c.data) + row);
      return c.type == YQ_INT32 ? (uint64_t)(int64_t)(int32_t)v : (uint64_t)v;
    }
    case 8: return (uint64_t)__ldg(reinterpret_cast<const unsigned long long*>(c.data) + row);
    default: return (uint64_t)(uint8_t)c.data[row];
  }
}

__device__ __forceinline__ bool cell_null(const JCol& c, uint32_t row) { return c.nulls && c.nulls[row]; }

// Normalised equality/hash key: -0.0 folds into +0.0 so they join.
__device__ __forceinline__ uint64_t hash_key(const JCol& c, uint32_t row) {
  uint64_t v = cell_u64(c, row);
  if (c.type == YQ_FLOAT32 && ((uint32_t)v & 0x7fffffffu) == 0u) v = 0;
  if (c.type == YQ_FLOAT64 && (v & 0x7fffffffffffffffull) == 0ull) v = 0;
  return v;
}

__device__ __forceinline__ uint32_t hash_bucket(uint64_t k, uint32_t nb) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return (uint32_t)k & (nb - 1u);
}

}  // namespace yq
