// Single-pass decoupled look-back over tiles (Merrill & Garland) with a
// bounded wait. Tile ids come from an atomic counter, so every predecessor of
// a tile is already resident when the tile waits on it; the bound only guards
// against a broken invariant, and running out of it sets an error flag and
// publishes an inclusive value so that no successor waits forever.
#pragma once

#include "yq_common.cuh"

namespace yq {

constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagIncl = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// Called by all 32 lanes of one warp. Publishes `agg` for `tile`, walks back
// over predecessors and returns the exclusive prefix of this tile (all lanes).
__device__ __forceinline__ unsigned long long tile_lookback(unsigned long long* status, uint32_t tile,
                                                            unsigned long long agg, uint32_t* err) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_relaxed_u64(status, kFlagIncl | agg);
    return 0ull;
  }
  if (lane == 0) st_relaxed_u64(status + tile, kFlagAgg | agg);
  unsigned long long excl = 0;
  long long base = (long long)tile - 1;
  uint32_t spins = 0;
  bool timed_out = false;
  for (;;) {
    const long long j = base - lane;
    unsigned long long s = (j >= 0) ? ld_relaxed_u64(status + j) : kFlagIncl;
    const unsigned long long flag = s & ~kValMask;
    if (__any_sync(0xffffffffu, flag == 0ull)) {
      // Give up at the bound, or early once another tile has already failed.
      if (++spins > kSpinLimit || ((spins & 63u) == 0u && ld_relaxed_u32(err) != 0u)) {
        timed_out = true;
        break;
      }
      __nanosleep(spins < 64 ? 32 : 256);
      continue;
    }
    const uint32_t incl = __ballot_sync(0xffffffffu, flag == kFlagIncl);
    if (incl) {
      const int first = __ffs(incl) - 1;  // nearest predecessor with an inclusive value
      excl += warp_sum_u64(lane <= first ? (s & kValMask) : 0ull);
      break;
    }
    excl += warp_sum_u64(s & kValMask);
    base -= 32;
  }
  if (timed_out) {
    if (lane == 0) atomicOr(err, kErrTimeout);
    excl = 0;
  }
  if (lane == 0) st_relaxed_u64(status + tile, kFlagIncl | ((excl + agg) & kValMask));
  return excl;
}

}  // namespace yq
