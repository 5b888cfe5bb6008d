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

// Predecessor words read per lane and round: a warp looks at a window of 128
// predecessors per memory round trip. Many tiles finish together, so the
// nearest inclusive value can lie a whole wave of tiles back; a wide window
// reaches it in one or two round trips.
constexpr int kLookbackPerLane = 4;
constexpr int kLookbackWindow = 32 * kLookbackPerLane;

// Called by all 32 lanes of one warp. Publishes `agg` for `tile`, walks back
// over predecessors and returns the exclusive prefix of this tile (all lanes).
// `limit` bounds the polls of one unpublished word (kSpinLimit unless a test
// lowers it); running out sets kErrTimeout in *err.
// Window position p (0 = nearest predecessor) is word base - p, read by lane
// p / kLookbackPerLane. The walk waits while a word nearer than the nearest
// inclusive one is unpublished; otherwise it adds the window's values up to
// and including that inclusive word and stops, or adds the whole window and
// moves it back.
__device__ __forceinline__ unsigned long long tile_lookback(unsigned long long* status, uint32_t tile,
                                                            unsigned long long agg, uint32_t* err,
                                                            uint32_t limit = kSpinLimit) {
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
    unsigned long long w[kLookbackPerLane];
#pragma unroll
    for (int i = 0; i < kLookbackPerLane; ++i) {
      const long long j = base - (long long)(lane * kLookbackPerLane + i);
      w[i] = (j >= 0) ? ld_relaxed_u64(status + j) : kFlagIncl;  // before tile 0: inclusive 0
    }
    int fz = kLookbackPerLane, fi = kLookbackPerLane;  // this lane's first unpublished / inclusive word
#pragma unroll
    for (int i = kLookbackPerLane - 1; i >= 0; --i) {
      const unsigned long long flag = w[i] & ~kValMask;
      if (flag == 0ull) fz = i;
      if (flag == kFlagIncl) fi = i;
    }
    const uint32_t zl = __ballot_sync(0xffffffffu, fz < kLookbackPerLane);
    const uint32_t il = __ballot_sync(0xffffffffu, fi < kLookbackPerLane);
    const int lz = zl ? __ffs(zl) - 1 : 0, li = il ? __ffs(il) - 1 : 0;
    const int fz_at = __shfl_sync(0xffffffffu, fz, lz), fi_at = __shfl_sync(0xffffffffu, fi, li);
    const int gz = zl ? lz * kLookbackPerLane + fz_at : kLookbackWindow;
    const int gi = il ? li * kLookbackPerLane + fi_at : kLookbackWindow;
    if (gz < gi) {
      // Give up at the bound, or early once another tile has already failed.
      if (++spins > limit || ((spins & 63u) == 0u && ld_relaxed_u32(err) != 0u)) {
        timed_out = true;
        break;
      }
      __nanosleep(spins < 64 ? 32 : 256);
      continue;
    }
    unsigned long long part = 0;
#pragma unroll
    for (int i = 0; i < kLookbackPerLane; ++i)
      if (lane * kLookbackPerLane + i <= gi) part += w[i] & kValMask;
    excl += warp_sum_u64(part);
    if (gi < kLookbackWindow) break;
    base -= kLookbackWindow;
  }
  if (timed_out) {
    if (lane == 0) atomicOr(err, kErrTimeout);
    excl = 0;
  }
  if (lane == 0) st_relaxed_u64(status + tile, kFlagIncl | ((excl + agg) & kValMask));
  return excl;
}

}  // namespace yq
