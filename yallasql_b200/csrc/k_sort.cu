// Stable LSD radix argsort for ORDER BY (sm_100a), onesweep style
// (Adinets & Merrill, "Onesweep: A Faster Least Significant Digit Radix Sort
// for GPUs", 2022): one upfront histogram kernel computes every pass's digit
// counts; each pass is then a single kernel that ranks a tile's digits with
// warp ballots, obtains the tile's global digit offsets through a decoupled
// look-back over tiles, and scatters through a shared-memory staging buffer so
// global writes are contiguous per digit run.
//
// Replaces BoundRefSortExpression + int_to_uint32/float_to_uint32 +
// launch_radix_sort (radix_sort_local_kerenl, launch_prefix_sum,
// radix_sort_shuffle per 4-bit pass) + move_rows_batch
// (include/engine/operators/expressions/bound_ref_sort.hpp:26-64,
//  src/kernels/radix_sort_utils.cu:4-53, src/kernels/radix_sort_kernel.cu:65-178,
//  include/kernels/radix_sort_kernel.hpp:26-73, include/kernels/move_rows_kernel.hpp:51-83).
//
// Segmented: rows are split into independent segments (sorted runs); tiles
// never straddle a segment and the look-back stops at a segment's first tile,
// so all 4 MB batches of a table (or all tasks of a batch) sort in one set of
// launches. A single global sort is the one-segment case.
#include <string.h>
#include <map>
#include <mutex>
#include <vector>
#include "yq_sort.cuh"

namespace yq {

constexpr int kSortBlock = 256;
constexpr uint32_t kStatAgg = 1u << 30;
constexpr uint32_t kStatIncl = 2u << 30;
constexpr uint32_t kStatMask = (1u << 30) - 1u;
constexpr uint32_t kMaxSortRows = (1u << 30) - 1u;

struct SegInfo {
  const uint32_t* seg_start;   // nseg + 1 row offsets
  const uint32_t* tile_start;  // nseg + 1 tile offsets
  const uint32_t* tile_seg;    // segment of every tile (null: binary search of tile_start)
  int32_t nseg;
};

template <int KW, int D>
__device__ __forceinline__ uint32_t digit_of(const uint32_t (&k)[KW], int shift) {
  const int w = shift >> 5, o = shift & 31;
  uint32_t lo = 0u, hi = 0u;
#pragma unroll
  for (int j = 0; j < KW; ++j) {
    if (j == w) lo = k[j];
    if (j == w + 1) hi = k[j];
  }
  uint32_t v = lo >> o;
  if (o + D > 32) v |= hi << (32 - o);
  return v & ((1u << D) - 1u);
}

__device__ __forceinline__ int find_segment(const SegInfo& g, uint32_t tile) {
  if (g.tile_seg) return (int)__ldg(g.tile_seg + tile);  // one load instead of a chain of dependent ones
  int lo = 0, hi = g.nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(g.tile_start + mid) <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------- histogram
// Each block owns a contiguous range of tiles; per-segment counts for every
// pass accumulate in shared memory and are flushed when the segment changes.
template <int KW, int D>
__global__ void __launch_bounds__(kSortBlock) k_sort_histogram(const KeySrc src, const SegInfo seg, uint32_t tile_rows,
                                                               uint32_t ntiles, uint32_t* __restrict__ hist) {
  constexpr int RADIX = 1 << D;
  constexpr int P = (KW * 32 + D - 1) / D;
  extern __shared__ uint32_t s_hist[];  // [P][RADIX]
  const int lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < P * RADIX; i += kSortBlock) s_hist[i] = 0u;
  __syncthreads();
  const uint32_t per = ceil_div<uint32_t>(ntiles, gridDim.x);
  const uint32_t t0 = blockIdx.x * per;
  const uint32_t t1 = min(ntiles, t0 + per);
  int cur = -1;
  for (uint32_t t = t0; t < t1; ++t) {
    const int sg = find_segment(seg, t);
    if (sg != cur) {
      if (cur >= 0) {
        __syncthreads();
        uint32_t* h = hist + (size_t)cur * P * RADIX;
        for (int i = threadIdx.x; i < P * RADIX; i += kSortBlock) {
          if (s_hist[i]) atomicAdd(h + i, s_hist[i]);
          s_hist[i] = 0u;
        }
        __syncthreads();
      }
      cur = sg;
    }
    const uint32_t lt = t - __ldg(seg.tile_start + sg);
    const uint32_t r0 = __ldg(seg.seg_start + sg) + lt * tile_rows;
    const uint32_t r1 = min(__ldg(seg.seg_start + sg + 1), r0 + tile_rows);
    for (uint32_t base = r0; base < r1; base += kSortBlock) {
      const uint32_t e = base + threadIdx.x;
      const bool valid = e < r1;
      uint32_t k[KW];
      const uint32_t row = valid ? (src.in_perm ? __ldg(src.in_perm + e) : e) : 0u;
      if (valid) make_key<KW>(src, row, k);
      else {
#pragma unroll
        for (int j = 0; j < KW; ++j) k[j] = 0u;
      }
      if (src.lossy) {  // the key column is read here anyway: flag values the key words cannot restore
        const bool l = valid && !(src.nulls && src.nulls[row]) &&
                       key_value_lossy(src.type, src.data + (size_t)row * src.width);
        if (__any_sync(0xffffffffu, l) && lane == 0) atomicOr(src.lossy, 1u);
      }
      const uint32_t vb = __ballot_sync(0xffffffffu, valid);
      const int first = __ffs(vb) - 1;
      // One vote per key: when every valid lane of the warp holds the same key
      // (all-equal columns, heavy Zipf heads) lane `first` counts them all.
      // Every lane executes the shuffle (full mask), valid or not.
      bool same = true;
#pragma unroll
      for (int j = 0; j < KW; ++j) {
        const uint32_t kf = __shfl_sync(0xffffffffu, k[j], first < 0 ? 0 : first);
        same &= (!valid || k[j] == kf);
      }
      if (__all_sync(0xffffffffu, same)) {
        if (lane == first) {
#pragma unroll
          for (int p = 0; p < P; ++p) atomicAdd(&s_hist[p * RADIX + digit_of<KW, D>(k, p * D)], (uint32_t)__popc(vb));
        }
      } else if (valid) {
#pragma unroll
        for (int p = 0; p < P; ++p) atomicAdd(&s_hist[p * RADIX + digit_of<KW, D>(k, p * D)], 1u);
      }
    }
  }
  __syncthreads();
  if (cur >= 0) {
    uint32_t* h = hist + (size_t)cur * P * RADIX;
    for (int i = threadIdx.x; i < P * RADIX; i += kSortBlock)
      if (s_hist[i]) atomicAdd(h + i, s_hist[i]);
  }
}

// --------------------------------------------------------------- onesweep
struct SweepParams {
  const uint32_t* keys_in;  // null on a key's first pass (keys come from src)
  const uint32_t* vals_in;  // null on a key's first pass (vals = source row)
  uint32_t* keys_out;       // null on the last pass
  uint32_t* vals_out;
  KeySrc src;
  SegInfo seg;
  const uint32_t* hist;  // [nseg][P][RADIX] of this key
  uint32_t* status;      // [ntiles][RADIX], zero on entry
  uint32_t* tile_counter;
  uint32_t* err;
  int32_t pass;          // index of this pass's digit (bit offset = pass * D)
  int32_t npass;         // P
};

// Blocks per SM the registers are sized for: four for the variants whose
// keys, values and ranks fit 64 registers without spilling (one key word, up
// to 12 items per thread, or 8 items of two words), three otherwise.
// Blocks of 512 threads get half as many blocks per SM and blocks of 128
// twice as many, so the per-thread register budget stays the same.
constexpr int sweep_min_blocks(int kw, int d, int items) { return (kw * items <= 12 && d == 8) || (kw == 2 && items <= 8 && d == 8) ? 4 : 3; }
constexpr int sweep_min_blocks(int kw, int d, int items, int block) {
  return block == 256 ? sweep_min_blocks(kw, d, items)
                      : (block > 256 ? (sweep_min_blocks(kw, d, items) + 1) / 2 : 2 * sweep_min_blocks(kw, d, items));
}

// BLOCK threads, ITEMS keys per thread: a tile of BLOCK * ITEMS rows. Every
// digit has its own thread in the per-digit steps (RADIX <= BLOCK).
template <int KW, int D, int ITEMS, int BLOCK>
__global__ void __launch_bounds__(BLOCK, sweep_min_blocks(KW, D, ITEMS, BLOCK)) k_sort_onesweep(const __grid_constant__ SweepParams S) {
  constexpr int RADIX = 1 << D;
  constexpr int NW = BLOCK / 32;
  constexpr uint32_t TILE = BLOCK * ITEMS;
  static_assert(RADIX <= BLOCK, "one digit per thread");

  extern __shared__ uint32_t smem[];
  uint32_t* s_whist = smem;                       // [NW][RADIX]
  uint32_t* s_tile_base = s_whist + NW * RADIX;   // [RADIX]
  uint32_t* s_glob = s_tile_base + RADIX;         // [RADIX]
  uint32_t* s_scan = s_glob + RADIX;              // [NW + 1]
  uint32_t* s_misc = s_scan + NW + 1;             // [4]
  uint32_t* s_keys = s_misc + 4;                  // [TILE][KW]
  uint32_t* s_vals = s_keys + TILE * KW;          // [TILE]

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_misc[0] = atomicAdd(S.tile_counter, 1u);
  for (int i = threadIdx.x; i < NW * RADIX; i += BLOCK) s_whist[i] = 0u;
  __syncthreads();
  const uint32_t tile = s_misc[0];
  const int sg = find_segment(S.seg, tile);
  const uint32_t lt = tile - __ldg(S.seg.tile_start + sg);
  const uint32_t seg0 = __ldg(S.seg.seg_start + sg);
  const uint32_t seg1 = __ldg(S.seg.seg_start + sg + 1);
  const uint32_t r0 = seg0 + lt * TILE;
  const uint32_t tile_n = min(TILE, seg1 - r0);
  const int shift = S.pass * D;

  // 1. load (warp-striped: element = r0 + warp*ITEMS*32 + k*32 + lane)
  uint32_t key[ITEMS][KW];
  uint32_t val[ITEMS];
  uint32_t rank[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t off = (uint32_t)(warp * ITEMS * 32 + k * 32 + lane);
    const uint32_t e = r0 + off;
    const bool valid = off < tile_n;
    if (valid) {
      if (S.keys_in) {
        if (KW == 1) {
          key[k][0] = __ldg(S.keys_in + e);
        } else if (KW == 2) {
          uint2 q = __ldg(reinterpret_cast<const uint2*>(S.keys_in) + e);
          key[k][0] = q.x;
          key[k][KW > 1 ? 1 : 0] = q.y;
        } else {
#pragma unroll
          for (int j = 0; j < KW; j += 4) {
            uint4 q = ldg_nc_v4(S.keys_in + (size_t)e * KW + j);
            key[k][j] = q.x;
            key[k][j + 1 < KW ? j + 1 : 0] = q.y;
            key[k][j + 2 < KW ? j + 2 : 0] = q.z;
            key[k][j + 3 < KW ? j + 3 : 0] = q.w;
          }
        }
        val[k] = __ldg(S.vals_in + e);
      } else {
        const uint32_t row = S.src.in_perm ? __ldg(S.src.in_perm + e) : e;
        make_key<KW>(S.src, row, key[k]);
        val[k] = row;
      }
    } else {
#pragma unroll
      for (int j = 0; j < KW; ++j) key[k][j] = 0u;
      val[k] = 0u;
    }
  }

  // 2. warp-level stable ranking (order within a warp = (k, lane))
  const uint32_t lt_mask = lanemask_lt();
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t off = (uint32_t)(warp * ITEMS * 32 + k * 32 + lane);
    const bool valid = off < tile_n;
    uint32_t peers = __ballot_sync(0xffffffffu, valid);
    const uint32_t dk = digit_of<KW, D>(key[k], shift);
#pragma unroll
    for (int b = 0; b < D; ++b) {
      const bool bit = (dk >> b) & 1u;
      const uint32_t bb = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bb : ~bb;
    }
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0u;
    if (valid && lane == leader) {
      old = s_whist[warp * RADIX + dk];
      s_whist[warp * RADIX + dk] = old + __popc(peers);
    }
    old = __shfl_sync(0xffffffffu, old, leader < 0 ? 0 : leader);
    rank[k] = old + __popc(peers & lt_mask);
    __syncwarp();
  }
  __syncthreads();

  // 3. per-digit: warp offsets, tile count, global digit base of the segment
  const int t = threadIdx.x;
  uint32_t tile_count = 0u, seg_count = 0u;
  if (t < RADIX) {
    for (int w = 0; w < NW; ++w) {
      const uint32_t c = s_whist[w * RADIX + t];
      s_whist[w * RADIX + t] = tile_count;
      tile_count += c;
    }
    seg_count = __ldg(S.hist + ((size_t)sg * S.npass + S.pass) * RADIX + t);
  }
  uint32_t total;
  const uint32_t tile_excl = block_exclusive_sum<BLOCK>(t < RADIX ? tile_count : 0u, s_scan, total);
  const uint32_t seg_excl = block_exclusive_sum<BLOCK>(t < RADIX ? seg_count : 0u, s_scan, total);

  // 4. decoupled look-back per digit over the segment's earlier tiles
  if (t < RADIX) {
    s_tile_base[t] = tile_excl;
    uint32_t* st = S.status + (size_t)tile * RADIX + t;
    uint32_t excl = 0u;
    if (lt == 0) {
      st_relaxed_u32(st, kStatIncl | tile_count);
    } else {
      st_relaxed_u32(st, kStatAgg | tile_count);
      const uint32_t* p = st - RADIX;
      uint32_t back = lt;
      uint32_t spins = 0;
      while (back > 0) {
        const uint32_t v = ld_relaxed_u32(p);
        const uint32_t f = v & ~kStatMask;
        if (f == 0u) {
          if (++spins > kSpinLimit || ((spins & 63u) == 0u && ld_relaxed_u32(S.err) != 0u)) {
            atomicOr(S.err, kErrTimeout);
            break;
          }
          __nanosleep(spins < 64 ? 32 : 128);
          continue;
        }
        excl += v & kStatMask;
        if (f == kStatIncl) break;
        p -= RADIX;
        --back;
      }
      st_relaxed_u32(st, kStatIncl | ((excl + tile_count) & kStatMask));
    }
    s_glob[t] = seg0 + seg_excl + excl;
  }
  __syncthreads();

  // 5. stage the tile in shared memory in digit order
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t off = (uint32_t)(warp * ITEMS * 32 + k * 32 + lane);
    if (off < tile_n) {
      const uint32_t dk = digit_of<KW, D>(key[k], shift);
      const uint32_t lp = s_tile_base[dk] + s_whist[warp * RADIX + dk] + rank[k];
      if (lp >= tile_n) {
        atomicOr(S.err, kErrBounds);
        continue;
      }
#pragma unroll
      for (int j = 0; j < KW; ++j) s_keys[lp * KW + j] = key[k][j];
      s_vals[lp] = val[k];
    }
  }
  __syncthreads();

  // 6. contiguous scatter per digit run
  for (uint32_t i = threadIdx.x; i < tile_n; i += BLOCK) {
    uint32_t kk[KW];
#pragma unroll
    for (int j = 0; j < KW; ++j) kk[j] = s_keys[i * KW + j];
    const uint32_t d = digit_of<KW, D>(kk, shift);
    const uint32_t g = s_glob[d] + (i - s_tile_base[d]);
    if (g < seg0 || g >= seg1) {  // offsets inconsistent with the histogram: skip, report
      atomicOr(S.err, kErrBounds);
      continue;
    }
    if (S.keys_out) {
      if (KW == 1) {
        S.keys_out[g] = kk[0];
      } else if (KW == 2) {
        reinterpret_cast<uint2*>(S.keys_out)[g] = make_uint2(kk[0], kk[KW > 1 ? 1 : 0]);
      } else {
#pragma unroll
        for (int j = 0; j < KW; j += 4)
          *reinterpret_cast<uint4*>(S.keys_out + (size_t)g * KW + j) =
              make_uint4(kk[j], kk[j + 1 < KW ? j + 1 : 0], kk[j + 2 < KW ? j + 2 : 0], kk[j + 3 < KW ? j + 3 : 0]);
      }
    }
    S.vals_out[g] = s_vals[i];
  }
}

// Which passes change the order, decided on the device so the host reads 16
// bytes per pass instead of every segment's histogram. Per pass p:
// sum[4p] = 1 while every non-empty segment's keys share one digit,
// sum[4p+1] / sum[4p+2] = the least / greatest such digit, sum[4p+3] = 1 when a
// non-empty segment exists. Block (p, b): its warps take segments
// b*64 + warp, + 8, ...; a warp's lanes look at 8 bins each.
__global__ void k_pass_summary_init(int32_t* sum, int P) {
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    sum[4 * p] = 1;
    sum[4 * p + 1] = 0x7fffffff;
    sum[4 * p + 2] = -1;
    sum[4 * p + 3] = 0;
  }
}

__global__ void k_pass_summary(const uint32_t* __restrict__ hist, const uint32_t* __restrict__ seg_start, int nseg,
                               int P, int R, int32_t* sum) {
  const int p = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g_end = min(nseg, (int)(blockIdx.y + 1) * 64);
  for (int g = blockIdx.y * 64 + warp; g < g_end; g += blockDim.x / 32) {
    const uint32_t len = __ldg(seg_start + g + 1) - __ldg(seg_start + g);
    if (len == 0) continue;
    const uint32_t* hp = hist + ((size_t)g * P + p) * R;
    int one = -1;
    for (int d = lane; d < R; d += 32)
      if (__ldg(hp + d) == len) one = d;  // at most one bin can hold every key
    const uint32_t hit = __ballot_sync(0xffffffffu, one >= 0);
    if (lane == 0) {
      atomicOr(sum + 4 * p + 3, 1);
      if (!hit) atomicAnd(sum + 4 * p, 0);
    }
    if (hit && lane == __ffs(hit) - 1) {
      atomicMin(sum + 4 * p + 1, one);
      atomicMax(sum + 4 * p + 2, one);
    }
  }
}

// tile_seg[t] = the segment tile t belongs to: block g fills segment g's tiles.
__global__ void k_fill_tile_seg(const uint32_t* __restrict__ tile_start, int nseg, uint32_t* __restrict__ tile_seg) {
  for (int g = blockIdx.x; g < nseg; g += gridDim.x) {
    const uint32_t t0 = __ldg(tile_start + g), t1 = __ldg(tile_start + g + 1);
    for (uint32_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) tile_seg[t] = (uint32_t)g;
  }
}

__global__ void k_iota_segments(uint32_t* out, const uint32_t* in_perm, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = in_perm ? in_perm[i] : i;
}

// Number of significant 4-byte words of a text column (index of the last
// nonzero word + 1 over all rows).
__global__ void k_text_words(const char* data, const uint8_t* nulls, int width, uint32_t n, uint32_t* out) {
  uint32_t best = 0;
  const int words = width >> 2;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    if (nulls && nulls[r]) continue;
    const uint32_t* p = reinterpret_cast<const uint32_t*>(data + (size_t)r * width);
    for (int j = words - 1; j >= (int)best; --j)
      if (__ldg(p + j)) {
        best = j + 1;
        break;
      }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, d));
  if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

// ------------------------------------------------------------------ gather
struct GatherCol {
  const char* src;
  const uint8_t* src_nulls;
  char* dst;
  uint8_t* dst_nulls;
  const uint32_t* only_if;  // non-null: the column moves only when *only_if != 0
  int32_t width;
};
struct GatherParams {
  GatherCol c[YQ_MAX_BATCH_COLUMNS];
  int32_t ncols;
};

__device__ __forceinline__ void copy_bytes(char* dst, const char* src, int width) {
  if (width == 4) *reinterpret_cast<uint32_t*>(dst) = __ldg(reinterpret_cast<const uint32_t*>(src));
  else if (width == 8)
    *reinterpret_cast<unsigned long long*>(dst) = __ldg(reinterpret_cast<const unsigned long long*>(src));
  else if (width == 1) *dst = *src;
  else if ((width & 15) == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0)
    for (int i = 0; i < width; i += 16) *reinterpret_cast<uint4*>(dst + i) = ldg_nc_v4(src + i);
  else
    for (int i = 0; i < width; i += 4)
      *reinterpret_cast<uint32_t*>(dst + i) = __ldg(reinterpret_cast<const uint32_t*>(src + i));
}

// Column-parallel gather: blockIdx.y picks the column, each thread moves
// kGatherItems rows of it with all random loads issued before any store, so
// a warp keeps 8 x 32 independent sector reads in flight.
constexpr int kGatherItems = 8;

template <typename V>
__device__ __forceinline__ void gather_rows(const V* __restrict__ src, V* __restrict__ dst,
                                            const uint32_t* __restrict__ perm, uint32_t i0, uint32_t n) {
  uint32_t r[kGatherItems];
  V v[kGatherItems];
#pragma unroll
  for (int k = 0; k < kGatherItems; ++k) {
    const uint32_t i = i0 + k * 256;
    r[k] = i < n ? __ldg(perm + i) : 0xffffffffu;
  }
#pragma unroll
  for (int k = 0; k < kGatherItems; ++k)
    if (r[k] < n) v[k] = __ldg(src + r[k]);
#pragma unroll
  for (int k = 0; k < kGatherItems; ++k)
    if (r[k] < n) dst[i0 + k * 256] = v[k];
}

__global__ void __launch_bounds__(256) k_gather_cols(const __grid_constant__ GatherParams G,
                                                     const uint32_t* __restrict__ perm, uint32_t n) {
  const GatherCol& g = G.c[blockIdx.y];
  if (g.only_if && *g.only_if == 0u) return;
  for (uint32_t base = blockIdx.x * (256u * kGatherItems); base < n; base += gridDim.x * (256u * kGatherItems)) {
    const uint32_t i0 = base + threadIdx.x;
    switch (g.width) {
      case 4:
        gather_rows<uint32_t>(reinterpret_cast<const uint32_t*>(g.src), reinterpret_cast<uint32_t*>(g.dst), perm, i0, n);
        break;
      case 8:
        gather_rows<unsigned long long>(reinterpret_cast<const unsigned long long*>(g.src),
                                        reinterpret_cast<unsigned long long*>(g.dst), perm, i0, n);
        break;
      case 16:
        gather_rows<uint4>(reinterpret_cast<const uint4*>(g.src), reinterpret_cast<uint4*>(g.dst), perm, i0, n);
        break;
      case 1:
        gather_rows<uint8_t>(reinterpret_cast<const uint8_t*>(g.src), reinterpret_cast<uint8_t*>(g.dst), perm, i0, n);
        break;
      default:
        for (int k = 0; k < kGatherItems; ++k) {
          const uint32_t i = i0 + k * 256;
          if (i >= n) break;
          const uint32_t r = __ldg(perm + i);
          if (r < n) copy_bytes(g.dst + (size_t)i * g.width, g.src + (size_t)r * g.width, g.width);
        }
    }
    if (g.dst_nulls) {
      for (int k = 0; k < kGatherItems; ++k) {
        const uint32_t i = i0 + k * 256;
        if (i >= n) break;
        const uint32_t r = __ldg(perm + i);
        if (r < n) g.dst_nulls[i] = g.src_nulls ? g.src_nulls[r] : 0;
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_gather(const __grid_constant__ GatherParams G, const uint32_t* __restrict__ perm,
                                                uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t r = __ldg(perm + i);
    if (r >= n) continue;  // perm must be a permutation of [0, n): skip anything else
    for (int c = 0; c < G.ncols; ++c) {
      const GatherCol& g = G.c[c];
      if (g.only_if && *g.only_if == 0u) continue;
      copy_bytes(g.dst + (size_t)i * g.width, g.src + (size_t)r * g.width, g.width);
      if (g.dst_nulls) g.dst_nulls[i] = g.src_nulls ? g.src_nulls[r] : 0;
    }
  }
}

// -------------------------------------------------------------- host side
struct SortShape {
  int kw;     // key words (1, 2, 4, 8)
  int vwords;
  int null_word;
};

static int key_value_words(const yq_column& c) {
  switch (c.type) {
    case YQ_INT32:
    case YQ_FLOAT32:
    case YQ_BOOL: return 1;
    case YQ_INT64:
    case YQ_DATETIME:
    case YQ_FLOAT64: return 2;
    case YQ_TEXT: return c.width / 4;
    default: return -1;
  }
}

static bool valid_key_column(const yq_column& c) {
  if (!c.data) return false;
  switch (c.type) {
    case YQ_INT32:
    case YQ_FLOAT32: return c.width == 4;
    case YQ_INT64:
    case YQ_DATETIME:
    case YQ_FLOAT64: return c.width == 8;
    case YQ_BOOL: return c.width == 1;
    case YQ_TEXT: return c.width >= 4 && c.width <= YQ_MAX_TEXT_WIDTH && c.width % 4 == 0;
    default: return false;
  }
}

static int round_kw(int w) { return w <= 1 ? 1 : (w <= 2 ? 2 : (w <= 4 ? 4 : (w <= 8 ? 8 : -1))); }

template <int KW, int D, int ITEMS, int BLOCK>
static size_t sweep_smem() {
  constexpr int RADIX = 1 << D;
  constexpr int NW = BLOCK / 32;
  return sizeof(uint32_t) * ((size_t)NW * RADIX + 2 * RADIX + NW + 1 + 4 + (size_t)BLOCK * ITEMS * (KW + 1));
}

template <int KW, int D, int ITEMS, int BLOCK>
static int launch_sweep(const SweepParams& P, uint32_t ntiles, cudaStream_t s) {
  const size_t smem = sweep_smem<KW, D, ITEMS, BLOCK>();
  YQ_TRY(kernel_allow_smem((const void*)k_sort_onesweep<KW, D, ITEMS, BLOCK>, smem));
  k_sort_onesweep<KW, D, ITEMS, BLOCK><<<ntiles, BLOCK, smem, s>>>(P);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

template <int KW, int D>
static int launch_hist(const KeySrc& src, const SegInfo& seg, uint32_t tile_rows, uint32_t ntiles, uint32_t* hist,
                       cudaStream_t s) {
  constexpr int P = (KW * 32 + D - 1) / D;
  const size_t smem = sizeof(uint32_t) * P * (1 << D);
  YQ_TRY(kernel_allow_smem((const void*)k_sort_histogram<KW, D>, smem));
  int grid = sm_count() * 4;
  if ((uint32_t)grid > ntiles) grid = (int)ntiles;
  if (grid < 1) grid = 1;
  k_sort_histogram<KW, D><<<grid, kSortBlock, smem, s>>>(src, seg, tile_rows, ntiles, hist);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

// Dispatch table over (KW, D, ITEMS, BLOCK).
struct SortKernels {
  int (*hist)(const KeySrc&, const SegInfo&, uint32_t, uint32_t, uint32_t*, cudaStream_t);
  int (*sweep)(const SweepParams&, uint32_t, cudaStream_t);
  int items;
  int block;
  uint32_t tile_rows() const { return (uint32_t)(items * block); }
};

template <int KW, int D, int ITEMS, int BLOCK = kSortBlock>
static SortKernels make_kernels() {
  SortKernels k;
  k.hist = &launch_hist<KW, D>;
  k.sweep = &launch_sweep<KW, D, ITEMS, BLOCK>;
  k.items = ITEMS;
  k.block = BLOCK;
  return k;
}

// Instantiated (key words, digit bits, items per thread, block threads)
// variants; items = 0 picks the default for (kw, d) and block = 0 the
// 256-thread block. Every variant's tile (items x block) is at least
// min_tile_rows(kw), which sizes the look-back status.
static bool pick_kernels(int kw, int d, int items, int block, SortKernels& k) {
  if (block == 512) {
    switch (kw * 10000 + d * 100 + items) {
      case 10808: case 10800: k = make_kernels<1, 8, 8, 512>(); return true;
      case 10812: k = make_kernels<1, 8, 12, 512>(); return true;
      case 20808: case 20800: k = make_kernels<2, 8, 8, 512>(); return true;
      default: return false;
    }
  }
  if (block == 128) {
    switch (kw * 10000 + d * 100 + items) {
      case 10616: case 10600: k = make_kernels<1, 6, 16, 128>(); return true;
      case 10416: case 10400: k = make_kernels<1, 4, 16, 128>(); return true;
      case 20616: case 20600: k = make_kernels<2, 6, 16, 128>(); return true;
      default: return false;
    }
  }
  if (block != 0 && block != kSortBlock) return false;
  switch (kw * 10000 + d * 100 + items) {
    case 10816: k = make_kernels<1, 8, 16>(); return true;
    case 10812: case 10800: k = make_kernels<1, 8, 12>(); return true;  // 12 items: four blocks per SM
    case 10808: k = make_kernels<1, 8, 8>(); return true;
    case 10616: case 10600: k = make_kernels<1, 6, 16>(); return true;
    case 10416: case 10400: k = make_kernels<1, 4, 16>(); return true;
    case 20812: case 20800: k = make_kernels<2, 8, 12>(); return true;
    case 20808: k = make_kernels<2, 8, 8>(); return true;
    case 20612: case 20600: k = make_kernels<2, 6, 12>(); return true;
    case 20412: case 20400: k = make_kernels<2, 4, 12>(); return true;
    case 40808: case 40800: k = make_kernels<4, 8, 8>(); return true;
    case 80804: case 80800: k = make_kernels<8, 8, 4>(); return true;
    default: return false;
  }
}
static bool pick_kernels(int kw, int d, int items, SortKernels& k) { return pick_kernels(kw, d, items, 0, k); }

// Fewest rows per tile any variant of key width kw uses (sizes the look-back
// status of the most tiles a tuned choice can make).
static uint32_t min_tile_rows(int kw) { return (uint32_t)kSortBlock * (kw == 8 ? 4 : 8); }

// Autotuned variant per (key words, log2 of rows per segment).
struct TunedSort {
  int d = 8, items = 0, block = 0;
};
static std::mutex g_tune_mu;
static std::map<std::pair<int, int>, TunedSort> g_tuned;

static int rows_bucket(uint32_t rows, int nseg) {
  uint32_t avg = nseg > 0 ? rows / (uint32_t)nseg : rows;
  int b = 0;
  while (avg > 1) {
    avg >>= 1;
    ++b;
  }
  return b;
}

static TunedSort tuned_choice(int kw, uint32_t rows, int nseg) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find({kw, rows_bucket(rows, nseg)});
  if (it == g_tuned.end()) return TunedSort{};
  return it->second;
}

struct SegPlan {
  std::vector<uint32_t> seg;    // nseg + 1
  std::vector<uint32_t> tiles;  // nseg + 1
  uint32_t ntiles = 0;
};

static void plan_segments(const uint32_t* offsets, int nseg, uint32_t tile_rows, SegPlan& sp) {
  sp.seg.assign(offsets, offsets + nseg + 1);
  sp.tiles.resize(nseg + 1);
  uint32_t t = 0;
  for (int i = 0; i < nseg; ++i) {
    sp.tiles[i] = t;
    const uint32_t len = offsets[i + 1] - offsets[i];
    t += ceil_div<uint32_t>(len, tile_rows);
  }
  sp.tiles[nseg] = t;
  sp.ntiles = t;
}

// One key of a (possibly multi-key) segmented sort: perm_in (null = identity) -> perm_out.

// Resolved plan for one key: words, digit width, tiling.
struct KeyPlan {
  SortShape sh;
  int D, P, R;
  SortKernels K;
  uint32_t tile_rows, ntiles;
};

// want_d / want_items / want_block = 0: the autotuned choice for this key
// width and segment size (yq_sort_autotune), else 8-bit digits with the
// default items and 256-thread blocks. `sizing`: tile count for the smallest
// tile any variant uses (workspace bound).
static int plan_key(const yq_column& c, int vwords_override, int want_d, int want_items, int want_block,
                    const uint32_t* seg_offsets, int nseg, KeyPlan& kp, bool sizing = false,
                    int null_word_override = -1) {
  kp.sh.vwords = vwords_override >= 0 ? vwords_override : key_value_words(c);
  kp.sh.null_word = null_word_override >= 0 ? null_word_override : c.nulls != nullptr;
  kp.sh.kw = round_kw(kp.sh.vwords + kp.sh.null_word);
  if (kp.sh.kw < 0) return YQ_ERR_UNSUPPORTED;
  kp.D = want_d;
  int items = want_items, block = want_block;
  if (kp.D == 0) {
    const TunedSort t = tuned_choice(kp.sh.kw, seg_offsets[nseg] - seg_offsets[0], nseg);
    kp.D = t.d;
    if (items == 0) items = t.items;
    if (block == 0) block = t.block;
  }
  if (!pick_kernels(kp.sh.kw, kp.D, items, block, kp.K)) {
    kp.D = 8;
    if (!pick_kernels(kp.sh.kw, 8, 0, kp.K)) return YQ_ERR_UNSUPPORTED;
  }
  kp.P = (kp.sh.kw * 32 + kp.D - 1) / kp.D;
  kp.R = 1 << kp.D;
  kp.tile_rows = sizing ? min_tile_rows(kp.sh.kw) : kp.K.tile_rows();
  kp.ntiles = 0;
  for (int i = 0; i < nseg; ++i) kp.ntiles += ceil_div<uint32_t>(seg_offsets[i + 1] - seg_offsets[i], kp.tile_rows);
  return YQ_OK;
}

// Workspace: [seg offsets][tile offsets][histograms][look-back status per pass]
//            [counters][keys A/B][vals A/B][perm between keys]
int sort_key_words_max(const yq_column& c) {
  int vw = key_value_words(c);
  if (vw < 0) return -1;
  if (c.type == YQ_TEXT && vw > 8 - (c.nulls ? 1 : 0)) vw = 8 - (c.nulls ? 1 : 0);
  return round_kw(vw + (c.nulls ? 1 : 0));
}

// Key words of every row in row order (a key whose passes all fall out: its
// sorted order is the row order).
template <int KW>
__global__ void k_make_keys(const KeySrc src, uint32_t* __restrict__ out, uint32_t rows) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    uint32_t k[KW];
    make_key<KW>(src, src.in_perm ? __ldg(src.in_perm + r) : r, k);
#pragma unroll
    for (int j = 0; j < KW; ++j) out[(size_t)r * KW + j] = k[j];
  }
}

static int launch_make_keys(int kw, const KeySrc& src, uint32_t* out, uint32_t rows, cudaStream_t s) {
  const int grid = sm_count() * 8;
  switch (kw) {
    case 1: k_make_keys<1><<<grid, 256, 0, s>>>(src, out, rows); break;
    case 2: k_make_keys<2><<<grid, 256, 0, s>>>(src, out, rows); break;
    case 4: k_make_keys<4><<<grid, 256, 0, s>>>(src, out, rows); break;
    case 8: k_make_keys<8><<<grid, 256, 0, s>>>(src, out, rows); break;
    default: return YQ_ERR_UNSUPPORTED;
  }
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int sort_segments_impl(const KeyJob* jobs, int njobs, uint32_t rows, const uint32_t* seg_offsets_host, int nseg,
                       uint32_t* out_perm, const yq_sort_config* cfg, void* workspace, size_t workspace_bytes,
                       cudaStream_t s, size_t* size_only, uint32_t* keys_out, int* kw_out, bool defer_err,
                       uint32_t** err_out, uint32_t* high_out) {
  if (keys_out && (njobs != 1 || !kw_out)) return YQ_ERR_INVALID_ARG;
  if (kw_out) *kw_out = 0;
  if (high_out) memset(high_out, 0, 8 * sizeof(uint32_t));
  if (njobs <= 0 || nseg <= 0 || !seg_offsets_host) return YQ_ERR_INVALID_ARG;
  if (rows > kMaxSortRows) return YQ_ERR_UNSUPPORTED;
  if (seg_offsets_host[0] != 0 || seg_offsets_host[nseg] != rows) return YQ_ERR_INVALID_ARG;
  for (int i = 0; i < nseg; ++i)
    if (seg_offsets_host[i + 1] < seg_offsets_host[i]) return YQ_ERR_INVALID_ARG;
  const int want_d = cfg ? cfg->digit_bits : 0;
  const int want_items = cfg ? cfg->items_per_thread : 0;
  const int want_block = cfg ? cfg->block_threads : 0;
  if (want_d != 0 && want_d != 4 && want_d != 6 && want_d != 8) return YQ_ERR_INVALID_ARG;
  if (want_items < 0 || want_items > 16) return YQ_ERR_INVALID_ARG;
  if (want_block != 0 && want_block != 128 && want_block != 256 && want_block != 512) return YQ_ERR_INVALID_ARG;
  const bool keep_trivial = cfg && cfg->keep_trivial;

  // Size buffers for the widest plan any key can take (text keys are sized
  // for their full slot, up to 8 words; their significant width is measured
  // on the device before they are sorted).
  size_t max_kw = 1, max_hist = 1, max_status = 1, max_tiles = 1;
  for (int j = 0; j < njobs; ++j) {
    const yq_column& c = jobs[j].key;
    if (!valid_key_column(c)) return YQ_ERR_INVALID_ARG;
    KeyPlan kp;
    int vw = key_value_words(c);
    if (c.type == YQ_TEXT && vw > 8 - (c.nulls ? 1 : 0)) vw = 8 - (c.nulls ? 1 : 0);
    // Sized for 8-bit digits (the largest passes x bins) and the fewest items
    // per thread (the most tiles), which bound every variant's buffers.
    int st = plan_key(c, vw, 8, 0, 0, seg_offsets_host, nseg, kp, true);
    if (st != YQ_OK) return st;
    // For a text key this is the plan at its full (clamped) width, which
    // bounds every narrower plan: fewer words mean fewer passes and larger tiles.
    max_kw = kp.sh.kw > (int)max_kw ? kp.sh.kw : max_kw;
    const size_t h = (size_t)nseg * kp.P * kp.R, sz = (size_t)kp.P * kp.ntiles * kp.R;
    if (h > max_hist) max_hist = h;
    if (sz > max_status) max_status = sz;
    if (kp.ntiles > max_tiles) max_tiles = kp.ntiles;
  }

  WsSize w;
  w.add<uint32_t>(nseg + 1);
  w.add<uint32_t>(nseg + 1);
  w.add<uint32_t>(max_hist);
  w.add<uint32_t>(max_status);
  w.add<uint32_t>(80 + 4 * 64);
  w.add<uint32_t>((size_t)rows * max_kw);
  w.add<uint32_t>((size_t)rows * max_kw);
  w.add<uint32_t>(rows);
  w.add<uint32_t>(rows);
  w.add<uint32_t>(rows);
  w.add<uint32_t>(max_tiles + 1);  // segment of every tile
  if (size_only) {
    *size_only = w.total();
    return YQ_OK;
  }
  if (!out_perm) return YQ_ERR_INVALID_ARG;
  if (rows == 0) return YQ_OK;

  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, w.total(), s));
  uint32_t* d_seg = ws.take<uint32_t>(nseg + 1);
  uint32_t* d_tiles = ws.take<uint32_t>(nseg + 1);
  uint32_t* d_hist = ws.take<uint32_t>(max_hist);
  uint32_t* d_status = ws.take<uint32_t>(max_status);
  uint32_t* d_misc = ws.take<uint32_t>(80 + 4 * 64);  // [0..63] tile counters, [64] error, [65] text words,
                                                       // [66..] pass summary
  uint32_t* d_keys[2] = {ws.take<uint32_t>((size_t)rows * max_kw), ws.take<uint32_t>((size_t)rows * max_kw)};
  uint32_t* d_vals[2] = {ws.take<uint32_t>(rows), ws.take<uint32_t>(rows)};
  uint32_t* d_perm_tmp = ws.take<uint32_t>(rows);
  uint32_t* d_tile_seg = ws.take<uint32_t>(max_tiles + 1);
  // tile offsets of a plan on the device, with the segment of every tile
  auto upload_tiles = [&](const SegPlan& p) -> int {
    YQ_TRY(h2d_async(d_tiles, p.tiles.data(), (nseg + 1) * sizeof(uint32_t), s));
    if (p.ntiles > max_tiles) return YQ_ERR_UNSUPPORTED;
    const int g = nseg < 4096 ? nseg : 4096;
    k_fill_tile_seg<<<g, 256, 0, s>>>(d_tiles, nseg, d_tile_seg);
    YQ_CHECK_LAUNCH();
    return YQ_OK;
  };
  uint32_t* d_err = d_misc + 64;
  uint32_t* d_textw = d_misc + 65;
  YQ_TRY_CUDA(cudaMemsetAsync(d_misc, 0, 80 * sizeof(uint32_t), s));

  const uint32_t* perm_in = nullptr;  // order from the less significant keys (null = identity)
  for (int jj = njobs - 1; jj >= 0; --jj) {
    const KeyJob& job = jobs[jj];
    const yq_column& c = job.key;
    int vw = -1;
    if (c.type == YQ_TEXT) {
      // Only the significant prefix of the slot takes part: trailing all-zero
      // words are equal for every row.
      uint32_t tw = 0;
      YQ_TRY_CUDA(cudaMemsetAsync(d_textw, 0, sizeof(uint32_t), s));
      k_text_words<<<sm_count() * 4, 256, 0, s>>>(static_cast<const char*>(c.data), c.nulls, c.width, rows, d_textw);
      YQ_CHECK_LAUNCH();
      YQ_TRY(d2h_sync(&tw, d_textw, sizeof(uint32_t), s));
      vw = (int)tw;
      if (vw == 0 && !c.nulls) continue;  // every key equal: order unchanged
    }
    // A text key longer than one pass's key (8 words, 7 with a NULL word) is
    // sorted as a chain of chunk keys, its last chunk first (stable LSD over
    // chunks): chunk 0 holds the leading words and the NULL word; NULL rows
    // read as zero in the other chunks, so their order among themselves is
    // kept. Every chunk reads the same slots at an offset (row stride = width).
    const int lead = 8 - (c.nulls ? 1 : 0);
    int nchunks = 1;
    if (c.type == YQ_TEXT && vw > lead) {
      if (keys_out) return YQ_ERR_UNSUPPORTED;  // merges carry one key of at most 8 words
      nchunks = 1 + (vw - lead + 7) / 8;
    }
    for (int ch = nchunks - 1; ch >= 0; --ch) {
    yq_column cc = c;
    int cvw = vw;
    int cnull = c.nulls != nullptr;
    if (nchunks > 1) {
      const int w0 = ch == 0 ? 0 : lead + (ch - 1) * 8;
      const int w1 = ch == 0 ? lead : (w0 + 8 < vw ? w0 + 8 : vw);
      cc.data = const_cast<char*>(static_cast<const char*>(c.data)) + 4 * w0;
      cvw = w1 - w0;
      cnull = (ch == 0 && c.nulls) ? 1 : 0;
    }
    KeyPlan kp;
    YQ_TRY(plan_key(cc, cvw, want_d, want_items, want_block, seg_offsets_host, nseg, kp, false, cnull));
    SegPlan sp;
    plan_segments(seg_offsets_host, nseg, kp.tile_rows, sp);
    YQ_TRY(h2d_async(d_seg, sp.seg.data(), (nseg + 1) * sizeof(uint32_t), s));
    YQ_TRY(upload_tiles(sp));
    YQ_TRY_CUDA(cudaMemsetAsync(d_hist, 0, (size_t)nseg * kp.P * kp.R * sizeof(uint32_t), s));
    YQ_TRY_CUDA(cudaMemsetAsync(d_status, 0, (size_t)kp.P * sp.ntiles * kp.R * sizeof(uint32_t), s));
    YQ_TRY_CUDA(cudaMemsetAsync(d_misc, 0, 64 * sizeof(uint32_t), s));

    KeySrc src;
    src.data = static_cast<const char*>(cc.data);
    src.nulls = c.nulls;
    src.in_perm = perm_in;
    src.type = c.type;
    src.width = c.width;
    src.vwords = kp.sh.vwords;
    src.desc = job.desc;
    src.nulls_first = job.nulls_first;
    src.null_word = kp.sh.null_word;
    src.lossy = nchunks == 1 ? job.lossy : nullptr;
    SegInfo seg;
    seg.seg_start = d_seg;
    seg.tile_start = d_tiles;
    seg.tile_seg = d_tile_seg;
    seg.nseg = nseg;
    {
      // algorithmic bytes: each key read once (+ the incoming permutation)
      ProfScope ps("sort_histogram", s, (double)rows * (c.width + (perm_in ? 4 : 0)));
      YQ_TRY(kp.K.hist(src, seg, kp.tile_rows, sp.ntiles, d_hist, s));
    }

    std::vector<int> passes;
    KeyPlan kq = kp;  // the passes' plan: kp, or fewer key words when the leading ones are shared
    uint32_t high[8] = {0};
    if (keep_trivial) {
      for (int p = 0; p < kp.P; ++p) passes.push_back(p);
    } else {
      // A pass whose digit is the same for every key of every segment leaves
      // the order unchanged and is skipped. common[p] = that digit when it is
      // also the same across segments, else -1.
      if (kp.P > 64) return YQ_ERR_UNSUPPORTED;
      int32_t* d_sum = reinterpret_cast<int32_t*>(d_misc + 66);  // [4 * P] summary words (P <= 64 here)
      k_pass_summary_init<<<1, 64, 0, s>>>(d_sum, kp.P);
      YQ_CHECK_LAUNCH();
      k_pass_summary<<<dim3((unsigned)kp.P, (unsigned)ceil_div(nseg, 64)), 256, 0, s>>>(d_hist, d_seg, nseg, kp.P,
                                                                                          kp.R, d_sum);
      YQ_CHECK_LAUNCH();
      int32_t sum[4 * 64];
      YQ_TRY(d2h_sync(sum, d_sum, (size_t)kp.P * 4 * sizeof(int32_t), s));
      std::vector<int> common(kp.P, -1);
      for (int p = 0; p < kp.P; ++p) {
        const bool trivial = sum[4 * p] != 0;
        // -2: no non-empty segment; -1: segments disagree on the digit
        const int digit = !sum[4 * p + 3] ? -2 : (sum[4 * p + 1] == sum[4 * p + 2] ? sum[4 * p + 1] : -1);
        if (!trivial) passes.push_back(p);
        else common[p] = digit;
      }
      // Leading words whose every digit is common to all rows: the passes
      // keep the words below them (a kernel width of 1, 2 or 4 words).
      if (32 % kp.D == 0 && !passes.empty()) {
        const int ppw = 32 / kp.D;
        int shared = 0;
        for (int w = kp.sh.kw - 1; w >= 1; --w) {
          bool all = true;
          for (int q = 0; q < ppw && all; ++q) all = common[w * ppw + q] >= 0;
          if (!all) break;
          ++shared;
        }
        const int kw_eff = round_kw(kp.sh.kw - shared);
        if (kw_eff > 0 && kw_eff < kp.sh.kw && pick_kernels(kw_eff, kp.D, 0, kq.K)) {
          kq.sh.kw = kw_eff;
          kq.P = kw_eff * ppw;
          kq.tile_rows = kq.K.tile_rows();
          for (int w = kw_eff; w < kp.sh.kw; ++w)
            for (int q = 0; q < ppw; ++q) high[w - kw_eff] |= (uint32_t)common[w * ppw + q] << (q * kp.D);
          std::vector<int> kept;
          for (int p : passes)
            if (p < kq.P) kept.push_back(p);
          passes.swap(kept);
        } else {
          kq = kp;
        }
      }
    }
    if (keys_out) *kw_out = kq.sh.kw;
    if (high_out) memcpy(high_out, high, sizeof(high));
    if (passes.empty()) {  // order unchanged by this key
      if (keys_out) YQ_TRY(launch_make_keys(kq.sh.kw, src, keys_out, rows, s));
      continue;
    }
    if (kq.sh.kw != kp.sh.kw) {  // tiles of the narrower kernels
      plan_segments(seg_offsets_host, nseg, kq.tile_rows, sp);
      YQ_TRY(upload_tiles(sp));
      YQ_TRY_CUDA(cudaMemsetAsync(d_status, 0, passes.size() * sp.ntiles * kq.R * sizeof(uint32_t), s));
    }
    if (passes.size() > 64) return YQ_ERR_UNSUPPORTED;
    uint32_t* dst_perm = (perm_in == out_perm) ? d_perm_tmp : out_perm;
    for (size_t i = 0; i < passes.size(); ++i) {
      const bool first = (i == 0), last = (i + 1 == passes.size());
      SweepParams Sp;
      Sp.keys_in = first ? nullptr : d_keys[(i - 1) & 1];
      Sp.vals_in = first ? nullptr : d_vals[(i - 1) & 1];
      Sp.keys_out = last ? keys_out : d_keys[i & 1];
      Sp.vals_out = last ? dst_perm : d_vals[i & 1];
      Sp.src = src;
      Sp.seg = seg;
      Sp.hist = d_hist;
      Sp.status = d_status + (size_t)i * sp.ntiles * kq.R;
      Sp.tile_counter = d_misc + i;
      Sp.err = d_err;
      Sp.pass = passes[i];
      Sp.npass = kp.P;
      // algorithmic bytes: keys + row ids in, keys + row ids out (the first
      // pass reads the raw key (+ incoming permutation), the last writes ids only)
      const double kb = 4.0 * kq.sh.kw;
      const double in_b = first ? (double)c.width + (perm_in ? 4.0 : 0.0) : kb + 4.0;
      const double out_b = (last && !keys_out) ? 4.0 : kb + 4.0;
      ProfScope ps("sort_onesweep", s, (double)rows * (in_b + out_b));
      YQ_TRY(kq.K.sweep(Sp, sp.ntiles, s));
    }
    perm_in = dst_perm;
    }  // chunks of a long text key
  }
  if (perm_in != out_perm) {
    if (perm_in) {
      YQ_TRY_CUDA(cudaMemcpyAsync(out_perm, perm_in, (size_t)rows * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    } else {
      k_iota_segments<<<sm_count() * 4, 256, 0, s>>>(out_perm, nullptr, rows);
      YQ_CHECK_LAUNCH();
    }
  }
  if (err_out) *err_out = d_err;
  if (!keep_trivial && !defer_err) {
    uint32_t err = 0;
    YQ_TRY(d2h_sync(&err, d_err, sizeof(uint32_t), s));
    if (err & kErrTimeout) return YQ_ERR_TIMEOUT;
    if (err & kErrBounds) return YQ_ERR_INVALID_ARG;
  }
  return YQ_OK;
}

// Gather used by yq_gather and yq_order_by (see yq_sort.cuh).
int gather_impl(const yq_column* in, int32_t ncols, const uint32_t* perm, uint32_t rows, const yq_column* out,
                const uint32_t* const* only_if, cudaStream_t s) {
  if (ncols < 0 || ncols > YQ_MAX_BATCH_COLUMNS || (ncols > 0 && (!in || !out)) || (rows > 0 && !perm))
    return YQ_ERR_INVALID_ARG;
  if (rows == 0 || ncols == 0) return YQ_OK;
  GatherParams G;
  memset(&G, 0, sizeof(G));
  G.ncols = ncols;
  for (int c = 0; c < ncols; ++c) {
    if (!in[c].data || !out[c].data || in[c].width != out[c].width || in[c].width <= 0) return YQ_ERR_INVALID_ARG;
    if (in[c].width != 1 && in[c].width % 4 != 0) return YQ_ERR_INVALID_ARG;
    G.c[c].src = static_cast<const char*>(in[c].data);
    G.c[c].src_nulls = in[c].nulls;
    G.c[c].dst = static_cast<char*>(out[c].data);
    G.c[c].dst_nulls = const_cast<uint8_t*>(out[c].nulls);
    G.c[c].width = in[c].width;
    G.c[c].only_if = only_if ? only_if[c] : nullptr;
  }
  // Aligned columns (16-byte text slots, 4/8-byte values) take the
  // column-parallel kernel; others the row-parallel one.
  bool aligned = true;
  for (int c = 0; c < ncols; ++c)
    aligned &= ((reinterpret_cast<uintptr_t>(G.c[c].src) | reinterpret_cast<uintptr_t>(G.c[c].dst)) &
                (uintptr_t)(G.c[c].width >= 16 ? 15 : (G.c[c].width >= 8 ? 7 : (G.c[c].width >= 4 ? 3 : 0)))) == 0;
  double row_bytes = 4.0;  // permutation
  for (int c = 0; c < ncols; ++c)
    if (!only_if || !only_if[c]) row_bytes += 2.0 * in[c].width + (out[c].nulls ? 2.0 : 0.0);
  ProfScope ps("gather", s, (double)rows * row_bytes);
  if (aligned) {
    const uint32_t tiles = ceil_div<uint32_t>(rows, 256u * kGatherItems);
    const uint32_t cap = (uint32_t)sm_count() * 8;
    dim3 grid(tiles < cap ? tiles : cap, (unsigned)ncols);
    k_gather_cols<<<grid, 256, 0, s>>>(G, perm, rows);
  } else {
    int grid = (int)ceil_div<uint32_t>(rows, 256);
    const int cap = sm_count() * 16;
    if (grid > cap) grid = cap;
    k_gather<<<grid, 256, 0, s>>>(G, perm, rows);
  }
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

}  // namespace yq

using namespace yq;

extern "C" {

size_t yq_sort_workspace_size(const yq_column* key, uint32_t rows) {
  if (!key) return 0;
  KeyJob j{*key, 0, 0};
  uint32_t offs[2] = {0, rows};
  size_t bytes = 0;
  if (sort_segments_impl(&j, 1, rows, offs, 1, nullptr, nullptr, nullptr, 0, nullptr, &bytes) != YQ_OK) return 0;
  return bytes;
}

int yq_sort_indices(const yq_column* key, uint32_t rows, int32_t descending, int32_t nulls_first, uint32_t* out_perm,
                    const yq_sort_config* config, void* workspace, size_t workspace_bytes, void* stream) {
  if (!key) return YQ_ERR_INVALID_ARG;
  KeyJob j{*key, descending != 0, nulls_first != 0};
  uint32_t offs[2] = {0, rows};
  return sort_segments_impl(&j, 1, rows, offs, 1, out_perm, config, workspace, workspace_bytes, as_stream(stream),
                            nullptr);
}

int yq_sort_indices_multi(const yq_column* keys, const int32_t* descending, const int32_t* nulls_first, int32_t nkeys,
                          uint32_t rows, uint32_t* out_perm, const yq_sort_config* config, void* workspace,
                          size_t workspace_bytes, void* stream) {
  if (!keys || nkeys <= 0 || nkeys > YQ_MAX_BATCH_COLUMNS) return YQ_ERR_INVALID_ARG;
  std::vector<KeyJob> jobs(nkeys);
  for (int i = 0; i < nkeys; ++i) {
    jobs[i].key = keys[i];
    jobs[i].desc = descending ? descending[i] != 0 : 0;
    jobs[i].nulls_first = nulls_first ? nulls_first[i] != 0 : 0;
  }
  uint32_t offs[2] = {0, rows};
  return sort_segments_impl(jobs.data(), nkeys, rows, offs, 1, out_perm, config, workspace, workspace_bytes,
                            as_stream(stream), nullptr);
}

size_t yq_sort_segments_workspace_size(const yq_column* key, uint32_t rows, const uint32_t* seg_offsets, int32_t nseg) {
  if (!key) return 0;
  KeyJob j{*key, 0, 0};
  size_t bytes = 0;
  if (sort_segments_impl(&j, 1, rows, seg_offsets, nseg, nullptr, nullptr, nullptr, 0, nullptr, &bytes) != YQ_OK)
    return 0;
  return bytes;
}

int yq_sort_segments(const yq_column* key, uint32_t rows, const uint32_t* seg_offsets, int32_t nseg, int32_t descending,
                     int32_t nulls_first, uint32_t* out_perm, const yq_sort_config* config, void* workspace,
                     size_t workspace_bytes, void* stream) {
  if (!key) return YQ_ERR_INVALID_ARG;
  KeyJob j{*key, descending != 0, nulls_first != 0};
  return sort_segments_impl(&j, 1, rows, seg_offsets, nseg, out_perm, config, workspace, workspace_bytes,
                            as_stream(stream), nullptr);
}

int yq_sort_autotune(const yq_column* key, uint32_t rows, const uint32_t* seg_offsets, int32_t nseg,
                     int32_t descending, yq_sort_config* best, void* stream) {
  if (!key || !seg_offsets || nseg <= 0 || !best || !valid_key_column(*key)) return YQ_ERR_INVALID_ARG;
  const int kw = round_kw(key_value_words(*key) + (key->nulls ? 1 : 0));
  if (kw < 0) return YQ_ERR_UNSUPPORTED;
  // Every instantiated (digit bits, items per thread, block threads) variant
  // of this key width.
  std::vector<TunedSort> cand;
  for (int d : {8, 6, 4})
    for (int it : {16, 12, 8, 4})
      for (int b : {256, 512, 128}) {
        SortKernels k;
        if (pick_kernels(kw, d, it, b, k) && k.items == it && k.block == b) cand.push_back(TunedSort{d, it, b});
      }
  if (cand.empty()) return YQ_ERR_UNSUPPORTED;
  cudaStream_t s = as_stream(stream);
  KeyJob j{*key, descending != 0, 0};
  size_t wsb = 0;
  YQ_TRY(sort_segments_impl(&j, 1, rows, seg_offsets, nseg, nullptr, nullptr, nullptr, 0, nullptr, &wsb));
  void* ws = nullptr;
  uint32_t* perm = nullptr;
  YQ_TRY_CUDA(cudaMallocAsync(&ws, wsb, s));
  YQ_TRY_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&perm), (size_t)(rows ? rows : 1) * 4, s));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  YQ_TRY_CUDA(cudaEventCreate(&e0));
  YQ_TRY_CUDA(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  TunedSort pick = cand[0];
  int status = YQ_OK;
  for (const auto& c : cand) {
    yq_sort_config cfg{c.d, c.items, c.block, 1};
    status = sort_segments_impl(&j, 1, rows, seg_offsets, nseg, perm, &cfg, ws, wsb, s, nullptr);  // warm-up
    if (status != YQ_OK) break;
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3 && status == YQ_OK; ++r)
      status = sort_segments_impl(&j, 1, rows, seg_offsets, nseg, perm, &cfg, ws, wsb, s, nullptr);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (status == YQ_OK && ms < best_ms) {
      best_ms = ms;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(ws, s);
  cudaFreeAsync(perm, s);
  if (status != YQ_OK) return status;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[{kw, rows_bucket(rows, nseg)}] = pick;
  }
  best->digit_bits = pick.d;
  best->items_per_thread = pick.items;
  best->block_threads = pick.block;
  best->keep_trivial = 0;
  return YQ_OK;
}

int yq_gather(const yq_column* in, int32_t ncols, const uint32_t* perm, uint32_t rows, yq_column* out, void* stream) {
  return gather_impl(in, ncols, perm, rows, out, nullptr, as_stream(stream));
}

}  // extern "C"
