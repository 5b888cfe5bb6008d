// Out-of-core ORDER BY: merge path over sorted runs (sm_100a).
//
// Replaces OrderOperator::merge_two_runs / load_in_buffer / shift_buffer and
// merge_sorted_array_kernel_v1 + move_one_col_merge
// (src/engine/operators/order_operator.cpp:14-220, src/kernels/merge_batchs.cu:14-148,
//  src/kernels/move_rows_kernel.cu:73-105). The reference walks two runs with a
// host loop of BUFFER_SZ windows (D2D copies per column and a blocking D2H per
// window); here one launch merges every pair of runs of a level:
//   1. k_merge_partition: one thread per output tile finds the tile's co-rank
//      (how many outputs come from run A) by binary search on the merge path;
//   2. k_merge_tiles: each block stages its slice of both runs' keys in shared
//      memory with 1-D TMA bulk copies (cp.async.bulk, no multicast) completing
//      on an mbarrier, merges there (ties take run A, so the merge is stable),
//      and moves every payload column with coalesced writes.
#include <string.h>
#include <map>
#include <mutex>
#include <vector>
#include "yq_sort.cuh"

namespace yq {

constexpr int kMergeBlock = 256;
constexpr int kMergeItems = 8;
constexpr uint32_t kMergeTile = kMergeBlock * kMergeItems;  // outputs per block
constexpr uint32_t kFromB = 0x80000000u;

struct MergePair {
  uint32_t a0, m;  // run A rows [a0, a0 + m)
  uint32_t b0, n;  // run B rows [b0, b0 + n)
  uint32_t out0;   // output row of the pair's first element
  uint32_t tile0;  // first global tile of the pair
};

struct MergeCol {
  const char* src;
  const uint8_t* src_nulls;
  char* dst;
  uint8_t* dst_nulls;
  int32_t width;
  int32_t vec;  // src and dst aligned to `width`: cells move as one 4/8/16-byte word
};

struct MergeParams {
  KeySrc key;
  MergeCol c[YQ_MAX_BATCH_COLUMNS];
  int32_t ncols;
  int32_t npairs;
  uint32_t ntiles;
  int32_t staged;  // stage key slices in shared memory (key width <= 32 bytes)
  const MergePair* pairs;
  uint32_t* split;  // co-rank of each tile's first output
  uint32_t* err;
};

__device__ __forceinline__ int pair_of_tile(const MergePair* pairs, int npairs, uint32_t tile) {
  int lo = 0, hi = npairs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&pairs[mid].tile0) <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int KW>
__device__ __forceinline__ void key_at(const KeySrc& s, uint32_t row, uint32_t (&k)[KW]) {
  make_key<KW>(s, row, k);
}

// Merge-path co-rank: number of A elements among the first k outputs,
// ties taken from A. A = rows [a0, a0+m), B = rows [b0, b0+n) of the key column.
template <int KW>
__device__ uint32_t corank_global(const KeySrc& s, uint32_t a0, uint32_t m, uint32_t b0, uint32_t n, uint32_t k) {
  uint32_t lo = k > n ? k - n : 0u, hi = k < m ? k : m;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    uint32_t ka[KW], kb[KW];
    key_at<KW>(s, a0 + mid, ka);
    key_at<KW>(s, b0 + (k - mid - 1), kb);
    if (key_le<KW>(ka, kb)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

template <int KW>
__global__ void k_merge_partition(const __grid_constant__ MergeParams M) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M.ntiles) return;
  const int q = pair_of_tile(M.pairs, M.npairs, t);
  const MergePair p = M.pairs[q];
  const uint32_t k = (t - p.tile0) * kMergeTile;
  M.split[t] = corank_global<KW>(M.key, p.a0, p.m, p.b0, p.n, k);
}

// Stage the raw key bytes of rows [r0, r1) into `dst` so that row r lands at
// dst + (r*W - floor16(r0*W)) relative to the 16-byte-aligned window start.
// The aligned interior goes through TMA, the ragged ends through plain loads.
// Returns the TMA bytes issued (thread 0 only issues).
__device__ __forceinline__ uint32_t stage_rows(char* dst, const char* col, int W, uint32_t r0, uint32_t r1,
                                               uint64_t* bar, bool issue) {
  if (r1 <= r0) return 0u;
  const uintptr_t g0 = reinterpret_cast<uintptr_t>(col) + (uintptr_t)r0 * W;
  const uintptr_t g1 = reinterpret_cast<uintptr_t>(col) + (uintptr_t)r1 * W;
  const uintptr_t base = g0 & ~(uintptr_t)15;
  const uintptr_t in0 = (g0 + 15) & ~(uintptr_t)15;
  const uintptr_t in1 = g1 & ~(uintptr_t)15;
  uint32_t tma = 0;
  if (in1 > in0) {
    tma = (uint32_t)(in1 - in0);
    if (issue) tma_load_1d(dst + (in0 - base), reinterpret_cast<const void*>(in0), tma, bar);
  }
  // ragged head [g0, min(in0, g1)) and tail [max(in1, in0), g1), 4 bytes at a time
  const uintptr_t h1 = in0 < g1 ? in0 : g1;
  for (uintptr_t a = g0 + threadIdx.x * 4; a < h1; a += kMergeBlock * 4)
    *reinterpret_cast<uint32_t*>(dst + (a - base)) = *reinterpret_cast<const uint32_t*>(a);
  const uintptr_t t0 = in1 > in0 ? in1 : (in0 < g1 ? in0 : g1);
  for (uintptr_t a = t0 + threadIdx.x * 4; a < g1; a += kMergeBlock * 4)
    *reinterpret_cast<uint32_t*>(dst + (a - base)) = *reinterpret_cast<const uint32_t*>(a);
  return tma;
}

__device__ __forceinline__ void copy_cell(char* dst, const char* src, int width) {
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

// Move kMergeItems cells of one column (value type V, widths 4/8/16).
template <typename V>
__device__ __forceinline__ void move_items(const MergeCol& mc, const uint32_t (&rows)[kMergeItems], uint32_t out_base) {
  const V* src = reinterpret_cast<const V*>(mc.src);
  V* dst = reinterpret_cast<V*>(mc.dst);
  V v[kMergeItems];
#pragma unroll
  for (int i = 0; i < kMergeItems; ++i)
    if (rows[i] != 0xffffffffu) v[i] = __ldg(src + rows[i]);
#pragma unroll
  for (int i = 0; i < kMergeItems; ++i)
    if (rows[i] != 0xffffffffu) dst[out_base + threadIdx.x + i * kMergeBlock] = v[i];
}

template <int KW>
__global__ void __launch_bounds__(kMergeBlock) k_merge_tiles(const __grid_constant__ MergeParams M) {
  extern __shared__ __align__(128) char smem[];
  const uint32_t t = blockIdx.x;
  const int q = pair_of_tile(M.pairs, M.npairs, t);
  const MergePair p = M.pairs[q];
  const uint32_t lt = t - p.tile0;
  const uint32_t total = p.m + p.n;
  const uint32_t k0 = lt * kMergeTile;
  const uint32_t k1 = min(k0 + kMergeTile, total);
  const uint32_t cnt = k1 - k0;
  const uint32_t i0 = M.split[t];
  const bool last_of_pair = (q + 1 < M.npairs) ? (t + 1 >= M.pairs[q + 1].tile0) : (t + 1 >= M.ntiles);
  const uint32_t i1 = last_of_pair ? p.m : M.split[t + 1];
  const uint32_t j0 = k0 - i0, j1 = k1 - i1;
  const uint32_t ma = i1 - i0, nb = j1 - j0;
  if (i1 < i0 || j1 < j0 || ma + nb != cnt || i1 > p.m || j1 > p.n) {  // inconsistent split: report, write nothing
    if (threadIdx.x == 0) atomicOr(M.err, kErrBounds);
    return;
  }

  const int W = M.key.width;
  uint32_t* s_src = reinterpret_cast<uint32_t*>(smem);                 // [kMergeTile]
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kMergeTile * 4);  // mbarrier
  char* sA = smem + kMergeTile * 4 + 128;
  char* sB = sA + kMergeTile * W + 32;
  const char* col = M.key.data;
  const uintptr_t abase = (reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.a0 + i0) * W) & ~(uintptr_t)15;
  const uintptr_t bbase = (reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.b0 + j0) * W) & ~(uintptr_t)15;
  const uint32_t aoff = (uint32_t)(reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.a0 + i0) * W - abase);
  const uint32_t boff = (uint32_t)(reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.b0 + j0) * W - bbase);

  if (M.staged) {
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    // Thread 0 computes the TMA byte count first (arrive.expect_tx), then issues.
    uint32_t bytes = 0;
    if (threadIdx.x == 0) {
      const uintptr_t ga0 = reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.a0 + i0) * W;
      const uintptr_t ga1 = reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.a0 + i1) * W;
      const uintptr_t gb0 = reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.b0 + j0) * W;
      const uintptr_t gb1 = reinterpret_cast<uintptr_t>(col) + (uintptr_t)(p.b0 + j1) * W;
      const uintptr_t ia0 = (ga0 + 15) & ~(uintptr_t)15, ia1 = ga1 & ~(uintptr_t)15;
      const uintptr_t ib0 = (gb0 + 15) & ~(uintptr_t)15, ib1 = gb1 & ~(uintptr_t)15;
      if (ma && ia1 > ia0) bytes += (uint32_t)(ia1 - ia0);
      if (nb && ib1 > ib0) bytes += (uint32_t)(ib1 - ib0);
      if (bytes) mbar_arrive_expect_tx(bar, bytes);
    }
    stage_rows(sA, col, W, p.a0 + i0, p.a0 + i1, bar, threadIdx.x == 0 && bytes);
    stage_rows(sB, col, W, p.b0 + j0, p.b0 + j1, bar, threadIdx.x == 0 && bytes);
    __shared__ uint32_t s_bytes;
    if (threadIdx.x == 0) s_bytes = bytes;
    __syncthreads();
    if (s_bytes) {
      uint32_t spins = 0;
      bool done = mbar_try_wait(bar, 0);
      while (!done && ++spins < kSpinLimit) done = mbar_try_wait(bar, 0);
      if (!done) {
        // Report, then give the copy one more bounded wait before leaving.
        if (threadIdx.x == 0) atomicOr(M.err, kErrTimeout);
        for (uint32_t s2 = 0; s2 < kSpinLimit && !mbar_try_wait(bar, 0); ++s2) {
        }
        return;
      }
    }
  }

  auto keyA = [&](uint32_t x, uint32_t (&k)[KW]) {
    const uint32_t row = p.a0 + i0 + x;
    const bool nul = M.key.nulls && M.key.nulls[row];
    if (M.staged) make_key_ptr<KW>(M.key, sA + aoff + (size_t)x * W, nul, k);
    else make_key<KW>(M.key, row, k);
  };
  auto keyB = [&](uint32_t x, uint32_t (&k)[KW]) {
    const uint32_t row = p.b0 + j0 + x;
    const bool nul = M.key.nulls && M.key.nulls[row];
    if (M.staged) make_key_ptr<KW>(M.key, sB + boff + (size_t)x * W, nul, k);
    else make_key<KW>(M.key, row, k);
  };

  // Each thread merges kMergeItems consecutive outputs of the tile.
  const uint32_t kk = threadIdx.x * kMergeItems;
  if (kk < cnt) {
    uint32_t lo = kk > nb ? kk - nb : 0u, hi = kk < ma ? kk : ma;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      uint32_t ka[KW], kb[KW];
      keyA(mid, ka);
      keyB(kk - mid - 1, kb);
      if (key_le<KW>(ka, kb)) lo = mid + 1;
      else hi = mid;
    }
    uint32_t ia = lo, jb = kk - lo;
    uint32_t ka[KW], kb[KW];
    if (ia < ma) keyA(ia, ka);
    if (jb < nb) keyB(jb, kb);
#pragma unroll
    for (int x = 0; x < kMergeItems; ++x) {
      if (kk + x >= cnt) break;
      const bool takeA = ia < ma && (jb >= nb || key_le<KW>(ka, kb));
      if (takeA) {
        s_src[kk + x] = ia++;
        if (ia < ma) keyA(ia, ka);
      } else {
        s_src[kk + x] = kFromB | jb++;
        if (jb < nb) keyB(jb, kb);
      }
    }
  }
  __syncthreads();

  // Move every column (key included) for the tile's outputs: the source row
  // of each output is resolved once, then per column all kMergeItems loads
  // are issued before the (coalesced) stores.
  const uint32_t out_base = p.out0 + k0;
  uint32_t rows[kMergeItems];
#pragma unroll
  for (int i = 0; i < kMergeItems; ++i) {
    const uint32_t x = threadIdx.x + i * kMergeBlock;
    rows[i] = 0xffffffffu;
    if (x < cnt) {
      const uint32_t s = s_src[x];
      rows[i] = (s & kFromB) ? p.b0 + j0 + (s & ~kFromB) : p.a0 + i0 + s;
    }
  }
  for (int c = 0; c < M.ncols; ++c) {
    const MergeCol& mc = M.c[c];
    switch (mc.vec ? mc.width : 0) {
      case 4: move_items<uint32_t>(mc, rows, out_base); break;
      case 8: move_items<unsigned long long>(mc, rows, out_base); break;
      case 16: move_items<uint4>(mc, rows, out_base); break;
      default:
#pragma unroll
        for (int i = 0; i < kMergeItems; ++i)
          if (rows[i] != 0xffffffffu)
            copy_cell(mc.dst + (size_t)(out_base + threadIdx.x + i * kMergeBlock) * mc.width,
                      mc.src + (size_t)rows[i] * mc.width, mc.width);
    }
    if (mc.dst_nulls) {
#pragma unroll
      for (int i = 0; i < kMergeItems; ++i)
        if (rows[i] != 0xffffffffu)
          mc.dst_nulls[out_base + threadIdx.x + i * kMergeBlock] = mc.src_nulls ? mc.src_nulls[rows[i]] : 0;
    }
  }
}

static int merge_kw(const yq_column& c) {
  int vw;
  switch (c.type) {
    case YQ_INT32:
    case YQ_FLOAT32:
    case YQ_BOOL: vw = 1; break;
    case YQ_INT64:
    case YQ_DATETIME:
    case YQ_FLOAT64: vw = 2; break;
    case YQ_TEXT: vw = c.width / 4; break;
    default: return -1;
  }
  const int w = vw + (c.nulls ? 1 : 0);
  return w <= 1 ? 1 : (w <= 2 ? 2 : (w <= 4 ? 4 : (w <= 8 ? 8 : -1)));
}

template <int KW>
static int launch_merge(const MergeParams& M, cudaStream_t s, double bytes) {
  const int W = M.key.width;
  const size_t smem = (size_t)kMergeTile * 4 + 128 + (M.staged ? 2 * ((size_t)kMergeTile * W + 32) : 0);
  YQ_TRY(kernel_allow_smem((const void*)k_merge_tiles<KW>, smem));
  {
    ProfScope ps("merge_partition", s, 0.0);
    k_merge_partition<KW><<<ceil_div<uint32_t>(M.ntiles, 128), 128, 0, s>>>(M);
    YQ_CHECK_LAUNCH();
  }
  ProfScope ps("merge_tiles", s, bytes);
  k_merge_tiles<KW><<<M.ntiles, kMergeBlock, smem, s>>>(M);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}


// ===================================================== merges of key words
// ORDER BY over sorted runs as the radix sort leaves them: each row is its
// order-preserving key words (yq_keys.cuh) plus its row id, so the merge
// compares unsigned words only. A level is two launches: the partition kernel
// gives every output tile its A and B windows (the merge-path co-rank at its
// first output; the next tile's gives its end); the tile kernel is persistent, and thread 0 of a block
// starts the bulk copies of the key and id windows of the tiles kRawStages - 1
// ahead of the one the block merges, so the copies overlap the merging. A
// level whose ids are the row positions (right after the first gather level)
// copies no ids.
// Windows are copied from their 16-byte aligned hull (buffers are padded).
constexpr int kRawStages = 3;

struct RawPair {
  uint32_t a0, m, b0, n, tile0;
};

// A tile's windows. The partition kernel searches one co-rank per tile (at
// the tile's first output): `i0` is it, and `done` says whether na / nb are
// final (the pair's last tile, whose end co-rank is the pair's A length);
// otherwise the tile kernel completes them from the next tile's i0.
struct RawTile {
  uint32_t a_row, na, b_row, nb, out0, cnt, i0, done;
};

__device__ __forceinline__ RawTile raw_tile_fix(RawTile d, uint32_t next_i0) {
  if (!d.done) {
    d.na = next_i0 - d.i0;
    d.nb = d.cnt - d.na;
  }
  return d;
}

// Decoding of key words back into the key column's values (the last level
// writes the sorted key column itself instead of its words).
struct KeyDecode {
  char* out;        // null: no decode
  int32_t type;
  int32_t vwords;   // value words (text: significant slot words)
  int32_t width;    // slot width (text)
  int32_t desc;
  uint32_t high[8];  // key words above the merged ones, shared by every row (key form)
};

struct RawLevel {
  const uint32_t* keys_in;  // [rows][KW] words
  const uint32_t* ids_in;   // [rows]
  uint32_t* keys_out;       // null: the level writes row ids only
  KeyDecode dec;
  uint32_t* ids_out;
  const RawPair* pairs;
  int32_t npairs;
  uint32_t ntiles;
  RawTile* tiles;  // [ntiles], written by the partition kernel
  uint32_t* err;
};

__device__ __forceinline__ int raw_pair_of_tile(const RawPair* pairs, int npairs, uint32_t tile) {
  int lo = 0, hi = npairs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&pairs[mid].tile0) <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int KW>
__device__ __forceinline__ void raw_key_g(const uint32_t* keys, uint32_t row, uint32_t (&k)[KW]) {
#pragma unroll
  for (int j = 0; j < KW; ++j) k[j] = __ldg(keys + (size_t)row * KW + j);
}

// Number of A rows among the first k outputs of pair p (ties from A).
template <int KW>
__device__ __forceinline__ uint32_t raw_corank(const uint32_t* keys, const RawPair& p, uint32_t k) {
  uint32_t lo = k > p.n ? k - p.n : 0u, hi = k < p.m ? k : p.m;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    uint32_t ka[KW], kb[KW];
    raw_key_g<KW>(keys, p.a0 + mid, ka);
    raw_key_g<KW>(keys, p.b0 + (k - mid - 1), kb);
    if (key_le<KW>(ka, kb)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Tile t's merge-path co-rank at its first output, one thread per tile (the
// tile's end co-rank is the next tile's start). Finding the co-ranks in the
// tile kernel's blocks instead, all of a block's tiles before its first merge,
// measured 70 us per level slower than this launch.
template <int KW, int ITEMS>
__global__ void k_merge_raw_partition(const __grid_constant__ RawLevel L) {
  constexpr uint32_t TILE = kMergeBlock * ITEMS;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L.ntiles) return;
  const RawPair p = L.pairs[raw_pair_of_tile(L.pairs, L.npairs, t)];
  const uint32_t total = p.m + p.n;
  const uint32_t k0 = (t - p.tile0) * TILE;
  const uint32_t k1 = min(k0 + TILE, total);
  if (k0 >= total) {  // a descriptor with no work (never produced by the host plan)
    L.tiles[t] = RawTile{0, 0, 0, 0, 0, 0, 0, 1};
    atomicOr(L.err, kErrBounds);
    return;
  }
  const uint32_t i0 = raw_corank<KW>(L.keys_in, p, k0);
  RawTile d;
  d.a_row = p.a0 + i0;
  d.b_row = p.b0 + (k0 - i0);
  d.out0 = p.a0 + k0;
  d.cnt = k1 - k0;
  d.i0 = i0;
  d.done = k1 == total;  // the end co-rank of a pair's last tile is p.m; others take the next tile's i0
  d.na = d.done ? p.m - i0 : 0u;
  d.nb = d.done ? d.cnt - d.na : 0u;
  L.tiles[t] = d;
}

// Where a tile's windows sit inside its stage slot.
struct RawSlot {
  uint32_t na, nb, cnt, out0;
  uint32_t ka, kb, ia, ib;  // byte offsets of the first A / B key and id in the slot
  uint32_t a_row, b_row;    // first A / B row (the ids themselves when the level has no id input)
};

// ITEMS outputs per thread: a tile of kMergeBlock * ITEMS outputs. Variants
// (KW, ITEMS) whose kRawStages slots fit the 227 KB of shared memory:
// ITEMS 4 and 8 for every key width, 16 for one and two key words.
template <int KW, int ITEMS>
struct RawGeom {
  static constexpr uint32_t W = 4u * KW;
  static constexpr uint32_t TILE = kMergeBlock * ITEMS;
  static constexpr uint32_t kreg = TILE * W + 64;  // keys of both windows + alignment slack
  static constexpr uint32_t ireg = TILE * 4 + 64;  // ids of both windows + alignment slack
  static constexpr uint32_t slot = kreg + ireg;
  static constexpr size_t smem = (size_t)kRawStages * slot + kRawStages * 8;
};

// Copy rows [r0, r0 + n) (w bytes each) from their 16-byte hull; returns the
// byte offset of row r0 inside the copy and advances `off` / `bytes`.
__device__ __forceinline__ uint32_t raw_window(unsigned char* region, uint32_t& off, const void* base, uint32_t r0,
                                               uint32_t n, uint32_t w, uint64_t* bar, uint32_t& bytes, bool issue) {
  if (n == 0) return off;
  const uintptr_t g0 = reinterpret_cast<uintptr_t>(base) + (uintptr_t)r0 * w;
  const uintptr_t g1 = g0 + (uintptr_t)n * w;
  const uintptr_t h0 = g0 & ~(uintptr_t)15, h1 = (g1 + 15) & ~(uintptr_t)15;
  const uint32_t at = off + (uint32_t)(g0 - h0);
  if (issue) tma_load_1d(region + off, reinterpret_cast<const void*>(h0), (uint32_t)(h1 - h0), bar);
  bytes += (uint32_t)(h1 - h0);
  off += (uint32_t)(h1 - h0);
  return at;
}

// Thread 0: start the copies of tile descriptor d into `slot`.
template <int KW, int ITEMS>
__device__ __forceinline__ void raw_issue(const RawLevel& L, const RawTile& d, int slot, unsigned char* smem,
                                          RawSlot* s_slot) {
  using G = RawGeom<KW, ITEMS>;
  unsigned char* kreg = smem + (size_t)slot * G::slot;
  unsigned char* ireg = kreg + G::kreg;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + (size_t)kRawStages * G::slot) + slot;
  uint32_t bytes = 0, ko = 0, io = 0;
  // sizes first (expect_tx before the copies)
  RawSlot r;
  r.na = d.na;
  r.nb = d.nb;
  r.cnt = d.cnt;
  r.out0 = d.out0;
  r.a_row = d.a_row;
  r.b_row = d.b_row;
  {
    uint32_t k2 = 0, i2 = 0, b2 = 0;
    r.ka = raw_window(kreg, k2, L.keys_in, d.a_row, d.na, G::W, bar, b2, false);
    r.kb = raw_window(kreg, k2, L.keys_in, d.b_row, d.nb, G::W, bar, b2, false);
    if (L.ids_in) {  // no id input: every row's id is its row number
      r.ia = raw_window(ireg, i2, L.ids_in, d.a_row, d.na, 4u, bar, b2, false);
      r.ib = raw_window(ireg, i2, L.ids_in, d.b_row, d.nb, 4u, bar, b2, false);
    } else {
      r.ia = r.ib = 0u;
    }
    mbar_arrive_expect_tx(bar, b2);
  }
  s_slot[slot] = r;
  raw_window(kreg, ko, L.keys_in, d.a_row, d.na, G::W, bar, bytes, true);
  raw_window(kreg, ko, L.keys_in, d.b_row, d.nb, G::W, bar, bytes, true);
  if (L.ids_in) {
    raw_window(ireg, io, L.ids_in, d.a_row, d.na, 4u, bar, bytes, true);
    raw_window(ireg, io, L.ids_in, d.b_row, d.nb, 4u, bar, bytes, true);
  }
}

template <int KW>
__device__ __forceinline__ void raw_key_s(const unsigned char* p, uint32_t (&k)[KW]) {
  if constexpr (KW == 1) {
    k[0] = *reinterpret_cast<const uint32_t*>(p);
  } else if constexpr (KW == 2) {
    const uint2 v = *reinterpret_cast<const uint2*>(p);
    k[0] = v.x;
    k[1] = v.y;
  } else {
#pragma unroll
    for (int j = 0; j < KW; j += 4) {
      const uint4 v = *reinterpret_cast<const uint4*>(p + 4 * j);
      k[j] = v.x;
      k[j + 1] = v.y;
      k[j + 2] = v.z;
      k[j + 3] = v.w;
    }
  }
}

template <int KW>
__device__ __forceinline__ void raw_key_store(uint32_t* out, size_t row, const uint32_t (&k)[KW]) {
  if constexpr (KW == 1) {
    out[row] = k[0];
  } else if constexpr (KW == 2) {
    reinterpret_cast<uint2*>(out)[row] = make_uint2(k[0], k[1]);
  } else {
#pragma unroll
    for (int j = 0; j < KW; j += 4)
      *reinterpret_cast<uint4*>(out + row * KW + j) = make_uint4(k[j], k[j + 1], k[j + 2], k[j + 3]);
  }
}

// Inverse of make_key_ptr for a key without nulls (exact when the column holds
// no -0.0, non-canonical NaN or bool byte other than 0/1: see key_value_lossy).
template <int KW>
__device__ __forceinline__ void decode_store(const KeyDecode& d, size_t row, const uint32_t (&k0)[KW]) {
  // the whole key: the merged words, then the words every row shares
  uint32_t k[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t w = j < KW ? k0[j < KW ? j : 0] : d.high[j >= KW ? j - KW : 0];
    k[j] = (d.desc && j < d.vwords) ? ~w : w;
  }
  switch (d.type) {
    case YQ_INT32: reinterpret_cast<uint32_t*>(d.out)[row] = k[0] ^ 0x80000000u; break;
    case YQ_FLOAT32: reinterpret_cast<uint32_t*>(d.out)[row] = (k[0] & 0x80000000u) ? (k[0] & 0x7fffffffu) : ~k[0]; break;
    case YQ_BOOL: reinterpret_cast<uint8_t*>(d.out)[row] = (uint8_t)(k[0] & 1u); break;
    case YQ_INT64:
    case YQ_DATETIME: reinterpret_cast<uint2*>(d.out)[row] = make_uint2(k[0], k[1] ^ 0x80000000u); break;
    case YQ_FLOAT64: {
      unsigned long long b = ((unsigned long long)k[1] << 32) | k[0];
      b = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
      reinterpret_cast<unsigned long long*>(d.out)[row] = b;
      break;
    }
    default: {  // TEXT: word i of the slot = bswap(k[vwords - 1 - i]); later words are zero
      uint32_t* w = reinterpret_cast<uint32_t*>(d.out + row * (size_t)d.width);
      for (int i = 0; i < (d.width >> 2); ++i) {
        uint32_t v = 0u;
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (i < d.vwords && j == d.vwords - 1 - i) v = bswap(k[j]);
        w[i] = v;
      }
    }
  }
}

template <int KW, int ITEMS>
__global__ void __launch_bounds__(kMergeBlock) k_merge_raw_tiles(const __grid_constant__ RawLevel L) {
  using G = RawGeom<KW, ITEMS>;
  extern __shared__ __align__(128) unsigned char raw_smem[];
  __shared__ RawSlot s_slot[kRawStages];
  uint64_t* bars = reinterpret_cast<uint64_t*>(raw_smem + (size_t)kRawStages * G::slot);
  const uint32_t NT = L.ntiles, GR = gridDim.x;
  if (threadIdx.x == 0)
    for (int s = 0; s < kRawStages; ++s) mbar_init(bars + s, 1);
  __syncthreads();
  RawTile next{};
  uint32_t next_i1 = 0u;  // the following tile's first co-rank (ends `next` unless it is done)
  if (threadIdx.x == 0) {
    for (int j = 0; j < kRawStages - 1; ++j) {
      const uint32_t t = blockIdx.x + (uint32_t)j * GR;
      if (t < NT)
        raw_issue<KW, ITEMS>(L, raw_tile_fix(L.tiles[t], t + 1 < NT ? L.tiles[t + 1].i0 : 0u), j, raw_smem, s_slot);
    }
    const uint32_t t = blockIdx.x + (uint32_t)(kRawStages - 1) * GR;
    if (t < NT) {
      next = L.tiles[t];
      next_i1 = t + 1 < NT ? L.tiles[t + 1].i0 : 0u;
    }
  }
  int slot = 0;
  uint32_t parity = 0;
  for (uint32_t t = blockIdx.x; t < NT; t += GR) {
    __syncthreads();  // every thread is done with the previous tile: its slot is free
    if (threadIdx.x == 0) {
      const uint32_t tn = t + (uint32_t)(kRawStages - 1) * GR;
      const int ns = slot == 0 ? kRawStages - 1 : slot - 1;
      if (tn < NT) {
        raw_issue<KW, ITEMS>(L, raw_tile_fix(next, next_i1), ns, raw_smem, s_slot);
        const uint32_t tf = tn + GR;  // descriptor for the next issue, loaded a tile ahead
        if (tf < NT) {
          next = L.tiles[tf];
          next_i1 = tf + 1 < NT ? L.tiles[tf + 1].i0 : 0u;
        }
      }
    }
    mbar_wait_bounded(bars + slot, parity, L.err);
    const RawSlot r = s_slot[slot];
    const unsigned char* kreg = raw_smem + (size_t)slot * G::slot;
    const unsigned char* ireg = kreg + G::kreg;
    const unsigned char* kA = kreg + r.ka;
    const unsigned char* kB = kreg + r.kb;

    // Each thread merges ITEMS consecutive outputs of the tile in
    // registers and stores them itself: a warp's stores cover one contiguous
    // run of 32 x ITEMS outputs (16-byte stores when aligned).
    const uint32_t kk = threadIdx.x * ITEMS;
    if (kk < r.cnt) {
      uint32_t lo = kk > r.nb ? kk - r.nb : 0u, hi = kk < r.na ? kk : r.na;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        uint32_t ka[KW], kb[KW];
        raw_key_s<KW>(kA + (size_t)mid * G::W, ka);
        raw_key_s<KW>(kB + (size_t)(kk - mid - 1) * G::W, kb);
        if (key_le<KW>(ka, kb)) lo = mid + 1;
        else hi = mid;
      }
      uint32_t ia = lo, jb = kk - lo;
      uint32_t ka[KW], kb[KW];
#pragma unroll
      for (int j = 0; j < KW; ++j) ka[j] = kb[j] = 0u;
      if (ia < r.na) raw_key_s<KW>(kA + (size_t)ia * G::W, ka);
      if (jb < r.nb) raw_key_s<KW>(kB + (size_t)jb * G::W, kb);
      const uint32_t* idA = reinterpret_cast<const uint32_t*>(ireg + r.ia);
      const uint32_t* idB = reinterpret_cast<const uint32_t*>(ireg + r.ib);
      uint32_t okey[ITEMS][KW], oid[ITEMS];
      const uint32_t m = r.cnt - kk < (uint32_t)ITEMS ? r.cnt - kk : (uint32_t)ITEMS;
#pragma unroll
      for (int x = 0; x < ITEMS; ++x) {
        if ((uint32_t)x >= m) break;
        const bool takeA = ia < r.na && (jb >= r.nb || key_le<KW>(ka, kb));
        if (takeA) {
#pragma unroll
          for (int j = 0; j < KW; ++j) okey[x][j] = ka[j];
          oid[x] = L.ids_in ? idA[ia] : r.a_row + ia;
          ++ia;
          if (ia < r.na) raw_key_s<KW>(kA + (size_t)ia * G::W, ka);
        } else {
#pragma unroll
          for (int j = 0; j < KW; ++j) okey[x][j] = kb[j];
          oid[x] = L.ids_in ? idB[jb] : r.b_row + jb;
          ++jb;
          if (jb < r.nb) raw_key_s<KW>(kB + (size_t)jb * G::W, kb);
        }
      }
      const size_t o0 = (size_t)r.out0 + kk;
      if (m == (uint32_t)ITEMS && (o0 & 3u) == 0u) {
#pragma unroll
        for (int x = 0; x < ITEMS; x += 4)
          *reinterpret_cast<uint4*>(L.ids_out + o0 + x) = make_uint4(oid[x], oid[x + 1], oid[x + 2], oid[x + 3]);
      } else {
#pragma unroll
        for (int x = 0; x < ITEMS; ++x)
          if ((uint32_t)x < m) L.ids_out[o0 + x] = oid[x];
      }
      if (L.keys_out) {
        if (KW == 1 && m == (uint32_t)ITEMS && (o0 & 3u) == 0u) {
#pragma unroll
          for (int x = 0; x < ITEMS; x += 4)
            *reinterpret_cast<uint4*>(L.keys_out + o0 + x) =
                make_uint4(okey[x][0], okey[x + 1][0], okey[x + 2][0], okey[x + 3][0]);
        } else {
#pragma unroll
          for (int x = 0; x < ITEMS; ++x)
            if ((uint32_t)x < m) raw_key_store<KW>(L.keys_out, o0 + x, okey[x]);
        }
      } else if (L.dec.out) {
#pragma unroll
        for (int x = 0; x < ITEMS; ++x)
          if ((uint32_t)x < m) decode_store<KW>(L.dec, o0 + x, okey[x]);
      }
    }
    if (++slot == kRawStages) {
      slot = 0;
      parity ^= 1u;
    }
  }
}

template <int KW, int ITEMS>
static int launch_raw_level(const RawLevel& L, cudaStream_t s, double bytes) {
  using G = RawGeom<KW, ITEMS>;
  static_assert(G::smem <= 227 * 1024, "stage slots exceed shared memory");
  YQ_TRY(kernel_allow_smem((const void*)k_merge_raw_tiles<KW, ITEMS>, G::smem));
  const int cap = kernel_blocks_per_sm((const void*)k_merge_raw_tiles<KW, ITEMS>, kMergeBlock, G::smem) * sm_count();
  {
    ProfScope ps("merge_partition", s, 0.0);
    k_merge_raw_partition<KW, ITEMS><<<ceil_div<uint32_t>(L.ntiles, 128), 128, 0, s>>>(L);
    YQ_CHECK_LAUNCH();
  }
  const int grid = (int)(L.ntiles < (uint32_t)cap ? L.ntiles : (uint32_t)cap);
  ProfScope ps("merge_tiles", s, bytes);
  k_merge_raw_tiles<KW, ITEMS><<<grid, kMergeBlock, G::smem, s>>>(L);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

static bool merge_items_ok(int kw, int items) {
  return items == 4 || items == 8 || (items == 16 && kw <= 2);
}

static int launch_raw_level_items(int kw, int items, const RawLevel& L, cudaStream_t s, double bytes) {
  switch (kw * 100 + items) {
    case 104: return launch_raw_level<1, 4>(L, s, bytes);
    case 108: return launch_raw_level<1, 8>(L, s, bytes);
    case 116: return launch_raw_level<1, 16>(L, s, bytes);
    case 204: return launch_raw_level<2, 4>(L, s, bytes);
    case 208: return launch_raw_level<2, 8>(L, s, bytes);
    case 216: return launch_raw_level<2, 16>(L, s, bytes);
    case 404: return launch_raw_level<4, 4>(L, s, bytes);
    case 408: return launch_raw_level<4, 8>(L, s, bytes);
    case 804: return launch_raw_level<8, 4>(L, s, bytes);
    case 808: return launch_raw_level<8, 8>(L, s, bytes);
    default: return YQ_ERR_UNSUPPORTED;
  }
}

// Merge-path tile (outputs per thread) per (key words, log2 of rows), set by
// yq_order_by_autotune; kMergeItems where none was tuned.
static std::mutex g_merge_tune_mu;
static std::map<std::pair<int, int>, int> g_merge_tuned;

static int log2_rows(uint32_t rows) {
  int b = 0;
  while (rows > 1) {
    rows >>= 1;
    ++b;
  }
  return b;
}

static int merge_items_for(int kw, uint32_t rows) {
  std::lock_guard<std::mutex> lk(g_merge_tune_mu);
  auto it = g_merge_tuned.find({kw, log2_rows(rows)});
  return it == g_merge_tuned.end() ? kMergeItems : it->second;
}

// Merge levels of one ORDER BY: host plan of every level's pairs.
struct OrderPlan {
  std::vector<RawPair> pairs;         // all levels, back to back
  std::vector<int> level_first;       // first pair of each level (+ end)
  std::vector<uint32_t> level_tiles;  // tiles per level
};

static void plan_order_levels(const uint32_t* offsets, int nruns, uint32_t tile, OrderPlan& P) {
  std::vector<uint32_t> offs(offsets, offsets + nruns + 1);
  P.pairs.clear();
  P.level_first.clear();
  P.level_tiles.clear();
  while (offs.size() > 2) {
    P.level_first.push_back((int)P.pairs.size());
    uint32_t tiles = 0;
    std::vector<uint32_t> next;
    const int runs = (int)offs.size() - 1;
    for (int r = 0; r < runs; r += 2) {
      RawPair p;
      p.a0 = offs[r];
      p.m = offs[r + 1] - offs[r];
      p.b0 = offs[r + 1];
      p.n = (r + 1 < runs) ? offs[r + 2] - offs[r + 1] : 0u;
      p.tile0 = tiles;
      next.push_back(offs[r]);
      const uint32_t t = ceil_div<uint32_t>(p.m + p.n, tile);
      if (t == 0) continue;  // empty pair
      tiles += t;
      P.pairs.push_back(p);
    }
    next.push_back(offs.back());
    offs.swap(next);
    P.level_tiles.push_back(tiles);
  }
  P.level_first.push_back((int)P.pairs.size());
}

struct OrderWs {
  size_t sort_bytes = 0;
  int kw_max = 0;
  uint32_t max_tiles = 0;
  size_t npairs = 0;
};

// Two-level gather: with many runs over a table larger than L2, one gather by
// the merged row ids reads every cell at a random row of the whole table
// (each 4-16-byte cell costs a DRAM sector or more). Instead every column is
// first gathered run by run into sorted-run order (the rows a run reads lie
// within that run, so the in-flight window stays in L2), the row ids become
// positions in that layout, and after the merges the final gather reads each
// run's rows in increasing order: hundreds of sequential streams whose
// sectors L2 serves until every cell of them is used.
constexpr double kTwoLevelGatherBytes = 64.0 * 1024 * 1024;

static bool two_level_gather(const yq_batch& in, int nruns) {
  if (nruns < 2) return false;
  double b = 0;
  for (int c = 0; c < in.ncols; ++c) b += (double)in.rows * (in.columns[c].width + (in.columns[c].nulls ? 1 : 0));
  return b >= kTwoLevelGatherBytes;
}

// The sorted-run copy of every column (same widths, nulls where the input has them).
static void stage_ws_layout(const yq_batch& in, WsSize& w) {
  for (int c = 0; c < in.ncols; ++c) {
    w.add<char>((size_t)in.rows * in.columns[c].width + 16);
    if (in.columns[c].nulls) w.add<uint8_t>((size_t)in.rows + 16);
  }
}

__global__ void k_iota(uint32_t* __restrict__ ids, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) ids[i] = i;
}

static int order_ws_layout(const yq_column& key, uint32_t rows, const uint32_t* offsets, int nruns, OrderWs& o,
                           WsSize& w) {
  o.kw_max = sort_key_words_max(key);
  if (o.kw_max < 0) return YQ_ERR_INVALID_ARG;
  KeyJob j{key, 0, 0};
  YQ_TRY(sort_segments_impl(&j, 1, rows, offsets, nruns, nullptr, nullptr, nullptr, 0, nullptr, &o.sort_bytes));
  o.max_tiles = ceil_div<uint32_t>(rows, kMergeBlock * 4u) + (uint32_t)nruns + 1;  // the smallest merge tile
  o.npairs = (size_t)nruns + 64;
  w.add<char>(o.sort_bytes);
  w.add<uint32_t>((size_t)rows * o.kw_max + 16);  // keys, two buffers
  w.add<uint32_t>((size_t)rows * o.kw_max + 16);
  w.add<uint32_t>((size_t)rows + 16);  // row ids, two buffers
  w.add<uint32_t>((size_t)rows + 16);
  w.add<RawPair>(o.npairs);
  w.add<RawTile>(o.max_tiles);
  w.add<uint32_t>(4);
  return YQ_OK;
}

}  // namespace yq

using namespace yq;

extern "C" size_t yq_order_by_workspace_size(const yq_column* key, uint32_t rows, const uint32_t* run_offsets,
                                             int32_t nruns) {
  if (!key || !run_offsets || nruns <= 0) return 0;
  OrderWs o;
  WsSize w;
  if (order_ws_layout(*key, rows, run_offsets, nruns, o, w) != YQ_OK) return 0;
  return w.total();
}

extern "C" size_t yq_order_by_batch_workspace_size(const yq_batch* in, int32_t key_col, const uint32_t* run_offsets,
                                                   int32_t nruns) {
  if (!in || !run_offsets || nruns <= 0 || key_col < 0 || key_col >= in->ncols) return 0;
  OrderWs o;
  WsSize w;
  if (order_ws_layout(in->columns[key_col], in->rows, run_offsets, nruns, o, w) != YQ_OK) return 0;
  if (two_level_gather(*in, nruns)) stage_ws_layout(*in, w);
  return w.total();
}

// Many independent ORDER BY tasks: task g owns rows [seg[g], seg[g+1]);
// one segmented sort orders every task and one gather moves every column.
extern "C" size_t yq_order_by_segments_workspace_size(const yq_column* key, uint32_t rows, const uint32_t* seg_offsets,
                                                      int32_t nseg) {
  if (!key || !seg_offsets || nseg <= 0) return 0;
  KeyJob j{*key, 0, 0};
  size_t sort_bytes = 0;
  if (sort_segments_impl(&j, 1, rows, seg_offsets, nseg, nullptr, nullptr, nullptr, 0, nullptr, &sort_bytes) != YQ_OK)
    return 0;
  WsSize w;
  w.add<uint32_t>(4);
  w.add<char>(sort_bytes);
  w.add<uint32_t>((size_t)rows + 16);
  return w.total();
}

static int order_by_segments_impl(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                                  const uint32_t* seg_offsets, int32_t nseg, yq_batch* out, uint32_t* perm_out,
                                  const yq_sort_config* config, void* workspace, size_t workspace_bytes,
                                  void* stream) {
  if (!in || !out || !seg_offsets || nseg <= 0 || key_col < 0 || key_col >= in->ncols || out->ncols != in->ncols ||
      in->ncols > YQ_MAX_BATCH_COLUMNS)
    return YQ_ERR_INVALID_ARG;
  const uint32_t rows = in->rows;
  if (seg_offsets[0] != 0 || seg_offsets[nseg] != rows) return YQ_ERR_INVALID_ARG;
  for (int c = 0; c < in->ncols; ++c)
    if (in->columns[c].type != out->columns[c].type || in->columns[c].width != out->columns[c].width)
      return YQ_ERR_INVALID_ARG;
  const bool no_wait = config && config->keep_trivial;
  if (no_wait && !workspace) return YQ_ERR_INVALID_ARG;  // the error word lives in the caller's workspace
  cudaStream_t s = as_stream(stream);
  const size_t need = yq_order_by_segments_workspace_size(&in->columns[key_col], rows, seg_offsets, nseg);
  if (need == 0) return YQ_ERR_INVALID_ARG;
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, need, s));
  uint32_t* d_err = ws.take<uint32_t>(4);
  KeyJob j{in->columns[key_col], descending != 0, nulls_first != 0};
  size_t sort_bytes = 0;
  YQ_TRY(sort_segments_impl(&j, 1, rows, seg_offsets, nseg, nullptr, nullptr, nullptr, 0, nullptr, &sort_bytes));
  char* sort_ws = ws.take<char>(sort_bytes);
  uint32_t* perm = ws.take<uint32_t>((size_t)rows + 16);
  if (perm_out) perm = perm_out;  // the caller keeps the permutation
  if (rows == 0) return YQ_OK;
  uint32_t* sort_err = nullptr;
  YQ_TRY(sort_segments_impl(&j, 1, rows, seg_offsets, nseg, perm, config, sort_ws, sort_bytes, s, nullptr, nullptr,
                            nullptr, true, &sort_err));
  yq_column outs[YQ_MAX_BATCH_COLUMNS];
  for (int c = 0; c < in->ncols; ++c) outs[c] = out->columns[c];
  YQ_TRY(yq_gather(in->columns, in->ncols, perm, rows, outs, s));
  YQ_TRY_CUDA(cudaMemcpyAsync(d_err, sort_err, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  if (no_wait) return YQ_OK;
  uint32_t e = 0;
  YQ_TRY(d2h_sync(&e, d_err, sizeof(uint32_t), s));
  if (e & kErrTimeout) return YQ_ERR_TIMEOUT;
  if (e & kErrBounds) return YQ_ERR_INVALID_ARG;
  return YQ_OK;
}

extern "C" int yq_order_by_segments(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                                    const uint32_t* seg_offsets, int32_t nseg, yq_batch* out,
                                    const yq_sort_config* config, void* workspace, size_t workspace_bytes,
                                    void* stream) {
  return order_by_segments_impl(in, key_col, descending, nulls_first, seg_offsets, nseg, out, nullptr, config,
                                workspace, workspace_bytes, stream);
}

extern "C" int yq_order_by_segments_perm(const yq_batch* in, int32_t key_col, int32_t descending,
                                         int32_t nulls_first, const uint32_t* seg_offsets, int32_t nseg,
                                         yq_batch* out, uint32_t* perm_out, const yq_sort_config* config,
                                         void* workspace, size_t workspace_bytes, void* stream) {
  if (!perm_out) return YQ_ERR_INVALID_ARG;
  return order_by_segments_impl(in, key_col, descending, nulls_first, seg_offsets, nseg, out, perm_out, config,
                                workspace, workspace_bytes, stream);
}

// merge_items: outputs per thread of the merge tiles (0 = the tuned or default
// choice); *kw_used (optional): the key words the merge levels compared.
static int order_by_run(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                        const uint32_t* run_offsets, int32_t nruns, yq_batch* out, void* workspace,
                        size_t workspace_bytes, void* stream, int merge_items, int* kw_used = nullptr) {
  if (!in || !out || !run_offsets || nruns <= 0 || key_col < 0 || key_col >= in->ncols || out->ncols != in->ncols ||
      in->ncols > YQ_MAX_BATCH_COLUMNS)
    return YQ_ERR_INVALID_ARG;
  const uint32_t rows = in->rows;
  if (run_offsets[0] != 0 || run_offsets[nruns] != rows) return YQ_ERR_INVALID_ARG;
  for (int r = 0; r < nruns; ++r)
    if (run_offsets[r + 1] < run_offsets[r]) return YQ_ERR_INVALID_ARG;
  for (int c = 0; c < in->ncols; ++c) {
    const yq_column& a = in->columns[c];
    const yq_column& b = out->columns[c];
    if (a.type != b.type || a.width != b.width || (rows > 0 && (!a.data || !b.data))) return YQ_ERR_INVALID_ARG;
  }
  if (rows == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  const yq_column& key = in->columns[key_col];
  OrderWs o;
  WsSize wsz;
  YQ_TRY(order_ws_layout(key, rows, run_offsets, nruns, o, wsz));
  const size_t base_bytes = wsz.total();
  // The sorted-run copy needs more workspace: used when the caller's holds it
  // (yq_order_by_batch_workspace_size) or the library allocates.
  bool staged = two_level_gather(*in, nruns);
  if (staged) {
    stage_ws_layout(*in, wsz);
    if (workspace && workspace_bytes < wsz.total()) staged = false;
  }
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, staged ? wsz.total() : base_bytes, s));
  char* sort_ws = ws.take<char>(o.sort_bytes);
  uint32_t* keys[2] = {ws.take<uint32_t>((size_t)rows * o.kw_max + 16), ws.take<uint32_t>((size_t)rows * o.kw_max + 16)};
  uint32_t* ids[2] = {ws.take<uint32_t>((size_t)rows + 16), ws.take<uint32_t>((size_t)rows + 16)};
  RawPair* d_pairs = ws.take<RawPair>(o.npairs);
  RawTile* d_tiles = ws.take<RawTile>(o.max_tiles);
  uint32_t* d_err = ws.take<uint32_t>(4);
  yq_column stage[YQ_MAX_BATCH_COLUMNS];
  if (staged)
    for (int c = 0; c < in->ncols; ++c) {
      stage[c] = in->columns[c];
      stage[c].data = ws.take<char>((size_t)rows * in->columns[c].width + 16);
      stage[c].nulls = in->columns[c].nulls ? ws.take<uint8_t>((size_t)rows + 16) : nullptr;
    }
  YQ_TRY_CUDA(cudaMemsetAsync(d_err, 0, 4 * sizeof(uint32_t), s));

  // 1. every run sorted; the sort hands over its key words and row ids, and
  // its histogram pass flags key values the key words cannot restore
  const bool may_decode = nruns > 1 && !key.nulls && key.type != YQ_TEXT;
  uint32_t* d_lossy = d_err + 1;
  KeyJob job{key, descending != 0, nulls_first != 0};
  if (may_decode && (key.type == YQ_FLOAT32 || key.type == YQ_FLOAT64 || key.type == YQ_BOOL)) job.lossy = d_lossy;
  int kw = 0;
  uint32_t* sort_err = nullptr;
  uint32_t high[8];
  YQ_TRY(sort_segments_impl(&job, 1, rows, run_offsets, nruns, ids[0], nullptr, sort_ws, o.sort_bytes, s, nullptr,
                            keys[0], &kw, true, &sort_err, high));
  // The last merge level writes the key column itself when the key has no
  // nulls; the gather then moves the key column only if some value would not
  // round-trip through its key words (flag set on the device).
  const bool decode = kw > 0 && may_decode;
  const uint32_t* only_if[YQ_MAX_BATCH_COLUMNS] = {nullptr};
  if (decode) only_if[key_col] = d_lossy;  // zero unless a value would not round-trip
  // 1b. two-level gather, first level: every column into sorted-run order;
  // the row ids become positions in that copy, so the first merge level
  // reads no ids (a row's id is its position)
  const bool merged = kw > 0 && nruns > 1;
  staged = staged && merged;
  bool ids_are_positions = false;
  if (staged) {
    YQ_TRY(gather_impl(in->columns, in->ncols, ids[0], rows, stage, only_if, s));
    ids_are_positions = true;
  }
  // 2. merge levels over (key words, row id)
  int cur = 0;
  if (merged) {
    if (kw_used) *kw_used = kw;
    const int mi = merge_items ? merge_items : merge_items_for(kw, rows);
    if (!merge_items_ok(kw, mi)) return YQ_ERR_UNSUPPORTED;
    OrderPlan P;
    plan_order_levels(run_offsets, nruns, kMergeBlock * (uint32_t)mi, P);
    if (P.pairs.size() > o.npairs) return YQ_ERR_UNSUPPORTED;
    YQ_TRY(h2d_async(d_pairs, P.pairs.data(), P.pairs.size() * sizeof(RawPair), s));
    const int levels = (int)P.level_tiles.size();
    for (int l = 0; l < levels; ++l) {
      const bool last = l + 1 == levels;
      RawLevel L;
      L.keys_in = keys[cur];
      L.ids_in = ids_are_positions ? nullptr : ids[cur];
      L.keys_out = last ? nullptr : keys[cur ^ 1];
      memset(&L.dec, 0, sizeof(L.dec));
      if (last && decode) {
        L.dec.out = static_cast<char*>(out->columns[key_col].data);
        L.dec.type = key.type;
        L.dec.vwords = key.type == YQ_INT32 || key.type == YQ_FLOAT32 || key.type == YQ_BOOL ? 1 : 2;
        L.dec.width = key.width;
        L.dec.desc = descending != 0;
        memcpy(L.dec.high, high, sizeof(high));
      }
      L.ids_out = ids[cur ^ 1];
      L.pairs = d_pairs + P.level_first[l];
      L.npairs = P.level_first[l + 1] - P.level_first[l];
      L.ntiles = P.level_tiles[l];
      L.tiles = d_tiles;
      L.err = d_err;
      if (L.ntiles > o.max_tiles) return YQ_ERR_UNSUPPORTED;
      if (L.ntiles == 0) continue;
      // algorithmic bytes: key words + id in and out (ids only out on the
      // last level; no ids in when they are the row positions)
      const double bytes =
          (double)rows * (4.0 * kw + (L.ids_in ? 4.0 : 0.0) + (last ? 4.0 : 4.0 * kw + 4.0));
      YQ_TRY(launch_raw_level_items(kw, mi, L, s, bytes));
      ids_are_positions = false;
      cur ^= 1;
    }
  }
  if (ids_are_positions) {  // no level ran: the final gather still needs the positions written out
    k_iota<<<sm_count() * 4, 256, 0, s>>>(ids[cur], rows);
    YQ_CHECK_LAUNCH();
  }
  // 3. every column (the key included) gathered once by the final row ids
  YQ_TRY(gather_impl(staged ? stage : in->columns, in->ncols, ids[cur], rows, out->columns, only_if, s));
  uint32_t err[2] = {0, 0};
  YQ_TRY(d2h_sync(&err[0], sort_err, sizeof(uint32_t), s));
  YQ_TRY(d2h_sync(&err[1], d_err, sizeof(uint32_t), s));
  const uint32_t e = err[0] | err[1];
  if (e & kErrTimeout) return YQ_ERR_TIMEOUT;
  if (e & kErrBounds) return YQ_ERR_INVALID_ARG;
  return YQ_OK;
}

extern "C" int yq_order_by(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                           const uint32_t* run_offsets, int32_t nruns, yq_batch* out, void* workspace,
                           size_t workspace_bytes, void* stream) {
  return order_by_run(in, key_col, descending, nulls_first, run_offsets, nruns, out, workspace, workspace_bytes,
                      stream, 0);
}

extern "C" int yq_order_by_tiled(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                                 const uint32_t* run_offsets, int32_t nruns, yq_batch* out, int32_t merge_items,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  if (merge_items != 0 && merge_items != 4 && merge_items != 8 && merge_items != 16) return YQ_ERR_INVALID_ARG;
  return order_by_run(in, key_col, descending, nulls_first, run_offsets, nruns, out, workspace, workspace_bytes,
                      stream, merge_items);
}

extern "C" int yq_order_by_autotune(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                                    const uint32_t* run_offsets, int32_t nruns, yq_sort_config* best_sort,
                                    int32_t* best_merge_items, void* stream) {
  if (!in || !run_offsets || nruns <= 0 || key_col < 0 || key_col >= in->ncols || in->ncols > YQ_MAX_BATCH_COLUMNS ||
      !best_sort || !best_merge_items)
    return YQ_ERR_INVALID_ARG;
  cudaStream_t s = as_stream(stream);
  // run formation: the sort's own tuner over the runs as segments
  YQ_TRY(yq_sort_autotune(&in->columns[key_col], in->rows, run_offsets, nruns, descending, best_sort, stream));
  *best_merge_items = kMergeItems;
  const int kw = sort_key_words_max(in->columns[key_col]);
  if (nruns < 2 || in->rows == 0 || kw <= 0) return YQ_OK;
  // merge levels: time the whole ORDER BY for each merge tile (an output
  // batch and a workspace of its own, freed before returning)
  yq_column oc[YQ_MAX_BATCH_COLUMNS];
  void* bufs[2 * YQ_MAX_BATCH_COLUMNS + 1] = {nullptr};
  int nb = 0;
  int status = YQ_OK;
  for (int c = 0; c < in->ncols && status == YQ_OK; ++c) {
    oc[c] = in->columns[c];
    void* d = nullptr;
    void* n = nullptr;
    if (cudaMallocAsync(&d, (size_t)in->rows * oc[c].width + 16, s) != cudaSuccess) status = YQ_ERR_ALLOC;
    bufs[nb++] = d;
    if (status == YQ_OK && oc[c].nulls && cudaMallocAsync(&n, (size_t)in->rows + 16, s) != cudaSuccess)
      status = YQ_ERR_ALLOC;
    bufs[nb++] = n;
    oc[c].data = d;
    oc[c].nulls = static_cast<const uint8_t*>(n);
  }
  yq_batch out{oc, in->ncols, in->rows};
  const size_t wsb = yq_order_by_batch_workspace_size(in, key_col, run_offsets, nruns);
  void* ws = nullptr;
  if (status == YQ_OK && (wsb == 0 || cudaMallocAsync(&ws, wsb, s) != cudaSuccess)) status = YQ_ERR_ALLOC;
  bufs[nb++] = ws;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (status == YQ_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    status = YQ_ERR_CUDA;
  float best_ms = 1e30f;
  int pick = kMergeItems;
  int kw_merge = 0;
  for (int items : {8, 4, 16}) {
    if (status != YQ_OK) break;
    if (!merge_items_ok(kw, items)) continue;
    status = order_by_run(in, key_col, descending, nulls_first, run_offsets, nruns, &out, ws, wsb, stream, items,
                          &kw_merge);
    if (status != YQ_OK) break;
    cudaEventRecord(e0, s);
    for (int r = 0; r < 2 && status == YQ_OK; ++r)
      status = order_by_run(in, key_col, descending, nulls_first, run_offsets, nruns, &out, ws, wsb, stream, items);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (status == YQ_OK && ms < best_ms) {
      best_ms = ms;
      pick = items;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  for (int i = 0; i < nb; ++i)
    if (bufs[i]) cudaFreeAsync(bufs[i], s);
  if (status != YQ_OK) return status;
  if (kw_merge > 0) {  // keyed by the key words the merge levels compare
    std::lock_guard<std::mutex> lk(g_merge_tune_mu);
    g_merge_tuned[{kw_merge, log2_rows(in->rows)}] = pick;
  }
  *best_merge_items = pick;
  return YQ_OK;
}

namespace yq {
}  // namespace yq

using namespace yq;

extern "C" {

size_t yq_merge_workspace_size(uint32_t total_rows, int32_t nruns) {
  if (nruns < 0) return 0;
  const size_t npairs = (size_t)(nruns + 1) / 2;
  const size_t tiles = ceil_div<size_t>(total_rows, kMergeTile) + npairs;
  WsSize w;
  w.add<MergePair>(npairs + 1);
  w.add<uint32_t>(tiles + 1);
  w.add<uint32_t>(4);
  return w.total();
}

int yq_merge_pass(const yq_column* cols, int32_t ncols, int32_t key_col, int32_t descending, int32_t nulls_first,
                  const uint32_t* run_offsets, int32_t nruns, yq_column* out, void* workspace, size_t workspace_bytes,
                  void* stream) {
  if (!cols || !out || ncols <= 0 || ncols > YQ_MAX_BATCH_COLUMNS || key_col < 0 || key_col >= ncols || nruns < 0 ||
      (nruns > 0 && !run_offsets))
    return YQ_ERR_INVALID_ARG;
  if (nruns == 0) return YQ_OK;
  for (int r = 0; r < nruns; ++r)
    if (run_offsets[r + 1] < run_offsets[r]) return YQ_ERR_INVALID_ARG;
  const yq_column& kc = cols[key_col];
  const int kw = merge_kw(kc);
  if (kw < 0) return kc.type == YQ_TEXT ? YQ_ERR_UNSUPPORTED : YQ_ERR_INVALID_ARG;
  MergeParams M;
  memset(&M, 0, sizeof(M));
  double row_bytes = 0;
  for (int c = 0; c < ncols; ++c) {
    if (!cols[c].data || !out[c].data || cols[c].width != out[c].width || cols[c].type != out[c].type ||
        cols[c].width <= 0 || (cols[c].width != 1 && cols[c].width % 4))
      return YQ_ERR_INVALID_ARG;
    M.c[c].src = static_cast<const char*>(cols[c].data);
    M.c[c].src_nulls = cols[c].nulls;
    M.c[c].dst = static_cast<char*>(out[c].data);
    M.c[c].dst_nulls = const_cast<uint8_t*>(out[c].nulls);
    M.c[c].width = cols[c].width;
    {
      const int w = cols[c].width;
      const uintptr_t a = reinterpret_cast<uintptr_t>(cols[c].data) | reinterpret_cast<uintptr_t>(out[c].data);
      M.c[c].vec = (w == 4 || w == 8 || w == 16) && (a % (uintptr_t)w) == 0;
    }
    row_bytes += 2.0 * cols[c].width + (out[c].nulls ? 2.0 : 0.0);
  }
  M.ncols = ncols;
  M.key.data = static_cast<const char*>(kc.data);
  M.key.nulls = kc.nulls;
  M.key.in_perm = nullptr;
  M.key.type = kc.type;
  M.key.width = kc.width;
  M.key.vwords = kc.type == YQ_TEXT ? kc.width / 4 : (kc.width == 8 ? 2 : 1);
  M.key.desc = descending != 0;
  M.key.nulls_first = nulls_first != 0;
  M.key.null_word = kc.nulls != nullptr;
  M.staged = (kc.width <= 32 && (kc.width == 4 || kc.width == 8 || kc.width % 16 == 0) &&
              (reinterpret_cast<uintptr_t>(kc.data) & 15u) == 0);

  std::vector<MergePair> pairs;
  uint32_t tiles = 0;
  for (int r = 0; r < nruns; r += 2) {
    MergePair p;
    p.a0 = run_offsets[r];
    p.m = run_offsets[r + 1] - run_offsets[r];
    p.b0 = run_offsets[r + 1];
    p.n = (r + 1 < nruns) ? run_offsets[r + 2] - run_offsets[r + 1] : 0u;
    p.out0 = p.a0;
    p.tile0 = tiles;
    const uint32_t t = ceil_div<uint32_t>(p.m + p.n, kMergeTile);
    if (t == 0) continue;  // empty pair
    tiles += t;
    pairs.push_back(p);
  }
  if (tiles == 0) return YQ_OK;
  const uint32_t total_rows = run_offsets[nruns] - run_offsets[0];
  cudaStream_t s = as_stream(stream);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_merge_workspace_size(total_rows + (uint32_t)run_offsets[0], nruns), s));
  MergePair* d_pairs = ws.take<MergePair>(pairs.size() + 1);
  uint32_t* d_split = ws.take<uint32_t>((size_t)tiles + 1);
  uint32_t* d_err = ws.take<uint32_t>(4);
  YQ_TRY_CUDA(cudaMemcpyAsync(d_pairs, pairs.data(), pairs.size() * sizeof(MergePair), cudaMemcpyHostToDevice, s));
  YQ_TRY_CUDA(cudaMemsetAsync(d_err, 0, 4 * sizeof(uint32_t), s));
  M.npairs = (int)pairs.size();
  M.ntiles = tiles;
  M.pairs = d_pairs;
  M.split = d_split;
  M.err = d_err;
  const double bytes = (double)total_rows * row_bytes;
  switch (kw) {
    case 1: YQ_TRY(launch_merge<1>(M, s, bytes)); break;
    case 2: YQ_TRY(launch_merge<2>(M, s, bytes)); break;
    case 4: YQ_TRY(launch_merge<4>(M, s, bytes)); break;
    default: YQ_TRY(launch_merge<8>(M, s, bytes)); break;
  }
  uint32_t err = 0;
  YQ_TRY(d2h_sync(&err, d_err, sizeof(uint32_t), s));
  if (err & kErrTimeout) return YQ_ERR_TIMEOUT;
  if (err & kErrBounds) return YQ_ERR_INVALID_ARG;
  return YQ_OK;
}

}  // extern "C"
