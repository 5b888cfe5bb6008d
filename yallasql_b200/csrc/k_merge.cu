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
#include <vector>
#include "yq_keys.cuh"

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
  static size_t attr = 0;
  if (smem > 48 * 1024 && smem > attr) {
    YQ_TRY_CUDA(cudaFuncSetAttribute(k_merge_tiles<KW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = smem;
  }
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
  YQ_TRY_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  YQ_TRY_CUDA(cudaStreamSynchronize(s));
  if (err & kErrTimeout) return YQ_ERR_TIMEOUT;
  if (err & kErrBounds) return YQ_ERR_INVALID_ARG;
  return YQ_OK;
}

}  // extern "C"
