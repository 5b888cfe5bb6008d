// Inner join (nested-loop semantics), cross product and the fused star-join
// aggregate for sm_100a.
//
// Replaces ComparisonJoinExpression / ConjunctionJoinExpression with
// outer_join_batches (one thread per (l, r) pair, one global atomic per match)
// and and_join_batches (P1 x P2 intersection of pair lists), move_rows_join
// per output column, and CrossProductOperator's per-column replication
// (include/engine/operators/filters/comparison_join.hpp:70-236,
//  src/kernels/comparison_operators_kernel.cu:6-54,136-167,
//  src/kernels/move_rows_kernel.cu:8-30, include/engine/operators/join_operator.hpp:36-265,
//  include/engine/operators/cross_product_operator.hpp:87-125, src/kernels/cross_product_kernel.cu:8-27).
//
// All conditions are evaluated in one kernel and pairs come out in a fixed
// order (left row ascending, then right row ascending):
//  - equality path: the right side's equality key is bucketed once into a
//    stably ordered hash table that every block copies into shared memory;
//    each left row probes its bucket, checks the remaining conditions, counts,
//    and after a decoupled look-back over tiles writes its pairs;
//  - nested-loop path: a warp per left row sweeps the right rows 32 at a time,
//    ballots the matches and appends them with popc offsets (coalesced);
//  - no condition: the cross product is written directly, left-major.
#include <string.h>
#include <vector>
#include "vm_host.cuh"
#include "row_kernels.cuh"
#include "yq_jit.cuh"
#include "yq_sort.cuh"

namespace yq {

constexpr int kJoinBlock = 256;
constexpr int kJoinItems = 4;
constexpr uint32_t kJoinTile = kJoinBlock * kJoinItems;
constexpr uint32_t kHashMaxRows = 8192;  // right rows that fit the shared-memory table
constexpr int kMaxConds = 8;
constexpr int kMaxJoinOut = YQ_MAX_PROJECTIONS;

struct JCond {
  JCol l, r;
  int32_t cmp;
};

struct JOut {
  const char* src;
  const uint8_t* src_nulls;
  char* dst;
  uint8_t* dst_nulls;
  int32_t width;
  int32_t side;  // 0 = left, 1 = right
};

struct JoinParams {
  JCond cond[kMaxConds];
  int32_t ncond;
  // OR of ANDs: condition i belongs to disjunct group[i]; a pair matches when
  // every condition of at least one group holds. ngroups <= 1: one conjunction.
  int8_t group[kMaxConds];
  int32_t ngroups;
  int32_t eq;  // index of the equality condition used for hashing (-1: nested loop)
  JOut out[kMaxJoinOut];
  int32_t nout;          // 0: write pairs
  uint32_t* out_left;    // pair output (nout == 0)
  uint32_t* out_right;
  unsigned long long capacity;
  uint32_t L, R;
  // hash table (equality path)
  const uint32_t* bstart;  // nbuckets + 1
  const unsigned long long* hkeys;
  const uint32_t* hrows;
  uint32_t nbuckets, hrows_n;
  unsigned long long* status;
  uint32_t* tile_counter;
  unsigned long long* total;
  uint32_t* err;
  const uint32_t* counts;  // typed nested loop: matches per left row, counted up front (null: count in the kernel)
  char* vdst[2];           // typed nested loop writing the condition's own values: left / right output (or null)
};


__device__ __forceinline__ bool cmp_holds(int s, int op) {
  switch (op) {
    case YQ_LT: return s < 0;
    case YQ_LE: return s <= 0;
    case YQ_GT: return s > 0;
    case YQ_GE: return s >= 0;
    case YQ_EQ: return s == 0;
    default: return s != 0;
  }
}

// Three-way compare of left row l and right row r for one condition; false
// when either side is NULL (an SQL comparison with NULL is not TRUE).
__device__ __forceinline__ bool cond_holds(const JCond& c, uint32_t l, uint32_t r) {
  if (cell_null(c.l, l) || cell_null(c.r, r)) return false;
  int s;
  if (c.l.type == YQ_TEXT) {
    const uint32_t* p = reinterpret_cast<const uint32_t*>(c.l.data + (size_t)l * c.l.width);
    const uint32_t* q = reinterpret_cast<const uint32_t*>(c.r.data + (size_t)r * c.r.width);
    const int pw = c.l.width >> 2, qw = c.r.width >> 2, n = pw > qw ? pw : qw;
    s = 0;
    for (int i = 0; i < n && s == 0; ++i) {
      const uint32_t a = i < pw ? __byte_perm(__ldg(p + i), 0, 0x0123) : 0u;
      const uint32_t b = i < qw ? __byte_perm(__ldg(q + i), 0, 0x0123) : 0u;
      s = (a > b) - (a < b);
    }
  } else {
    const uint64_t a = cell_u64(c.l, l), b = cell_u64(c.r, r);
    switch (c.l.type) {
      case YQ_FLOAT32: {
        const float x = __uint_as_float((uint32_t)a), y = __uint_as_float((uint32_t)b);
        s = (x > y) - (x < y);
        break;
      }
      case YQ_FLOAT64: {
        const double x = __longlong_as_double((long long)a), y = __longlong_as_double((long long)b);
        s = (x > y) - (x < y);
        break;
      }
      default: {
        const int64_t x = (int64_t)a, y = (int64_t)b;
        s = (x > y) - (x < y);
      }
    }
    if (c.l.type == YQ_FLOAT32 || c.l.type == YQ_FLOAT64) {
      // NaN never satisfies a comparison
      const bool nan_a = c.l.type == YQ_FLOAT32 ? isnan(__uint_as_float((uint32_t)a))
                                                : isnan(__longlong_as_double((long long)a));
      const bool nan_b = c.l.type == YQ_FLOAT32 ? isnan(__uint_as_float((uint32_t)b))
                                                : isnan(__longlong_as_double((long long)b));
      if (nan_a || nan_b) return c.cmp == YQ_NE;
    }
  }
  return cmp_holds(s, c.cmp);
}

// A disjunction of conjunctions: a group fails at its first condition that
// does not hold (a comparison with a NULL side does not hold), later
// conditions of a failed group are skipped, and the pair matches while some
// group has not failed. Only TRUE selects a pair, so this two-valued
// evaluation gives the rows SQL's three-valued OR/AND selects.
__device__ __forceinline__ bool any_group(const JoinParams& J, uint32_t l, uint32_t r) {
  const uint32_t all = (1u << J.ngroups) - 1u;
  uint32_t failed = 0u;
  for (int i = 0; i < J.ncond; ++i) {
    const uint32_t bit = 1u << J.group[i];
    if (!(failed & bit) && !cond_holds(J.cond[i], l, r)) {
      failed |= bit;
      if (failed == all) return false;
    }
  }
  return true;
}

__device__ __forceinline__ bool all_conds(const JoinParams& J, uint32_t l, uint32_t r, int skip) {
  if (J.ngroups > 1) return any_group(J, l, r);
  for (int i = 0; i < J.ncond; ++i)
    if (i != skip && !cond_holds(J.cond[i], l, r)) return false;
  return true;
}

__device__ __forceinline__ void copy_cell_j(char* dst, const char* src, int width) {
  if (width == 4) *reinterpret_cast<uint32_t*>(dst) = __ldg(reinterpret_cast<const uint32_t*>(src));
  else if (width == 8)
    *reinterpret_cast<unsigned long long*>(dst) = __ldg(reinterpret_cast<const unsigned long long*>(src));
  else if (width == 1) *dst = *src;
  else
    for (int i = 0; i < width; i += 4)
      *reinterpret_cast<uint32_t*>(dst + i) = __ldg(reinterpret_cast<const uint32_t*>(src + i));
}

__device__ __forceinline__ void emit_pair(const JoinParams& J, unsigned long long pos, uint32_t l, uint32_t r) {
  if (pos >= J.capacity) return;
  if (J.nout == 0) {
    J.out_left[pos] = l;
    J.out_right[pos] = r;
    return;
  }
  for (int o = 0; o < J.nout; ++o) {
    const JOut& w = J.out[o];
    const uint32_t row = w.side ? r : l;
    copy_cell_j(w.dst + (size_t)pos * w.width, w.src + (size_t)row * w.width, w.width);
    if (w.dst_nulls) w.dst_nulls[pos] = w.src_nulls ? w.src_nulls[row] : 0;
  }
}

// ------------------------------------------------------------ hash build
// One block buckets the right rows (optionally only those passing a
// predicate) by hash of the equality key; within a bucket rows stay in
// ascending row order, so probing yields right rows in ascending order.
struct BuildParams {
  VmProgram P;        // predicate over the right batch (pred_len == 0: all rows)
  int32_t pred_len;
  JCol key;
  uint32_t R;
  uint32_t nbuckets;
  uint32_t* bstart;   // [nbuckets + 1]
  unsigned long long* hkeys;
  uint32_t* hrows;
  uint32_t* counts;   // [0] rows kept, [1] duplicate keys seen
};


constexpr int kBuildBlock = 1024;

__global__ void __launch_bounds__(kBuildBlock) k_hash_build(const __grid_constant__ BuildParams B) {
  extern __shared__ uint32_t sb[];
  uint32_t* s_cnt = sb;                        // [nbuckets] counts, then cursors
  uint32_t* s_rows = s_cnt + B.nbuckets;       // [R] kept rows in order
  uint32_t* s_warp = s_rows + kHashMaxRows;    // [33]
  __shared__ uint32_t s_kept;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t i = threadIdx.x; i < B.nbuckets; i += kBuildBlock) s_cnt[i] = 0;
  if (threadIdx.x == 0) s_kept = 0;
  __syncthreads();
  // 1. stable compaction of the rows passing the predicate
  for (uint32_t base = 0; base < B.R; base += kBuildBlock * ITEMS) {
    const uint32_t row0 = base + threadIdx.x * ITEMS;
    uint32_t inr = 0;
    if (row0 < B.R) inr = (B.R - row0 >= (uint32_t)ITEMS) ? 0xfu : ((1u << (B.R - row0)) - 1u);
    SelEmit E;
    E.sel = inr;
    if (B.pred_len > 0) {
      Ctx X;
      X.tile0 = base;
      X.lr = threadIdx.x * ITEMS;
      X.inr = inr;
      X.stage = 0;
      X.vec_ok = (base & 15u) == 0u;
      Stack S;
      run_vm<false>(B.P, 0, B.pred_len, X, S, E);
    }
    // key NULLs never join
    for (int k = 0; k < ITEMS; ++k)
      if ((E.sel >> k & 1u) && cell_null(B.key, row0 + k)) E.sel &= ~(1u << k);
    uint32_t total;
    const uint32_t excl = block_exclusive_sum<kBuildBlock>(__popc(E.sel), s_warp, total);
    uint32_t pos = s_kept + excl;
    for (int k = 0; k < ITEMS; ++k)
      if (E.sel >> k & 1u) {
        if (pos < kHashMaxRows) s_rows[pos] = row0 + k;
        ++pos;
      }
    __syncthreads();
    if (threadIdx.x == 0) s_kept += total;
    __syncthreads();
  }
  const uint32_t kept = min(s_kept, kHashMaxRows);
  // 2. bucket counts and starts
  for (uint32_t i = threadIdx.x; i < kept; i += kBuildBlock)
    atomicAdd(&s_cnt[hash_bucket(hash_key(B.key, s_rows[i]), B.nbuckets)], 1u);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (uint32_t b = 0; b < B.nbuckets; ++b) {
      const uint32_t c = s_cnt[b];
      B.bstart[b] = run;
      s_cnt[b] = run;  // becomes the insertion cursor
      run += c;
    }
    B.bstart[B.nbuckets] = run;
    B.counts[0] = s_kept;
  }
  __syncthreads();
  // 3. stable scatter: rows in ascending order, one warp at a time
  for (uint32_t base = 0; base < kept; base += kBuildBlock) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < kept;
    const uint32_t row = valid ? s_rows[i] : 0u;
    const uint64_t key = valid ? hash_key(B.key, row) : 0ull;
    const uint32_t b = valid ? hash_bucket(key, B.nbuckets) : 0xffffffffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, b) & __ballot_sync(0xffffffffu, valid);
    const uint32_t rank = __popc(peers & lanemask_lt());
    for (int w = 0; w < kBuildBlock / 32; ++w) {
      if (warp == w && valid) {
        const uint32_t slot = s_cnt[b] + rank;
        B.hkeys[slot] = key;
        B.hrows[slot] = row;
        __syncwarp(peers);
        if (rank == 0) s_cnt[b] += __popc(peers);
      }
      __syncthreads();
    }
  }
  __syncthreads();
  // 4. duplicate keys (the fused aggregate needs unique dimension keys)
  for (uint32_t b = threadIdx.x; b < B.nbuckets; b += kBuildBlock) {
    const uint32_t s0 = B.bstart[b], s1 = B.bstart[b + 1];
    for (uint32_t x = s0; x < s1; ++x)
      for (uint32_t y = x + 1; y < s1; ++y)
        if (B.hkeys[x] == B.hkeys[y]) atomicAdd(&B.counts[1], 1u);
  }
  (void)lane;
}

// ------------------------------------------------------ equality probing
struct ProbeSmem {
  uint32_t* bstart;
  unsigned long long* keys;
  uint32_t* rows;
};

__device__ __forceinline__ ProbeSmem load_table(const JoinParams& J, uint32_t* sm) {
  ProbeSmem t;
  t.bstart = sm;
  t.keys = reinterpret_cast<unsigned long long*>(sm + ((J.nbuckets + 2) & ~1u));
  t.rows = reinterpret_cast<uint32_t*>(t.keys + J.hrows_n);
  for (uint32_t i = threadIdx.x; i <= J.nbuckets; i += blockDim.x) t.bstart[i] = __ldg(J.bstart + i);
  for (uint32_t i = threadIdx.x; i < J.hrows_n; i += blockDim.x) {
    t.keys[i] = __ldg(J.hkeys + i);
    t.rows[i] = __ldg(J.hrows + i);
  }
  __syncthreads();
  return t;
}

__global__ void __launch_bounds__(kJoinBlock) k_join_hash(const __grid_constant__ JoinParams J) {
  extern __shared__ uint32_t sm[];
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kJoinBlock / 32 + 1];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(J.tile_counter, 1u);
  const ProbeSmem T = load_table(J, sm);
  const uint32_t tile = s_tile;
  const uint32_t l0 = tile * kJoinTile + threadIdx.x * kJoinItems;
  const JCond& ec = J.cond[J.eq];
  // pass 1: count
  uint32_t cnt = 0;
  for (int k = 0; k < kJoinItems; ++k) {
    const uint32_t l = l0 + k;
    if (l >= J.L || cell_null(ec.l, l)) continue;
    const uint64_t key = hash_key(ec.l, l);
    const uint32_t b = hash_bucket(key, J.nbuckets);
    for (uint32_t x = T.bstart[b]; x < T.bstart[b + 1]; ++x)
      if (T.keys[x] == key && all_conds(J, l, T.rows[x], J.eq)) ++cnt;
  }
  uint32_t total;
  const uint32_t excl = block_exclusive_sum<kJoinBlock>(cnt, s_warp, total);
  if (threadIdx.x < 32) {
    const unsigned long long p = tile_lookback(J.status, tile, total, J.err);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  unsigned long long pos = s_prefix + excl;
  // pass 2: write
  if (cnt) {
    for (int k = 0; k < kJoinItems; ++k) {
      const uint32_t l = l0 + k;
      if (l >= J.L || cell_null(ec.l, l)) continue;
      const uint64_t key = hash_key(ec.l, l);
      const uint32_t b = hash_bucket(key, J.nbuckets);
      for (uint32_t x = T.bstart[b]; x < T.bstart[b + 1]; ++x)
        if (T.keys[x] == key && all_conds(J, l, T.rows[x], J.eq)) emit_pair(J, pos++, l, T.rows[x]);
    }
  }
  if (tile == gridDim.x - 1 && threadIdx.x == 0) *J.total = s_prefix + total;
}

// ------------------------------------------------------------ nested loop
constexpr int kNlRowsPerWarp = 4;
constexpr uint32_t kNlTile = (kJoinBlock / 32) * kNlRowsPerWarp;  // left rows per block

__global__ void __launch_bounds__(kJoinBlock) k_join_nested(const __grid_constant__ JoinParams J) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_cnt[kNlTile];
  __shared__ uint32_t s_warp[kJoinBlock / 32 + 1];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(J.tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = lanemask_lt();
  // pass 1: per left row, count the matching right rows (warp ballots)
  for (int i = 0; i < kNlRowsPerWarp; ++i) {
    const uint32_t slot = warp * kNlRowsPerWarp + i;
    const uint32_t l = tile * kNlTile + slot;
    uint32_t c = 0;
    if (l < J.L)
      for (uint32_t r0 = 0; r0 < J.R; r0 += 32) {
        const uint32_t r = r0 + lane;
        const bool m = r < J.R && all_conds(J, l, r, -1);
        c += __popc(__ballot_sync(0xffffffffu, m));
      }
    if (lane == 0) s_cnt[slot] = c;
  }
  __syncthreads();
  const uint32_t mine = threadIdx.x < kNlTile ? s_cnt[threadIdx.x] : 0u;
  uint32_t total;
  const uint32_t excl = block_exclusive_sum<kJoinBlock>(mine, s_warp, total);
  if (threadIdx.x < kNlTile) s_cnt[threadIdx.x] = excl;  // row offset within the tile
  if (threadIdx.x < 32) {
    const unsigned long long p = tile_lookback(J.status, tile, total, J.err);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  // pass 2: write matches, 32 right rows per ballot, consecutive positions
  for (int i = 0; i < kNlRowsPerWarp; ++i) {
    const uint32_t slot = warp * kNlRowsPerWarp + i;
    const uint32_t l = tile * kNlTile + slot;
    if (l >= J.L) continue;
    unsigned long long pos = s_prefix + s_cnt[slot];
    for (uint32_t r0 = 0; r0 < J.R; r0 += 32) {
      const uint32_t r = r0 + lane;
      const bool m = r < J.R && all_conds(J, l, r, -1);
      const uint32_t bal = __ballot_sync(0xffffffffu, m);
      if (m) emit_pair(J, pos + __popc(bal & lt), l, r);
      pos += __popc(bal);
    }
  }
  if (tile == gridDim.x - 1 && threadIdx.x == 0) *J.total = s_prefix + total;
}

// Nested loop for one comparison of two columns of the same fixed-width
// numeric type without nulls (the common inequality join): the right column
// is staged in shared memory kNlChunk rows at a time, each warp holds its
// kNlRowsPerWarp left values in registers, and every right value a lane
// loads is compared with all of them, so a comparison costs a compare, a
// ballot and a popc. IEEE comparisons give the SQL results for NaN (only <>
// holds) and for -0.0 = +0.0. Same tiles, look-back and output order (left
// row major, right rows ascending) as k_join_nested.
constexpr uint32_t kNlChunk = 4096;

template <typename T, int OP>
__device__ __forceinline__ bool nl_cmp(T a, T b) {
  if constexpr (OP == YQ_LT) return a < b;
  else if constexpr (OP == YQ_LE) return a <= b;
  else if constexpr (OP == YQ_GT) return a > b;
  else if constexpr (OP == YQ_GE) return a >= b;
  else if constexpr (OP == YQ_EQ) return a == b;
  else return a != b;
}

// Matches per left row of one typed comparison, from the right column sorted
// ascending with its NaNs (float columns) at the end, `nvalid` values before
// them: two binary searches per left row instead of a pass over the right
// side. A NaN compares false except under <>, as in nl_cmp.
template <typename T>
__device__ __forceinline__ bool nan_of(T v) {
  return v != v;
}

template <typename T>
__global__ void k_join_count_valid(const T* __restrict__ sorted, uint32_t R, uint32_t* nvalid) {
  uint32_t nan = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x)
    nan += nan_of(__ldg(sorted + i)) ? 1u : 0u;
  for (int d = 16; d > 0; d >>= 1) nan += __shfl_xor_sync(0xffffffffu, nan, d);
  if ((threadIdx.x & 31) == 0 && nan) atomicSub(nvalid, nan);
}

template <typename T, int OP>
__global__ void k_join_count_sorted(const T* __restrict__ lcol, uint32_t L, const T* __restrict__ sorted,
                                    const uint32_t* __restrict__ nvalid_p, uint32_t R, uint32_t* __restrict__ counts) {
  const uint32_t nvalid = *nvalid_p;
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < L; l += gridDim.x * blockDim.x) {
    const T v = __ldg(lcol + l);
    uint32_t c;
    if (nan_of(v)) {
      c = OP == YQ_NE ? R : 0u;
    } else {
      uint32_t lo = 0, hi = nvalid;  // first position holding a value >= v
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(sorted + mid) < v) lo = mid + 1;
        else hi = mid;
      }
      const uint32_t lb = lo;
      hi = nvalid;  // first position holding a value > v
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (!(v < __ldg(sorted + mid))) lo = mid + 1;
        else hi = mid;
      }
      const uint32_t ub = lo;
      if constexpr (OP == YQ_LT) c = nvalid - ub;
      else if constexpr (OP == YQ_LE) c = nvalid - lb;
      else if constexpr (OP == YQ_GT) c = lb;
      else if constexpr (OP == YQ_GE) c = ub;
      else if constexpr (OP == YQ_EQ) c = ub - lb;
      else c = R - (ub - lb);
    }
    counts[l] = c;
  }
}

// Outputs of a join that are all 4- or 8-byte cells without null bytes (at
// most kSimpleOut of them, e.g. one column of each side): the typed kernel
// writes them directly, reading each left row's cells once.
constexpr int kSimpleOut = 2;

__device__ __forceinline__ unsigned long long cell_bits(const char* p, int w) {
  return w == 8 ? __ldg(reinterpret_cast<const unsigned long long*>(p)) : (unsigned long long)__ldg(reinterpret_cast<const uint32_t*>(p));
}

// MODE 0: writes (left row, right row) pairs; 1: writes up to kSimpleOut
// 4- or 8-byte cells of either side; 2: the outputs are the condition's own
// two columns (SELECT a.x, b.y ... WHERE a.x < b.y), written from registers.
template <typename T, int OP, int MODE>
__global__ void __launch_bounds__(kJoinBlock) k_join_nested_typed(const __grid_constant__ JoinParams J) {
  constexpr bool SIMPLE = MODE == 1;
  __shared__ T s_r[kNlChunk];
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_cnt[kNlTile];
  __shared__ uint32_t s_warp[kJoinBlock / 32 + 1];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(J.tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = lanemask_lt();
  const JCond& c = J.cond[0];
  const T* lcol = reinterpret_cast<const T*>(c.l.data);
  const T* rcol = reinterpret_cast<const T*>(c.r.data);
  T lv[kNlRowsPerWarp];
  bool lok[kNlRowsPerWarp];
#pragma unroll
  for (int i = 0; i < kNlRowsPerWarp; ++i) {
    const uint32_t l = tile * kNlTile + warp * kNlRowsPerWarp + i;
    lok[i] = l < J.L;
    lv[i] = lok[i] ? __ldg(lcol + l) : T(0);
  }
  // pass 1: matches per left row (counted up front from the sorted right
  // side when J.counts is given, else here over the whole right side)
  if (J.counts) {
    if (lane == 0)
#pragma unroll
      for (int i = 0; i < kNlRowsPerWarp; ++i)
        s_cnt[warp * kNlRowsPerWarp + i] = lok[i] ? __ldg(J.counts + tile * kNlTile + warp * kNlRowsPerWarp + i) : 0u;
  } else {
    uint32_t cnt[kNlRowsPerWarp];
#pragma unroll
    for (int i = 0; i < kNlRowsPerWarp; ++i) cnt[i] = 0;
    for (uint32_t r0 = 0; r0 < J.R; r0 += kNlChunk) {
      const uint32_t n = min(kNlChunk, J.R - r0);
      __syncthreads();
      for (uint32_t x = threadIdx.x; x < n; x += kJoinBlock) s_r[x] = __ldg(rcol + r0 + x);
      __syncthreads();
      // per-lane counts (one predicated add a comparison), summed over the warp below
      for (uint32_t x = lane; x < n; x += 32) {
        const T rv = s_r[x];
#pragma unroll
        for (int i = 0; i < kNlRowsPerWarp; ++i) cnt[i] += (lok[i] && nl_cmp<T, OP>(lv[i], rv)) ? 1u : 0u;
      }
    }
#pragma unroll
    for (int i = 0; i < kNlRowsPerWarp; ++i)
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) cnt[i] += __shfl_xor_sync(0xffffffffu, cnt[i], d);
    if (lane == 0)
#pragma unroll
      for (int i = 0; i < kNlRowsPerWarp; ++i) s_cnt[warp * kNlRowsPerWarp + i] = cnt[i];
  }
  __syncthreads();
  const uint32_t mine = threadIdx.x < kNlTile ? s_cnt[threadIdx.x] : 0u;
  uint32_t total;
  const uint32_t excl = block_exclusive_sum<kJoinBlock>(mine, s_warp, total);
  if (threadIdx.x < kNlTile) s_cnt[threadIdx.x] = excl;  // row offset within the tile
  if (threadIdx.x < 32) {
    const unsigned long long p = tile_lookback(J.status, tile, total, J.err);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  // pass 2: write the matches, consecutive positions per left row
  unsigned long long pos[kNlRowsPerWarp];
#pragma unroll
  for (int i = 0; i < kNlRowsPerWarp; ++i) pos[i] = s_prefix + s_cnt[warp * kNlRowsPerWarp + i];
  unsigned long long lcell[kNlRowsPerWarp][SIMPLE ? kSimpleOut : 1];  // left-side output cells of each row
  const bool room = s_prefix + total <= J.capacity;  // every pair of this tile fits: no per-pair check
  T* const vl = reinterpret_cast<T*>(J.vdst[0]);
  T* const vr = reinterpret_cast<T*>(J.vdst[1]);
  uint32_t from_rv = 0u;  // outputs that are the condition's right column: written from the staged value
  if constexpr (SIMPLE) {
#pragma unroll
    for (int o = 0; o < kSimpleOut; ++o)
      if (o < J.nout && J.out[o].side == 1 && J.out[o].src == static_cast<const char*>(c.r.data) &&
          J.out[o].width == (int)sizeof(T))
        from_rv |= 1u << o;
#pragma unroll
    for (int i = 0; i < kNlRowsPerWarp; ++i)
#pragma unroll
      for (int o = 0; o < kSimpleOut; ++o) {
        const uint32_t l = tile * kNlTile + warp * kNlRowsPerWarp + i;
        lcell[i][o] = (o < J.nout && J.out[o].side == 0 && lok[i])
                          ? cell_bits(J.out[o].src + (size_t)l * J.out[o].width, J.out[o].width) : 0ull;
      }
  }
  for (uint32_t r0 = 0; r0 < J.R; r0 += kNlChunk) {
    const uint32_t n = min(kNlChunk, J.R - r0);
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < n; x += kJoinBlock) s_r[x] = __ldg(rcol + r0 + x);
    __syncthreads();
    for (uint32_t x = lane; x < ((n + 31) & ~31u); x += 32) {
      const bool ok = x < n;
      const T rv = ok ? s_r[x] : T(0);
#pragma unroll
      for (int i = 0; i < kNlRowsPerWarp; ++i) {
        const bool m = ok && lok[i] && nl_cmp<T, OP>(lv[i], rv);
        const uint32_t bal = __ballot_sync(0xffffffffu, m);
        if (m) {
          const unsigned long long at = pos[i] + __popc(bal & lt);
          if constexpr (SIMPLE) {
            if (room || at < J.capacity) {
#pragma unroll
              for (int o = 0; o < kSimpleOut; ++o) {
                if (o >= J.nout) break;
                const JOut& w = J.out[o];
                unsigned long long rb = 0ull;
                if (from_rv >> o & 1u) {
                  if constexpr (sizeof(T) == 8) rb = *reinterpret_cast<const unsigned long long*>(&rv);
                  else rb = (unsigned long long)*reinterpret_cast<const uint32_t*>(&rv);
                }
                const unsigned long long v =
                    !w.side ? lcell[i][o] : ((from_rv >> o & 1u) ? rb : cell_bits(w.src + (size_t)(r0 + x) * w.width, w.width));
                if (w.width == 8) reinterpret_cast<unsigned long long*>(w.dst)[at] = v;
                else reinterpret_cast<uint32_t*>(w.dst)[at] = (uint32_t)v;
              }
            }
          } else if constexpr (MODE == 2) {
            if (room || at < J.capacity) {
              if (vl) vl[at] = lv[i];
              if (vr) vr[at] = rv;
            }
          } else {
            emit_pair(J, at, tile * kNlTile + warp * kNlRowsPerWarp + i, r0 + x);
          }
        }
        pos[i] += __popc(bal);
      }
    }
  }
  if (tile == gridDim.x - 1 && threadIdx.x == 0) *J.total = s_prefix + total;
}

template <typename T, int MODE>
static void launch_nested_typed_op(int op, unsigned grid, const JoinParams& J, cudaStream_t s) {
  switch (op) {
    case YQ_LT: k_join_nested_typed<T, YQ_LT, MODE><<<grid, kJoinBlock, 0, s>>>(J); break;
    case YQ_LE: k_join_nested_typed<T, YQ_LE, MODE><<<grid, kJoinBlock, 0, s>>>(J); break;
    case YQ_GT: k_join_nested_typed<T, YQ_GT, MODE><<<grid, kJoinBlock, 0, s>>>(J); break;
    case YQ_GE: k_join_nested_typed<T, YQ_GE, MODE><<<grid, kJoinBlock, 0, s>>>(J); break;
    case YQ_EQ: k_join_nested_typed<T, YQ_EQ, MODE><<<grid, kJoinBlock, 0, s>>>(J); break;
    default: k_join_nested_typed<T, YQ_NE, MODE><<<grid, kJoinBlock, 0, s>>>(J); break;
  }
}

template <typename T>
static void launch_nested_typed(int op, unsigned grid, JoinParams J, cudaStream_t s) {
  bool simple = J.nout >= 1 && J.nout <= kSimpleOut;
  for (int o = 0; o < J.nout && simple; ++o) simple = (J.out[o].width == 4 || J.out[o].width == 8) && !J.out[o].dst_nulls;
  // the outputs are the condition's own left and right columns, each at most once
  bool values = simple;
  J.vdst[0] = J.vdst[1] = nullptr;
  for (int o = 0; o < J.nout && values; ++o) {
    const JOut& w = J.out[o];
    const JCol& cc = w.side ? J.cond[0].r : J.cond[0].l;
    values = w.src == cc.data && w.width == (int)sizeof(T) && !J.vdst[w.side];
    if (values) J.vdst[w.side] = w.dst;
  }
  if (values) launch_nested_typed_op<T, 2>(op, grid, J, s);
  else if (simple) launch_nested_typed_op<T, 1>(op, grid, J, s);
  else launch_nested_typed_op<T, 0>(op, grid, J, s);
}

// ------------------------------------------------------- cross product
// Every (l, r), left-major: output row l*R + r.
__global__ void __launch_bounds__(256) k_cross_fill(const __grid_constant__ JoinParams J) {
  const unsigned long long n = (unsigned long long)J.L * J.R;
  const unsigned long long lim = n < J.capacity ? n : J.capacity;
  for (unsigned long long p = blockIdx.x * 256ull + threadIdx.x; p < lim; p += (unsigned long long)gridDim.x * 256ull) {
    const uint32_t l = (uint32_t)(p / J.R), r = (uint32_t)(p % J.R);
    emit_pair(J, p, l, r);
  }
}

template <bool STAGED>
__global__ void __launch_bounds__(kRowBlock, 2) k_join_aggregate(const __grid_constant__ JAParams F, uint32_t n,
                                                                 Acc* __restrict__ partials, uint32_t* ticket,
                                                                 Acc* state) {
  join_aggregate_body<STAGED, InterpRunner>(F, n, partials, ticket, state);
}

// ---------------------------------------------------------------- host
static bool join_col_ok(const yq_column& c) {
  if (!c.data) return false;
  return ProgramBuilder::valid_column(c);
}

static JCol jcol(const yq_column& c) {
  JCol j;
  j.data = static_cast<const char*>(c.data);
  j.nulls = c.nulls;
  j.type = c.type;
  j.width = c.width;
  return j;
}

static bool hashable(int t) {
  return t == YQ_INT32 || t == YQ_INT64 || t == YQ_DATETIME || t == YQ_FLOAT32 || t == YQ_FLOAT64 || t == YQ_BOOL;
}

static uint32_t pow2_at_least(uint32_t x) {
  uint32_t p = 16;
  while (p < x) p <<= 1;
  return p;
}

static size_t table_smem(uint32_t nbuckets, uint32_t nrows, bool with_rows) {
  return sizeof(uint32_t) * ((nbuckets + 2) & ~1u) + sizeof(unsigned long long) * nrows +
         (with_rows ? sizeof(uint32_t) * nrows : 0);
}

static int build_table(const yq_batch* right, const yq_program* pred, const yq_constants* consts, int key_col,
                       uint32_t nbuckets, uint32_t* bstart, unsigned long long* hkeys, uint32_t* hrows,
                       uint32_t* counts, cudaStream_t s) {
  BuildParams B;
  memset(&B, 0, sizeof(B));
  ProgramBuilder PB;
  YQ_TRY(PB.set_columns(right->columns, right->ncols));
  YQ_TRY(PB.set_constants(consts));
  if (pred && pred->len > 0) {
    int t = -1;
    YQ_TRY(PB.append(pred, t));
    if (t != YQ_BOOL) return YQ_ERR_INVALID_ARG;
    YQ_TRY(PB.emit(OP_EMIT_PRED, 0, 0, YQ_BOOL));
  }
  YQ_TRY(PB.finalize());
  memcpy(&B.P, &PB.P, sizeof(VmProgram));
  B.pred_len = PB.len;
  B.key = jcol(right->columns[key_col]);
  B.R = right->rows;
  B.nbuckets = nbuckets;
  B.bstart = bstart;
  B.hkeys = hkeys;
  B.hrows = hrows;
  B.counts = counts;
  const size_t smem = sizeof(uint32_t) * (nbuckets + kHashMaxRows + 40);
  YQ_TRY(kernel_allow_smem((const void*)k_hash_build, smem));
  ProfScope ps("join_hash_build", s, (double)right->rows * right->columns[key_col].width);
  k_hash_build<<<1, kBuildBlock, smem, s>>>(B);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

// The typed nested loop counts each left row's matches up front when the
// right side is at least this long: one sort of the right key and two
// binary searches per left row, instead of a comparison pass over L x R.
constexpr uint32_t kCountFirstRows = 4096;

// Sort workspace for a right side of R rows (an 8-byte key bounds the typed
// path's 4- and 8-byte keys). Sizing reads no column data: the placeholder
// pointer only has to be non-null.
static size_t count_sort_bytes(uint32_t R) {
  yq_column dummy{reinterpret_cast<void*>(static_cast<uintptr_t>(256)), nullptr, YQ_INT64, 8};
  KeyJob j{dummy, 0, 0};
  uint32_t offs[2] = {0, R};
  size_t sb = 0;
  if (sort_segments_impl(&j, 1, R, offs, 1, nullptr, nullptr, nullptr, 0, nullptr, &sb) != YQ_OK) return 0;
  return sb;
}

struct CountWs {
  char* sort_ws;
  size_t sort_bytes;
  uint32_t* perm;     // [R]
  char* sorted;       // [R] values of the right key, ascending
  uint32_t* nvalid;   // [1] values before the NaNs
  uint32_t* counts;   // [L]
};

static void count_ws_layout(uint32_t L, uint32_t R, size_t sort_bytes, WsSize& w) {
  w.add<char>(sort_bytes);
  w.add<uint32_t>(R ? R : 1);
  w.add<unsigned long long>(R ? R : 1);
  w.add<uint32_t>(4);
  w.add<uint32_t>(L ? L : 1);
}

template <typename T>
static int count_matches_typed(const JoinParams& J, const CountWs& c, cudaStream_t s) {
  const JCond& c0 = J.cond[0];
  const yq_column rc{const_cast<char*>(c0.r.data), nullptr, c0.r.type, c0.r.width};
  KeyJob j{rc, 0, 0};
  uint32_t offs[2] = {0, J.R};
  YQ_TRY(sort_segments_impl(&j, 1, J.R, offs, 1, c.perm, nullptr, c.sort_ws, c.sort_bytes, s, nullptr));
  const yq_column sc{c.sorted, nullptr, rc.type, rc.width};
  YQ_TRY(gather_impl(&rc, 1, c.perm, J.R, &sc, nullptr, s));
  const uint32_t R = J.R;
  YQ_TRY(h2d_async(c.nvalid, &R, sizeof(R), s));
  const int grid = sm_count() * 4;
  const T* sorted = reinterpret_cast<const T*>(c.sorted);
  const T* lcol = reinterpret_cast<const T*>(c0.l.data);
  k_join_count_valid<T><<<grid, 256, 0, s>>>(sorted, J.R, c.nvalid);
  YQ_CHECK_LAUNCH();
  switch (c0.cmp) {
    case YQ_LT: k_join_count_sorted<T, YQ_LT><<<grid, 256, 0, s>>>(lcol, J.L, sorted, c.nvalid, R, c.counts); break;
    case YQ_LE: k_join_count_sorted<T, YQ_LE><<<grid, 256, 0, s>>>(lcol, J.L, sorted, c.nvalid, R, c.counts); break;
    case YQ_GT: k_join_count_sorted<T, YQ_GT><<<grid, 256, 0, s>>>(lcol, J.L, sorted, c.nvalid, R, c.counts); break;
    case YQ_GE: k_join_count_sorted<T, YQ_GE><<<grid, 256, 0, s>>>(lcol, J.L, sorted, c.nvalid, R, c.counts); break;
    case YQ_EQ: k_join_count_sorted<T, YQ_EQ><<<grid, 256, 0, s>>>(lcol, J.L, sorted, c.nvalid, R, c.counts); break;
    default: k_join_count_sorted<T, YQ_NE><<<grid, 256, 0, s>>>(lcol, J.L, sorted, c.nvalid, R, c.counts); break;
  }
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

// Shared by yq_join_pairs / yq_join_project.
static int join_impl(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds, const int32_t* disjunct,
                     int32_t ncond, const yq_join_output* outputs, int32_t nout, yq_column* out, uint32_t* out_left,
                     uint32_t* out_right, uint64_t capacity, uint64_t* count_host, void* workspace,
                     size_t workspace_bytes, cudaStream_t s) {
  if (!left || !right || ncond < 0 || ncond > kMaxConds || (ncond > 0 && !conds) || nout < 0 || nout > kMaxJoinOut ||
      (nout > 0 && (!outputs || !out)))
    return YQ_ERR_INVALID_ARG;
  JoinParams J;
  memset(&J, 0, sizeof(J));
  J.L = left->rows;
  J.R = right->rows;
  J.ncond = ncond;
  J.eq = -1;
  J.ngroups = 1;
  if (disjunct && ncond > 0) {  // groups numbered 0..G-1, each used by some condition
    int g = 0;
    uint32_t used = 0u;
    for (int i = 0; i < ncond; ++i) {
      if (disjunct[i] < 0 || disjunct[i] >= kMaxConds) return YQ_ERR_INVALID_ARG;
      J.group[i] = (int8_t)disjunct[i];
      used |= 1u << disjunct[i];
      g = disjunct[i] + 1 > g ? disjunct[i] + 1 : g;
    }
    if (used != (1u << g) - 1u) return YQ_ERR_INVALID_ARG;
    J.ngroups = g;
  }
  for (int i = 0; i < ncond; ++i) {
    const yq_join_cond& c = conds[i];
    if (c.left_col < 0 || c.left_col >= left->ncols || c.right_col < 0 || c.right_col >= right->ncols ||
        c.cmp < YQ_LT || c.cmp > YQ_NE)
      return YQ_ERR_INVALID_ARG;
    const yq_column& a = left->columns[c.left_col];
    const yq_column& b = right->columns[c.right_col];
    if (!join_col_ok(a) || !join_col_ok(b) || a.type != b.type) return YQ_ERR_INVALID_ARG;
    J.cond[i].l = jcol(a);
    J.cond[i].r = jcol(b);
    J.cond[i].cmp = c.cmp;
    if (J.eq < 0 && J.ngroups == 1 && c.cmp == YQ_EQ && hashable(a.type)) J.eq = i;
  }
  for (int o = 0; o < nout; ++o) {
    const yq_join_output& w = outputs[o];
    const yq_batch* side = w.side ? right : left;
    if (w.column < 0 || w.column >= side->ncols) return YQ_ERR_INVALID_ARG;
    const yq_column& c = side->columns[w.column];
    if (!join_col_ok(c) || out[o].type != c.type || out[o].width != c.width || !out[o].data) return YQ_ERR_INVALID_ARG;
    J.out[o].src = static_cast<const char*>(c.data);
    J.out[o].src_nulls = c.nulls;
    J.out[o].dst = static_cast<char*>(out[o].data);
    J.out[o].dst_nulls = const_cast<uint8_t*>(out[o].nulls);
    J.out[o].width = c.width;
    J.out[o].side = w.side;
  }
  J.nout = nout;
  if (nout == 0 && capacity > 0 && (!out_left || !out_right)) return YQ_ERR_INVALID_ARG;
  J.out_left = out_left;
  J.out_right = out_right;
  J.capacity = capacity;

  if (J.L == 0 || J.R == 0) {
    if (count_host) *count_host = 0;
    return YQ_OK;
  }
  if (ncond == 0) {  // cross product: size known up front
    const unsigned long long n = (unsigned long long)J.L * J.R;
    double row_bytes = nout == 0 ? 8.0 : 0.0;
    for (int o = 0; o < nout; ++o) row_bytes += J.out[o].width + (J.out[o].dst_nulls ? 1 : 0);
    ProfScope ps("cross_product", s, (double)(n < capacity ? n : capacity) * row_bytes);
    const unsigned long long lim = n < capacity ? n : capacity;
    int grid = (int)((lim + 255) / 256);
    const int cap = sm_count() * 16;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    k_cross_fill<<<grid, 256, 0, s>>>(J);
    YQ_CHECK_LAUNCH();
    if (count_host) *count_host = n;
    return n > capacity ? YQ_ERR_CAPACITY : YQ_OK;
  }

  const bool use_hash = J.eq >= 0 && J.R <= kHashMaxRows;
  const uint32_t nbuckets = use_hash ? pow2_at_least(J.R) : 0u;
  const uint32_t ntiles = use_hash ? ceil_div<uint32_t>(J.L, kJoinTile) : ceil_div<uint32_t>(J.L, kNlTile);
  const JCond& t0 = J.cond[0];
  const bool typed = !use_hash && J.ncond == 1 && J.ngroups == 1 && t0.l.type == t0.r.type && !t0.l.nulls &&
                     !t0.r.nulls && t0.l.width == t0.r.width &&
                     (t0.l.type == YQ_INT32 || t0.l.type == YQ_FLOAT32 || t0.l.type == YQ_INT64 ||
                      t0.l.type == YQ_DATETIME || t0.l.type == YQ_FLOAT64);
  const size_t sort_bytes = typed && J.R >= kCountFirstRows ? count_sort_bytes(J.R) : 0;
  const bool count_first = sort_bytes != 0;  // else (a right side too long to sort) the kernel counts
  WsSize w;
  w.add<uint32_t>(nbuckets + 1);
  w.add<unsigned long long>(use_hash ? J.R : 1);
  w.add<uint32_t>(use_hash ? J.R : 1);
  w.add<unsigned long long>((size_t)ntiles + 1);
  w.add<uint32_t>(8);
  w.add<unsigned long long>(2);
  if (count_first) count_ws_layout(J.L, J.R, sort_bytes, w);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, w.total(), s));
  uint32_t* d_bstart = ws.take<uint32_t>(nbuckets + 1);
  unsigned long long* d_hkeys = ws.take<unsigned long long>(use_hash ? J.R : 1);
  uint32_t* d_hrows = ws.take<uint32_t>(use_hash ? J.R : 1);
  J.status = ws.take<unsigned long long>((size_t)ntiles + 1);
  uint32_t* d_misc = ws.take<uint32_t>(8);  // [0] tile counter [1] err [2..3] build counts
  J.total = ws.take<unsigned long long>(2);
  J.tile_counter = d_misc;
  J.err = d_misc + 1;
  CountWs cw{};
  if (count_first) {
    cw.sort_ws = ws.take<char>(sort_bytes);
    cw.sort_bytes = sort_bytes;
    cw.perm = ws.take<uint32_t>(J.R ? J.R : 1);
    cw.sorted = reinterpret_cast<char*>(ws.take<unsigned long long>(J.R ? J.R : 1));
    cw.nvalid = ws.take<uint32_t>(4);
    cw.counts = ws.take<uint32_t>(J.L ? J.L : 1);
  }
  YQ_TRY_CUDA(cudaMemsetAsync(J.status, 0, ((size_t)ntiles + 1) * sizeof(unsigned long long), s));
  YQ_TRY_CUDA(cudaMemsetAsync(d_misc, 0, 8 * sizeof(uint32_t), s));
  YQ_TRY_CUDA(cudaMemsetAsync(J.total, 0, 2 * sizeof(unsigned long long), s));
  double out_row_bytes = nout == 0 ? 8.0 : 0.0;
  for (int o = 0; o < nout; ++o) out_row_bytes += J.out[o].width + (J.out[o].dst_nulls ? 1 : 0);
  if (use_hash) {
    YQ_TRY(build_table(right, nullptr, nullptr, conds[J.eq].right_col, nbuckets, d_bstart, d_hkeys, d_hrows,
                       d_misc + 2, s));
    J.bstart = d_bstart;
    J.hkeys = d_hkeys;
    J.hrows = d_hrows;
    J.nbuckets = nbuckets;
    J.hrows_n = J.R;
    const size_t smem = table_smem(nbuckets, J.R, true);
    YQ_TRY(kernel_allow_smem((const void*)k_join_hash, smem));
    ProfScope ps("join_hash_probe", s, (double)J.L * left->columns[conds[J.eq].left_col].width);
    k_join_hash<<<ntiles, kJoinBlock, smem, s>>>(J);
    YQ_CHECK_LAUNCH();
  } else {
    ProfScope ps("join_nested_loop", s, (double)J.L * J.R * 0.0);
    const JCond& c0 = J.cond[0];
    if (typed) {
      if (count_first) {
        switch (c0.l.type) {
          case YQ_INT32: YQ_TRY(count_matches_typed<int32_t>(J, cw, s)); break;
          case YQ_FLOAT32: YQ_TRY(count_matches_typed<float>(J, cw, s)); break;
          case YQ_FLOAT64: YQ_TRY(count_matches_typed<double>(J, cw, s)); break;
          default: YQ_TRY(count_matches_typed<long long>(J, cw, s)); break;  // INT64, DATETIME
        }
        J.counts = cw.counts;
      }
      switch (c0.l.type) {
        case YQ_INT32: launch_nested_typed<int32_t>(c0.cmp, ntiles, J, s); break;
        case YQ_FLOAT32: launch_nested_typed<float>(c0.cmp, ntiles, J, s); break;
        case YQ_FLOAT64: launch_nested_typed<double>(c0.cmp, ntiles, J, s); break;
        default: launch_nested_typed<long long>(c0.cmp, ntiles, J, s); break;  // INT64, DATETIME
      }
    } else {
      k_join_nested<<<ntiles, kJoinBlock, 0, s>>>(J);
    }
    YQ_CHECK_LAUNCH();
  }
  unsigned long long h_total = 0;
  uint32_t h_err = 0;
  YQ_TRY(d2h_sync(&h_total, J.total, sizeof(h_total), s));
  YQ_TRY(d2h_sync(&h_err, J.err, sizeof(h_err), s));
  if (count_host) *count_host = h_total;
  if (h_err & kErrTimeout) return YQ_ERR_TIMEOUT;
  return h_total > capacity ? YQ_ERR_CAPACITY : YQ_OK;
}

}  // namespace yq

using namespace yq;

extern "C" {

size_t yq_join_workspace_size(uint32_t left_rows, uint32_t right_rows) {
  const uint32_t nb = pow2_at_least(right_rows);
  const uint32_t ntiles = ceil_div<uint32_t>(left_rows, kNlTile);
  WsSize w;
  w.add<uint32_t>(nb + 1);
  w.add<unsigned long long>(right_rows ? right_rows : 1);
  w.add<uint32_t>(right_rows ? right_rows : 1);
  w.add<unsigned long long>((size_t)ntiles + 1);
  w.add<uint32_t>(8);
  w.add<unsigned long long>(2);
  if (right_rows >= kCountFirstRows) count_ws_layout(left_rows, right_rows, count_sort_bytes(right_rows), w);
  return w.total();
}

int yq_join_pairs(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds, int32_t ncond,
                  uint32_t* out_left, uint32_t* out_right, uint64_t capacity, uint64_t* count_host, void* workspace,
                  size_t workspace_bytes, void* stream) {
  return join_impl(left, right, conds, nullptr, ncond, nullptr, 0, nullptr, out_left, out_right, capacity,
                   count_host, workspace, workspace_bytes, as_stream(stream));
}

int yq_join_project(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds, int32_t ncond,
                    const yq_join_output* outputs, int32_t nout, yq_column* out, uint64_t capacity,
                    uint64_t* count_host, void* workspace, size_t workspace_bytes, void* stream) {
  if (nout <= 0) return YQ_ERR_INVALID_ARG;
  return join_impl(left, right, conds, nullptr, ncond, outputs, nout, out, nullptr, nullptr, capacity, count_host,
                   workspace, workspace_bytes, as_stream(stream));
}

int yq_join_pairs_or(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds, const int32_t* disjunct,
                     int32_t ncond, uint32_t* out_left, uint32_t* out_right, uint64_t capacity, uint64_t* count_host,
                     void* workspace, size_t workspace_bytes, void* stream) {
  if (ncond <= 0 || !disjunct) return YQ_ERR_INVALID_ARG;
  return join_impl(left, right, conds, disjunct, ncond, nullptr, 0, nullptr, out_left, out_right, capacity,
                   count_host, workspace, workspace_bytes, as_stream(stream));
}

int yq_join_project_or(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds,
                       const int32_t* disjunct, int32_t ncond, const yq_join_output* outputs, int32_t nout,
                       yq_column* out, uint64_t capacity, uint64_t* count_host, void* workspace,
                       size_t workspace_bytes, void* stream) {
  if (nout <= 0 || ncond <= 0 || !disjunct) return YQ_ERR_INVALID_ARG;
  return join_impl(left, right, conds, disjunct, ncond, outputs, nout, out, nullptr, nullptr, capacity, count_host,
                   workspace, workspace_bytes, as_stream(stream));
}

size_t yq_join_aggregate_workspace_size(uint32_t fact_rows, uint32_t dim_rows, int32_t nagg) {
  (void)fact_rows;
  (void)nagg;
  const uint32_t nb = pow2_at_least(dim_rows);
  WsSize w;
  w.add<uint32_t>(nb + 1);
  w.add<unsigned long long>(dim_rows ? dim_rows : 1);
  w.add<uint32_t>(dim_rows ? dim_rows : 1);
  w.add<uint32_t>(8);
  w.add<Acc>((size_t)sm_count() * 8 * YQ_MAX_AGGREGATES);
  return w.total();
}

}  // extern "C"

// The fact side of a star-join aggregate: predicate and aggregate inputs as
// one program over the fact columns.
static int join_agg_params(const yq_batch* fact, const yq_program* fact_predicate, int32_t fact_key,
                           const yq_constants* constants, const yq_agg_spec* aggs, int32_t nagg, JAParams& F) {
  memset(&F, 0, sizeof(F));
  {
    ProgramBuilder B;
    YQ_TRY(B.set_columns(fact->columns, fact->ncols));
    YQ_TRY(B.set_constants(constants));
    if (fact_predicate && fact_predicate->len > 0) {
      int t = -1;
      YQ_TRY(B.append(fact_predicate, t));
      if (t != YQ_BOOL) return YQ_ERR_INVALID_ARG;
      YQ_TRY(B.emit(OP_EMIT_PRED, 0, 0, YQ_BOOL));
    }
    const int pred_end = B.len;
    for (int a = 0; a < nagg; ++a) {
      const yq_agg_spec& g = aggs[a];
      if (g.kind < YQ_AGG_COUNT_STAR || g.kind > YQ_AGG_MAX) return YQ_ERR_INVALID_ARG;
      const bool flt = (g.input_type == YQ_FLOAT32 || g.input_type == YQ_FLOAT64);
      uint8_t upd;
      switch (g.kind) {
        case YQ_AGG_COUNT_STAR: upd = UPD_COUNT_STAR; break;
        case YQ_AGG_COUNT: upd = UPD_COUNT; break;
        case YQ_AGG_SUM:
        case YQ_AGG_AVG: upd = flt ? UPD_SUM_F : UPD_SUM_I; break;
        case YQ_AGG_MIN: upd = flt ? UPD_MIN_F : UPD_MIN_I; break;
        default: upd = flt ? UPD_MAX_F : UPD_MAX_I; break;
      }
      F.A.upd[a] = upd;
      if (g.kind == YQ_AGG_COUNT_STAR) continue;
      int t = -1;
      YQ_TRY(B.append(&g.input, t));
      if (g.kind != YQ_AGG_COUNT && t != g.input_type) return YQ_ERR_INVALID_ARG;
      YQ_TRY(B.emit(OP_EMIT_AGG, (uint8_t)a, upd, (uint8_t)t));
    }
    YQ_TRY(B.finalize());
    F.fkey_col = fact_key;
    if (!plan_stages(B.P, B.used_cols | (1u << fact_key), F.SP)) F.SP.nstages = 0;
    memcpy(&F.P, &B.P, sizeof(VmProgram));
    F.pred_end = B.remap[pred_end];
    F.pc_end = B.len;
    F.A.nagg = nagg;
  }
  return YQ_OK;
}

// Probe launch over a built dimension table (nbuckets buckets, `kept` rows).
static int join_agg_launch(JAParams& F, const yq_batch* fact, int32_t fact_key, uint32_t nbuckets, uint32_t kept,
                           uint32_t* d_bstart, unsigned long long* d_hkeys, Acc* partials, uint32_t* d_misc,
                           void* state, cudaStream_t s) {
  const yq_column& fk = fact->columns[fact_key];
  const int grid_cap = sm_count() * 8;
  const uint32_t counts[1] = {kept};
  F.fkey = jcol(fk);
  F.nbuckets = nbuckets;
  F.hrows_n = counts[0];
  F.bstart = d_bstart;
  F.hkeys = d_hkeys;
  const size_t table = table_smem(nbuckets, counts[0], false);
  // The ring leaves room for the table; with too few stages left the kernel
  // reads the fact columns from global memory.
  const size_t budget = kStageBudget + 8 * 1024;
  if (F.SP.nstages && stage_smem_bytes(F.SP) + table > budget) {
    const int fit = (int)((budget > table ? budget - table : 0) / (F.SP.stage_bytes + 8));
    F.SP.nstages = fit >= 2 ? (fit > kStageMax ? kStageMax : fit) : 0;
  }
  const bool staged = F.SP.nstages > 0;
  F.table_off = (uint32_t)align_up(stage_smem_bytes(F.SP), 16);
  const size_t smem = F.table_off + table;
  const void* kern = staged ? (const void*)k_join_aggregate<true> : (const void*)k_join_aggregate<false>;
  YQ_TRY(kernel_allow_smem(kern, smem));
  int per_sm = kernel_blocks_per_sm(kern, kRowBlock, smem);
  if (per_sm > 8) per_sm = 8;
  const uint32_t tiles = ceil_div<uint32_t>(fact->rows, kStepRows);
  int grid = sm_count() * per_sm;
  if ((uint32_t)grid > tiles) grid = (int)tiles;
  const double row_bytes = row_bytes_of(F.P, program_columns(F.P, F.pc_end, 1u << fact_key));
  const void* jk = jit_kernel(JIT_JOIN_AGG, staged, F.P, F.pred_end, F.pc_end);
  ProfScope ps("join_aggregate", s, (double)fact->rows * row_bytes);
  if (jk) {
    size_t jsmem = smem;
    if (staged) {  // ring depth for the specialised kernel's occupancy, table after it
      F.SP.nstages = jit_stages(jk, F.SP.stage_bytes, F.SP.nstages, table);
      F.table_off = (uint32_t)align_up(stage_smem_bytes(F.SP), 16);
      jsmem = F.table_off + table;
    }
    uint32_t n = fact->rows;
    Acc* st = static_cast<Acc*>(state);
    void* args[] = {&F, &n, &partials, &d_misc, &st};
    return jit_launch(jk, grid_cap, tiles, jsmem, args, s);
  }
  if (staged)
    k_join_aggregate<true><<<grid, kRowBlock, smem, s>>>(F, fact->rows, partials, d_misc, static_cast<Acc*>(state));
  else
    k_join_aggregate<false><<<grid, kRowBlock, smem, s>>>(F, fact->rows, partials, d_misc, static_cast<Acc*>(state));
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}


extern "C" {

int yq_join_aggregate(const yq_batch* fact, const yq_program* fact_predicate, int32_t fact_key, const yq_batch* dim,
                      const yq_program* dim_predicate, int32_t dim_key, const yq_constants* constants,
                      const yq_agg_spec* aggs, int32_t nagg, void* state, void* workspace, size_t workspace_bytes,
                      void* stream) {
  if (!fact || !dim || !state || fact_key < 0 || fact_key >= fact->ncols || dim_key < 0 || dim_key >= dim->ncols ||
      nagg < 0 || nagg > YQ_MAX_AGGREGATES || (nagg > 0 && !aggs))
    return YQ_ERR_INVALID_ARG;
  const yq_column& fk = fact->columns[fact_key];
  const yq_column& dk = dim->columns[dim_key];
  if (!join_col_ok(fk) || !join_col_ok(dk) || fk.type != dk.type || !hashable(fk.type)) return YQ_ERR_INVALID_ARG;
  if (dim->rows > kHashMaxRows) return YQ_ERR_UNSUPPORTED;
  cudaStream_t s = as_stream(stream);
  JAParams F;
  YQ_TRY(join_agg_params(fact, fact_predicate, fact_key, constants, aggs, nagg, F));
  if (fact->rows == 0 || nagg == 0) return YQ_OK;
  const uint32_t nbuckets = pow2_at_least(dim->rows ? dim->rows : 1);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_join_aggregate_workspace_size(fact->rows, dim->rows, nagg), s));
  uint32_t* d_bstart = ws.take<uint32_t>(nbuckets + 1);
  unsigned long long* d_hkeys = ws.take<unsigned long long>(dim->rows ? dim->rows : 1);
  uint32_t* d_hrows = ws.take<uint32_t>(dim->rows ? dim->rows : 1);
  uint32_t* d_misc = ws.take<uint32_t>(8);  // [0] ticket [2] kept rows [3] duplicate keys
  const int grid_cap = sm_count() * 8;
  Acc* partials = ws.take<Acc>((size_t)grid_cap * YQ_MAX_AGGREGATES);
  YQ_TRY_CUDA(cudaMemsetAsync(d_misc, 0, 8 * sizeof(uint32_t), s));
  YQ_TRY(build_table(dim, dim_predicate, constants, dim_key, nbuckets, d_bstart, d_hkeys, d_hrows, d_misc + 2, s));
  uint32_t counts[2] = {0, 0};
  YQ_TRY(d2h_sync(counts, d_misc + 2, sizeof(counts), s));
  if (counts[1] != 0) return YQ_ERR_UNSUPPORTED;  // dimension keys repeat: use yq_join_pairs + an aggregate
  return join_agg_launch(F, fact, fact_key, nbuckets, counts[0], d_bstart, d_hkeys, partials, d_misc, state, s);
}

// ------------------------------------------------ prepared dimension table
// Table layout: [8 counters][bucket starts nb+1][keys dim_rows][rows dim_rows].
static size_t dim_table_layout(uint32_t dim_rows, WsSize& w) {
  const uint32_t nb = pow2_at_least(dim_rows ? dim_rows : 1);
  w.add<uint32_t>(8);
  w.add<uint32_t>(nb + 1);
  w.add<unsigned long long>(dim_rows ? dim_rows : 1);
  w.add<uint32_t>(dim_rows ? dim_rows : 1);
  return w.total();
}

size_t yq_join_dim_table_size(uint32_t dim_rows) {
  WsSize w;
  return dim_table_layout(dim_rows, w);
}

int yq_join_dim_table_build(const yq_batch* dim, const yq_program* dim_predicate, int32_t dim_key,
                            const yq_constants* constants, void* table, size_t table_bytes, uint32_t* kept,
                            void* stream) {
  if (!dim || !table || !kept || dim_key < 0 || dim_key >= dim->ncols) return YQ_ERR_INVALID_ARG;
  const yq_column& dk = dim->columns[dim_key];
  if (!join_col_ok(dk) || !hashable(dk.type)) return YQ_ERR_INVALID_ARG;
  if (dim->rows > kHashMaxRows) return YQ_ERR_UNSUPPORTED;
  if (table_bytes < yq_join_dim_table_size(dim->rows)) return YQ_ERR_CAPACITY;
  cudaStream_t s = as_stream(stream);
  const uint32_t nbuckets = pow2_at_least(dim->rows ? dim->rows : 1);
  Workspace ws;
  YQ_TRY(ws.acquire(table, table_bytes, yq_join_dim_table_size(dim->rows), s));
  uint32_t* d_misc = ws.take<uint32_t>(8);
  uint32_t* d_bstart = ws.take<uint32_t>(nbuckets + 1);
  unsigned long long* d_hkeys = ws.take<unsigned long long>(dim->rows ? dim->rows : 1);
  uint32_t* d_hrows = ws.take<uint32_t>(dim->rows ? dim->rows : 1);
  YQ_TRY_CUDA(cudaMemsetAsync(d_misc, 0, 8 * sizeof(uint32_t), s));
  YQ_TRY(build_table(dim, dim_predicate, constants, dim_key, nbuckets, d_bstart, d_hkeys, d_hrows, d_misc + 2, s));
  uint32_t counts[2] = {0, 0};
  YQ_TRY(d2h_sync(counts, d_misc + 2, sizeof(counts), s));
  if (counts[1] != 0) return YQ_ERR_UNSUPPORTED;
  *kept = counts[0];
  return YQ_OK;
}

size_t yq_join_aggregate_prepared_workspace_size(int32_t nagg) {
  (void)nagg;
  WsSize w;
  w.add<uint32_t>(8);
  w.add<Acc>((size_t)sm_count() * 8 * YQ_MAX_AGGREGATES);
  return w.total();
}

int yq_join_aggregate_prepared(const yq_batch* fact, const yq_program* fact_predicate, int32_t fact_key,
                               const void* table, uint32_t dim_rows, uint32_t kept, int32_t key_type,
                               const yq_constants* constants, const yq_agg_spec* aggs, int32_t nagg, void* state,
                               void* workspace, size_t workspace_bytes, void* stream) {
  if (!fact || !table || !state || fact_key < 0 || fact_key >= fact->ncols || nagg < 0 ||
      nagg > YQ_MAX_AGGREGATES || (nagg > 0 && !aggs) || kept > dim_rows || dim_rows > kHashMaxRows)
    return YQ_ERR_INVALID_ARG;
  const yq_column& fk = fact->columns[fact_key];
  if (!join_col_ok(fk) || fk.type != key_type || !hashable(fk.type)) return YQ_ERR_INVALID_ARG;
  cudaStream_t s = as_stream(stream);
  JAParams F;
  YQ_TRY(join_agg_params(fact, fact_predicate, fact_key, constants, aggs, nagg, F));
  if (fact->rows == 0 || nagg == 0) return YQ_OK;
  const uint32_t nbuckets = pow2_at_least(dim_rows ? dim_rows : 1);
  const size_t tbytes = yq_join_dim_table_size(dim_rows);
  Workspace tw;  // the caller's table, carved as yq_join_dim_table_build laid it out
  YQ_TRY(tw.acquire(const_cast<void*>(table), tbytes, tbytes, s));
  tw.take<uint32_t>(8);
  uint32_t* d_bstart = tw.take<uint32_t>(nbuckets + 1);
  unsigned long long* d_hkeys = tw.take<unsigned long long>(dim_rows ? dim_rows : 1);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_join_aggregate_prepared_workspace_size(nagg), s));
  uint32_t* d_misc = ws.take<uint32_t>(8);
  Acc* partials = ws.take<Acc>((size_t)sm_count() * 8 * YQ_MAX_AGGREGATES);
  YQ_TRY_CUDA(cudaMemsetAsync(d_misc, 0, 8 * sizeof(uint32_t), s));
  return join_agg_launch(F, fact, fact_key, nbuckets, kept, d_bstart, d_hkeys, partials, d_misc, state, s);
}

}  // extern "C"
