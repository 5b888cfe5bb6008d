// GROUP BY with aggregates: one row per distinct key.
//
// The reference plans GROUP BY but ignores the groups: AggregateOperator
// folds every row into one accumulator (include/engine/operators/
// aggregate_operator.hpp:84-104). This follows SQL (DuckDB) semantics instead:
// NULL keys form one group; aggregates skip NULL inputs; SUM/AVG/MIN/MAX over
// no non-NULL input is NULL; COUNT(*) counts rows, COUNT(col) non-NULL values;
// float sums accumulate in FP64.
//
// Sort-based, all on the device:
//   yq_sort_indices   stable LSD radix argsort of the key (NULLs last)
//   k_group_heads     head flag at every sorted position whose key differs
//                     from the one before it (-0.0 equals +0.0, NaNs equal)
//   yq_prefix_sum_mask  -> group index of every sorted position, group count
//   k_group_keys      each group's key into the output
//   k_group_tiles     tiles of 2,048 sorted positions (8 a thread), values
//                     read through the permutation: each thread folds its
//                     positions in order, a segmented scan over the block's
//                     threads (fixed tree) completes every group that starts
//                     and ends in the tile and writes its output row; a group
//                     crossing the tile's edges leaves a partial record
//   k_group_span      each group that crosses tiles, from the tile where it
//                     starts: its tiles' partial records folded in tile order
//                     (fixed tree), output row written
// No atomics: every floating-point sum is added in an order fixed by the
// data's sorted layout, so a query gives the same bits on every run.
#include <climits>

#include "yq_common.cuh"
#include "yq_sort.cuh"

using namespace yq;

namespace {

constexpr int kGroupThreads = 256;

// Key equality of two rows (canonical floats, NULL == NULL).
__device__ __forceinline__ bool same_key(const yq_column& k, uint32_t a, uint32_t b) {
  if (k.nulls) {
    const bool na = k.nulls[a] != 0, nb = k.nulls[b] != 0;
    if (na || nb) return na == nb;
  }
  switch (k.type) {
    case YQ_INT32: return static_cast<const int32_t*>(k.data)[a] == static_cast<const int32_t*>(k.data)[b];
    case YQ_FLOAT32: {
      const float x = static_cast<const float*>(k.data)[a], y = static_cast<const float*>(k.data)[b];
      return x == y || (x != x && y != y);
    }
    case YQ_FLOAT64: {
      const double x = static_cast<const double*>(k.data)[a], y = static_cast<const double*>(k.data)[b];
      return x == y || (x != x && y != y);
    }
    case YQ_TEXT: {
      const uint32_t* p = reinterpret_cast<const uint32_t*>(static_cast<const char*>(k.data) + (size_t)a * k.width);
      const uint32_t* q = reinterpret_cast<const uint32_t*>(static_cast<const char*>(k.data) + (size_t)b * k.width);
      for (int i = 0; i < k.width / 4; ++i)
        if (p[i] != q[i]) return false;
      return true;
    }
    default: return static_cast<const long long*>(k.data)[a] == static_cast<const long long*>(k.data)[b];
  }
}

__global__ void k_group_heads(const yq_column key, const uint32_t* __restrict__ perm, uint32_t rows,
                              uint8_t* __restrict__ head) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x)
    head[i] = (i == 0 || !same_key(key, perm[i], perm[i - 1])) ? 1 : 0;
}

// First input row of every tile of sorted positions (the tiles run in the
// order of these rows: see yq_group_by).
__global__ void k_tile_first_row(const uint32_t* __restrict__ perm, uint32_t ntiles, uint32_t tile_rows,
                                 uint32_t* __restrict__ first) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x)
    first[t] = __ldg(perm + (size_t)t * tile_rows);
}

// Head flags from the sorted key words (kw words a row, in sorted order): a
// sequential read instead of two reads through the permutation. Key words
// already equate -0.0 with +0.0 and every NaN, and carry the NULL flag.
__global__ void k_group_heads_words(const uint32_t* __restrict__ words, int kw, uint32_t rows,
                                    uint8_t* __restrict__ head) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    bool h = i == 0;
    for (int j = 0; j < kw && !h; ++j) h = __ldg(words + (size_t)i * kw + j) != __ldg(words + (size_t)(i - 1) * kw + j);
    head[i] = h ? 1 : 0;
  }
}

__global__ void k_group_keys(const yq_column key, const uint32_t* __restrict__ perm, uint32_t rows,
                             const uint8_t* __restrict__ head, const uint32_t* __restrict__ incl, yq_column out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    if (!head[i]) continue;
    const uint32_t g = incl[i] - 1, r = perm[i];
    const char* src = static_cast<const char*>(key.data) + (size_t)r * key.width;
    char* dst = static_cast<char*>(out.data) + (size_t)g * key.width;
    for (int b = 0; b < key.width; b += 4) *reinterpret_cast<uint32_t*>(dst + b) = *reinterpret_cast<const uint32_t*>(src + b);
    if (out.nulls) const_cast<uint8_t*>(out.nulls)[g] = key.nulls ? key.nulls[r] : 0;
  }
}

struct GAgg {
  const void* data;      // input column (COUNT_STAR: none)
  const uint8_t* nulls;
  int32_t type;          // input type
  int32_t kind;          // yq_agg_kind
};

struct GroupParams {
  GAgg a[YQ_MAX_AGGREGATES];
  int32_t nagg;
  uint32_t rows;
  const uint32_t* perm;
  const uint32_t* incl;  // inclusive scan of the head flags: group = incl - 1
  uint32_t* starts;      // [groups + 1] first sorted position of every group; starts[groups] = rows
  yq_column out[YQ_MAX_AGGREGATES];  // aggregate output columns
  unsigned long long* rec;  // [tiles][2][nagg][2]: head / tail partial (count, value) of every tile
  const uint32_t* tile_order;  // [tiles] the tile block b works on (null: tile b)
  uint32_t* tail_group;     // [tiles] group of the tile's tail record
  uint32_t* tile_flags;     // [tiles] kHeadRec | kTailRec | kTailStarted (set with atomicOr)
  uint32_t* err;
};

constexpr uint32_t kGroupItems = 8;
constexpr uint32_t kGroupTile = kGroupThreads * kGroupItems;  // 2,048 sorted positions
constexpr uint32_t kHeadRec = 1, kTailRec = 2, kTailStarted = 4;

// Order-preserving signed 64-bit key of a double (NaN above +inf, one NaN).
__device__ __forceinline__ long long ordered(double d) {
  unsigned long long u = d != d ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(d);
  u = (u >> 63) ? ~u : (u | (1ull << 63));
  return (long long)(u ^ (1ull << 63));
}
__device__ __forceinline__ double unordered(long long k) {
  unsigned long long u = (unsigned long long)k ^ (1ull << 63);
  u = (u >> 63) ? (u & ~(1ull << 63)) : ~u;
  return __longlong_as_double((long long)u);
}

__device__ __forceinline__ bool is_float(int32_t t) { return t == YQ_FLOAT32 || t == YQ_FLOAT64; }

// Input value r of an aggregate as int64 or double.
__device__ __forceinline__ long long in_int(const GAgg& a, uint32_t r) {
  return a.type == YQ_INT32 ? (long long)static_cast<const int32_t*>(a.data)[r]
                            : static_cast<const long long*>(a.data)[r];
}
__device__ __forceinline__ double in_dbl(const GAgg& a, uint32_t r) {
  return a.type == YQ_FLOAT32 ? (double)static_cast<const float*>(a.data)[r] : static_cast<const double*>(a.data)[r];
}

// One aggregate's partial state: a count and a 64-bit value (int64 sum,
// double sum bits, or the ordered key of MIN / MAX).
struct GPart {
  unsigned long long cnt;
  unsigned long long v;
};

__device__ __forceinline__ GPart part_identity(int kind) {
  return GPart{0ull, kind == YQ_AGG_MIN ? (unsigned long long)LLONG_MAX
                     : kind == YQ_AGG_MAX ? (unsigned long long)LLONG_MIN : 0ull};
}

__device__ __forceinline__ GPart part_combine(int kind, bool flt, GPart a, GPart b) {
  GPart c;
  c.cnt = a.cnt + b.cnt;
  switch (kind) {
    case YQ_AGG_SUM:
    case YQ_AGG_AVG:
      c.v = flt ? (unsigned long long)__double_as_longlong(__longlong_as_double((long long)a.v) +
                                                           __longlong_as_double((long long)b.v))
                : a.v + b.v;
      break;
    case YQ_AGG_MIN: c.v = (long long)a.v < (long long)b.v ? a.v : b.v; break;
    case YQ_AGG_MAX: c.v = (long long)a.v > (long long)b.v ? a.v : b.v; break;
    default: c.v = 0ull; break;
  }
  return c;
}

__device__ __forceinline__ void part_add_row(const GAgg& a, bool flt, GPart& p, uint32_t r) {
  if (a.kind == YQ_AGG_COUNT_STAR) {
    ++p.cnt;
    return;
  }
  if (a.nulls && a.nulls[r]) return;
  ++p.cnt;
  if (a.kind == YQ_AGG_SUM || a.kind == YQ_AGG_AVG) {
    if (flt) p.v = (unsigned long long)__double_as_longlong(__longlong_as_double((long long)p.v) + in_dbl(a, r));
    else p.v += (unsigned long long)in_int(a, r);
  } else if (a.kind == YQ_AGG_MIN || a.kind == YQ_AGG_MAX) {
    const long long k = flt ? ordered(in_dbl(a, r)) : in_int(a, r);
    if (a.kind == YQ_AGG_MIN ? k < (long long)p.v : k > (long long)p.v) p.v = (unsigned long long)k;
  }
}

// Output row g of aggregate a from its complete state.
__device__ __forceinline__ void part_write(const GAgg& a, const yq_column& o, uint32_t g, GPart p) {
  const bool flt = is_float(a.type);
  const bool null = p.cnt == 0 && a.kind != YQ_AGG_COUNT && a.kind != YQ_AGG_COUNT_STAR;
  if (o.nulls) const_cast<uint8_t*>(o.nulls)[g] = null ? 1 : 0;
  switch (a.kind) {
    case YQ_AGG_COUNT:
    case YQ_AGG_COUNT_STAR: static_cast<long long*>(o.data)[g] = (long long)p.cnt; break;
    case YQ_AGG_SUM:
      if (flt) static_cast<double*>(o.data)[g] = null ? 0.0 : __longlong_as_double((long long)p.v);
      else static_cast<long long*>(o.data)[g] = null ? 0 : (long long)p.v;
      break;
    case YQ_AGG_AVG: {
      const double sum = flt ? __longlong_as_double((long long)p.v) : (double)(long long)p.v;
      static_cast<double*>(o.data)[g] = null ? 0.0 : sum / (double)p.cnt;
      break;
    }
    default: {  // MIN / MAX in the input type
      const long long k = (long long)p.v;
      if (a.type == YQ_INT32) static_cast<int32_t*>(o.data)[g] = null ? 0 : (int32_t)k;
      else if (a.type == YQ_FLOAT32) static_cast<float*>(o.data)[g] = null ? 0.0f : (float)unordered(k);
      else if (a.type == YQ_FLOAT64) static_cast<double*>(o.data)[g] = null ? 0.0 : unordered(k);
      else static_cast<long long*>(o.data)[g] = null ? 0 : k;
      break;
    }
  }
}

__device__ __forceinline__ GPart shfl_up_part(GPart p, int d) {
  return GPart{__shfl_up_sync(0xffffffffu, p.cnt, d), __shfl_up_sync(0xffffffffu, p.v, d)};
}

// Inclusive segmented scan over the block's threads in thread order (a
// thread's flag restarts the running state); fixed combine tree. Returns the
// inclusive state and flag; excl / excl_flag = the same up to the thread before.
__device__ __forceinline__ void block_seg_scan(int kind, bool flt, bool flag, GPart x, GPart& incl, bool& incl_flag,
                                               GPart& excl, bool& excl_flag, GPart* s_part, uint32_t* s_flag) {
  constexpr int NW = kGroupThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  GPart v = x;
  bool f = flag;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const GPart u = shfl_up_part(v, d);
    const bool uf = __shfl_up_sync(0xffffffffu, f, d);
    if (lane >= d) {
      if (!f) v = part_combine(kind, flt, u, v);
      f = f || uf;
    }
  }
  if (lane == 31) {
    s_part[warp] = v;
    s_flag[warp] = f;
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // warp prefixes in warp order (exclusive), one thread: fixed order
    GPart run = part_identity(kind);
    bool rf = false;
    for (int w = 0; w < NW; ++w) {
      const GPart wv = s_part[w];
      const bool wf = s_flag[w] != 0u;
      s_part[NW + w] = run;
      s_flag[NW + w] = rf;
      run = wf ? wv : part_combine(kind, flt, run, wv);
      rf = rf || wf;
    }
  }
  __syncthreads();
  const GPart wp = s_part[NW + warp];
  const bool wpf = s_flag[NW + warp] != 0u;
  // lane-level exclusive value within the warp
  GPart le = shfl_up_part(v, 1);
  bool lef = __shfl_up_sync(0xffffffffu, f, 1);
  if (lane == 0) {
    le = part_identity(kind);
    lef = false;
  }
  incl = f ? v : part_combine(kind, flt, wp, v);
  incl_flag = f || wpf;
  excl = lef ? le : (lane == 0 ? wp : part_combine(kind, flt, wp, le));
  excl_flag = lef || wpf;
  __syncthreads();
}

__global__ void __launch_bounds__(kGroupThreads) k_group_tiles(const __grid_constant__ GroupParams P) {
  __shared__ GPart s_part[2 * (kGroupThreads / 32)];
  __shared__ uint32_t s_flag[2 * (kGroupThreads / 32)];
  const uint32_t tile = P.tile_order ? __ldg(P.tile_order + blockIdx.x) : blockIdx.x;
  const uint32_t tile0 = tile * kGroupTile;
  const uint32_t tile_end = min(P.rows, tile0 + kGroupTile);
  const uint32_t p0 = tile0 + threadIdx.x * kGroupItems;
  const uint32_t n = p0 < tile_end ? min(kGroupItems, tile_end - p0) : 0u;  // valid positions of this thread
  // A tile inside one group (with few groups, nearly every tile): every
  // aggregate folds over the whole tile by a fixed-order block reduction,
  // with one barrier instead of a segmented scan per aggregate.
  if (tile0 < tile_end && __ldg(P.incl + tile0) == __ldg(P.incl + tile_end - 1)) {
    __shared__ GPart s_u[YQ_MAX_AGGREGATES][kGroupThreads / 32];
    const uint32_t G = __ldg(P.incl + tile0) - 1u;
    const bool starts = tile0 == 0 || __ldg(P.incl + tile0 - 1) - 1u != G;
    const bool ends = tile_end == P.rows || __ldg(P.incl + tile_end) - 1u != G;
    if (threadIdx.x == 0 && starts) P.starts[G] = tile0;
    uint32_t rr[kGroupItems];
#pragma unroll
    for (int q = 0; q < (int)kGroupItems; ++q) rr[q] = (uint32_t)q < n ? __ldg(P.perm + p0 + q) : 0u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = 0; j < P.nagg; ++j) {
      const GAgg& a = P.a[j];
      const bool flt = is_float(a.type);
      GPart acc = part_identity(a.kind);
#pragma unroll
      for (int q = 0; q < (int)kGroupItems; ++q)
        if ((uint32_t)q < n) part_add_row(a, flt, acc, rr[q]);
      // fixed tree: lanes pairwise in index order
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const GPart o{__shfl_down_sync(0xffffffffu, acc.cnt, d), __shfl_down_sync(0xffffffffu, acc.v, d)};
        if ((lane & (2 * d - 1)) == 0) acc = part_combine(a.kind, flt, acc, o);
      }
      if (lane == 0) s_u[j][warp] = acc;
    }
    __syncthreads();
    if ((int)threadIdx.x < P.nagg) {  // thread j: aggregate j, warps in order
      const int j = threadIdx.x;
      const GAgg& a = P.a[j];
      const bool flt = is_float(a.type);
      GPart tot = s_u[j][0];
      for (int w = 1; w < kGroupThreads / 32; ++w) tot = part_combine(a.kind, flt, tot, s_u[j][w]);
      unsigned long long* head_rec = P.rec + ((size_t)tile * 2 * P.nagg + j) * 2;
      unsigned long long* tail_rec = P.rec + ((size_t)tile * 2 * P.nagg + P.nagg + j) * 2;
      if (starts && ends) {
        part_write(a, P.out[j], G, tot);
      } else if (ends) {  // the group began before this tile and ends at its last position
        head_rec[0] = tot.cnt;
        head_rec[1] = tot.v;
      } else {  // the group goes on past this tile
        tail_rec[0] = tot.cnt;
        tail_rec[1] = tot.v;
      }
    }
    if (threadIdx.x == 0 && P.nagg > 0 && !(starts && ends)) {
      if (ends) {
        atomicOr(P.tile_flags + tile, kHeadRec);
      } else {
        P.tail_group[tile] = G;
        atomicOr(P.tile_flags + tile, kTailRec | (starts ? kTailStarted : 0u));
      }
    }
    return;
  }
  uint32_t g[kGroupItems], r[kGroupItems];
#pragma unroll
  for (int q = 0; q < (int)kGroupItems; ++q) {
    g[q] = (uint32_t)q < n ? __ldg(P.incl + p0 + q) - 1u : 0u;
    r[q] = (uint32_t)q < n ? __ldg(P.perm + p0 + q) : 0u;
  }
  const uint32_t prev_g = p0 > 0 && n ? __ldg(P.incl + p0 - 1) - 1u : 0xffffffffu;
  const uint32_t last = n ? p0 + n - 1 : 0u;
  const uint32_t next_g = n && last + 1 < P.rows ? __ldg(P.incl + last + 1) - 1u : 0xffffffffu;
  // group starts
#pragma unroll
  for (int q = 0; q < (int)kGroupItems; ++q)
    if ((uint32_t)q < n && (q == 0 ? g[0] != prev_g : g[q] != g[q - 1])) P.starts[g[q]] = p0 + q;
  const bool starts_here = n && g[0] != prev_g;
  bool boundary = false;  // a group starts inside (after the first position)
#pragma unroll
  for (int q = 1; q < (int)kGroupItems; ++q) boundary |= (uint32_t)q < n && g[q] != g[q - 1];
  uint32_t g_last = 0u;
#pragma unroll
  for (int q = 0; q < (int)kGroupItems; ++q)
    if ((uint32_t)q + 1 == n) g_last = g[q];
  const bool ends_here = n && next_g != g_last;
  const bool tile_last = n && last + 1 == tile_end;  // the tile's last valid position is this thread's
  for (int j = 0; j < P.nagg; ++j) {
    const GAgg& a = P.a[j];
    const bool flt = is_float(a.type);
    GPart first = part_identity(a.kind), cur = part_identity(a.kind);
    uint32_t cg = g[0];
    int seg = 0;  // segments closed so far in this thread
#pragma unroll
    for (int q = 0; q < (int)kGroupItems; ++q) {
      if ((uint32_t)q >= n) break;
      if (q > 0 && g[q] != cg) {  // the segment of group cg ends before position q
        if (seg == 0) first = cur;                         // the thread's first segment
        else part_write(a, P.out[j], cg, cur);             // an inner segment: complete here
        if (seg == 0 && starts_here) part_write(a, P.out[j], cg, cur);  // first segment began here too
        ++seg;
        cg = g[q];
        cur = part_identity(a.kind);
      }
      part_add_row(a, flt, cur, r[q]);
    }
    // thread element of the scan: the running state of the thread's last segment
    GPart inc, exc;
    bool inc_f, exc_f;
    block_seg_scan(a.kind, flt, n == 0 || starts_here || boundary, cur, inc, inc_f, exc, exc_f, s_part, s_flag);
    if (n == 0) continue;
    unsigned long long* head_rec = P.rec + ((size_t)tile * 2 * P.nagg + j) * 2;
    unsigned long long* tail_rec = P.rec + ((size_t)tile * 2 * P.nagg + P.nagg + j) * 2;
    if (boundary && !starts_here) {
      // the first segment continues a group from earlier threads and ends here
      const GPart tot = part_combine(a.kind, flt, exc, first);
      if (exc_f) {
        part_write(a, P.out[j], g[0], tot);
      } else {  // the group began before this tile: the tile's head record
        head_rec[0] = tot.cnt;
        head_rec[1] = tot.v;
        if (j == 0) atomicOr(P.tile_flags + tile, kHeadRec);
      }
    }
    // the last segment: its state up to here is the inclusive scan value
    if (ends_here) {
      if (inc_f) {
        part_write(a, P.out[j], g_last, inc);
      } else {
        head_rec[0] = inc.cnt;
        head_rec[1] = inc.v;
        if (j == 0) atomicOr(P.tile_flags + tile, kHeadRec);
      }
    } else if (tile_last) {  // the group goes on past this tile
      tail_rec[0] = inc.cnt;
      tail_rec[1] = inc.v;
      if (j == 0) {
        P.tail_group[tile] = g_last;
        atomicOr(P.tile_flags + tile, kTailRec | (inc_f ? kTailStarted : 0u));
      }
    }
  }
}

// One block per tile: the group that starts in this tile and runs past it.
__global__ void __launch_bounds__(kGroupThreads) k_group_span(const __grid_constant__ GroupParams P, uint32_t ntiles) {
  __shared__ GPart s_red[kGroupThreads / 32];
  const uint32_t t = blockIdx.x;
  const uint32_t fl = P.tile_flags[t];
  if (!(fl & kTailRec) || !(fl & kTailStarted)) return;
  const uint32_t g = P.tail_group[t];
  const uint32_t end = P.starts[g + 1];
  if (end == 0 || end > P.rows) {
    if (threadIdx.x == 0) atomicOr(P.err, 2u);
    return;
  }
  const uint32_t tb = (end - 1) / kGroupTile;
  if (tb <= t || tb >= ntiles || !(P.tile_flags[tb] & kHeadRec)) {
    if (threadIdx.x == 0) atomicOr(P.err, 2u);
    return;
  }
  const uint32_t n = tb - t + 1;  // contributions: tail(t), tail(t+1..tb-1), head(tb)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = 0; j < P.nagg; ++j) {
    const GAgg& a = P.a[j];
    const bool flt = is_float(a.type);
    GPart acc = part_identity(a.kind);
    for (uint32_t k = threadIdx.x; k < n; k += kGroupThreads) {
      const uint32_t tt = t + k;
      const unsigned long long* rec =
          P.rec + ((size_t)tt * 2 * P.nagg + (k + 1 == n ? 0 : P.nagg) + j) * 2;  // head of tb, else tail
      acc = part_combine(a.kind, flt, acc, GPart{rec[0], rec[1]});
    }
    // fixed tree: lanes pairwise in index order, then warps in order
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const GPart o{__shfl_down_sync(0xffffffffu, acc.cnt, d), __shfl_down_sync(0xffffffffu, acc.v, d)};
      if ((lane & (2 * d - 1)) == 0) acc = part_combine(a.kind, flt, acc, o);
    }
    if (lane == 0) s_red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      GPart tot = s_red[0];
      for (int w = 1; w < kGroupThreads / 32; ++w) tot = part_combine(a.kind, flt, tot, s_red[w]);
      part_write(a, P.out[j], g, tot);
    }
    __syncthreads();
  }
}

int out_type(int32_t kind, int32_t in) {
  switch (kind) {
    case YQ_AGG_COUNT:
    case YQ_AGG_COUNT_STAR: return YQ_INT64;
    case YQ_AGG_SUM: return (in == YQ_FLOAT32 || in == YQ_FLOAT64) ? YQ_FLOAT64 : YQ_INT64;
    case YQ_AGG_AVG: return YQ_FLOAT64;
    default: return in;
  }
}

int type_width(int32_t t) { return (t == YQ_INT32 || t == YQ_FLOAT32) ? 4 : 8; }

unsigned grid_for(uint64_t n, unsigned per_block) {
  const uint64_t g = (n + per_block - 1) / per_block;
  return (unsigned)(g < 1 ? 1 : (g > 65535 ? 65535 : g));
}

}  // namespace

extern "C" {

// Sort workspace for ordering `ntiles` tiles by their first row (4-byte keys).
// Sizing reads no column data: the placeholder pointer only has to be non-null.
static size_t tile_order_sort_bytes(uint32_t ntiles) {
  const yq_column c{reinterpret_cast<void*>(static_cast<uintptr_t>(256)), nullptr, YQ_INT32, 4};
  return yq_sort_workspace_size(&c, ntiles);
}

size_t yq_group_by_workspace_size(const yq_column* key, uint32_t rows, int32_t nagg, uint32_t capacity) {
  if (!key) return 0;
  const size_t tiles = ((size_t)rows + kGroupTile - 1) / kGroupTile + 1;
  WsSize w;
  w.add<uint8_t>(yq_sort_workspace_size(key, rows));
  w.add<uint32_t>((size_t)rows + 1);          // permutation
  const int kwm = sort_key_words_max(*key);
  w.add<uint32_t>((size_t)rows * (kwm > 0 ? kwm : 1) + 16);  // sorted key words
  w.add<uint8_t>((size_t)rows + 16);          // head flags
  w.add<uint32_t>((size_t)rows + 1);          // group of every sorted position
  w.add<uint8_t>(yq_prefix_sum_workspace_size(rows));
  w.add<uint32_t>((size_t)capacity + 2);      // group starts
  w.add<unsigned long long>(tiles * 4 * (size_t)(nagg > 0 ? nagg : 1));  // tile head / tail records
  w.add<uint32_t>(tiles);                     // tail group of every tile
  w.add<uint32_t>(2 * tiles);                 // first row of every tile, tile order
  w.add<uint8_t>(tile_order_sort_bytes((uint32_t)tiles));
  w.add<uint32_t>(tiles);                     // tile flags
  w.add<uint32_t>(4);                         // error word
  return w.total();
}

int yq_group_by(const yq_batch* batch, int32_t key_col, const yq_group_agg* aggs, int32_t nagg, yq_column* out,
                uint32_t capacity, uint32_t* groups, void* workspace, size_t workspace_bytes, void* stream) {
  if (!batch || !groups || !out || nagg < 0 || nagg > YQ_MAX_AGGREGATES || key_col < 0 ||
      key_col >= batch->ncols || (nagg && !aggs))
    return YQ_ERR_INVALID_ARG;
  *groups = 0;
  const yq_column key = batch->columns[key_col];
  const uint32_t rows = batch->rows;
  if (!(key.type == YQ_INT32 || key.type == YQ_INT64 || key.type == YQ_DATETIME || key.type == YQ_FLOAT32 ||
        key.type == YQ_FLOAT64 || key.type == YQ_TEXT))
    return YQ_ERR_UNSUPPORTED;
  if (out[0].type != key.type || out[0].width != key.width || (rows && !out[0].data)) return YQ_ERR_INVALID_ARG;
  GroupParams P;
  memset(&P, 0, sizeof(P));
  P.nagg = nagg;
  P.rows = rows;
  for (int j = 0; j < nagg; ++j) {
    const yq_group_agg& g = aggs[j];
    const bool star = g.kind == YQ_AGG_COUNT_STAR;
    if (g.kind < YQ_AGG_COUNT_STAR || g.kind > YQ_AGG_MAX) return YQ_ERR_INVALID_ARG;
    if (!star && (g.column < 0 || g.column >= batch->ncols)) return YQ_ERR_INVALID_ARG;
    const yq_column in = star ? yq_column{nullptr, nullptr, YQ_INT64, 8} : batch->columns[g.column];
    const int it = in.type;
    const bool numeric = it == YQ_INT32 || it == YQ_INT64 || it == YQ_FLOAT32 || it == YQ_FLOAT64;
    if (!star && g.kind != YQ_AGG_COUNT && !(numeric || (it == YQ_DATETIME && (g.kind == YQ_AGG_MIN ||
                                                                              g.kind == YQ_AGG_MAX))))
      return YQ_ERR_UNSUPPORTED;
    const int ot = out_type(g.kind, it);
    const yq_column& o = out[1 + j];
    if (o.type != ot || o.width != type_width(ot) || (rows && !o.data)) return YQ_ERR_INVALID_ARG;
    if (!o.nulls && g.kind != YQ_AGG_COUNT && g.kind != YQ_AGG_COUNT_STAR && rows) return YQ_ERR_INVALID_ARG;
    P.a[j] = GAgg{in.data, in.nulls, it, g.kind};
    P.out[j] = o;
  }
  if (rows == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_group_by_workspace_size(&key, rows, nagg, capacity), s));
  const uint32_t ntiles = (uint32_t)(((size_t)rows + kGroupTile - 1) / kGroupTile);
  const size_t sort_ws = yq_sort_workspace_size(&key, rows);
  void* d_sort = ws.take<uint8_t>(sort_ws);
  uint32_t* perm = ws.take<uint32_t>((size_t)rows + 1);
  const int kwm = sort_key_words_max(key);
  uint32_t* words = ws.take<uint32_t>((size_t)rows * (kwm > 0 ? kwm : 1) + 16);
  uint8_t* head = ws.take<uint8_t>((size_t)rows + 16);
  uint32_t* incl = ws.take<uint32_t>((size_t)rows + 1);
  void* scan_ws = ws.take<uint8_t>(yq_prefix_sum_workspace_size(rows));
  uint32_t* starts = ws.take<uint32_t>((size_t)capacity + 2);
  unsigned long long* rec = ws.take<unsigned long long>(((size_t)ntiles + 1) * 4 * (size_t)(nagg > 0 ? nagg : 1));
  uint32_t* tail_group = ws.take<uint32_t>((size_t)ntiles + 1);
  uint32_t* first_row = ws.take<uint32_t>((size_t)ntiles + 1);
  uint32_t* tile_order = ws.take<uint32_t>((size_t)ntiles + 1);
  const size_t order_ws_bytes = tile_order_sort_bytes(ntiles + 1);
  void* order_ws = ws.take<uint8_t>(order_ws_bytes);
  uint32_t* tile_flags = ws.take<uint32_t>((size_t)ntiles + 1);
  uint32_t* d_err = ws.take<uint32_t>(4);
  // The sort skips the passes whose digit every key shares (a key of few
  // distinct values sorts in one or two passes) and hands over its key words
  // in sorted order; a text key too long for one pass's words sorts without
  // them, and its heads compare the rows through the permutation.
  KeyJob job{key, 0, 0};
  const uint32_t offs[2] = {0, rows};
  int kw = 0;
  int st = sort_segments_impl(&job, 1, rows, offs, 1, perm, nullptr, d_sort, sort_ws, s, nullptr, words, &kw);
  const bool have_words = st == YQ_OK;
  if (st == YQ_ERR_UNSUPPORTED)
    st = sort_segments_impl(&job, 1, rows, offs, 1, perm, nullptr, d_sort, sort_ws, s, nullptr);
  YQ_TRY(st);
  if (have_words) {
    ProfScope ps("group_heads", s, (double)rows * 4.0 * (kw > 0 ? kw : 1));
    k_group_heads_words<<<grid_for(rows, kGroupThreads), kGroupThreads, 0, s>>>(words, kw, rows, head);
    YQ_CHECK_LAUNCH();
  } else {
    ProfScope ps("group_heads", s, (double)rows * (key.width + 4));
    k_group_heads<<<grid_for(rows, kGroupThreads), kGroupThreads, 0, s>>>(key, perm, rows, head);
    YQ_CHECK_LAUNCH();
  }
  YQ_TRY(yq_prefix_sum_mask(head, incl, rows, scan_ws, yq_prefix_sum_workspace_size(rows), stream));
  uint32_t G = 0;
  YQ_TRY(d2h_sync(&G, incl + rows - 1, sizeof(G), s));
  *groups = G;
  if (G > capacity) return YQ_ERR_CAPACITY;
  P.perm = perm;
  P.incl = incl;
  P.starts = starts;
  P.rec = rec;
  P.tail_group = tail_group;
  P.tile_flags = tile_flags;
  P.err = d_err;
  k_group_keys<<<grid_for(rows, kGroupThreads), kGroupThreads, 0, s>>>(key, perm, rows, head, incl, out[0]);
  YQ_CHECK_LAUNCH();
  if (nagg) {
    const uint32_t end_word[1] = {rows};
    YQ_TRY(h2d_async(starts + G, end_word, sizeof(uint32_t), s));  // starts[G] = rows
    YQ_TRY_CUDA(cudaMemsetAsync(tile_flags, 0, ((size_t)ntiles + 1) * sizeof(uint32_t), s));
    YQ_TRY_CUDA(cudaMemsetAsync(d_err, 0, 4 * sizeof(uint32_t), s));
    double in_bytes = 8.0 * rows;  // group index + permutation
    for (int j = 0; j < nagg; ++j)
      if (P.a[j].data) in_bytes += (double)rows * (type_width(P.a[j].type) + (P.a[j].nulls ? 1 : 0));
    // Tiles run in the order of their first input row. The rows of one group
    // ascend through its sorted positions, so the tiles resident together
    // (one stretch of every group) read values from one stretch of rows,
    // which L2 then holds for all of them; in position order they would be
    // one group's tiles reading rows spread over the whole table. The
    // results do not depend on the order: each tile writes its own records.
    if (ntiles >= 64) {
      k_tile_first_row<<<grid_for(ntiles, kGroupThreads), kGroupThreads, 0, s>>>(perm, ntiles, kGroupTile, first_row);
      YQ_CHECK_LAUNCH();
      const yq_column fc{first_row, nullptr, YQ_INT32, 4};
      KeyJob oj{fc, 0, 0};
      const uint32_t oo[2] = {0, ntiles};
      YQ_TRY(sort_segments_impl(&oj, 1, ntiles, oo, 1, tile_order, nullptr, order_ws, order_ws_bytes, s, nullptr));
      P.tile_order = tile_order;
    }
    {
      ProfScope ps("group_accumulate", s, in_bytes);
      k_group_tiles<<<ntiles, kGroupThreads, 0, s>>>(P);
      YQ_CHECK_LAUNCH();
      k_group_span<<<ntiles, kGroupThreads, 0, s>>>(P, ntiles);
      YQ_CHECK_LAUNCH();
    }
    uint32_t err = 0;
    YQ_TRY(d2h_sync(&err, d_err, sizeof(err), s));
    if (err) return YQ_ERR_INVALID_ARG;
  }
  return YQ_OK;
}

}  // extern "C"
