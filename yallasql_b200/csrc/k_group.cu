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
//   k_group_accumulate  32 consecutive sorted positions a thread, values read
//                     through the permutation; a run of one group is folded in
//                     registers and flushed with one atomic per aggregate
//   k_group_finalize  accumulators -> output values and NULL bytes
#include <climits>

#include "yq_common.cuh"

using namespace yq;

namespace {

constexpr int kGroupThreads = 256;
constexpr int kGroupRun = 32;  // sorted positions per thread in the accumulate pass

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
  unsigned long long* count;  // per group: rows (COUNT_STAR) or non-NULL inputs
  unsigned long long* value;  // per group: int64 sum, double sum (bits), or ordered MIN/MAX key
};

struct GroupParams {
  GAgg a[YQ_MAX_AGGREGATES];
  int32_t nagg;
  uint32_t rows;
  const uint32_t* perm;
  const uint32_t* incl;  // inclusive scan of the head flags: group = incl - 1
};

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

__device__ __forceinline__ void flush(const GAgg& a, uint32_t g, unsigned long long cnt, long long isum, double dsum,
                                      long long best) {
  if (cnt == 0) return;
  atomicAdd(a.count + g, cnt);
  switch (a.kind) {
    case YQ_AGG_SUM:
    case YQ_AGG_AVG:
      if (is_float(a.type)) atomicAdd(reinterpret_cast<double*>(a.value + g), dsum);
      else atomicAdd(a.value + g, (unsigned long long)isum);
      break;
    case YQ_AGG_MIN: atomicMin(reinterpret_cast<long long*>(a.value + g), best); break;
    case YQ_AGG_MAX: atomicMax(reinterpret_cast<long long*>(a.value + g), best); break;
    default: break;
  }
}

__global__ void __launch_bounds__(kGroupThreads) k_group_accumulate(const __grid_constant__ GroupParams P) {
  const uint64_t t = (uint64_t)blockIdx.x * kGroupThreads + threadIdx.x;
  const uint64_t lo = t * kGroupRun;
  if (lo >= P.rows) return;
  const uint32_t hi = (uint32_t)(lo + kGroupRun < P.rows ? lo + kGroupRun : P.rows);
  for (int j = 0; j < P.nagg; ++j) {  // aggregates one at a time: the warp's lanes run the same one
    const GAgg& a = P.a[j];
    uint32_t g = P.incl[lo] - 1;
    unsigned long long cnt = 0;
    long long isum = 0, best = a.kind == YQ_AGG_MIN ? LLONG_MAX : LLONG_MIN;
    double dsum = 0.0;
    for (uint32_t i = (uint32_t)lo; i < hi; ++i) {
      const uint32_t gi = P.incl[i] - 1;
      if (gi != g) {
        flush(a, g, cnt, isum, dsum, best);
        g = gi;
        cnt = 0;
        isum = 0;
        dsum = 0.0;
        best = a.kind == YQ_AGG_MIN ? LLONG_MAX : LLONG_MIN;
      }
      if (a.kind == YQ_AGG_COUNT_STAR) { ++cnt; continue; }
      const uint32_t r = P.perm[i];
      if (a.nulls && a.nulls[r]) continue;
      ++cnt;
      if (a.kind == YQ_AGG_SUM || a.kind == YQ_AGG_AVG) {
        if (is_float(a.type)) dsum += in_dbl(a, r);
        else isum += in_int(a, r);
      } else if (a.kind == YQ_AGG_MIN || a.kind == YQ_AGG_MAX) {
        const long long k = is_float(a.type) ? ordered(in_dbl(a, r)) : in_int(a, r);
        best = a.kind == YQ_AGG_MIN ? (k < best ? k : best) : (k > best ? k : best);
      }
    }
    flush(a, g, cnt, isum, dsum, best);
  }
}

__global__ void k_group_init(const __grid_constant__ GroupParams P, uint32_t groups) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += gridDim.x * blockDim.x)
    for (int j = 0; j < P.nagg; ++j) {
      P.a[j].count[g] = 0;
      P.a[j].value[g] = P.a[j].kind == YQ_AGG_MIN ? (unsigned long long)LLONG_MAX
                        : P.a[j].kind == YQ_AGG_MAX ? (unsigned long long)LLONG_MIN : 0ull;
    }
}

__global__ void k_group_finalize(const __grid_constant__ GroupParams P, uint32_t groups, const yq_column* out_dev) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += gridDim.x * blockDim.x)
    for (int j = 0; j < P.nagg; ++j) {
      const GAgg& a = P.a[j];
      const yq_column o = out_dev[1 + j];
      const unsigned long long cnt = a.count[g], v = a.value[g];
      const bool null = cnt == 0 && a.kind != YQ_AGG_COUNT && a.kind != YQ_AGG_COUNT_STAR;
      if (o.nulls) const_cast<uint8_t*>(o.nulls)[g] = null ? 1 : 0;
      switch (a.kind) {
        case YQ_AGG_COUNT:
        case YQ_AGG_COUNT_STAR: static_cast<long long*>(o.data)[g] = (long long)cnt; break;
        case YQ_AGG_SUM:
          if (is_float(a.type)) static_cast<double*>(o.data)[g] = null ? 0.0 : __longlong_as_double((long long)v);
          else static_cast<long long*>(o.data)[g] = null ? 0 : (long long)v;
          break;
        case YQ_AGG_AVG: {
          const double s = is_float(a.type) ? __longlong_as_double((long long)v) : (double)(long long)v;
          static_cast<double*>(o.data)[g] = null ? 0.0 : s / (double)cnt;
          break;
        }
        default: {  // MIN / MAX in the input type
          const long long k = (long long)v;
          if (a.type == YQ_INT32) static_cast<int32_t*>(o.data)[g] = null ? 0 : (int32_t)k;
          else if (a.type == YQ_FLOAT32) static_cast<float*>(o.data)[g] = null ? 0.0f : (float)unordered(k);
          else if (a.type == YQ_FLOAT64) static_cast<double*>(o.data)[g] = null ? 0.0 : unordered(k);
          else static_cast<long long*>(o.data)[g] = null ? 0 : k;
          break;
        }
      }
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

size_t yq_group_by_workspace_size(const yq_column* key, uint32_t rows, int32_t nagg, uint32_t capacity) {
  if (!key) return 0;
  WsSize w;
  w.add<uint8_t>(yq_sort_workspace_size(key, rows));
  w.add<uint32_t>((size_t)rows + 1);          // permutation
  w.add<uint8_t>((size_t)rows + 16);          // head flags
  w.add<uint32_t>((size_t)rows + 1);          // group of every sorted position
  w.add<uint8_t>(yq_prefix_sum_workspace_size(rows));
  w.add<unsigned long long>((size_t)2 * (nagg > 0 ? nagg : 1) * ((size_t)capacity + 1));  // accumulators
  w.add<yq_column>(YQ_MAX_AGGREGATES + 1);
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
    P.a[j] = GAgg{in.data, in.nulls, it, g.kind, nullptr, nullptr};
  }
  if (rows == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_group_by_workspace_size(&key, rows, nagg, capacity), s));
  const size_t sort_ws = yq_sort_workspace_size(&key, rows);
  void* d_sort = ws.take<uint8_t>(sort_ws);
  uint32_t* perm = ws.take<uint32_t>((size_t)rows + 1);
  uint8_t* head = ws.take<uint8_t>((size_t)rows + 16);
  uint32_t* incl = ws.take<uint32_t>((size_t)rows + 1);
  void* scan_ws = ws.take<uint8_t>(yq_prefix_sum_workspace_size(rows));
  unsigned long long* acc = ws.take<unsigned long long>((size_t)2 * (nagg > 0 ? nagg : 1) * ((size_t)capacity + 1));
  yq_column* out_dev = ws.take<yq_column>(YQ_MAX_AGGREGATES + 1);
  yq_sort_config cfg{0, 0, 256, 1};  // every pass kept: no host read-back inside the sort
  YQ_TRY(yq_sort_indices(&key, rows, 0, 0, perm, &cfg, d_sort, sort_ws, stream));
  {
    ProfScope ps("group_heads", s, (double)rows * (key.width + 4));
    k_group_heads<<<grid_for(rows, kGroupThreads), kGroupThreads, 0, s>>>(key, perm, rows, head);
    YQ_CHECK_LAUNCH();
  }
  YQ_TRY(yq_prefix_sum_mask(head, incl, rows, scan_ws, yq_prefix_sum_workspace_size(rows), stream));
  uint32_t G = 0;
  YQ_TRY_CUDA(cudaMemcpyAsync(&G, incl + rows - 1, sizeof(G), cudaMemcpyDeviceToHost, s));
  YQ_TRY_CUDA(cudaStreamSynchronize(s));
  *groups = G;
  if (G > capacity) return YQ_ERR_CAPACITY;
  for (int j = 0; j < nagg; ++j) {
    P.a[j].count = acc + (size_t)2 * j * ((size_t)capacity + 1);
    P.a[j].value = P.a[j].count + capacity + 1;
  }
  P.perm = perm;
  P.incl = incl;
  YQ_TRY(h2d_async(out_dev, out, sizeof(yq_column) * (size_t)(nagg + 1), s));
  k_group_keys<<<grid_for(rows, kGroupThreads), kGroupThreads, 0, s>>>(key, perm, rows, head, incl, out[0]);
  YQ_CHECK_LAUNCH();
  if (nagg) {
    k_group_init<<<grid_for(G, kGroupThreads), kGroupThreads, 0, s>>>(P, G);
    YQ_CHECK_LAUNCH();
    double in_bytes = 4.0 * rows;
    for (int j = 0; j < nagg; ++j)
      if (P.a[j].data) in_bytes += (double)rows * (type_width(P.a[j].type) + (P.a[j].nulls ? 1 : 0));
    {
      ProfScope ps("group_accumulate", s, in_bytes);
      const uint64_t threads = ((uint64_t)rows + kGroupRun - 1) / kGroupRun;
      k_group_accumulate<<<(unsigned)((threads + kGroupThreads - 1) / kGroupThreads), kGroupThreads, 0, s>>>(P);
      YQ_CHECK_LAUNCH();
    }
    k_group_finalize<<<grid_for(G, kGroupThreads), kGroupThreads, 0, s>>>(P, G, out_dev);
    YQ_CHECK_LAUNCH();
  }
  return YQ_OK;
}

}  // extern "C"
