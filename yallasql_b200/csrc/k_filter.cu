// WHERE + aggregates and WHERE + projection (stream compaction) for sm_100a.
//
// Replaces the reference's per-node launches (comparison -> conjunction ->
// prefix_sum_mask -> move_rows_filter per column, then cast -> mul ->
// reduction per aggregate; include/engine/operators/filter_operator.hpp:31-98,
// include/engine/operators/expressions/aggregate.hpp:55-284,
// src/kernels/reduction_kernel.cu:79-185) with one kernel per operator that
// keeps every intermediate in registers.
#include "vm_host.cuh"
#include "yq_lookback.cuh"

namespace yq {

constexpr int kRowBlock = 256;
constexpr uint32_t kRowTile = kRowBlock * ITEMS;  // 1024 rows per tile

// ================================================================ aggregate
struct FAParams {
  VmProgram P;
  int32_t pc_end;
  int32_t nagg;
  uint8_t upd[YQ_MAX_AGGREGATES];
};

struct AggEmit {
  uint32_t sel;
  Acc acc[YQ_MAX_AGGREGATES];
  __device__ __forceinline__ void pred(uint32_t bits) { sel &= bits; }
  __device__ __forceinline__ void agg(int a, int upd, int t, const Val& x) {
    switch (a) {
#define YQ_AGG_CASE(k) \
  case k: acc_update(acc[k], upd, t, x, sel); break;
      YQ_AGG_CASE(0) YQ_AGG_CASE(1) YQ_AGG_CASE(2) YQ_AGG_CASE(3)
      YQ_AGG_CASE(4) YQ_AGG_CASE(5) YQ_AGG_CASE(6) YQ_AGG_CASE(7)
#undef YQ_AGG_CASE
      default: break;
    }
  }
  __device__ __forceinline__ void proj(int, const Val&) {}
};

__device__ __forceinline__ uint32_t in_range_bits(uint32_t row0, uint32_t n) {
  if (row0 >= n) return 0u;
  const uint32_t left = n - row0;
  return left >= (uint32_t)ITEMS ? ((1u << ITEMS) - 1u) : ((1u << left) - 1u);
}

struct AggInitParams {
  int32_t nagg;
  uint8_t upd[YQ_MAX_AGGREGATES];
};

__global__ void k_agg_state_init(Acc* state, const AggInitParams p) {
  const int a = threadIdx.x;
  if (a < p.nagg) acc_init(state[a], p.upd[a]);
}

__global__ void __launch_bounds__(kRowBlock) k_filter_aggregate(const __grid_constant__ FAParams F, uint32_t n,
                                                                Acc* __restrict__ partials, uint32_t* ticket,
                                                                Acc* __restrict__ state) {
  AggEmit E;
#pragma unroll
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) acc_init(E.acc[a], a < F.nagg ? F.upd[a] : UPD_COUNT);

  const uint32_t ntiles = ceil_div<uint32_t>(n, kRowTile);
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t row0 = tile * kRowTile + threadIdx.x * ITEMS;
    const uint32_t inr = in_range_bits(row0, n);
    E.sel = inr;
    Stack S;
    run_vm(F.P, 0, F.pc_end, row0, inr, inr == 0xfu, S, E);
#pragma unroll
    for (int a = 0; a < YQ_MAX_AGGREGATES; ++a)
      if (a < F.nagg && F.upd[a] == UPD_COUNT_STAR) E.acc[a].cnt += __popc(E.sel);
  }

  // Block reduction: warp shuffles, then warps in order.
  __shared__ Acc s_acc[kRowBlock / 32][YQ_MAX_AGGREGATES];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) {
    if (a < F.nagg) {
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) acc_shfl_down(E.acc[a], d, F.upd[a]);
      if (lane == 0) s_acc[warp][a] = E.acc[a];
    }
  }
  __syncthreads();
  if (threadIdx.x < F.nagg) {
    const int a = threadIdx.x;
    Acc t = s_acc[0][a];
    for (int w = 1; w < kRowBlock / 32; ++w) acc_combine(t, s_acc[w][a], F.upd[a]);
    partials[blockIdx.x * YQ_MAX_AGGREGATES + a] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < F.nagg) {
    // Fold the per-block partials in block order: the result does not depend
    // on which block finished last.
    const int a = threadIdx.x;
    const int upd = F.upd[a];
    Acc t;
    acc_init(t, upd);
    for (uint32_t b = 0; b < gridDim.x; ++b) {
      const Acc* p = partials + b * YQ_MAX_AGGREGATES + a;
      Acc q;
      q.cnt = __ldcg(&p->cnt);
      q.i = __ldcg(&p->i);
      q.f = __ldcg(&p->f);
      acc_combine(t, q, upd);
    }
    Acc s = state[a];
    acc_combine(s, t, upd);
    state[a] = s;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// Bytes per row of every input column a program references (plus null bytes).
static double referenced_row_bytes(const VmProgram& P, int len) {
  bool used[YQ_MAX_BATCH_COLUMNS] = {false};
  for (int i = 0; i < len; ++i) {
    const Insn& I = P.code[i];
    switch (I.op & OP_MASK) {
      case OP_COL: used[I.a] = true; break;
      case OP_ARITH_COL:
      case OP_CMP_COL_CONST:
      case OP_AND_CMP_COL_CONST: used[I.b] = true; break;
      case OP_CMP_COL_COL: used[I.b] = true; used[I.imm] = true; break;
      default: break;
    }
  }
  double b = 0;
  for (int c = 0; c < P.ncols; ++c)
    if (used[c]) b += P.cols[c].width + (P.cols[c].nulls ? 1 : 0);
  return b;
}

static int occupancy_grid(const void* kernel, int block, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * sm_count();
}

static uint8_t agg_update_code(int kind, int t) {
  const bool flt = (t == YQ_FLOAT32 || t == YQ_FLOAT64);
  switch (kind) {
    case YQ_AGG_COUNT_STAR: return UPD_COUNT_STAR;
    case YQ_AGG_COUNT: return UPD_COUNT;
    case YQ_AGG_SUM:
    case YQ_AGG_AVG: return flt ? UPD_SUM_F : UPD_SUM_I;
    case YQ_AGG_MIN: return flt ? UPD_MIN_F : UPD_MIN_I;
    default: return flt ? UPD_MAX_F : UPD_MAX_I;
  }
}

static int check_aggs(const yq_agg_spec* aggs, int nagg) {
  if (nagg < 0 || nagg > YQ_MAX_AGGREGATES || (nagg > 0 && !aggs)) return YQ_ERR_INVALID_ARG;
  for (int a = 0; a < nagg; ++a) {
    if (aggs[a].kind < YQ_AGG_COUNT_STAR || aggs[a].kind > YQ_AGG_MAX) return YQ_ERR_INVALID_ARG;
    if (aggs[a].kind != YQ_AGG_COUNT_STAR && aggs[a].kind != YQ_AGG_COUNT) {
      const int t = aggs[a].input_type;
      if (t != YQ_INT32 && t != YQ_FLOAT32 && t != YQ_INT64 && t != YQ_DATETIME && t != YQ_FLOAT64 && t != YQ_BOOL)
        return YQ_ERR_INVALID_ARG;
    }
  }
  return YQ_OK;
}

// Builds the VM program: predicate (+EMIT_PRED) then each aggregate's input (+EMIT_AGG).
static int build_agg_program(ProgramBuilder& B, const yq_program* predicate, const yq_agg_spec* aggs, int nagg,
                             uint8_t* upd) {
  if (predicate && predicate->len > 0) {
    int t = -1;
    YQ_TRY(B.append(predicate, t));
    if (t != YQ_BOOL) return YQ_ERR_INVALID_ARG;
    YQ_TRY(B.emit(OP_EMIT_PRED, 0, 0, YQ_BOOL));
  }
  for (int a = 0; a < nagg; ++a) {
    upd[a] = agg_update_code(aggs[a].kind, aggs[a].input_type);
    if (aggs[a].kind == YQ_AGG_COUNT_STAR) continue;
    int t = -1;
    YQ_TRY(B.append(&aggs[a].input, t));
    if (aggs[a].kind != YQ_AGG_COUNT && t != aggs[a].input_type) return YQ_ERR_INVALID_ARG;
    YQ_TRY(B.emit(OP_EMIT_AGG, (uint8_t)a, upd[a], (uint8_t)t));
  }
  B.finalize();
  return YQ_OK;
}

int launch_filter_aggregate(const FAParams& F, uint32_t rows, Acc* partials, uint32_t* ticket, Acc* state, int grid,
                            cudaStream_t s) {
  ProfScope ps("filter_aggregate", s, (double)rows * referenced_row_bytes(F.P, F.pc_end));
  k_filter_aggregate<<<grid, kRowBlock, 0, s>>>(F, rows, partials, ticket, state);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int filter_aggregate_grid(uint32_t rows) {
  static int cap = 0;
  if (!cap) cap = occupancy_grid((const void*)k_filter_aggregate, kRowBlock, 0);
  const int tiles = (int)ceil_div<uint32_t>(rows, kRowTile);
  return tiles < cap ? (tiles > 0 ? tiles : 1) : cap;
}

int prepare_filter_aggregate(const yq_batch* batch, const yq_program* predicate, const yq_constants* constants,
                             const yq_agg_spec* aggs, int32_t nagg, FAParams* F) {
  if (!batch || !F) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  ProgramBuilder B;
  YQ_TRY(B.set_columns(batch->columns, batch->ncols));
  YQ_TRY(B.set_constants(constants));
  uint8_t upd[YQ_MAX_AGGREGATES] = {0};
  YQ_TRY(build_agg_program(B, predicate, aggs, nagg, upd));
  memcpy(&F->P, &B.P, sizeof(VmProgram));
  F->pc_end = B.len;
  F->nagg = nagg;
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) F->upd[a] = a < nagg ? upd[a] : UPD_COUNT;
  return YQ_OK;
}

// ================================================================ project
struct DevOut {
  char* data;
  uint8_t* nulls;
  int32_t width;
  int32_t src_col;  // >= 0: copy of this input column
};

struct FPParams {
  VmProgram P;
  int32_t pred_end;
  int32_t proj_end;
  int32_t nproj;
  uint32_t capacity;
  DevOut out[YQ_MAX_PROJECTIONS];
};

__device__ __forceinline__ void store_slot(char* base, uint32_t pos, int width, uint64_t v) {
  if (width == 4) reinterpret_cast<uint32_t*>(base)[pos] = (uint32_t)v;
  else if (width == 8) reinterpret_cast<unsigned long long*>(base)[pos] = v;
  else reinterpret_cast<uint8_t*>(base)[pos] = (uint8_t)v;
}

struct ProjEmit {
  uint32_t sel;
  uint32_t pos;
  const FPParams* F;
  __device__ __forceinline__ void pred(uint32_t bits) { sel &= bits; }
  __device__ __forceinline__ void agg(int, int, int, const Val&) {}
  __device__ __forceinline__ void proj(int p, const Val& x) {
    const DevOut& o = F->out[p];
    uint32_t q = pos;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if (sel & (1u << k)) {
        if (q < F->capacity) {
          store_slot(o.data, q, o.width, x.v[k]);
          if (o.nulls) o.nulls[q] = (x.valid >> k & 1u) ? 0 : 1;
        }
        ++q;
      }
    }
  }
};

__device__ __forceinline__ void copy_value(char* dst, const char* src, int width) {
  if (width == 4) {
    *reinterpret_cast<uint32_t*>(dst) = __ldg(reinterpret_cast<const uint32_t*>(src));
  } else if (width == 8) {
    *reinterpret_cast<unsigned long long*>(dst) = __ldg(reinterpret_cast<const unsigned long long*>(src));
  } else if (width == 1) {
    *dst = *src;
  } else if ((width & 15) == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
    for (int i = 0; i < width; i += 16)
      *reinterpret_cast<uint4*>(dst + i) = ldg_nc_v4(src + i);
  } else {
    for (int i = 0; i < width; i += 4)
      *reinterpret_cast<uint32_t*>(dst + i) = __ldg(reinterpret_cast<const uint32_t*>(src + i));
  }
}

__global__ void __launch_bounds__(kRowBlock) k_filter_project(const __grid_constant__ FPParams F, uint32_t n,
                                                              uint32_t* tile_counter,
                                                              unsigned long long* __restrict__ status,
                                                              uint32_t* out_count, uint32_t* err) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kRowBlock / 32 + 1];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t row0 = tile * kRowTile + threadIdx.x * ITEMS;
  const uint32_t inr = in_range_bits(row0, n);
  const bool full = (inr == 0xfu);

  ProjEmit E;
  E.sel = inr;
  E.pos = 0;
  E.F = &F;
  Stack S;
  if (F.pred_end > 0) run_vm(F.P, 0, F.pred_end, row0, inr, full, S, E);

  uint32_t total;
  const uint32_t excl = block_exclusive_sum<kRowBlock>(__popc(E.sel), s_warp, total);
  if (threadIdx.x < 32) {
    unsigned long long p = tile_lookback(status, tile, total, err);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  const unsigned long long base = s_prefix;
  E.pos = (uint32_t)(base + excl);

  if (F.proj_end > F.pred_end) run_vm(F.P, F.pred_end, F.proj_end, row0, inr, full, S, E);
  for (int p = 0; p < F.nproj; ++p) {
    const DevOut& o = F.out[p];
    if (o.src_col < 0) continue;
    const DevCol& c = F.P.cols[o.src_col];
    uint32_t q = E.pos;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if (E.sel & (1u << k)) {
        if (q < F.capacity) {
          copy_value(o.data + (size_t)q * o.width, c.data + (size_t)(row0 + k) * c.width, c.width);
          if (o.nulls) o.nulls[q] = c.nulls ? c.nulls[row0 + k] : 0;
        }
        ++q;
      }
    }
  }
  if (tile == gridDim.x - 1 && threadIdx.x == 0) {
    const unsigned long long cnt = base + total;
    *out_count = cnt > 0xffffffffull ? 0xffffffffu : (uint32_t)cnt;
  }
}

}  // namespace yq

using namespace yq;

extern "C" {

size_t yq_agg_state_bytes(int32_t nagg) {
  if (nagg < 0) nagg = 0;
  return align_up((size_t)nagg * sizeof(Acc), 256);
}

int yq_agg_state_init(void* state, const yq_agg_spec* aggs, int32_t nagg, void* stream) {
  if (!state) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  if (nagg == 0) return YQ_OK;
  AggInitParams p;
  p.nagg = nagg;
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) p.upd[a] = a < nagg ? agg_update_code(aggs[a].kind, aggs[a].input_type) : 0;
  k_agg_state_init<<<1, 32, 0, as_stream(stream)>>>(static_cast<Acc*>(state), p);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

size_t yq_filter_aggregate_workspace_size(uint32_t rows, int32_t nagg) {
  (void)nagg;
  WsSize w;
  w.add<Acc>((size_t)filter_aggregate_grid(rows) * YQ_MAX_AGGREGATES);
  w.add<uint32_t>(4);
  return w.total();
}

int yq_filter_aggregate(const yq_batch* batch, const yq_program* predicate, const yq_constants* constants,
                        const yq_agg_spec* aggs, int32_t nagg, void* state, void* workspace, size_t workspace_bytes,
                        void* stream) {
  if (!batch || !state) return YQ_ERR_INVALID_ARG;
  FAParams F;
  YQ_TRY(prepare_filter_aggregate(batch, predicate, constants, aggs, nagg, &F));
  if (batch->rows == 0 || nagg == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  const int grid = filter_aggregate_grid(batch->rows);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_filter_aggregate_workspace_size(batch->rows, nagg), s));
  Acc* partials = ws.take<Acc>((size_t)grid * YQ_MAX_AGGREGATES);
  uint32_t* ticket = ws.take<uint32_t>(4);
  YQ_TRY_CUDA(cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s));
  return launch_filter_aggregate(F, batch->rows, partials, ticket, static_cast<Acc*>(state), grid, s);
}

int yq_agg_state_read(const void* state, const yq_agg_spec* aggs, int32_t nagg, yq_agg_result* out, void* stream) {
  if (!state || !out) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  Acc host[YQ_MAX_AGGREGATES];
  cudaStream_t s = as_stream(stream);
  YQ_TRY_CUDA(cudaMemcpyAsync(host, state, (size_t)nagg * sizeof(Acc), cudaMemcpyDeviceToHost, s));
  YQ_TRY_CUDA(cudaStreamSynchronize(s));
  for (int a = 0; a < nagg; ++a) {
    const Acc& h = host[a];
    yq_agg_result& r = out[a];
    const int kind = aggs[a].kind;
    const int t = aggs[a].input_type;
    const bool flt = (t == YQ_FLOAT32 || t == YQ_FLOAT64);
    r.kind = kind;
    r.count = h.cnt;
    r.i = 0;
    r.f = 0.0;
    r.is_null = 0;
    switch (kind) {
      case YQ_AGG_COUNT_STAR:
      case YQ_AGG_COUNT: r.i = h.cnt; break;
      case YQ_AGG_SUM:
        r.is_null = h.cnt == 0;
        if (flt) r.f = h.f;
        else r.i = h.i;
        break;
      case YQ_AGG_AVG:
        r.is_null = h.cnt == 0;
        if (h.cnt) r.f = flt ? h.f / (double)h.cnt : (double)h.i / (double)h.cnt;
        break;
      default:
        r.is_null = h.cnt == 0;
        if (flt) r.f = h.f;
        else r.i = h.i;
        break;
    }
  }
  return YQ_OK;
}

size_t yq_filter_project_workspace_size(uint32_t rows) {
  WsSize w;
  w.add<unsigned long long>((size_t)ceil_div<uint32_t>(rows, kRowTile) + 1);
  w.add<uint32_t>(4);
  return w.total();
}

int yq_filter_project(const yq_batch* batch, const yq_program* predicate, const yq_constants* constants,
                      const yq_projection* proj, int32_t nproj, yq_column* out, uint32_t capacity,
                      uint32_t* count_device, uint32_t* count_host, void* workspace, size_t workspace_bytes,
                      void* stream) {
  if (!batch || nproj < 0 || nproj > YQ_MAX_PROJECTIONS || (nproj > 0 && (!proj || !out))) return YQ_ERR_INVALID_ARG;
  cudaStream_t s = as_stream(stream);
  FPParams F;
  {
    ProgramBuilder B;
    YQ_TRY(B.set_columns(batch->columns, batch->ncols));
    YQ_TRY(B.set_constants(constants));
    if (predicate && predicate->len > 0) {
      int t = -1;
      YQ_TRY(B.append(predicate, t));
      if (t != YQ_BOOL) return YQ_ERR_INVALID_ARG;
      YQ_TRY(B.emit(OP_EMIT_PRED, 0, 0, YQ_BOOL));
    }
    F.pred_end = B.len;
    for (int p = 0; p < nproj; ++p) {
      DevOut& o = F.out[p];
      o.data = static_cast<char*>(out[p].data);
      o.nulls = const_cast<uint8_t*>(out[p].nulls);
      o.src_col = proj[p].column;
      if (!o.data && capacity > 0) return YQ_ERR_INVALID_ARG;
      if (proj[p].column >= 0) {
        if (proj[p].column >= batch->ncols) return YQ_ERR_INVALID_ARG;
        const yq_column& c = batch->columns[proj[p].column];
        if (out[p].type != c.type || out[p].width != c.width) return YQ_ERR_INVALID_ARG;
        o.width = c.width;
      } else {
        int t = -1;
        YQ_TRY(B.append(&proj[p].program, t));
        if (t != proj[p].out_type || t != out[p].type || !ProgramBuilder::valid_column(out[p])) return YQ_ERR_INVALID_ARG;
        o.width = out[p].width;
        YQ_TRY(B.emit(OP_EMIT_PROJ, (uint8_t)p, 0, (uint8_t)t));
      }
    }
    B.finalize();
    memcpy(&F.P, &B.P, sizeof(VmProgram));
    F.proj_end = B.len;
    F.nproj = nproj;
    F.capacity = capacity;
  }
  const uint32_t rows = batch->rows;
  if (rows == 0) {
    if (count_device) YQ_TRY_CUDA(cudaMemsetAsync(count_device, 0, sizeof(uint32_t), s));
    if (count_host) *count_host = 0;
    return YQ_OK;
  }
  const uint32_t ntiles = ceil_div<uint32_t>(rows, kRowTile);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_filter_project_workspace_size(rows), s));
  unsigned long long* status = ws.take<unsigned long long>((size_t)ntiles + 1);
  uint32_t* misc = ws.take<uint32_t>(4);  // [0] tile counter, [1] error, [2] count
  YQ_TRY_CUDA(cudaMemsetAsync(status, 0, ((size_t)ntiles + 1) * sizeof(unsigned long long), s));
  YQ_TRY_CUDA(cudaMemsetAsync(misc, 0, 4 * sizeof(uint32_t), s));
  uint32_t* cnt_dev = count_device ? count_device : misc + 2;
  {
    // algorithmic bytes: referenced input columns (outputs depend on selectivity)
    const double in_b = referenced_row_bytes(F.P, F.proj_end);
    ProfScope ps("filter_project", s, (double)rows * in_b);
    k_filter_project<<<ntiles, kRowBlock, 0, s>>>(F, rows, misc, status, cnt_dev, misc + 1);
    YQ_CHECK_LAUNCH();
  }
  if (count_host) {
    uint32_t h[2];
    YQ_TRY_CUDA(cudaMemcpyAsync(&h[0], cnt_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    YQ_TRY_CUDA(cudaMemcpyAsync(&h[1], misc + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    YQ_TRY_CUDA(cudaStreamSynchronize(s));
    *count_host = h[0];
    if (h[1] & kErrTimeout) return YQ_ERR_TIMEOUT;
    if (h[0] > capacity) return YQ_ERR_CAPACITY;
  }
  return YQ_OK;
}

}  // extern "C"

// =================================================== allocation-free variant
// yq_filter_project_noalloc runs the same kernel as yq_filter_project, but its
// look-back scratch is this file-scope device array instead of a workspace
// the caller passes or the library allocates. Layout: four 32-bit counters
// (tile counter, error word, row count, spare), then one 64-bit look-back
// status word per 1,024-row tile plus one.
#include <mutex>

namespace yq {

constexpr uint32_t kNoAllocTiles = YQ_FILTER_PROJECT_NOALLOC_MAX_ROWS / kRowTile;
constexpr size_t kNoAllocWords = 2 + (size_t)kNoAllocTiles + 1;  // 2 words hold the four counters

static __device__ __align__(256) unsigned long long g_filter_project_scratch[kNoAllocWords];

// Device address of the scratch array, looked up once per device with that
// device current (host code only sees a host-side stand-in for the symbol).
static int noalloc_scratch(unsigned long long** out) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  int dev = 0;
  YQ_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return YQ_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_filter_project_scratch);
    if (e != cudaSuccess || !p) {
      set_cuda_error(e);
      return YQ_ERR_CUDA;
    }
    addr[dev] = p;
  }
  *out = static_cast<unsigned long long*>(addr[dev]);
  return YQ_OK;
}

// Same validation and program build as yq_filter_project.
static int build_project_params(const yq_batch* batch, const yq_program* predicate, const yq_constants* constants,
                                const yq_projection* proj, int32_t nproj, yq_column* out, uint32_t capacity,
                                FPParams& F) {
  if (!batch || nproj < 0 || nproj > YQ_MAX_PROJECTIONS || (nproj > 0 && (!proj || !out))) return YQ_ERR_INVALID_ARG;
  ProgramBuilder B;
  YQ_TRY(B.set_columns(batch->columns, batch->ncols));
  YQ_TRY(B.set_constants(constants));
  if (predicate && predicate->len > 0) {
    int t = -1;
    YQ_TRY(B.append(predicate, t));
    if (t != YQ_BOOL) return YQ_ERR_INVALID_ARG;
    YQ_TRY(B.emit(OP_EMIT_PRED, 0, 0, YQ_BOOL));
  }
  F.pred_end = B.len;
  for (int p = 0; p < nproj; ++p) {
    DevOut& o = F.out[p];
    o.data = static_cast<char*>(out[p].data);
    o.nulls = const_cast<uint8_t*>(out[p].nulls);
    o.src_col = proj[p].column;
    if (!o.data && capacity > 0) return YQ_ERR_INVALID_ARG;
    if (proj[p].column >= 0) {
      if (proj[p].column >= batch->ncols) return YQ_ERR_INVALID_ARG;
      const yq_column& c = batch->columns[proj[p].column];
      if (out[p].type != c.type || out[p].width != c.width) return YQ_ERR_INVALID_ARG;
      o.width = c.width;
    } else {
      int t = -1;
      YQ_TRY(B.append(&proj[p].program, t));
      if (t != proj[p].out_type || t != out[p].type || !ProgramBuilder::valid_column(out[p])) return YQ_ERR_INVALID_ARG;
      o.width = out[p].width;
      YQ_TRY(B.emit(OP_EMIT_PROJ, (uint8_t)p, 0, (uint8_t)t));
    }
  }
  B.finalize();
  memcpy(&F.P, &B.P, sizeof(VmProgram));
  F.proj_end = B.len;
  F.nproj = nproj;
  F.capacity = capacity;
  return YQ_OK;
}

}  // namespace yq

extern "C" int yq_filter_project_noalloc(const yq_batch* batch, const yq_program* predicate,
                                         const yq_constants* constants, const yq_projection* proj, int32_t nproj,
                                         yq_column* out, uint32_t capacity, uint32_t* count_device,
                                         uint32_t* count_host, void* stream) {
  if (!batch) return YQ_ERR_INVALID_ARG;
  if (batch->rows > YQ_FILTER_PROJECT_NOALLOC_MAX_ROWS) return YQ_ERR_INVALID_ARG;  // scratch holds no more tiles
  FPParams F;
  YQ_TRY(build_project_params(batch, predicate, constants, proj, nproj, out, capacity, F));
  cudaStream_t s = as_stream(stream);
  const uint32_t rows = batch->rows;
  if (rows == 0) {
    if (count_device) YQ_TRY_CUDA(cudaMemsetAsync(count_device, 0, sizeof(uint32_t), s));
    if (count_host) *count_host = 0;
    return YQ_OK;
  }
  unsigned long long* scratch = nullptr;
  YQ_TRY(noalloc_scratch(&scratch));
  const uint32_t ntiles = ceil_div<uint32_t>(rows, kRowTile);
  uint32_t* misc = reinterpret_cast<uint32_t*>(scratch);  // [0] tile counter, [1] error, [2] count
  unsigned long long* status = scratch + 2;
  // The previous call's values are still there: clear what this call reads.
  YQ_TRY_CUDA(cudaMemsetAsync(scratch, 0, (2 + (size_t)ntiles + 1) * sizeof(unsigned long long), s));
  uint32_t* cnt_dev = count_device ? count_device : misc + 2;
  k_filter_project<<<ntiles, kRowBlock, 0, s>>>(F, rows, misc, status, cnt_dev, misc + 1);
  YQ_CHECK_LAUNCH();
  if (count_host) {
    uint32_t h[2];
    YQ_TRY_CUDA(cudaMemcpyAsync(&h[0], cnt_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    YQ_TRY_CUDA(cudaMemcpyAsync(&h[1], misc + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    YQ_TRY_CUDA(cudaStreamSynchronize(s));
    *count_host = h[0];
    if (h[1] & kErrTimeout) return YQ_ERR_TIMEOUT;
    if (h[0] > capacity) return YQ_ERR_CAPACITY;
  }
  return YQ_OK;
}
