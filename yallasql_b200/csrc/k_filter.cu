// WHERE + aggregates and WHERE + projection (stream compaction) for sm_100a.
//
// Replaces the reference's per-node launches (comparison -> conjunction ->
// prefix_sum_mask -> move_rows_filter per column, then cast -> mul ->
// reduction per aggregate; include/engine/operators/filter_operator.hpp:31-98,
// include/engine/operators/expressions/aggregate.hpp:55-284,
// src/kernels/reduction_kernel.cu:79-185) with one persistent kernel per
// operator that keeps every intermediate in registers. The columns a program
// reads are staged in shared memory a few steps ahead by bulk copies
// (yq_stage.cuh) when they are 16-byte aligned and fit; otherwise the kernel
// reads them from global memory directly.
#include <algorithm>
#include <vector>
#include "vm_host.cuh"
#include "row_kernels.cuh"
#include "yq_jit.cuh"

namespace yq {

// Persistent grid of a row kernel: resident blocks on every SM (per device,
// cached), no more than the steps.
static int resident_grid(const void* kernel, size_t dyn_smem, uint32_t steps) {
  const int cap = kernel_blocks_per_sm(kernel, kRowBlock, dyn_smem) * sm_count();
  const int g = (int)(steps < (uint32_t)cap ? steps : (uint32_t)cap);
  return g < 1 ? 1 : g;
}

static size_t max_row_grid() { return (size_t)sm_count() * 8; }

// ================================================================ aggregate

__global__ void k_agg_state_init(Acc* state, const AggParams p) {
  const int a = threadIdx.x;
  if (a < YQ_MAX_AGGREGATES) state[a] = Acc{0, acc_identity(a < p.nagg ? p.upd[a] : UPD_COUNT)};
  if (a == 0) *agg_state_err(state) = 0u;
}

// One block per state of a back-to-back array of states.
__global__ void k_agg_states_init(char* states, const AggParams p) {
  Acc* st = reinterpret_cast<Acc*>(states + (size_t)blockIdx.x * kAggStateBytes);
  const int a = threadIdx.x;
  if (a < YQ_MAX_AGGREGATES) st[a] = Acc{0, acc_identity(a < p.nagg ? p.upd[a] : UPD_COUNT)};
  if (a == 0) *agg_state_err(st) = 0u;
}

template <bool STAGED>
__global__ void __launch_bounds__(kRowBlock, 2) k_filter_aggregate(const __grid_constant__ FAParams F, uint32_t n,
                                                                   Acc* __restrict__ partials, uint32_t* ticket,
                                                                   Acc* state) {
  filter_aggregate_body<STAGED, InterpRunner>(F, n, partials, ticket, state);
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
  return B.finalize();
}

static int prepare_filter_aggregate(const yq_batch* batch, const yq_program* predicate, const yq_constants* constants,
                                    const yq_agg_spec* aggs, int32_t nagg, FAParams* F) {
  if (!batch || !F) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  ProgramBuilder B;
  YQ_TRY(B.set_columns(batch->columns, batch->ncols));
  YQ_TRY(B.set_constants(constants));
  uint8_t upd[YQ_MAX_AGGREGATES] = {0};
  YQ_TRY(build_agg_program(B, predicate, aggs, nagg, upd));
  if (!plan_stages(B.P, B.used_cols, F->SP)) F->SP.nstages = 0;
  memcpy(&F->P, &B.P, sizeof(VmProgram));
  F->pc_end = B.len;
  F->A.nagg = nagg;
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) F->A.upd[a] = a < nagg ? upd[a] : UPD_COUNT;
  return YQ_OK;
}

// Batches with fewer steps than about four per resident block (1M rows and
// less) skip the staging ring: every block then handles one or two steps, and
// setting up a ring (barriers, copies issued ahead) costs more than it hides.
static bool few_steps(uint32_t rows) { return ceil_div<uint32_t>(rows, kStepRows) < 12u * (uint32_t)sm_count(); }

static int launch_filter_aggregate(const FAParams& F0, uint32_t rows, Acc* partials, uint32_t* ticket, Acc* state,
                                   cudaStream_t s) {
  FAParams F = F0;
  if (few_steps(rows)) F.SP.nstages = 0;
  const bool staged = F.SP.nstages > 0;
  const void* kern = staged ? (const void*)k_filter_aggregate<true> : (const void*)k_filter_aggregate<false>;
  const size_t smem = stage_smem_bytes(F.SP);
  YQ_TRY(kernel_allow_smem(kern, smem));
  int grid = resident_grid(kern, smem, ceil_div<uint32_t>(rows, kStepRows));
  if ((size_t)grid > max_row_grid()) grid = (int)max_row_grid();
  const void* jk = jit_kernel(JIT_FILTER_AGG, staged, F.P, F.pc_end, F.pc_end);  // compiles once, outside the timing
  ProfScope ps("filter_aggregate", s, (double)rows * row_bytes_of(F.P, program_columns(F.P, F.pc_end, 0)));
  if (jk) {
    FAParams G = F;
    if (staged) G.SP.nstages = jit_stages(jk, G.SP.stage_bytes, G.SP.nstages);
    void* args[] = {&G, &rows, &partials, &ticket, &state};
    return jit_launch(jk, (int)max_row_grid(), ceil_div<uint32_t>(rows, kStepRows), stage_smem_bytes(G.SP), args, s);
  }
  if (staged)
    k_filter_aggregate<true><<<grid, kRowBlock, smem, s>>>(F, rows, partials, ticket, state);
  else
    k_filter_aggregate<false><<<grid, kRowBlock, 0, s>>>(F, rows, partials, ticket, state);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

// ======================================================= segmented aggregate

template <bool STAGED>
__global__ void __launch_bounds__(kRowBlock, 2) k_filter_aggregate_seg(const __grid_constant__ FASegParams Q) {
  filter_aggregate_seg_body<STAGED, InterpRunner>(Q);
}

// One block per task folds the task's step partials: thread t takes steps
// t, t + kFoldBlock, ... of the task, then the warps and the block combine
// them in a fixed order, so the result is deterministic.
constexpr int kFoldBlock = 256;

__global__ void __launch_bounds__(kFoldBlock) k_agg_seg_fold(const Acc* __restrict__ partials,
                                                             const uint32_t* __restrict__ step0, int nseg,
                                                             const AggParams A, Acc* states, const uint32_t* err) {
  __shared__ Acc s_acc[kFoldBlock / 32][YQ_MAX_AGGREGATES];
  const int g = blockIdx.x;
  if (g >= nseg) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Acc* st = reinterpret_cast<Acc*>(reinterpret_cast<char*>(states) + (size_t)g * kAggStateBytes);
  if (threadIdx.x == 0 && *err) *agg_state_err(st) |= *err;
  const uint32_t s0 = step0[g], s1 = step0[g + 1];
#pragma unroll
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) {
    if (a < A.nagg) {
      const int upd = A.upd[a];
      long long c = 0;
      unsigned long long v = acc_identity(upd);
      for (uint32_t s = s0 + threadIdx.x; s < s1; s += kFoldBlock) {
        const Acc p = partials[(size_t)s * YQ_MAX_AGGREGATES + a];
        c += p.cnt;
        v = acc_merge(upd, v, p.bits);
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, d);
        v = acc_merge(upd, v, __shfl_down_sync(0xffffffffu, v, d));
      }
      if (lane == 0) s_acc[warp][a] = Acc{c, v};
    }
  }
  __syncthreads();
  const int a = threadIdx.x;
  if (a >= A.nagg) return;
  const int upd = A.upd[a];
  Acc t = s_acc[0][a];
  for (int w = 1; w < kFoldBlock / 32; ++w) {
    t.cnt += s_acc[w][a].cnt;
    t.bits = acc_merge(upd, t.bits, s_acc[w][a].bits);
  }
  Acc cur = st[a];
  cur.cnt += t.cnt;
  cur.bits = acc_merge(upd, cur.bits, t.bits);
  st[a] = cur;
}

static uint32_t seg_steps(const uint32_t* begin, const uint32_t* end, int nseg, std::vector<uint32_t>& step0) {
  step0.resize((size_t)nseg + 1);
  uint32_t t = 0;
  for (int g = 0; g < nseg; ++g) {
    step0[g] = t;
    if (end[g] > begin[g]) t += ceil_div<uint32_t>(end[g], kStepRows) - begin[g] / kStepRows;
  }
  step0[nseg] = t;
  return t;
}

// ================================================================ project
template <bool STAGED>
__global__ void __launch_bounds__(kRowBlock, 2) k_filter_project(const __grid_constant__ FPParams F, uint32_t n,
                                                                 uint32_t* chunk_counter,
                                                                 unsigned long long* __restrict__ status,
                                                                 uint32_t* out_count, uint32_t* err) {
  filter_project_body<STAGED, InterpRunner>(F, n, chunk_counter, status, out_count, err);
}

// Validation and program build shared by yq_filter_project and its
// allocation-free variant.
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
  const int pred_end = B.len;
  uint32_t copy_mask = 0;
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
      copy_mask |= 1u << proj[p].column;
    } else {
      int t = -1;
      YQ_TRY(B.append(&proj[p].program, t));
      if (t != proj[p].out_type || t != out[p].type || !ProgramBuilder::valid_column(out[p])) return YQ_ERR_INVALID_ARG;
      o.width = out[p].width;
      YQ_TRY(B.emit(OP_EMIT_PROJ, (uint8_t)p, 0, (uint8_t)t));
    }
  }
  YQ_TRY(B.finalize());
  // Pass 0 stages what the predicate reads, pass 1 what the output reads.
  const int pe = B.remap[pred_end];
  if (!plan_stages2(B.P, program_columns_in(B.P, 0, pe, 0), program_columns_in(B.P, pe, B.len, copy_mask), F.SP))
    F.SP.nstages = 0;
  memcpy(&F.P, &B.P, sizeof(VmProgram));
  F.pred_end = B.remap[pred_end];
  F.proj_end = B.len;
  F.nproj = nproj;
  F.capacity = capacity;
  return YQ_OK;
}

// Launch over `rows` rows with look-back scratch `status` (one word per
// 1,024-row step plus one; a chunk of steps uses one) and `misc` = {chunk
// counter, error word} (both zeroed). Chunks are as long as keeps about eight
// of them per SM (at most 8 steps), so a batch still spreads over every SM.
static int launch_filter_project(FPParams& F, uint32_t rows, uint32_t* misc, unsigned long long* status,
                                 uint32_t* cnt_dev, cudaStream_t s, bool allow_jit = true) {
  const bool staged = F.SP.nstages > 0;
  F.csteps = std::max<uint32_t>(1u, std::min<uint32_t>(8u, ceil_div<uint32_t>(rows, kStepRows) / (8u * sm_count())));
  const void* kern = staged ? (const void*)k_filter_project<true> : (const void*)k_filter_project<false>;
  const size_t smem = stage_smem_bytes(F.SP);
  YQ_TRY(kernel_allow_smem(kern, smem));
  const int grid = resident_grid(kern, smem, ceil_div<uint32_t>(rows, kStepRows));
  uint32_t mask = program_columns(F.P, F.proj_end, 0);
  for (int p = 0; p < F.nproj; ++p)
    if (F.out[p].src_col >= 0) mask |= 1u << F.out[p].src_col;
  // algorithmic bytes: referenced input columns (outputs depend on selectivity)
  const void* jk = allow_jit ? jit_kernel(JIT_FILTER_PROJECT, staged, F.P, F.pred_end, F.proj_end, &F) : nullptr;
  ProfScope ps("filter_project", s, (double)rows * row_bytes_of(F.P, mask));
  if (jk) {
    uint32_t* err = misc + 1;
    if (staged) F.SP.nstages = jit_stages(jk, F.SP.stage_bytes, F.SP.nstages);
    void* args[] = {&F, &rows, &misc, &status, &cnt_dev, &err};
    return jit_launch(jk, 1 << 30, ceil_div<uint32_t>(rows, kStepRows), stage_smem_bytes(F.SP), args, s);
  }
  if (staged)
    k_filter_project<true><<<grid, kRowBlock, smem, s>>>(F, rows, misc, status, cnt_dev, misc + 1);
  else
    k_filter_project<false><<<grid, kRowBlock, 0, s>>>(F, rows, misc, status, cnt_dev, misc + 1);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

}  // namespace yq

using namespace yq;

extern "C" {

size_t yq_agg_state_bytes(int32_t nagg) {
  (void)nagg;
  return kAggStateBytes;
}

int yq_agg_state_init(void* state, const yq_agg_spec* aggs, int32_t nagg, void* stream) {
  if (!state) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  AggParams p;
  memset(&p, 0, sizeof(p));
  p.nagg = nagg;
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) p.upd[a] = a < nagg ? agg_update_code(aggs[a].kind, aggs[a].input_type) : 0;
  k_agg_state_init<<<1, 32, 0, as_stream(stream)>>>(static_cast<Acc*>(state), p);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

size_t yq_filter_aggregate_workspace_size(uint32_t rows, int32_t nagg) {
  (void)nagg;
  (void)rows;
  WsSize w;
  w.add<Acc>(max_row_grid() * YQ_MAX_AGGREGATES);
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
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_filter_aggregate_workspace_size(batch->rows, nagg), s));
  Acc* partials = ws.take<Acc>(max_row_grid() * YQ_MAX_AGGREGATES);
  uint32_t* ticket = ws.take<uint32_t>(4);
  YQ_TRY_CUDA(cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s));
  return launch_filter_aggregate(F, batch->rows, partials, ticket, static_cast<Acc*>(state), s);
}

int yq_agg_state_read(const void* state, const yq_agg_spec* aggs, int32_t nagg, yq_agg_result* out, void* stream) {
  if (!state || !out) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  Acc host[YQ_MAX_AGGREGATES + 1];
  cudaStream_t s = as_stream(stream);
  YQ_TRY(d2h_sync(host, state, sizeof(Acc) * YQ_MAX_AGGREGATES + sizeof(uint32_t), s));
  if (*agg_state_err(host)) return YQ_ERR_TIMEOUT;
  for (int a = 0; a < nagg; ++a) {
    const Acc& h = host[a];
    yq_agg_result& r = out[a];
    const int kind = aggs[a].kind;
    const int t = aggs[a].input_type;
    const bool flt = (t == YQ_FLOAT32 || t == YQ_FLOAT64);
    double hf;
    memcpy(&hf, &h.bits, sizeof(hf));
    const long long hi = (long long)h.bits;
    r.kind = kind;
    r.count = h.cnt;
    r.i = 0;
    r.f = 0.0;
    r.is_null = 0;
    switch (kind) {
      case YQ_AGG_COUNT_STAR:
      case YQ_AGG_COUNT: r.i = h.cnt; break;
      case YQ_AGG_AVG:
        r.is_null = h.cnt == 0;
        if (h.cnt) r.f = flt ? hf / (double)h.cnt : (double)hi / (double)h.cnt;
        break;
      default:  // SUM, MIN, MAX
        r.is_null = h.cnt == 0;
        if (flt) r.f = hf;
        else r.i = hi;
        break;
    }
  }
  return YQ_OK;
}

int yq_agg_states_init(void* states, int32_t count, const yq_agg_spec* aggs, int32_t nagg, void* stream) {
  if (!states || count < 0) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  if (count == 0) return YQ_OK;
  AggParams p;
  memset(&p, 0, sizeof(p));
  p.nagg = nagg;
  for (int a = 0; a < YQ_MAX_AGGREGATES; ++a) p.upd[a] = a < nagg ? agg_update_code(aggs[a].kind, aggs[a].input_type) : 0;
  k_agg_states_init<<<count, 32, 0, as_stream(stream)>>>(static_cast<char*>(states), p);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

int yq_agg_states_read(const void* states, int32_t count, const yq_agg_spec* aggs, int32_t nagg, yq_agg_result* out,
                       void* stream) {
  if (!states || !out || count < 0) return YQ_ERR_INVALID_ARG;
  YQ_TRY(check_aggs(aggs, nagg));
  if (count == 0) return YQ_OK;
  std::vector<char> host((size_t)count * kAggStateBytes);
  cudaStream_t s = as_stream(stream);
  YQ_TRY(d2h_sync(host.data(), states, host.size(), s));
  int status = YQ_OK;
  for (int g = 0; g < count; ++g) {
    Acc* st = reinterpret_cast<Acc*>(host.data() + (size_t)g * kAggStateBytes);
    if (*agg_state_err(st)) status = YQ_ERR_TIMEOUT;
    for (int a = 0; a < nagg; ++a) {
      const Acc& h = st[a];
      yq_agg_result& r = out[(size_t)g * nagg + a];
      const int kind = aggs[a].kind, t = aggs[a].input_type;
      const bool flt = (t == YQ_FLOAT32 || t == YQ_FLOAT64);
      double hf;
      memcpy(&hf, &h.bits, sizeof(hf));
      const long long hi = (long long)h.bits;
      r.kind = kind;
      r.count = h.cnt;
      r.i = 0;
      r.f = 0.0;
      r.is_null = 0;
      if (kind == YQ_AGG_COUNT_STAR || kind == YQ_AGG_COUNT) {
        r.i = h.cnt;
      } else if (kind == YQ_AGG_AVG) {
        r.is_null = h.cnt == 0;
        if (h.cnt) r.f = flt ? hf / (double)h.cnt : (double)hi / (double)h.cnt;
      } else {
        r.is_null = h.cnt == 0;
        if (flt) r.f = hf;
        else r.i = hi;
      }
    }
  }
  return status;
}

// Steps of nseg ranges: at most one per kStepRows window a range touches.
static size_t ranges_steps_bound(const uint32_t* begin, const uint32_t* end, int nseg) {
  size_t t = 0;
  for (int g = 0; g < nseg; ++g)
    if (end[g] > begin[g]) t += ceil_div<uint32_t>(end[g], kStepRows) - begin[g] / kStepRows;
  return t;
}

static size_t ranges_ws(size_t steps, int nseg) {
  WsSize w;
  w.add<uint32_t>((size_t)nseg + 1);
  w.add<uint32_t>((size_t)nseg + 1);
  w.add<uint32_t>((size_t)nseg + 1);
  w.add<Acc>((steps ? steps : 1) * YQ_MAX_AGGREGATES);
  w.add<uint32_t>(4);
  return w.total();
}

static int filter_aggregate_ranges(const yq_batch* batch, const uint32_t* begin, const uint32_t* end, int32_t nseg,
                                   const yq_program* predicate, const yq_constants* constants,
                                   const yq_agg_spec* aggs, int32_t nagg, void* states, void* workspace,
                                   size_t workspace_bytes, cudaStream_t s) {
  if (!batch || !states || nseg < 0 || (nseg > 0 && (!begin || !end))) return YQ_ERR_INVALID_ARG;
  if (nseg == 0) return YQ_OK;
  for (int g = 0; g < nseg; ++g)
    if (end[g] < begin[g] || end[g] > batch->rows) return YQ_ERR_INVALID_ARG;
  FASegParams Q;
  memset(&Q, 0, sizeof(Q));
  YQ_TRY(prepare_filter_aggregate(batch, predicate, constants, aggs, nagg, &Q.F));
  if (nagg == 0) return YQ_OK;
  std::vector<uint32_t> step0;
  const uint32_t nsteps = seg_steps(begin, end, nseg, step0);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, ranges_ws(nsteps, nseg), s));
  uint32_t* d_begin = ws.take<uint32_t>((size_t)nseg + 1);
  uint32_t* d_end = ws.take<uint32_t>((size_t)nseg + 1);
  uint32_t* d_step0 = ws.take<uint32_t>((size_t)nseg + 1);
  Acc* partials = ws.take<Acc>((nsteps ? nsteps : 1) * (size_t)YQ_MAX_AGGREGATES);
  uint32_t* d_err = ws.take<uint32_t>(4);
  YQ_TRY(h2d_async(d_begin, begin, (size_t)nseg * sizeof(uint32_t), s));
  YQ_TRY(h2d_async(d_end, end, (size_t)nseg * sizeof(uint32_t), s));
  YQ_TRY(h2d_async(d_step0, step0.data(), ((size_t)nseg + 1) * sizeof(uint32_t), s));
  YQ_TRY_CUDA(cudaMemsetAsync(d_err, 0, 4 * sizeof(uint32_t), s));
  Q.seg = d_begin;
  Q.seg_end = d_end;
  Q.step0 = d_step0;
  Q.nseg = nseg;
  Q.nsteps = nsteps;
  Q.partials = partials;
  Q.err = d_err;
  if (nsteps > 0) {
    const bool staged = Q.F.SP.nstages > 0;
    const void* kern =
        staged ? (const void*)k_filter_aggregate_seg<true> : (const void*)k_filter_aggregate_seg<false>;
    const size_t smem = stage_smem_bytes(Q.F.SP);
    YQ_TRY(kernel_allow_smem(kern, smem));
    const int grid = resident_grid(kern, smem, nsteps);
    double rows = 0;
    for (int g = 0; g < nseg; ++g) rows += end[g] - begin[g];
    const void* jk = jit_kernel(JIT_FILTER_AGG_SEG, staged, Q.F.P, Q.F.pc_end, Q.F.pc_end);
    ProfScope ps("filter_aggregate_seg", s, rows * row_bytes_of(Q.F.P, program_columns(Q.F.P, Q.F.pc_end, 0)));
    if (jk) {
      if (staged) Q.F.SP.nstages = jit_stages(jk, Q.F.SP.stage_bytes, Q.F.SP.nstages);
      void* args[] = {&Q};
      YQ_TRY(jit_launch(jk, (int)max_row_grid(), nsteps, stage_smem_bytes(Q.F.SP), args, s));
    } else if (staged)
      k_filter_aggregate_seg<true><<<grid, kRowBlock, smem, s>>>(Q);
    else
      k_filter_aggregate_seg<false><<<grid, kRowBlock, 0, s>>>(Q);
    YQ_CHECK_LAUNCH();
  }
  k_agg_seg_fold<<<nseg, kFoldBlock, 0, s>>>(partials, d_step0, nseg, Q.F.A, static_cast<Acc*>(states), d_err);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

size_t yq_filter_aggregate_segments_workspace_size(uint32_t rows, int32_t nseg) {
  if (nseg < 0) return 0;
  // every range touches at most one window more than its rows fill
  return ranges_ws((size_t)ceil_div<uint32_t>(rows, kStepRows) + (size_t)nseg, nseg);
}

int yq_filter_aggregate_segments(const yq_batch* batch, const uint32_t* seg_offsets, int32_t nseg,
                                 const yq_program* predicate, const yq_constants* constants, const yq_agg_spec* aggs,
                                 int32_t nagg, void* states, void* workspace, size_t workspace_bytes, void* stream) {
  if (!batch || nseg < 0 || (nseg > 0 && !seg_offsets)) return YQ_ERR_INVALID_ARG;
  if (nseg == 0) return YQ_OK;
  if (seg_offsets[0] != 0) return YQ_ERR_INVALID_ARG;
  return filter_aggregate_ranges(batch, seg_offsets, seg_offsets + 1, nseg, predicate, constants, aggs, nagg, states,
                                 workspace, workspace_bytes, as_stream(stream));
}

size_t yq_filter_aggregate_ranges_workspace_size(const uint32_t* begin, const uint32_t* end, int32_t nseg) {
  if (nseg < 0 || (nseg > 0 && (!begin || !end))) return 0;
  return ranges_ws(ranges_steps_bound(begin, end, nseg), nseg);
}

int yq_filter_aggregate_ranges(const yq_batch* batch, const uint32_t* begin, const uint32_t* end, int32_t nseg,
                               const yq_program* predicate, const yq_constants* constants, const yq_agg_spec* aggs,
                               int32_t nagg, void* states, void* workspace, size_t workspace_bytes, void* stream) {
  return filter_aggregate_ranges(batch, begin, end, nseg, predicate, constants, aggs, nagg, states, workspace,
                                 workspace_bytes, as_stream(stream));
}

size_t yq_filter_project_workspace_size(uint32_t rows) {
  WsSize w;
  w.add<unsigned long long>((size_t)ceil_div<uint32_t>(rows, kStepRows) + 1);
  w.add<uint32_t>(4);
  return w.total();
}

int yq_filter_project(const yq_batch* batch, const yq_program* predicate, const yq_constants* constants,
                      const yq_projection* proj, int32_t nproj, yq_column* out, uint32_t capacity,
                      uint32_t* count_device, uint32_t* count_host, void* workspace, size_t workspace_bytes,
                      void* stream) {
  cudaStream_t s = as_stream(stream);
  FPParams F;
  YQ_TRY(build_project_params(batch, predicate, constants, proj, nproj, out, capacity, F));
  const uint32_t rows = batch->rows;
  if (rows == 0) {
    if (count_device) YQ_TRY_CUDA(cudaMemsetAsync(count_device, 0, sizeof(uint32_t), s));
    if (count_host) *count_host = 0;
    return YQ_OK;
  }
  const uint32_t ntiles = ceil_div<uint32_t>(rows, kStepRows);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_filter_project_workspace_size(rows), s));
  unsigned long long* status = ws.take<unsigned long long>((size_t)ntiles + 1);
  uint32_t* misc = ws.take<uint32_t>(4);  // [0] chunk counter, [1] error, [2] count
  YQ_TRY_CUDA(cudaMemsetAsync(status, 0, ((size_t)ntiles + 1) * sizeof(unsigned long long), s));
  YQ_TRY_CUDA(cudaMemsetAsync(misc, 0, 4 * sizeof(uint32_t), s));
  uint32_t* cnt_dev = count_device ? count_device : misc + 2;
  YQ_TRY(launch_filter_project(F, rows, misc, status, cnt_dev, s));
  if (count_host) {
    uint32_t h[2];
    YQ_TRY(d2h_sync(&h[0], cnt_dev, sizeof(uint32_t), s));
    YQ_TRY(d2h_sync(&h[1], misc + 1, sizeof(uint32_t), s));
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
// (chunk counter, error word, row count, spare), then one 64-bit look-back
// status word per 1,024-row step plus one (a chunk of steps uses one).
#include <cuda.h>
#include <mutex>

namespace yq {

constexpr uint32_t kNoAllocTiles = YQ_FILTER_PROJECT_NOALLOC_MAX_ROWS / kStepRows;
constexpr size_t kNoAllocWords = 2 + (size_t)kNoAllocTiles + 1;  // 2 words hold the four counters

static __device__ __align__(256) unsigned long long g_filter_project_scratch[kNoAllocWords];

// Identity of the calling thread's current CUDA context, unique for the life
// of the process (cuCtxGetId, reached through the runtime's driver entry
// points so the library needs no link against the driver library); 0 when
// no context is current or the driver does not offer it.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

static unsigned long long current_context_id() {
  static std::once_flag once;
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array (host code only sees a host-side
// stand-in for the symbol). Looked up with the device current, once per
// device and context: after a device reset the device gets a new context in
// which the array may live elsewhere, so a changed context id (or none known)
// triggers a new lookup.
static int noalloc_scratch(unsigned long long** out) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  static unsigned long long ctx[64] = {0};
  int dev = 0;
  YQ_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return YQ_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(mu);
  const unsigned long long id = current_context_id();
  if (!addr[dev] || id == 0 || id != ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_filter_project_scratch);
    if (e != cudaSuccess || !p) {
      set_cuda_error(e);
      return YQ_ERR_CUDA;
    }
    addr[dev] = p;
    ctx[dev] = current_context_id();  // the lookup made the device's context current
  }
  *out = static_cast<unsigned long long*>(addr[dev]);
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
  const uint32_t ntiles = ceil_div<uint32_t>(rows, kStepRows);
  uint32_t* misc = reinterpret_cast<uint32_t*>(scratch);  // [0] chunk counter, [1] error, [2] count
  unsigned long long* status = scratch + 2;
  // The previous call's values are still there: clear what this call reads.
  YQ_TRY_CUDA(cudaMemsetAsync(scratch, 0, (2 + (size_t)ntiles + 1) * sizeof(unsigned long long), s));
  uint32_t* cnt_dev = count_device ? count_device : misc + 2;
  // the library's own kernel: loading a program-specialised one would allocate
  YQ_TRY(launch_filter_project(F, rows, misc, status, cnt_dev, s, false));
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
