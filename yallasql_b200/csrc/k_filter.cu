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
#include <vector>
#include "vm_host.cuh"
#include "yq_agg.cuh"
#include "yq_lookback.cuh"
#include "yq_stage.cuh"

namespace yq {

static int occupancy_grid(const void* kernel, int block, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * sm_count();
}

// Raise a kernel's dynamic shared memory limit (once per size) to `smem`.
static int allow_smem(const void* kernel, size_t smem, size_t& done) {
  if (smem > 48 * 1024 && smem > done) {
    YQ_TRY_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    done = smem;
  }
  return YQ_OK;
}

// Persistent grid of a row kernel: resident blocks, no more than the steps.
struct GridCache {
  int cap = 0;
  size_t smem = (size_t)-1;
  int grid(const void* kernel, size_t dyn_smem, uint32_t steps) {
    if (smem != dyn_smem) {
      cap = occupancy_grid(kernel, kRowBlock, dyn_smem);
      smem = dyn_smem;
    }
    int g = (int)(steps < (uint32_t)cap ? steps : (uint32_t)cap);
    return g < 1 ? 1 : g;
  }
};

static size_t max_row_grid() { return (size_t)sm_count() * 8; }

// ================================================================ aggregate
struct FAParams {
  VmProgram P;
  StagePlan SP;
  int32_t pc_end;
  AggParams A;
};

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
  uint32_t* err = agg_state_err(state);
  AggEmit E;
  agg_thread_init(E, F.A);
  uint32_t nsel = 0;
  const uint32_t ntiles = ceil_div<uint32_t>(n, kStepRows);
  const uint32_t G = gridDim.x;
  int S = 1;
  if constexpr (STAGED) {
    S = F.SP.nstages;
    stage_init(F.SP);
    if (threadIdx.x == 0)
      for (int j = 0; j < S - 1; ++j) {
        const uint32_t t = blockIdx.x + (uint32_t)j * G;
        if (t < ntiles) stage_start(F.SP, j, t * kStepRows, step_rows(t, n));
      }
  }
  int slot = 0;
  uint32_t parity = 0;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += G) {
    Ctx X;
    X.tile0 = tile * kStepRows;
    X.lr = threadIdx.x * ITEMS;
    X.inr = in_range_bits(X.tile0 + X.lr, n);
    X.stage = 0;
    X.vec_ok = (X.tile0 & 15u) == 0u;
    if constexpr (STAGED) {
      __syncthreads();  // every thread is done with the previous step: its slot is free
      if (threadIdx.x == 0) {
        const uint32_t t = tile + (uint32_t)(S - 1) * G;
        const int ns = slot == 0 ? S - 1 : slot - 1;
        if (t < ntiles) stage_start(F.SP, ns, t * kStepRows, step_rows(t, n));
      }
      stage_finish(F.SP, slot, parity, X.tile0, step_rows(tile, n), err);
      X.stage = (uint32_t)slot * F.SP.stage_bytes;
    }
    E.sel = X.inr;
    Stack St;
    run_vm<STAGED>(F.P, 0, F.pc_end, X, St, E);
    nsel += __popc(E.sel);
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
  agg_block_finish<kRowBlock>(E, nsel, F.A, partials, ticket, state);
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

static int launch_filter_aggregate(const FAParams& F, uint32_t rows, Acc* partials, uint32_t* ticket, Acc* state,
                                   cudaStream_t s) {
  const bool staged = F.SP.nstages > 0;
  const void* kern = staged ? (const void*)k_filter_aggregate<true> : (const void*)k_filter_aggregate<false>;
  const size_t smem = stage_smem_bytes(F.SP);
  static size_t done_smem = 0;
  YQ_TRY(allow_smem(kern, smem, done_smem));
  static GridCache gc[2];
  int grid = gc[staged ? 1 : 0].grid(kern, smem, ceil_div<uint32_t>(rows, kStepRows));
  if ((size_t)grid > max_row_grid()) grid = (int)max_row_grid();
  ProfScope ps("filter_aggregate", s, (double)rows * row_bytes_of(F.P, program_columns(F.P, F.pc_end, 0)));
  if (staged)
    k_filter_aggregate<true><<<grid, kRowBlock, smem, s>>>(F, rows, partials, ticket, state);
  else
    k_filter_aggregate<false><<<grid, kRowBlock, 0, s>>>(F, rows, partials, ticket, state);
  YQ_CHECK_LAUNCH();
  return YQ_OK;
}

// ======================================================= segmented aggregate
// Many independent filter+aggregate tasks in one launch: task g owns rows
// [seg[g], seg[g+1]) of the batch and its own aggregate state. Steps never
// straddle tasks; the persistent blocks walk the steps of all tasks as one
// queue (step -> task by binary search over the tasks' first steps), write
// one partial per step, and k_agg_seg_fold folds each task's partials in step
// order, so every task's result is deterministic and equal to the result of
// running it alone.
struct FASegParams {
  FAParams F;
  const uint32_t* seg;    // [nseg] first row of each task
  const uint32_t* seg_end;  // [nseg] end row of each task
  const uint32_t* step0;  // [nseg + 1] first step of each task
  int32_t nseg;
  uint32_t nsteps;
  Acc* partials;          // [nsteps][YQ_MAX_AGGREGATES]
  uint32_t* err;
};

__device__ __forceinline__ int seg_of_step(const uint32_t* step0, int nseg, uint32_t t) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(step0 + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Step t: task g's rows within the absolute step window of t (windows are
// kStepRows-aligned, so only a task's first and last steps are partial).
__device__ __forceinline__ void seg_step(const FASegParams& Q, uint32_t t, uint32_t& row0, uint32_t& rows) {
  const int g = seg_of_step(Q.step0, Q.nseg, t);
  const uint32_t s = __ldg(Q.seg + g), e = __ldg(Q.seg_end + g);
  const uint64_t base = ((uint64_t)(s / kStepRows) + (t - __ldg(Q.step0 + g))) * kStepRows;
  const uint64_t lo = base > s ? base : s;
  const uint64_t hi = base + kStepRows < e ? base + kStepRows : e;
  row0 = (uint32_t)lo;
  rows = (uint32_t)(hi - lo);
}

template <bool STAGED>
__global__ void __launch_bounds__(kRowBlock, 2) k_filter_aggregate_seg(const __grid_constant__ FASegParams Q) {
  const FAParams& F = Q.F;
  const uint32_t G = gridDim.x;
  int S = 1;
  if constexpr (STAGED) {
    S = F.SP.nstages;
    stage_init(F.SP);
    if (threadIdx.x == 0)
      for (int j = 0; j < S - 1; ++j) {
        const uint32_t t = blockIdx.x + (uint32_t)j * G;
        if (t < Q.nsteps) {
          uint32_t r0, nr;
          seg_step(Q, t, r0, nr);
          stage_start(F.SP, j, r0, nr);
        }
      }
  }
  int slot = 0;
  uint32_t parity = 0;
  for (uint32_t t = blockIdx.x; t < Q.nsteps; t += G) {
    uint32_t row0, rows;
    seg_step(Q, t, row0, rows);
    Ctx X;
    X.tile0 = row0;
    X.lr = threadIdx.x * ITEMS;
    X.inr = in_range_bits(X.lr, rows);
    X.stage = 0;
    X.vec_ok = (X.tile0 & 15u) == 0u;
    if constexpr (STAGED) {
      __syncthreads();  // every thread is done with the previous step: its slot is free
      if (threadIdx.x == 0) {
        const uint32_t tn = t + (uint32_t)(S - 1) * G;
        const int ns = slot == 0 ? S - 1 : slot - 1;
        if (tn < Q.nsteps) {
          uint32_t r0, nr;
          seg_step(Q, tn, r0, nr);
          stage_start(F.SP, ns, r0, nr);
        }
      }
      stage_finish(F.SP, slot, parity, row0, rows, Q.err);
      X.stage = (uint32_t)slot * F.SP.stage_bytes;
    }
    AggEmit E;
    agg_thread_init(E, F.A);
    E.sel = X.inr;
    Stack St;
    run_vm<STAGED>(F.P, 0, F.pc_end, X, St, E);
    agg_block_partial<kRowBlock>(E, __popc(E.sel), F.A, Q.partials + (size_t)t * YQ_MAX_AGGREGATES);
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
}

// One warp per task: aggregate a < nagg folds the task's step partials in order.
__global__ void k_agg_seg_fold(const Acc* __restrict__ partials, const uint32_t* __restrict__ step0, int nseg,
                               const AggParams A, Acc* states, const uint32_t* err) {
  const int g = blockIdx.x;
  const int a = threadIdx.x;
  if (g >= nseg) return;
  Acc* st = reinterpret_cast<Acc*>(reinterpret_cast<char*>(states) + (size_t)g * kAggStateBytes);
  if (a == 0 && *err) *agg_state_err(st) |= *err;
  if (a >= A.nagg) return;
  const int upd = A.upd[a];
  Acc t{0, acc_identity(upd)};
  for (uint32_t s = step0[g]; s < step0[g + 1]; ++s) {
    const Acc p = partials[(size_t)s * YQ_MAX_AGGREGATES + a];
    t.cnt += p.cnt;
    t.bits = acc_merge(upd, t.bits, p.bits);
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
struct DevOut {
  char* data;
  uint8_t* nulls;
  int32_t width;
  int32_t src_col;  // >= 0: copy of this input column
};

struct FPParams {
  VmProgram P;
  StagePlan SP;
  int32_t pred_end;
  int32_t proj_end;
  int32_t nproj;
  uint32_t capacity;
  DevOut out[YQ_MAX_PROJECTIONS];
};

struct ProjEmit {
  uint32_t sel;
  uint32_t pos;
  const FPParams* F;
  __device__ __forceinline__ void pred(uint32_t bits) { sel &= bits; }
  template <int K>
  __device__ __forceinline__ void agg(int, const Val&) {}
  template <int W>
  __device__ __forceinline__ void proj(int p, const Val& x) {
    const DevOut& o = F->out[p];
    uint32_t q = pos;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if (sel >> k & 1u) {
        if (q < F->capacity) {
          if constexpr (W == 0) reinterpret_cast<uint8_t*>(o.data)[q] = (uint8_t)((x.v[0] >> k) & 1u);
          else if constexpr (W == 1) reinterpret_cast<uint32_t*>(o.data)[q] = (uint32_t)x.v[k];
          else reinterpret_cast<unsigned long long*>(o.data)[q] = x.v[k];
          if (o.nulls) o.nulls[q] = (x.valid >> k & 1u) ? 0 : 1;
        }
        ++q;
      }
    }
  }
};

// One cell of `width` bytes; `src` is shared or global memory (generic).
__device__ __forceinline__ void copy_cell_any(char* dst, const char* src, int width) {
  if (width == 4) {
    *reinterpret_cast<uint32_t*>(dst) = *reinterpret_cast<const uint32_t*>(src);
  } else if (width == 8) {
    *reinterpret_cast<unsigned long long*>(dst) = *reinterpret_cast<const unsigned long long*>(src);
  } else if (width == 1) {
    *dst = *src;
  } else if ((width & 15) == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
    for (int i = 0; i < width; i += 16)
      *reinterpret_cast<uint4*>(dst + i) = *reinterpret_cast<const uint4*>(src + i);
  } else {
    for (int i = 0; i < width; i += 4)
      *reinterpret_cast<uint32_t*>(dst + i) = *reinterpret_cast<const uint32_t*>(src + i);
  }
}

// Projections that copy an input column: selected rows to positions pos, pos+1, ...
template <bool STAGED>
__device__ __forceinline__ void copy_source_columns(const FPParams& F, const Ctx& X, uint32_t sel, uint32_t pos) {
  for (int p = 0; p < F.nproj; ++p) {
    const DevOut& o = F.out[p];
    if (o.src_col < 0) continue;
    const DevCol& c = F.P.cols[o.src_col];
    uint32_t q = pos;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if (sel >> k & 1u) {
        if (q < F.capacity) {
          const uint32_t lr = X.lr + k;
          const char* src;
          uint8_t nul = 0;
          if constexpr (STAGED) {
            src = reinterpret_cast<const char*>(yq_dyn_smem + X.stage + c.soff + lr * (uint32_t)c.width);
            if (c.nulls) nul = yq_dyn_smem[X.stage + c.snoff + lr];
          } else {
            src = c.data + (size_t)(X.tile0 + lr) * c.width;
            if (c.nulls) nul = c.nulls[X.tile0 + lr];
          }
          copy_cell_any(o.data + (size_t)q * o.width, src, c.width);
          if (o.nulls) o.nulls[q] = nul;
        }
        ++q;
      }
    }
  }
}

// Tiles are claimed in order from a counter (a few steps ahead when staged),
// every block processes its claims in order, so each tile's predecessors are
// held by running blocks and the decoupled look-back always completes.
template <bool STAGED>
__global__ void __launch_bounds__(kRowBlock, 2) k_filter_project(const __grid_constant__ FPParams F, uint32_t n,
                                                                 uint32_t* tile_counter,
                                                                 unsigned long long* __restrict__ status,
                                                                 uint32_t* out_count, uint32_t* err) {
  __shared__ uint32_t s_tiles[kStageMax];
  __shared__ uint32_t s_warp[kRowBlock / 32 + 1];
  __shared__ unsigned long long s_prefix;
  const uint32_t ntiles = ceil_div<uint32_t>(n, kStepRows);
  int S = 1;
  if constexpr (STAGED) {
    S = F.SP.nstages;
    stage_init(F.SP);
  }
  if (threadIdx.x == 0)
    for (int j = 0; j < S - 1; ++j) {
      const uint32_t t = atomicAdd(tile_counter, 1u);
      s_tiles[j] = t;
      if constexpr (STAGED)
        if (t < ntiles) stage_start(F.SP, j, t * kStepRows, step_rows(t, n));
    }
  int slot = 0;
  uint32_t parity = 0;
  for (;;) {
    __syncthreads();  // every thread is done with the previous step
    if (threadIdx.x == 0) {
      const int ns = slot == 0 ? S - 1 : slot - 1;
      const uint32_t t = atomicAdd(tile_counter, 1u);
      s_tiles[ns] = t;
      if constexpr (STAGED)
        if (t < ntiles) stage_start(F.SP, ns, t * kStepRows, step_rows(t, n));
    }
    __syncthreads();
    const uint32_t tile = s_tiles[slot];
    if (tile >= ntiles) break;  // later claims are larger: no copy is in flight
    Ctx X;
    X.tile0 = tile * kStepRows;
    X.lr = threadIdx.x * ITEMS;
    X.inr = in_range_bits(X.tile0 + X.lr, n);
    X.stage = 0;
    X.vec_ok = (X.tile0 & 15u) == 0u;
    if constexpr (STAGED) {
      stage_finish(F.SP, slot, parity, X.tile0, step_rows(tile, n), err);
      X.stage = (uint32_t)slot * F.SP.stage_bytes;
    }
    ProjEmit E;
    E.sel = X.inr;
    E.pos = 0;
    E.F = &F;
    Stack St;
    if (F.pred_end > 0) run_vm<STAGED>(F.P, 0, F.pred_end, X, St, E);

    uint32_t total;
    const uint32_t excl = block_exclusive_sum<kRowBlock>(__popc(E.sel), s_warp, total);
    if (threadIdx.x < 32) {
      const unsigned long long p = tile_lookback(status, tile, total, err);
      if (threadIdx.x == 0) s_prefix = p;
    }
    __syncthreads();
    const unsigned long long base = s_prefix;
    E.pos = (uint32_t)(base + excl);
    if (F.proj_end > F.pred_end) run_vm<STAGED>(F.P, F.pred_end, F.proj_end, X, St, E);
    copy_source_columns<STAGED>(F, X, E.sel, E.pos);
    if (tile == ntiles - 1 && threadIdx.x == 0) {
      const unsigned long long cnt = base + total;
      *out_count = cnt > 0xffffffffull ? 0xffffffffu : (uint32_t)cnt;
    }
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
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
  if (!plan_stages(B.P, B.used_cols | copy_mask, F.SP)) F.SP.nstages = 0;
  memcpy(&F.P, &B.P, sizeof(VmProgram));
  F.pred_end = B.remap[pred_end];
  F.proj_end = B.len;
  F.nproj = nproj;
  F.capacity = capacity;
  return YQ_OK;
}

// Launch over `rows` rows with look-back scratch `status` (one word per tile
// plus one) and `misc` = {tile counter, error word} (both zeroed).
static int launch_filter_project(const FPParams& F, uint32_t rows, uint32_t* misc, unsigned long long* status,
                                 uint32_t* cnt_dev, cudaStream_t s) {
  const bool staged = F.SP.nstages > 0;
  const void* kern = staged ? (const void*)k_filter_project<true> : (const void*)k_filter_project<false>;
  const size_t smem = stage_smem_bytes(F.SP);
  static size_t done_smem = 0;
  YQ_TRY(allow_smem(kern, smem, done_smem));
  static GridCache gc[2];
  const int grid = gc[staged ? 1 : 0].grid(kern, smem, ceil_div<uint32_t>(rows, kStepRows));
  uint32_t mask = program_columns(F.P, F.proj_end, 0);
  for (int p = 0; p < F.nproj; ++p)
    if (F.out[p].src_col >= 0) mask |= 1u << F.out[p].src_col;
  // algorithmic bytes: referenced input columns (outputs depend on selectivity)
  ProfScope ps("filter_project", s, (double)rows * row_bytes_of(F.P, mask));
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
  YQ_TRY_CUDA(
      cudaMemcpyAsync(host, state, sizeof(Acc) * YQ_MAX_AGGREGATES + sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  YQ_TRY_CUDA(cudaStreamSynchronize(s));
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
  YQ_TRY_CUDA(cudaMemcpyAsync(host.data(), states, host.size(), cudaMemcpyDeviceToHost, s));
  YQ_TRY_CUDA(cudaStreamSynchronize(s));
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
    static size_t done_smem = 0;
    YQ_TRY(allow_smem(kern, smem, done_smem));
    static GridCache gc[2];
    const int grid = gc[staged ? 1 : 0].grid(kern, smem, nsteps);
    double rows = 0;
    for (int g = 0; g < nseg; ++g) rows += end[g] - begin[g];
    ProfScope ps("filter_aggregate_seg", s, rows * row_bytes_of(Q.F.P, program_columns(Q.F.P, Q.F.pc_end, 0)));
    if (staged)
      k_filter_aggregate_seg<true><<<grid, kRowBlock, smem, s>>>(Q);
    else
      k_filter_aggregate_seg<false><<<grid, kRowBlock, 0, s>>>(Q);
    YQ_CHECK_LAUNCH();
  }
  k_agg_seg_fold<<<nseg, 32, 0, s>>>(partials, d_step0, nseg, Q.F.A, static_cast<Acc*>(states), d_err);
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
  uint32_t* misc = ws.take<uint32_t>(4);  // [0] tile counter, [1] error, [2] count
  YQ_TRY_CUDA(cudaMemsetAsync(status, 0, ((size_t)ntiles + 1) * sizeof(unsigned long long), s));
  YQ_TRY_CUDA(cudaMemsetAsync(misc, 0, 4 * sizeof(uint32_t), s));
  uint32_t* cnt_dev = count_device ? count_device : misc + 2;
  YQ_TRY(launch_filter_project(F, rows, misc, status, cnt_dev, s));
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

constexpr uint32_t kNoAllocTiles = YQ_FILTER_PROJECT_NOALLOC_MAX_ROWS / kStepRows;
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
  uint32_t* misc = reinterpret_cast<uint32_t*>(scratch);  // [0] tile counter, [1] error, [2] count
  unsigned long long* status = scratch + 2;
  // The previous call's values are still there: clear what this call reads.
  YQ_TRY_CUDA(cudaMemsetAsync(scratch, 0, (2 + (size_t)ntiles + 1) * sizeof(unsigned long long), s));
  uint32_t* cnt_dev = count_device ? count_device : misc + 2;
  YQ_TRY(launch_filter_project(F, rows, misc, status, cnt_dev, s));
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
