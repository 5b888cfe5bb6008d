// Bodies of the row kernels that run an expression program: filter +
// aggregate, segmented filter + aggregate, filter + projection and the fused
// star-join aggregate (sm_100a).
//
// Each body is a device template over a program runner R. The library's
// kernels (k_filter.cu, k_join.cu) instantiate it with InterpRunner, which
// dispatches on the program's resolved opcodes at run time; a program-
// specialised kernel (jit.cu) instantiates the same body with a runner whose
// instruction list is compile-time constant, so the dispatch and the stack
// moves fold away and only the operations remain.
#pragma once

#include "yq_agg.cuh"
#include "yq_hash.cuh"
#include "yq_lookback.cuh"
#include "yq_stage.cuh"

namespace yq {

// Runs instructions [begin, end) of segment `seg` (0 = the predicate or the
// whole program, 1 = what follows the predicate) through the opcode switch.
struct FPParams;
struct ProjEmit;
template <bool STAGED>
__device__ __forceinline__ void copy_source_columns(const FPParams& F, const Ctx& X, const ProjEmit& E);

struct InterpRunner {
  template <bool STAGED, typename Emit>
  __device__ __forceinline__ static void run(const VmProgram& P, int seg, int begin, int end, const Ctx& X, Stack& S,
                                             Emit& E) {
    (void)seg;
    run_vm<STAGED>(P, begin, end, X, S, E);
  }
  // WHERE + projection: the projections that copy a source column.
  template <bool STAGED>
  __device__ __forceinline__ static void copies(const FPParams& F, const Ctx& X, const ProjEmit& E) {
    copy_source_columns<STAGED>(F, X, E);
  }
};

// ================================================================ aggregate
struct FAParams {
  VmProgram P;
  StagePlan SP;
  int32_t pc_end;
  AggParams A;
};

template <bool STAGED, typename R>
__device__ __forceinline__ void filter_aggregate_body(const FAParams& F, uint32_t n,
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
    R::template run<STAGED>(F.P, 0, 0, F.pc_end, X, St, E);
    nsel += __popc(E.sel);
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
  agg_block_finish<kRowBlock>(E, nsel, F.A, partials, ticket, state);
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

template <bool STAGED, typename R>
__device__ __forceinline__ void filter_aggregate_seg_body(const FASegParams& Q) {
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
    R::template run<STAGED>(F.P, 0, 0, F.pc_end, X, St, E);
    agg_block_partial<kRowBlock>(E, __popc(E.sel), F.A, Q.partials + (size_t)t * YQ_MAX_AGGREGATES);
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
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
  uint32_t csteps;  // 1,024-row steps per claimed chunk (1..8)
  DevOut out[YQ_MAX_PROJECTIONS];
};

// One warp's lists in the output pass: its selected rows in input order (row
// within the step) and, for the projection program being emitted, their values.
struct WarpOut {
  uint16_t rows[ITEMS * 32];
  unsigned long long vals[ITEMS * 32];
  uint8_t ok[ITEMS * 32];
};

// Output rows of a warp are consecutive: entry i of its lists goes to output
// row wbase + i, written by lane i % 32, so a warp's stores are coalesced
// whatever rows were selected.
struct ProjEmit {
  uint32_t sel;
  uint32_t pos;  // this thread's first output row
  const FPParams* F;
  WarpOut* W;             // this warp's lists (output pass only)
  uint32_t wbase, wcount;  // the warp's first output row and its selected rows
  uint32_t first;         // this thread's first entry in the lists
  __device__ __forceinline__ void pred(uint32_t bits) { sel &= bits; }
  template <int K>
  __device__ __forceinline__ void agg(int, const Val&) {}
  template <int WD>
  __device__ __forceinline__ void proj(int p, const Val& x) {
    const DevOut& o = F->out[p];
    uint32_t e = first;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if (sel >> k & 1u) {
        W->vals[e] = WD == 0 ? ((x.v[0] >> k) & 1u) : x.v[k];
        W->ok[e] = (uint8_t)((x.valid >> k) & 1u);
        ++e;
      }
    }
    __syncwarp();
    const uint32_t cap = F->capacity;
    for (uint32_t i = threadIdx.x & 31u; i < wcount; i += 32) {
      const uint32_t q = wbase + i;
      if (q >= cap) break;
      if constexpr (WD == 0) reinterpret_cast<uint8_t*>(o.data)[q] = (uint8_t)W->vals[i];
      else if constexpr (WD == 1) reinterpret_cast<uint32_t*>(o.data)[q] = (uint32_t)W->vals[i];
      else reinterpret_cast<unsigned long long*>(o.data)[q] = W->vals[i];
      if (o.nulls) o.nulls[q] = W->ok[i] ? 0 : 1;
    }
    __syncwarp();
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

// Projections that copy an input column: the warp's selected rows (listed in
// E.W->rows) to output rows E.wbase, E.wbase + 1, ..., lane i % 32 copying
// entry i.
template <bool STAGED>
__device__ __forceinline__ void copy_source_columns(const FPParams& F, const Ctx& X, const ProjEmit& E) {
  for (int p = 0; p < F.nproj; ++p) {
    const DevOut& o = F.out[p];
    if (o.src_col < 0) continue;
    const DevCol& c = F.P.cols[o.src_col];
    const uint32_t w = (uint32_t)c.width;
    for (uint32_t i = threadIdx.x & 31u; i < E.wcount; i += 32) {
      const uint32_t q = E.wbase + i;
      if (q >= F.capacity) break;
      const uint32_t lr = E.W->rows[i];
      const char* src;
      uint8_t nul = 0;
      if constexpr (STAGED) {
        src = reinterpret_cast<const char*>(yq_dyn_smem + X.stage + c.soff + lr * w);
        if (c.nulls) nul = yq_dyn_smem[X.stage + c.snoff + lr];
      } else {
        src = c.data + (size_t)(X.tile0 + lr) * w;
        if (c.nulls) nul = c.nulls[X.tile0 + lr];
      }
      copy_cell_any(o.data + (size_t)q * w, src, (int)w);
      if (o.nulls) o.nulls[q] = nul;
    }
  }
}

// One projection that copies source column C (W-byte cells) to output P, as
// copy_source_columns does for all of them; ON / SN: the output / the source
// has null bytes. The program-specialised kernels list their copies with
// these as compile-time constants.
template <bool STAGED, int P, int C, int W, bool ON, bool SN>
__device__ __forceinline__ void copy_column(const FPParams& F, const Ctx& X, const ProjEmit& E) {
  const DevOut& o = F.out[P];
  const DevCol& c = F.P.cols[C];
  for (uint32_t i = threadIdx.x & 31u; i < E.wcount; i += 32) {
    const uint32_t q = E.wbase + i;
    if (q >= F.capacity) break;
    const uint32_t lr = E.W->rows[i];
    const char* src;
    if constexpr (STAGED) src = reinterpret_cast<const char*>(yq_dyn_smem + X.stage + c.soff + lr * (uint32_t)W);
    else src = c.data + (size_t)(X.tile0 + lr) * W;
    copy_cell_any(o.data + (size_t)q * W, src, W);
    if constexpr (ON) {
      uint8_t nul = 0;
      if constexpr (SN) nul = STAGED ? yq_dyn_smem[X.stage + c.snoff + lr] : c.nulls[X.tile0 + lr];
      o.nulls[q] = nul;
    }
  }
}

// Rows are cut into chunks of F.csteps 1,024-row steps. Chunks are claimed in
// order from a counter (when the staging ring reaches the next one), and every
// block processes its claims in order, so each chunk's predecessors are held
// by running blocks and the decoupled look-back always completes.
//
// A chunk is 2 * csteps ring steps. The first csteps run the predicate over
// the staged predicate columns and keep each thread's 4 selection bits per
// step (at most 8 steps: one word). Then one block scan turns the per-step
// counts into output positions and one look-back gives the chunk's first
// output row, while the ring is already loading the same steps again with the
// columns the output reads (pass 1 of the stage plan; the chunk was just
// streamed, so these copies mostly hit L2). The last csteps run the
// projection programs and copy the source columns for the selected rows.
// Output rows keep input order.
template <bool STAGED, typename R>
__device__ __forceinline__ void filter_project_body(const FPParams& F, uint32_t n, uint32_t* chunk_counter,
                                                    unsigned long long* __restrict__ status, uint32_t* out_count,
                                                    uint32_t* err) {
  constexpr uint32_t Q = 8;  // claimed chunk ids kept: the current one through the one being prefetched
  __shared__ uint32_t s_claims[Q];
  __shared__ unsigned long long s_scan[2 * (kRowBlock / 32 + 1)];
  __shared__ unsigned long long s_prefix;
  __shared__ WarpOut s_out[kRowBlock / 32];
  const uint32_t nsteps = ceil_div<uint32_t>(n, kStepRows);
  const uint32_t C = F.csteps;  // 1..8
  const uint32_t V = 2 * C;     // ring steps per chunk
  const uint32_t nchunks = ceil_div<uint32_t>(nsteps, C);
  uint32_t S = 1;
  if constexpr (STAGED) {
    S = (uint32_t)F.SP.nstages;
    stage_init(F.SP);
  }
  // Thread 0: claim (at a chunk's first ring step) and start the copies of
  // the block's ring step pv: chunk number pv / V of this block, step
  // (pv % V) % C of it, pass (pv % V) / C.
  // The last chunk can end before its csteps: its missing steps of pass 0
  // come before its steps of pass 1, so each still completes its slot's
  // barrier phase (an arrive, no copy) and every slot keeps one phase per use.
  auto ahead = [&](uint32_t pv) {
    if (pv % V == 0) s_claims[(pv / V) % Q] = atomicAdd(chunk_counter, 1u);
    if constexpr (STAGED) {
      const uint32_t c = s_claims[(pv / V) % Q], r = pv % V, step = c * C + (r < C ? r : r - C);
      if (c < nchunks) {
        if (step < nsteps) stage_start(F.SP, (int)(pv % S), step * kStepRows, step_rows(step, n), r < C ? 0 : 1);
        else mbar_arrive(stage_bar(F.SP, (int)(pv % S)));
      }
    }
  };
  if (threadIdx.x == 0)
    for (uint32_t j = 0; j + 1 < S; ++j) ahead(j);
  uint32_t selmask = 0;
  unsigned long long ex_lo = 0, ex_hi = 0, tot_lo = 0, tot_hi = 0, run = 0;
  for (uint32_t v = 0;; ++v) {
    __syncthreads();  // every thread is done with the previous step: its slot is free
    if (threadIdx.x == 0) ahead(v + S - 1);
    if (S == 1) __syncthreads();  // the current chunk may have been claimed just now
    const uint32_t chunk = s_claims[(v / V) % Q];
    if (chunk >= nchunks) break;  // later claims are larger: no copy is in flight
    const uint32_t r = v % V, j = r < C ? r : r - C, step = chunk * C + j;
    const int pass = r < C ? 0 : 1;
    if (step < nsteps) {
      Ctx X;
      X.tile0 = step * kStepRows;
      X.lr = threadIdx.x * ITEMS;
      X.inr = in_range_bits(X.tile0 + X.lr, n);
      X.stage = 0;
      X.vec_ok = (X.tile0 & 15u) == 0u;
      if constexpr (STAGED) {
        const uint32_t slot = v % S;
        stage_finish(F.SP, (int)slot, (v / S) & 1u, X.tile0, step_rows(step, n), err, pass);
        X.stage = slot * F.SP.stage_bytes;
      }
      ProjEmit E;
      E.F = &F;
      E.W = nullptr;
      E.wbase = E.wcount = E.first = 0;
      Stack St;
      if (pass == 0) {
        E.sel = X.inr;
        E.pos = 0;
        if (F.pred_end > 0) R::template run<STAGED>(F.P, 0, 0, F.pred_end, X, St, E);
        selmask |= E.sel << (4 * j);
      } else {
        const uint32_t sh = 16u * (j & 3u);
        E.sel = (selmask >> (4 * j)) & 15u;
        E.pos = (uint32_t)(run + (((j < 4 ? ex_lo : ex_hi) >> sh) & 0xffffu));
        if (__any_sync(0xffffffffu, E.sel != 0u)) {
          E.W = &s_out[threadIdx.x >> 5];
          E.wbase = __shfl_sync(0xffffffffu, E.pos, 0);
          E.first = E.pos - E.wbase;
          E.wcount = __shfl_sync(0xffffffffu, E.first + (uint32_t)__popc(E.sel), 31);
          uint32_t e = E.first;
#pragma unroll
          for (int k = 0; k < ITEMS; ++k)
            if (E.sel >> k & 1u) E.W->rows[e++] = (uint16_t)(X.lr + k);
          __syncwarp();
          if (F.proj_end > F.pred_end) R::template run<STAGED>(F.P, 1, F.pred_end, F.proj_end, X, St, E);
          R::template copies<STAGED>(F, X, E);
        }
        run += ((j < 4 ? tot_lo : tot_hi) >> sh) & 0xffffu;
      }
    }
    if (r == C - 1) {
      // Predicate done for the chunk: per-step counts as 16-bit fields (steps
      // 0-3 in ex_lo, 4-7 in ex_hi), positions, look-back.
      ex_lo = ex_hi = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        ex_lo |= (unsigned long long)__popc((selmask >> (4 * k)) & 15u) << (16 * k);
        ex_hi |= (unsigned long long)__popc((selmask >> (4 * k + 16)) & 15u) << (16 * k);
      }
      block_exclusive_sum2<kRowBlock>(ex_lo, ex_hi, s_scan, tot_lo, tot_hi);
      unsigned long long total = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) total += ((tot_lo >> (16 * k)) & 0xffffu) + ((tot_hi >> (16 * k)) & 0xffffu);
      if (threadIdx.x < 32) {
        const unsigned long long p = tile_lookback(status, chunk, total, err);
        if (threadIdx.x == 0) s_prefix = p;
      }
      __syncthreads();
      run = s_prefix;
      if (chunk == nchunks - 1 && threadIdx.x == 0) {
        const unsigned long long cnt = run + total;
        *out_count = cnt > 0xffffffffull ? 0xffffffffu : (uint32_t)cnt;
      }
    }
    if (r == V - 1) selmask = 0;
  }
}

// ------------------------------------------------ fused star-join aggregate
struct JAParams {
  VmProgram P;  // fact predicate [0, pred_end) then aggregate inputs [pred_end, pc_end)
  StagePlan SP;
  int32_t pred_end, pc_end;
  AggParams A;
  int32_t fkey_col;  // fact key column (staged with the others when the ring is used)
  JCol fkey;
  uint32_t nbuckets, hrows_n;
  uint32_t table_off;  // byte offset of the dimension table in dynamic shared memory
  const uint32_t* bstart;
  const unsigned long long* hkeys;
};

// Normalised key from the raw bits of a cell (as hash_key).
__device__ __forceinline__ uint64_t norm_key(int type, uint64_t raw) {
  uint64_t v = raw;
  if (type == YQ_INT32) v = (uint64_t)(int64_t)(int32_t)(uint32_t)raw;
  if (type == YQ_FLOAT32 && ((uint32_t)v & 0x7fffffffu) == 0u) v = 0;
  if (type == YQ_FLOAT64 && (v & 0x7fffffffffffffffull) == 0ull) v = 0;
  return v;
}

template <bool STAGED, typename R>
__device__ __forceinline__ void join_aggregate_body(const JAParams& F, uint32_t n,
                                                                 Acc* __restrict__ partials, uint32_t* ticket,
                                                                 Acc* state) {
  uint32_t* s_bstart = reinterpret_cast<uint32_t*>(yq_dyn_smem + F.table_off);
  unsigned long long* s_keys =
      reinterpret_cast<unsigned long long*>(yq_dyn_smem + F.table_off + 4 * ((F.nbuckets + 2) & ~1u));
  for (uint32_t i = threadIdx.x; i <= F.nbuckets; i += kRowBlock) s_bstart[i] = __ldg(F.bstart + i);
  for (uint32_t i = threadIdx.x; i < F.hrows_n; i += kRowBlock) s_keys[i] = __ldg(F.hkeys + i);
  __syncthreads();

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
  const DevCol& kc = F.P.cols[F.fkey_col];
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
    if (F.pred_end > 0) R::template run<STAGED>(F.P, 0, 0, F.pred_end, X, St, E);
    // probe: keep rows whose key is present among the (unique) dimension keys
    const uint32_t knull = null_bits<STAGED>(kc, X);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if (!(E.sel >> k & 1u)) continue;
      bool hit = false;
      if (!(knull >> k & 1u)) {
        uint64_t key;
        if constexpr (STAGED) {
          const unsigned char* p = yq_dyn_smem + X.stage + kc.soff + (X.lr + k) * (uint32_t)kc.width;
          const uint64_t raw = kc.width == 8   ? *reinterpret_cast<const unsigned long long*>(p)
                               : kc.width == 4 ? (uint64_t)*reinterpret_cast<const uint32_t*>(p)
                                               : (uint64_t)*p;
          key = norm_key(kc.type, raw);
        } else {
          key = hash_key(F.fkey, X.tile0 + X.lr + k);
        }
        const uint32_t b = hash_bucket(key, F.nbuckets);
        for (uint32_t x = s_bstart[b]; x < s_bstart[b + 1] && !hit; ++x) hit = (s_keys[x] == key);
      }
      if (!hit) E.sel &= ~(1u << k);
    }
    R::template run<STAGED>(F.P, 1, F.pred_end, F.pc_end, X, St, E);
    nsel += __popc(E.sel);
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
  agg_block_finish<kRowBlock>(E, nsel, F.A, partials, ticket, state);
}

}  // namespace yq
