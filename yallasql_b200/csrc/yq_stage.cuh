// Shared-memory staging of column tiles for the row kernels (sm_100a).
//
// A block processes steps of kStepRows consecutive rows. The columns a
// program reads are laid out back to back in one stage (each column's
// kStepRows values, then its null bytes when it has them); a ring of 2-4
// stages in dynamic shared memory is filled by 1-D bulk copies
// (cp.async.bulk global -> shared, no multicast) that complete on one
// mbarrier per stage, so the copies of the next steps are in flight while the
// expression machine works on the current one. A step that is not full (the
// last rows of the batch) is copied with plain loads and zero padded.
#pragma once

#ifndef __CUDACC_RTC__
#include <string.h>
#endif
#include "yq_vm.cuh"

namespace yq {

constexpr int kRowBlock = 256;
constexpr uint32_t kStepRows = kRowBlock * ITEMS;  // 1024 rows per step
constexpr int kStageMax = 4;
// Dynamic shared memory one block may use for its ring (two blocks per SM).
constexpr size_t kStageBudget = 110 * 1024;

struct StageCopy {
  const char* src;     // first row of the column (16-byte aligned)
  uint32_t row_bytes;  // bytes per row
  uint32_t soff;       // offset in the stage
  uint32_t passes;     // bit p: copied on steps of pass p (a kernel that reads a step twice)
};

struct StagePlan {
  int32_t ncopy;
  int32_t nstages;       // 0 = columns are read from global memory
  uint32_t stage_bytes;  // bytes of one stage (multiple of 128)
  uint32_t tx_bytes[2];  // bytes a full step copies on pass 0 / pass 1
  StageCopy c[2 * YQ_MAX_BATCH_COLUMNS];
};

#ifndef __CUDACC_RTC__
// Lays the columns of pass0 | pass1 out in one stage (each at one offset for
// both passes) and sizes the ring; a step of pass p copies the columns of
// mask p. Returns false (nstages = 0) when a column or null array is not
// 16-byte aligned, when there is nothing to stage, or when fewer than two
// stages fit.
inline bool plan_stages2(VmProgram& P, uint32_t pass0, uint32_t pass1, StagePlan& SP) {
  memset(&SP, 0, sizeof(SP));
  const uint32_t mask = pass0 | pass1;
  uint32_t off = 0;
  int n = 0;
  for (int c = 0; c < P.ncols; ++c) {
    if (!(mask >> c & 1u)) continue;
    DevCol& d = P.cols[c];
    if (reinterpret_cast<uintptr_t>(d.data) & 15u) return false;
    const uint32_t passes = (pass0 >> c & 1u) | (pass1 >> c & 1u) << 1;
    const uint32_t row_bytes = kStepRows * (uint32_t)d.width;
    d.soff = off;
    SP.c[n++] = StageCopy{d.data, (uint32_t)d.width, off, passes};
    for (int p = 0; p < 2; ++p)
      if (passes >> p & 1u) SP.tx_bytes[p] += row_bytes;
    off += row_bytes;
    if (d.nulls) {
      if (reinterpret_cast<uintptr_t>(d.nulls) & 15u) return false;
      d.snoff = off;
      SP.c[n++] = StageCopy{reinterpret_cast<const char*>(d.nulls), 1u, off, passes};
      for (int p = 0; p < 2; ++p)
        if (passes >> p & 1u) SP.tx_bytes[p] += kStepRows;
      off += kStepRows;
    }
  }
  if (n == 0) return false;
  const uint32_t stage = (uint32_t)align_up(off, 128);
  int ns = (int)(kStageBudget / stage);
  if (ns > kStageMax) ns = kStageMax;
  if (ns < 2) {
    memset(&SP, 0, sizeof(SP));
    return false;
  }
  SP.ncopy = n;
  SP.nstages = ns;
  SP.stage_bytes = stage;
  return true;
}

// One pass over the columns of `mask`.
inline bool plan_stages(VmProgram& P, uint32_t mask, StagePlan& SP) { return plan_stages2(P, mask, 0u, SP); }
#endif

#ifndef __CUDACC_RTC__
inline size_t stage_smem_bytes(const StagePlan& SP) {
  return SP.nstages ? (size_t)SP.nstages * SP.stage_bytes + (size_t)SP.nstages * 8 : 0;
}
#endif

__device__ __forceinline__ uint64_t* stage_bar(const StagePlan& SP, int slot) {
  return reinterpret_cast<uint64_t*>(yq_dyn_smem + (size_t)SP.nstages * SP.stage_bytes) + slot;
}

__device__ __forceinline__ void stage_init(const StagePlan& SP) {
  if (threadIdx.x == 0)
    for (int s = 0; s < SP.nstages; ++s) mbar_init(stage_bar(SP, s), 1);
  __syncthreads();
}

// Thread 0: start the copies of pass `pass` of the full step at row `row0` into `slot`.
__device__ __forceinline__ void stage_issue(const StagePlan& SP, int slot, uint32_t row0, int pass) {
  uint64_t* bar = stage_bar(SP, slot);
  mbar_arrive_expect_tx(bar, SP.tx_bytes[pass]);
  unsigned char* dst = yq_dyn_smem + (size_t)slot * SP.stage_bytes;
  // A column the second pass reads again stays in L2 from its first read;
  // everything else streams through.
  const uint64_t keep = l2_evict_last_policy(), stream = l2_evict_first_policy();
  for (int i = 0; i < SP.ncopy; ++i) {
    const StageCopy& c = SP.c[i];
    if (c.passes >> pass & 1u)
      tma_load_1d_hint(dst + c.soff, c.src + (size_t)row0 * c.row_bytes, kStepRows * c.row_bytes, bar,
                       (pass == 0 && (c.passes & 2u)) ? keep : stream);
  }
}

// All threads: copy pass `pass` of a partial step of `rows` rows with plain
// loads, zero the rest.
__device__ __forceinline__ void stage_fill(const StagePlan& SP, int slot, uint32_t row0, uint32_t rows, int pass) {
  unsigned char* dst = yq_dyn_smem + (size_t)slot * SP.stage_bytes;
  for (int i = 0; i < SP.ncopy; ++i) {
    const StageCopy& c = SP.c[i];
    if (!(c.passes >> pass & 1u)) continue;
    const uint32_t valid = rows * c.row_bytes, total = kStepRows * c.row_bytes;
    const unsigned char* src = reinterpret_cast<const unsigned char*>(c.src) + (size_t)row0 * c.row_bytes;
    const bool words = (reinterpret_cast<uintptr_t>(src) & 3u) == 0u;
    for (uint32_t b = threadIdx.x * 4; b < total; b += blockDim.x * 4) {
      uint32_t w = 0;
      if (words && b + 4 <= valid) {
        w = *reinterpret_cast<const uint32_t*>(src + b);
      } else {
        for (uint32_t j = 0; j < 4; ++j)
          if (b + j < valid) w |= (uint32_t)src[b + j] << (8 * j);
      }
      *reinterpret_cast<uint32_t*>(dst + c.soff + b) = w;
    }
  }
}

// A step goes through bulk copies when it is full and starts on a 16-row
// boundary (every column's slice is then 16-byte aligned).
__device__ __forceinline__ bool step_bulk(uint32_t row0, uint32_t rows) {
  return rows == kStepRows && (row0 & 15u) == 0u;
}

// Thread 0: start the step of `rows` rows at `row0` in `slot`. A bulk step is
// copied by bulk copies; any other (the first or last rows of a batch or of a
// task) only completes the slot's barrier phase, and every thread fills it at
// stage_finish. Either way each use of a slot completes one phase.
__device__ __forceinline__ void stage_start(const StagePlan& SP, int slot, uint32_t row0, uint32_t rows,
                                            int pass = 0) {
  if (step_bulk(row0, rows)) stage_issue(SP, slot, row0, pass);
  else mbar_arrive(stage_bar(SP, slot));
}

// All threads: make the step in `slot` (ring pass parity `parity`) readable.
__device__ __forceinline__ void stage_finish(const StagePlan& SP, int slot, uint32_t parity, uint32_t row0,
                                             uint32_t rows, uint32_t* err, int pass = 0) {
  mbar_wait_bounded(stage_bar(SP, slot), parity, err);
  if (!step_bulk(row0, rows)) {
    stage_fill(SP, slot, row0, rows, pass);
    __syncthreads();
  }
}

// Rows of step `tile` of a batch of n rows.
__device__ __forceinline__ uint32_t step_rows(uint32_t tile, uint32_t n) {
  const uint32_t row0 = tile * kStepRows;
  return n - row0 < kStepRows ? n - row0 : kStepRows;
}

__device__ __forceinline__ uint32_t in_range_bits(uint32_t row0, uint32_t n) {
  if (row0 >= n) return 0u;
  const uint32_t left = n - row0;
  return left >= (uint32_t)ITEMS ? kItemsMask : ((1u << left) - 1u);
}

#ifndef __CUDACC_RTC__
// Columns an expression program reads (plus `extra`).
inline uint32_t program_columns_in(const VmProgram& P, int begin, int end, uint32_t extra) {
  uint32_t mask = extra;
  for (int i = begin; i < end; ++i) {
    const RInsn& I = P.code[i];
    if (I.opc < R_CONST) {
      mask |= 1u << I.a;
    } else if ((I.opc >= R_ARITH_COL && I.opc < R_ARITH_CONST) || (I.opc >= R_CMP_CC && I.opc < R_AND)) {
      mask |= 1u << I.b;
      if (I.opc >= R_CMP_CCOL) mask |= 1u << I.c;
    }
  }
  return mask;
}

inline uint32_t program_columns(const VmProgram& P, int end, uint32_t extra) {
  return program_columns_in(P, 0, end, extra);
}
#endif

#ifndef __CUDACC_RTC__
// Bytes per row of the columns in `mask` (plus null bytes).
inline double row_bytes_of(const VmProgram& P, uint32_t mask) {
  double b = 0;
  for (int c = 0; c < P.ncols; ++c)
    if (mask >> c & 1u) b += P.cols[c].width + (P.cols[c].nulls ? 1 : 0);
  return b;
}
#endif

}  // namespace yq
