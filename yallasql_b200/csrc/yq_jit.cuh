// Program-specialised row kernels (jit.cu): host interface.
#pragma once

#include "yq_vm.cuh"

namespace yq {

enum JitKind { JIT_FILTER_AGG = 0, JIT_FILTER_AGG_SEG = 1, JIT_FILTER_PROJECT = 2, JIT_JOIN_AGG = 3 };

// Kernel for `kind` (staged or not) that runs P's resolved instructions
// [0, seg0_end) as segment 0 and [seg0_end, end) as segment 1, compiled for
// this program (cached by its instruction words; constants stay parameters).
// Null when runtime compilation is switched off or unavailable, or failed:
// the caller then launches the interpreter kernel, which computes the same.
// For JIT_FILTER_PROJECT, `fp` lists the projections that copy a source
// column; the kernel copies them with their columns and widths as constants
// (they are part of the cache key).
struct FPParams;
const void* jit_kernel(JitKind kind, bool staged, const VmProgram& P, int seg0_end, int end,
                       const FPParams* fp = nullptr);

// Ring depth for `kernel` with stages of `stage_bytes`: of 2..kStageMax stages,
// the count that lets the most blocks share an SM, the deeper ring on a tie
// (a kernel with few registers then runs more blocks, each with a shallower
// ring). `nstages` (the plan made for the interpreter) when the occupancy
// cannot be queried or YQ_STAGE_FIT=0 is set in the environment. `extra`:
// dynamic shared memory the kernel keeps after the ring (16-byte aligned).
int jit_stages(const void* kernel, uint32_t stage_bytes, int nstages, size_t extra = 0);

// Launch helper for a kernel jit_kernel returned: raises its dynamic shared
// memory limit when needed and sizes a persistent grid (at most `steps`).
int jit_launch(const void* kernel, int max_grid, uint32_t steps, size_t smem, void** args, cudaStream_t s);

}  // namespace yq
