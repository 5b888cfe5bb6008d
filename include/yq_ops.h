/*
 * yq_ops.h — C ABI of the B200 (sm_100a) per-batch SQL operator kernels.
 *
 * This is the drop-in boundary for YallaSQL's kernel layer (`src/kernels/*.cu`,
 * declared in `include/kernels/*.hpp` of the reference) plus the fused per-batch
 * operator bodies that stitch those kernels together (FilterOperator::next,
 * ProjectionOperator::next, AggregateOperator::next, OrderOperator, JoinOperator,
 * CrossProductOperator in `include/engine/operators/*.hpp`).
 *
 * Conventions
 *  - Plain C: pointers, sizes and small POD structs only. No C++ or torch types.
 *  - Every column pointer is a DEVICE pointer. Nulls are one byte per row
 *    (nonzero = NULL), the reference's `NullBitSet::bitset` layout
 *    (include/null_bit_set.hpp:5-9); a NULL `nulls` pointer means "no nulls".
 *  - `stream` is a `cudaStream_t` passed as `void*` (NULL = legacy default stream).
 *    All work is stream ordered. Calls that must return a host value (a row
 *    count, a status read back from the device) synchronise that stream and say so.
 *  - Scratch: calls that need device scratch take (`workspace`, `workspace_bytes`).
 *    Passing workspace == NULL makes the library allocate it stream-ordered with
 *    cudaMallocAsync on `stream` and release it with cudaFreeAsync after the
 *    launch. The matching `*_workspace_size` function reports the bytes needed.
 *  - Every function returns a yq_status; nothing calls exit() (the reference's
 *    CUDA_CHECK exits the process, include/utils/macros.hpp:6-22).
 *  - Every device wait inside a kernel (decoupled look-back, mbarrier waits) is
 *    bounded; running out of the bound returns YQ_ERR_TIMEOUT and leaves the
 *    CUDA context usable.
 */
#ifndef YQ_OPS_H
#define YQ_OPS_H

#ifndef __CUDACC_RTC__ /* runtime-compiled kernels get these types from yq_common.cuh */
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define YQ_ABI_VERSION 1

/* ------------------------------------------------------------------ status */
typedef enum yq_status {
  YQ_OK = 0,
  YQ_ERR_INVALID_ARG = 1,   /* bad pointer / size / type combination            */
  YQ_ERR_UNSUPPORTED = 2,   /* valid request this build does not implement      */
  YQ_ERR_CAPACITY = 3,      /* output larger than the caller's capacity          */
  YQ_ERR_TIMEOUT = 4,       /* a bounded device wait ran out (error flag set)    */
  YQ_ERR_CUDA = 5,          /* a CUDA runtime call failed; see yq_last_cuda_error */
  YQ_ERR_ALLOC = 6          /* stream-ordered allocation failed                  */
} yq_status;

const char* yq_status_string(int status);
/* cudaError_t of the last failing CUDA call made by this library on this thread. */
int yq_last_cuda_error(void);
int yq_abi_version(void);

/* ------------------------------------------------------------------- types */
/* Values 0..3 equal the reference's DataType (include/enums/data_type.hpp:2-7):
 * INT, FLOAT, DATETIME (int64 epoch seconds), STRING (fixed NUL-padded slot). */
typedef enum yq_type {
  YQ_INT32 = 0,
  YQ_FLOAT32 = 1,
  YQ_DATETIME = 2,   /* int64 seconds since the epoch, UTC                     */
  YQ_TEXT = 3,       /* fixed-width slot, NUL padded, compared as unsigned bytes */
  YQ_INT64 = 4,      /* BIGINT (the reference folds it into INT32)             */
  YQ_FLOAT64 = 5,    /* DOUBLE (aggregate results, intermediate expressions)   */
  YQ_BOOL = 6        /* one byte, 0/1 (predicate masks)                        */
} yq_type;

/* One column of a batch. The reference's `Batch::columnData[i]` +
 * `Batch::nullset[i]->bitset` + `Column::{type,bytes}` (include/batch.hpp:21-60,
 * include/db/column.hpp:7-25). `width` is bytes per value: 4 for INT32/FLOAT32,
 * 8 for INT64/DATETIME/FLOAT64, 1 for BOOL, and the slot width for TEXT
 * (a multiple of 4 between 4 and 256; the reference's slot is 256 bytes). */
typedef struct yq_column {
  void* data;
  const uint8_t* nulls;
  int32_t type;
  int32_t width;
} yq_column;

typedef struct yq_batch {
  const yq_column* columns;
  int32_t ncols;
  uint32_t rows;
} yq_batch;

/* Comparison operators, in the order of the reference's functors
 * (include/kernels/comparison_operators_kernel.hpp:26-59): <, <=, >, >=, =, <>. */
typedef enum yq_cmp { YQ_LT = 0, YQ_LE = 1, YQ_GT = 2, YQ_GE = 3, YQ_EQ = 4, YQ_NE = 5 } yq_cmp;

/* Arithmetic (include/kernels/binary_operators_kernel.hpp:23-53). */
typedef enum yq_arith { YQ_ADD = 0, YQ_SUB = 1, YQ_MUL = 2, YQ_DIV = 3, YQ_MOD = 4 } yq_arith;

/* ---------------------------------------------------- expression programs
 * A compiled expression is a postfix program for a small stack machine that
 * every fused kernel evaluates per row in registers (stack depth 4). It is the
 * flattened form of the reference's `our::Expression` tree
 * (include/engine/operators/expressions/*.hpp): BoundRef -> YQ_OP_COL,
 * BoundValue -> YQ_OP_CONST, Cast -> YQ_OP_CAST, BoundFunc -> YQ_OP_ARITH,
 * Comparison -> YQ_OP_CMP / fused forms, Conjunction -> YQ_OP_AND / YQ_OP_OR.
 * Semantics are SQL three-valued logic: a comparison or arithmetic with a NULL
 * operand is NULL; a WHERE keeps only rows whose predicate is TRUE. */
typedef enum yq_opcode {
  YQ_OP_COL = 1,            /* push column `a` of the batch (typed by the column)  */
  YQ_OP_CONST = 2,          /* push constant `imm` of type `type`                  */
  YQ_OP_NULL = 3,           /* push NULL                                           */
  YQ_OP_CAST = 4,           /* top := CAST(top AS `a`); `type` = source type       */
  YQ_OP_ARITH = 5,          /* b=pop, a=pop, push a <op `a`> b; operands of `type` */
  YQ_OP_CMP = 6,            /* b=pop, a=pop, push a <cmp `a`> b as BOOL            */
  YQ_OP_CMP_COL_CONST = 7,  /* push column `b` <cmp `a`> constant `imm`            */
  YQ_OP_CMP_COL_COL = 8,    /* push column `b` <cmp `a`> column `imm`              */
  YQ_OP_AND = 9,
  YQ_OP_OR = 10,
  YQ_OP_NOT = 11,
  YQ_OP_IS_NULL = 12,
  YQ_OP_IS_NOT_NULL = 13,
  /* Fused forms (the loader also creates them from the plain sequences). */
  YQ_OP_ARITH_COL = 20,        /* top := top <op `a`> column `b` (loaded as `type`) */
  YQ_OP_ARITH_CONST = 21,      /* top := top <op `a`> constant `imm`                 */
  YQ_OP_AND_CMP_COL_CONST = 22 /* top := top AND (column `b` <cmp `a`> constant)     */
} yq_opcode;

typedef struct yq_insn {
  uint8_t op;     /* yq_opcode */
  uint8_t type;   /* operand type (yq_type)            */
  uint8_t a;      /* column / cmp / arith / cast target */
  uint8_t b;      /* column                             */
  int32_t imm;    /* constant index / second column     */
} yq_insn;

#define YQ_MAX_PROGRAM_INSNS 48
#define YQ_MAX_BATCH_COLUMNS 16
#define YQ_MAX_CONSTANTS 32
#define YQ_MAX_TEXT_CONSTANTS 4
#define YQ_MAX_TEXT_WIDTH 256
#define YQ_MAX_AGGREGATES 8
#define YQ_MAX_PROJECTIONS 12

typedef struct yq_program {
  const yq_insn* code;   /* host pointer */
  int32_t len;           /* 0 = empty program (a predicate that is always TRUE) */
} yq_program;

/* Constant pool shared by all programs of one call. Numeric constants are raw
 * 64-bit words: INT32/INT64/DATETIME hold the integer value, FLOAT32 holds the
 * float's bit pattern in the low 32 bits, FLOAT64 the double's bit pattern.
 * Text constants are `text_count` NUL-padded slots of `text_width` bytes. */
typedef struct yq_constants {
  const int64_t* values;
  int32_t count;
  const char* text;
  int32_t text_count;
  int32_t text_width;
} yq_constants;

/* ====================================================================
 * Fused per-batch operators (replace the operator bodies).
 * ==================================================================== */

/* ---- WHERE + aggregates: FilterOperator::next -> AggregateOperator::next
 * (include/engine/operators/filter_operator.hpp:31-98,
 *  include/engine/operators/aggregate_operator.hpp:30-81,
 *  include/engine/operators/expressions/aggregate.hpp:55-284,
 *  src/kernels/reduction_kernel.cu:79-185).
 * One kernel evaluates the predicate and each aggregate's input expression
 * per row and reduces with warp shuffles, a block reduction and one ticket
 * atomic per block; the last block folds the per-block partials in block
 * order, so results do not depend on scheduling. Float SUM/AVG accumulate in
 * FP64 (the reference keeps FP64 only for SUM and returns float32). Calls with
 * the same `state` accumulate across batches (the reference's accumulator
 * lives in AggregateExpression::accumlator). */
typedef enum yq_agg_kind {
  YQ_AGG_COUNT_STAR = 0,
  YQ_AGG_COUNT = 1,
  YQ_AGG_SUM = 2,
  YQ_AGG_AVG = 3,
  YQ_AGG_MIN = 4,
  YQ_AGG_MAX = 5
} yq_agg_kind;

typedef struct yq_agg_spec {
  int32_t kind;        /* yq_agg_kind */
  int32_t input_type;  /* yq_type of the input expression's value (ignored for COUNT_STAR) */
  yq_program input;    /* the aggregate's argument */
} yq_agg_spec;

/* Host view of one finished aggregate. COUNT/COUNT_STAR -> `i`; SUM of an
 * integer -> `i` (exact, int64); SUM/AVG of a float -> `f` (FP64); AVG of an
 * integer -> `f`; MIN/MAX -> `i` for integer/date inputs, `f` for float
 * inputs. `is_null` is set for SUM/AVG/MIN/MAX over zero rows. */
typedef struct yq_agg_result {
  int64_t i;
  double f;
  int64_t count;
  int32_t is_null;
  int32_t kind;
} yq_agg_result;

/* Device bytes of an accumulator for `nagg` aggregates (caller allocates). */
size_t yq_agg_state_bytes(int32_t nagg);
/* Reset an accumulator (stream ordered). */
int yq_agg_state_init(void* state, const yq_agg_spec* aggs, int32_t nagg, void* stream);
size_t yq_filter_aggregate_workspace_size(uint32_t rows, int32_t nagg);
int yq_filter_aggregate(const yq_batch* batch, const yq_program* predicate,
                        const yq_constants* constants, const yq_agg_spec* aggs,
                        int32_t nagg, void* state, void* workspace,
                        size_t workspace_bytes, void* stream);
/* Copy the accumulator to the host and finish AVG (sum / count in FP64).
 * Synchronises `stream`. */
int yq_agg_state_read(const void* state, const yq_agg_spec* aggs, int32_t nagg,
                      yq_agg_result* out, void* stream);

/* ---- WHERE + projection with stream compaction: FilterOperator::next +
 * ProjectionOperator::next (filter_operator.hpp:31-98, projection_operator.hpp:30-62,
 * src/kernels/prefix_sum_kernel.cu:106-157, src/kernels/move_rows_kernel.cu:33-49).
 * One single-pass kernel: predicate in registers, warp ballot/popc, a
 * decoupled look-back scan over tiles for the output offset, and the
 * projected columns written for the surviving rows in input order. */
typedef struct yq_projection {
  int32_t column;      /* >= 0: copy this input column (any type, nulls kept) */
  int32_t out_type;    /* when column < 0: result type of `program`           */
  yq_program program;  /* when column < 0: expression to evaluate             */
} yq_projection;

size_t yq_filter_project_workspace_size(uint32_t rows);
/* `out` has `nproj` columns with `capacity` rows of device storage each; an
 * output column's `nulls` may be NULL when the caller does not want null
 * flags. The surviving row count is written to `*count_device` (device,
 * optional) and, when `count_host` is not NULL, to `*count_host` after a
 * stream synchronisation. Returns YQ_ERR_CAPACITY (and the true count) when
 * more than `capacity` rows survive. */
int yq_filter_project(const yq_batch* batch, const yq_program* predicate,
                      const yq_constants* constants, const yq_projection* proj,
                      int32_t nproj, yq_column* out, uint32_t capacity,
                      uint32_t* count_device, uint32_t* count_host, void* workspace,
                      size_t workspace_bytes, void* stream);

/* ---- WHERE + projection that allocates nothing.
 * No counterpart in the reference: it exists for hosts that must not allocate
 * device memory inside the call — an engine that embeds this library and owns
 * every byte of device memory through its own fixed arena, or a serving loop
 * whose latency budget cannot absorb allocator calls and the synchronisation
 * they may bring. Same contract as yq_filter_project, except that the
 * look-back scratch is a static device array compiled into libyq_ops.so
 * (about 512 KiB, held by every GPU that loads the library until the process
 * exits), so batches are limited to YQ_FILTER_PROJECT_NOALLOC_MAX_ROWS rows;
 * larger batches are rejected with YQ_ERR_INVALID_ARG before any device work.
 * The first call on a device looks up that array's device address (once per
 * device and CUDA context, under a lock; a device reset gives the device a new
 * context, and the next call looks the address up again); make that first call
 * before any stream capture.
 * Every call shares the one array and clears the part it uses on `stream`, so
 * calls whose kernels overlap on the GPU (different streams, no ordering
 * between them) race and must not be issued.
 * It always runs the library's interpreter kernel: loading the
 * program-specialised kernel that yq_filter_project uses would itself
 * allocate, and the interpreter runs about 4x slower than that kernel. */
#define YQ_FILTER_PROJECT_NOALLOC_MAX_ROWS (1u << 26)
int yq_filter_project_noalloc(const yq_batch* batch, const yq_program* predicate,
                              const yq_constants* constants, const yq_projection* proj,
                              int32_t nproj, yq_column* out, uint32_t capacity,
                              uint32_t* count_device, uint32_t* count_host, void* stream);

/* ---- ORDER BY: stable LSD radix argsort.
 * Replaces BoundRefSortExpression + launch_radix_sort + move_rows_batch
 * (include/engine/operators/expressions/bound_ref_sort.hpp:26-64,
 *  src/kernels/radix_sort_utils.cu:4-53, src/kernels/radix_sort_kernel.cu:65-178,
 *  include/kernels/move_rows_kernel.hpp:51-83).
 * Keys are mapped to order-preserving unsigned words (signed bias, float
 * sign flip with -0.0 -> +0.0 and NaN canonicalised above +inf, big-endian
 * text words, DESC = bitwise NOT) inside the histogram and first scatter pass.
 * One upfront histogram computes every pass's digit counts; each pass is one
 * onesweep kernel (warp multisplit ranking, decoupled look-back over tiles,
 * shared-memory staging for coalesced scatter). Passes whose digit is the same
 * for every key are skipped (this reads the histogram back: the call
 * synchronises `stream` once). NULL keys sort last unless nulls_first. */
typedef struct yq_sort_config {
  int32_t digit_bits;        /* 4, 6 or 8; 0 = autotuned (yq_sort_autotune), else 8 */
  int32_t items_per_thread;  /* 0 = autotuned / the variant's default          */
  int32_t block_threads;     /* 128, 256 or 512; 0 = autotuned / 256          */
  int32_t keep_trivial;      /* 1 = never skip passes (no host read-back)      */
} yq_sort_config;

size_t yq_sort_workspace_size(const yq_column* key, uint32_t rows);
int yq_sort_indices(const yq_column* key, uint32_t rows, int32_t descending,
                    int32_t nulls_first, uint32_t* out_perm,
                    const yq_sort_config* config, void* workspace,
                    size_t workspace_bytes, void* stream);
/* Multi-key ORDER BY (keys[0] most significant); same contract. */
int yq_sort_indices_multi(const yq_column* keys, const int32_t* descending,
                          const int32_t* nulls_first, int32_t nkeys, uint32_t rows,
                          uint32_t* out_perm, const yq_sort_config* config,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Segmented form: rows [seg_offsets[s], seg_offsets[s+1]) are sorted
 * independently (seg_offsets is a host array of nseg+1 entries starting at 0
 * and ending at `rows`). `out_perm` holds global row ids; segment s's rows stay
 * inside its range. This is run formation for out-of-core ORDER BY (each 4 MB
 * batch is a segment; OrderOperator::firstPass, order_operator.hpp:89-121) in
 * one set of launches, and the batched form's ORDER BY tasks. */
size_t yq_sort_segments_workspace_size(const yq_column* key, uint32_t rows,
                                       const uint32_t* seg_offsets, int32_t nseg);
int yq_sort_segments(const yq_column* key, uint32_t rows, const uint32_t* seg_offsets,
                     int32_t nseg, int32_t descending, int32_t nulls_first,
                     uint32_t* out_perm, const yq_sort_config* config, void* workspace,
                     size_t workspace_bytes, void* stream);

/* out[c][i] = in[c][perm[i]] for every column c, nulls included
 * (move_one_col, src/kernels/move_rows_kernel.cu:52-70, all columns in one launch). */
int yq_gather(const yq_column* in, int32_t ncols, const uint32_t* perm, uint32_t rows,
              yq_column* out, void* stream);

/* ---- Out-of-core run merging: merge path.
 * Replaces merge_two_runs / load_in_buffer / shift_buffer and
 * merge_sorted_array_kernel_v1 + move_one_col_merge
 * (src/engine/operators/order_operator.cpp:14-220, src/kernels/merge_batchs.cu:14-148,
 *  src/kernels/move_rows_kernel.cu:73-105).
 * `cols` hold all runs back to back (run r = rows [run_offsets[r], run_offsets[r+1])).
 * One launch merges every pair (0,1), (2,3), ... of the level into `out`
 * (same layout; an odd last run is copied). Each block stages its slice of
 * both runs' keys in shared memory with 1-D TMA bulk copies, finds co-ranks
 * there, merges, and moves every payload column. Ties take the earlier run,
 * so merging sorted runs stays stable. `run_offsets` is a host array of
 * nruns+1 entries. */
size_t yq_merge_workspace_size(uint32_t total_rows, int32_t nruns);
int yq_merge_pass(const yq_column* cols, int32_t ncols, int32_t key_col,
                  int32_t descending, int32_t nulls_first, const uint32_t* run_offsets,
                  int32_t nruns, yq_column* out, void* workspace,
                  size_t workspace_bytes, void* stream);

/* ---- Out-of-core ORDER BY of one key: the whole operator in one call.
 * Replaces OrderOperator::firstPass + merge_all_sorted
 * (include/engine/operators/order_operator.hpp:89-193,
 *  src/engine/operators/order_operator.cpp:14-220): the rows of `in` arrive as
 * nruns sorted-on-arrival batches (run r = rows [run_offsets[r],
 * run_offsets[r+1]), host array). Every run is sorted by the segmented radix
 * sort, whose last pass also leaves each row's order-preserving key words;
 * the runs are then merged pairwise, level by level, as (key words, row id)
 * pairs by a persistent merge-path kernel that stages both windows of the
 * tiles ahead with 1-D bulk copies; finally every column is gathered once by
 * the merged row ids into `out` (same schema, at least in->rows rows).
 * Stable: equal keys keep their input order. The call waits for the device
 * once, at the end, to report errors.
 *
 * With many runs over a table larger than L2 the gather goes in two levels
 * when the workspace allows (or the library allocates it): the columns are
 * first gathered run by run into sorted-run order, and the final gather then
 * reads every run's rows in increasing order. yq_order_by_workspace_size is
 * the least workspace (one-level gather); yq_order_by_batch_workspace_size
 * includes the sorted-run copy of the batch's columns. */
size_t yq_order_by_workspace_size(const yq_column* key, uint32_t rows, const uint32_t* run_offsets,
                                  int32_t nruns);
size_t yq_order_by_batch_workspace_size(const yq_batch* in, int32_t key_col, const uint32_t* run_offsets,
                                        int32_t nruns);
int yq_order_by(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                const uint32_t* run_offsets, int32_t nruns, yq_batch* out, void* workspace,
                size_t workspace_bytes, void* stream);
/* yq_order_by with the merge-path tile given: merge_items outputs per
 * thread (4, 8 or 16; 16 needs a key of at most two words, else
 * YQ_ERR_UNSUPPORTED; 0 = the tuned or default choice). */
int yq_order_by_tiled(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                      const uint32_t* run_offsets, int32_t nruns, yq_batch* out, int32_t merge_items,
                      void* workspace, size_t workspace_bytes, void* stream);
/* Tunes yq_order_by for this input: the run-formation sort through
 * yq_sort_autotune (digit bits, items per thread, block threads; returned in
 * *best_sort) and the merge-path tile (outputs per thread, 4, 8 or 16; 16 for
 * keys of up to two words) by timing the whole ORDER BY once per tile; the
 * fastest tile is remembered for this key width and row count (log2) and
 * used by later yq_order_by calls. The reference fixes the merge tile at
 * compile time (ELE_PER_TH 6, src/kernels/merge_batchs.cu:8). Allocates its
 * own output and workspace (stream-ordered) and synchronises `stream`. */
int yq_order_by_autotune(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                         const uint32_t* run_offsets, int32_t nruns, yq_sort_config* best_sort,
                         int32_t* best_merge_items, void* stream);

/* ---- Batched forms: many independent tasks in one set of launches.
 * The tasks' rows sit back to back in one batch (task g = rows
 * [seg_offsets[g], seg_offsets[g+1]), host array); every launch walks the
 * steps of all tasks as one device-side queue, so hundreds of small tasks
 * cost a handful of launches instead of hundreds (the reference runs each
 * batch through its own launch sequence, operator.hpp:45-47).
 *
 * yq_filter_aggregate_segments: WHERE + aggregates per task into
 * states[g] = (char*)states + g * yq_agg_state_bytes(nagg), each initialised
 * by yq_agg_states_init. Results equal running each task alone up to the
 * summation order of float SUM/AVG (partials fold in a fixed order, so a
 * task's result is the same on every run).
 * yq_order_by_segments: ORDER BY per task (segmented radix sort + one gather).
 * With config->keep_trivial set it enqueues device work only and never waits
 * (it can be captured in a CUDA graph); an error is then left as a non-zero
 * 32-bit word at offset 0 of `workspace` (required in that mode).
 * yq_sort_autotune: times every instantiated (digit bits, items per thread,
 * block threads) variant on the given key and segments, remembers the fastest
 * for this key width and segment size (used whenever a sort's config leaves
 * those fields 0) and returns it. The reference fixes these at compile time:
 * OUR_RADIX 4 (include/kernels/radix_sort_kernel.hpp:9) and BLOCK_DIM 256
 * (include/kernels/constants.hpp:7). */
int yq_agg_states_init(void* states, int32_t count, const yq_agg_spec* aggs, int32_t nagg, void* stream);
int yq_agg_states_read(const void* states, int32_t count, const yq_agg_spec* aggs, int32_t nagg,
                       yq_agg_result* out, void* stream);
size_t yq_filter_aggregate_segments_workspace_size(uint32_t rows, int32_t nseg);
int yq_filter_aggregate_segments(const yq_batch* batch, const uint32_t* seg_offsets, int32_t nseg,
                                 const yq_program* predicate, const yq_constants* constants,
                                 const yq_agg_spec* aggs, int32_t nagg, void* states, void* workspace,
                                 size_t workspace_bytes, void* stream);
/* Same as yq_filter_aggregate_segments for tasks given as row ranges
 * [begin[g], end[g]) of the batch: ranges may leave gaps, repeat or overlap
 * (a serving loop co-launches pending queries over resident tables). */
size_t yq_filter_aggregate_ranges_workspace_size(const uint32_t* begin, const uint32_t* end, int32_t nseg);
int yq_filter_aggregate_ranges(const yq_batch* batch, const uint32_t* begin, const uint32_t* end, int32_t nseg,
                               const yq_program* predicate, const yq_constants* constants,
                               const yq_agg_spec* aggs, int32_t nagg, void* states, void* workspace,
                               size_t workspace_bytes, void* stream);
size_t yq_order_by_segments_workspace_size(const yq_column* key, uint32_t rows, const uint32_t* seg_offsets,
                                           int32_t nseg);
int yq_order_by_segments(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                         const uint32_t* seg_offsets, int32_t nseg, yq_batch* out, const yq_sort_config* config,
                         void* workspace, size_t workspace_bytes, void* stream);
/* The same, writing the permutation it gathers by into `perm_out` (`rows`
 * device words): a host that keeps it can serve a repeat of the query with
 * yq_gather alone (the serving loop keeps it as a resident intermediate). */
int yq_order_by_segments_perm(const yq_batch* in, int32_t key_col, int32_t descending, int32_t nulls_first,
                              const uint32_t* seg_offsets, int32_t nseg, yq_batch* out, uint32_t* perm_out,
                              const yq_sort_config* config, void* workspace, size_t workspace_bytes,
                              void* stream);
int yq_sort_autotune(const yq_column* key, uint32_t rows, const uint32_t* seg_offsets, int32_t nseg,
                     int32_t descending, yq_sort_config* best, void* stream);

/* ---- Inner join (nested loop semantics) and cross product.
 * Replaces ComparisonJoinExpression/ConjunctionJoinExpression +
 * outer_join_batches/and_join_batches + move_rows_join_kernel and
 * CrossProductOperator + cross_product_kernel
 * (include/engine/operators/filters/comparison_join.hpp:70-236,
 *  src/kernels/comparison_operators_kernel.cu:6-54,
 *  src/kernels/move_rows_kernel.cu:8-30,
 *  include/engine/operators/cross_product_operator.hpp:87-125,
 *  src/kernels/cross_product_kernel.cu:8-27).
 * All conditions are ANDed and evaluated in one kernel. Pairs are produced in
 * a deterministic order (left row ascending, then right row ascending); the
 * reference's order is unspecified (atomic slots), so parity is on the pair
 * multiset. An equality condition with a right side that fits in shared
 * memory is probed through a per-block hash table instead of a full scan. */
typedef struct yq_join_cond {
  int32_t left_col;
  int32_t right_col;
  int32_t cmp;        /* yq_cmp: left <cmp> right */
} yq_join_cond;

size_t yq_join_workspace_size(uint32_t left_rows, uint32_t right_rows);
/* Writes up to `capacity` pairs; `*count_host` receives the exact number of
 * matching pairs (synchronises `stream`). YQ_ERR_CAPACITY when it exceeds
 * `capacity` (the reference silently overflows, comparison_join.hpp:87). */
int yq_join_pairs(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds,
                  int32_t ncond, uint32_t* out_left, uint32_t* out_right,
                  uint64_t capacity, uint64_t* count_host, void* workspace,
                  size_t workspace_bytes, void* stream);

/* Output columns of a join or cross product: side 0 = left, 1 = right. */
typedef struct yq_join_output {
  int32_t side;
  int32_t column;
} yq_join_output;

/* Join and write the selected columns of each matching pair directly
 * (no pair list), warp-aggregated appends, same order as yq_join_pairs.
 * With ncond == 0 this is the cross product (left-major). */
int yq_join_project(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds,
                    int32_t ncond, const yq_join_output* outputs, int32_t nout,
                    yq_column* out, uint64_t capacity, uint64_t* count_host,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Join conditions as an OR of ANDs (the reference rejects OR in a join
 * condition, include/engine/operators/expressions/filters/conjunction_join.hpp:113-114,
 * and evaluates AND chains with and_join_batches,
 * src/kernels/comparison_operators_kernel.cu:24-54): condition i belongs to
 * disjunct group disjunct[i] (0..G-1, every group used); a pair matches when
 * all conditions of at least one group hold. A comparison with a NULL side
 * does not hold. Same output order, capacity and workspace contract as
 * yq_join_pairs / yq_join_project; always the nested-loop kernel. */
int yq_join_pairs_or(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds,
                     const int32_t* disjunct, int32_t ncond, uint32_t* out_left, uint32_t* out_right,
                     uint64_t capacity, uint64_t* count_host, void* workspace, size_t workspace_bytes,
                     void* stream);
int yq_join_project_or(const yq_batch* left, const yq_batch* right, const yq_join_cond* conds,
                       const int32_t* disjunct, int32_t ncond, const yq_join_output* outputs, int32_t nout,
                       yq_column* out, uint64_t capacity, uint64_t* count_host, void* workspace,
                       size_t workspace_bytes, void* stream);

/* Fused star-join aggregate: rows of `fact` passing `fact_predicate` are
 * probed against the rows of `dim` passing `dim_predicate` on
 * fact[fact_key] = dim[dim_key]; every match feeds the aggregates, whose input
 * programs read fact columns. Same accumulator contract as yq_filter_aggregate. */
size_t yq_join_aggregate_workspace_size(uint32_t fact_rows, uint32_t dim_rows, int32_t nagg);
int yq_join_aggregate(const yq_batch* fact, const yq_program* fact_predicate,
                      int32_t fact_key, const yq_batch* dim,
                      const yq_program* dim_predicate, int32_t dim_key,
                      const yq_constants* constants, const yq_agg_spec* aggs,
                      int32_t nagg, void* state, void* workspace,
                      size_t workspace_bytes, void* stream);

/* The same join against a dimension table prepared once and kept resident:
 * yq_join_dim_table_build hashes the rows of `dim` that pass `dim_predicate`
 * on `dim_key` into `table` (yq_join_dim_table_size bytes of device memory),
 * waits for it once and writes the number of rows it kept to *kept (host);
 * YQ_ERR_UNSUPPORTED when kept keys repeat. yq_join_aggregate_prepared then
 * probes that table from the fact side with no host synchronisation (the
 * reference rebuilds nothing either: it nests loops over every batch pair,
 * join_operator.hpp:36-100); `dim_rows`, `kept` and `key_type` are those of
 * the build. The table must stay valid while calls that read it run. */
size_t yq_join_dim_table_size(uint32_t dim_rows);
int yq_join_dim_table_build(const yq_batch* dim, const yq_program* dim_predicate, int32_t dim_key,
                            const yq_constants* constants, void* table, size_t table_bytes,
                            uint32_t* kept, void* stream);
size_t yq_join_aggregate_prepared_workspace_size(int32_t nagg);
int yq_join_aggregate_prepared(const yq_batch* fact, const yq_program* fact_predicate,
                               int32_t fact_key, const void* table, uint32_t dim_rows,
                               uint32_t kept, int32_t key_type, const yq_constants* constants,
                               const yq_agg_spec* aggs, int32_t nagg, void* state,
                               void* workspace, size_t workspace_bytes, void* stream);

/* ====================================================================
 * Reference-compatible element kernels: one entry per YallaSQL::Kernel::launch_*
 * so the reference's expression classes can forward to this library unchanged.
 * ==================================================================== */

/* An operand is a device vector of `n` values or, with is_scalar != 0, a device
 * pointer to one value broadcast over the batch (OperandType::SCALAR/VECTOR,
 * include/kernels/binary_operators_kernel.hpp:10-13). */
typedef struct yq_operand {
  const void* data;
  int32_t type;
  int32_t width;
  int32_t is_scalar;
} yq_operand;

/* launch_conditional_operators<T,Op> (comparison_operators_kernel.hpp:8):
 * mask[i] = (lhs <cmp> rhs) ^ negate; bytes 0/1. Null flags are not consulted
 * (the reference compares its null sentinels). */
int yq_compare(yq_operand lhs, yq_operand rhs, int32_t cmp, int32_t negate,
               uint8_t* out_mask, uint32_t n, void* stream);
/* launch_conditional_operators<bool, AND/OROperator>: 0 = AND, 1 = OR. */
int yq_logic(yq_operand lhs, yq_operand rhs, int32_t is_or, uint8_t* out_mask,
             uint32_t n, void* stream);
/* launch_binary_operators<T,Op> (binary_operators_kernel.hpp:16): typed
 * arithmetic; DIV/MOD by zero give 0 as in the reference's DivOperator/RemOperator. */
int yq_binary(yq_operand lhs, yq_operand rhs, int32_t arith, void* out, uint32_t n,
              void* stream);
/* launch_numerical_cast<S,D> (src/kernels/cast_operators_kernel.cu:23). */
int yq_cast(const void* src, int32_t src_type, void* dst, int32_t dst_type, uint32_t n,
            void* stream);
/* launch_prefix_sum_mask (include/kernels/prefix_sum.hpp:26): inclusive scan of
 * a 0/1 byte mask into uint32; single pass with a bounded decoupled look-back. */
size_t yq_prefix_sum_workspace_size(uint32_t n);
int yq_prefix_sum_mask(const uint8_t* mask, uint32_t* out, uint32_t n, void* workspace,
                       size_t workspace_bytes, void* stream);
/* Test hook for the bounded waits (no counterpart in the reference, whose
 * kernels wait without a bound or exit(1) on error): runs the library's
 * decoupled look-back as tile 1 of a chain whose tile 0 never publishes, with
 * the poll bound lowered to `spin_limit` (1 .. 2^22). Returns YQ_ERR_TIMEOUT
 * after the wait runs out, as every entry point built on that look-back does;
 * `workspace` is >= 64 bytes of device memory. */
int yq_debug_lookback_stall(uint32_t spin_limit, void* workspace, size_t workspace_bytes, void* stream);
/* launch_prefix_sum<uint32_t> (prefix_sum.hpp:29): inclusive scan of uint32. */
int yq_prefix_sum_u32(const uint32_t* in, uint32_t* out, uint32_t n, void* workspace,
                      size_t workspace_bytes, void* stream);
/* launch_move_rows_filter_kernel<T> (move_rows_kernel.hpp:19):
 * out[map[i]-1] = src[i] where mask[i] (map = inclusive scan of mask). */
int yq_move_rows_filter(const yq_column* src, const uint32_t* map, const uint8_t* mask,
                        uint32_t n, yq_column* out, void* stream);
/* lanch_move_rows_join_kernel<T> (move_rows_kernel.hpp:27): out[k] = src[pairs[2k+side]]. */
int yq_move_rows_join(const yq_column* src, const uint32_t* pairs, uint32_t npairs,
                      int32_t is_right, yq_column* out, void* stream);
/* launch_move_one_col_merge<T> (move_rows_kernel.hpp:35): out[i] = (fromA[i] ? A : B)[idx[i]],
 * written reversed when ascending == 0 as in the reference. */
int yq_move_rows_merge(const yq_column* a, const yq_column* b, const uint32_t* idx,
                       const uint8_t* from_a, int32_t ascending, uint32_t n,
                       yq_column* out, void* stream);
/* launch_reduction_operators<T,T_res,Op> and launch_reduction_count_notnull
 * (include/kernels/reduction_kernel.hpp:7-15): reduce `n` values (skipping rows
 * whose null byte is set) into *result with one atomic per block. kind is
 * YQ_AGG_SUM / MIN / MAX / COUNT; result type: SUM of FLOAT32 -> FLOAT64, SUM of
 * INT32 -> INT32 (wrapping, as the reference), otherwise the input type; COUNT -> INT32. */
int yq_reduce(const void* values, int32_t type, const uint8_t* nulls, uint32_t n,
              int32_t kind, void* result, void* stream);
/* Order-preserving key transforms (src/kernels/radix_sort_utils.cu:4-53):
 * INT32 -> x ^ 0x80000000, FLOAT32 -> sign flip; inverse = 1 restores.
 * INT64 / DATETIME -> x ^ 2^63 on each 64-bit value (dst holds two words per
 * value): the signed order of the result is the unsigned order of x, the
 * order the reference's sort gives int64 keys (radix_sort_kernel.cu:173). */
int yq_key_transform(const void* src, int32_t type, uint32_t* dst, uint32_t n,
                     int32_t inverse, void* stream);
/* launch_merge_sorted_array_kernel<T,Op> (include/kernels/merge_batchs.hpp:51):
 * merge the first k outputs of sorted A (m) and B (n); emit keys, source index
 * and from-A flag; *last_a (device) receives the co-rank of k in A. */
int yq_merge_path(const void* a, const void* b, int32_t type, int32_t width,
                  int32_t descending, uint32_t m, uint32_t n, uint32_t k, void* out_keys,
                  uint32_t* out_idx, uint8_t* out_from_a, int32_t* last_a, void* stream);
/* launch_cross_product_col<T> (cross_product_kernel.hpp:11): out[l*R + r] =
 * is_left ? col[l] : col[r] for l < left_rows, r < right_rows. */
int yq_cross_product_col(const yq_column* col, uint32_t left_rows, uint32_t right_rows,
                         int32_t is_left, yq_column* out, void* stream);

/* ---------------------------------------------------------------- GROUP BY
 * SELECT key, agg, ... GROUP BY key. The reference plans GROUP BY but folds
 * every row into one result (AggregateOperator ignores the groups,
 * include/engine/operators/aggregate_operator.hpp:84-104); this follows SQL
 * semantics: one output row per distinct key, NULL keys one group, in
 * ascending key order with the NULL group last (-0.0 equals +0.0, NaNs form
 * one group above +inf). Aggregates skip NULL inputs; COUNT(*) counts rows and
 * COUNT(col) non-NULL inputs (INT64); SUM of integers is INT64 (wrapping), of
 * floats FLOAT64 accumulated in FP64 (order of additions not fixed: within
 * 1e-15 relative between runs); AVG is FLOAT64; MIN/MAX keep the input type
 * (floats ordered -0.0 < +0.0, NaN above +inf). SUM/AVG/MIN/MAX over no
 * non-NULL input is NULL. */
typedef struct yq_group_agg {
  int32_t kind;    /* yq_agg_kind                              */
  int32_t column;  /* input column; ignored for YQ_AGG_COUNT_STAR */
} yq_group_agg;

size_t yq_group_by_workspace_size(const yq_column* key, uint32_t rows, int32_t nagg, uint32_t capacity);
/* out[0]: the key column (the key's type and width); out[1 + a]: aggregate a
 * (types above; a NULL-byte array is required except for COUNT). Every output
 * column has room for `capacity` rows. *groups = the number of groups; the
 * call synchronises `stream` to read it and returns YQ_ERR_CAPACITY (outputs
 * not written) when it exceeds `capacity`. Keys: INT32, INT64, DATETIME,
 * FLOAT32, FLOAT64, TEXT; aggregate inputs: the numeric types (DATETIME for
 * MIN/MAX/COUNT). */
int yq_group_by(const yq_batch* batch, int32_t key_col, const yq_group_agg* aggs, int32_t nagg, yq_column* out,
                uint32_t capacity, uint32_t* groups, void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- CSV scan
 * Device-side replacement of GetOperator::next's per-row loop
 * (src/engine/operators/get_operator.cpp:56-109): csv-parser's tokenizer
 * (vendor/csv-parser/csv.hpp:7063-7140, default format: ',' delimiter, '"'
 * quote, CR/LF newlines, blank lines skipped) and the per-field conversions
 * std::stoi / std::stof / getDateTime (strptime "%Y-%m-%d %H:%M:%S" + timegm,
 * include/enums/data_type_utils.hpp:24-44) / String::set
 * (include/kernels/string_kernel.hpp:16-31). `data` is the CSV text after the
 * header line, resident on the device; offsets are 32-bit, so one call takes
 * less than 4 GiB (the reference reads 4 MiB batches). */
#define YQ_CSV_MAX_FIELDS 64

/* A cell whose conversion throws in the reference (std::invalid_argument or
 * std::out_of_range from stoi/stof). The reference's process exits there; this
 * library writes 0 into the cell, finishes the batch and reports the first one. */
typedef struct yq_csv_error {
  uint64_t bad_cells;     /* cells that failed to convert                       */
  uint32_t first_row;     /* output row of the first                            */
  int32_t first_field;    /* its CSV field index, -1 when there is none         */
  int32_t kind;           /* 1: nothing converts (invalid_argument), 2: out of range */
} yq_csv_error;

size_t yq_csv_index_workspace_size(uint64_t nbytes);
/* Splits the text into records: the byte offset of each record's first byte
 * goes to record_starts[0..*records). Synchronises `stream` to read the count;
 * when it exceeds `capacity`, returns YQ_ERR_CAPACITY with *records = the count
 * and writes nothing (record_starts may be NULL to only count). */
int yq_csv_index(const uint8_t* data, uint64_t nbytes, uint32_t* record_starts, uint64_t capacity,
                 uint64_t* records, void* workspace, size_t workspace_bytes, void* stream);
size_t yq_csv_parse_workspace_size(uint32_t records);
/* Converts the records into typed columns. field_column[f] is the output
 * column of CSV field f (0 <= f < nfields, nfields = the header's field count)
 * or -1 when the field is not projected. Each output column has type INT32,
 * FLOAT32, DATETIME or TEXT (slot width multiple of 4, <= 256), room for
 * `records` rows, and a writable null-byte array: an empty field is NULL
 * (null byte 1, value INT_MIN / FLT_MIN / 0 / empty text, the sentinels of
 * get_operator.cpp:80-86). Records whose field count differs from nfields are
 * dropped, order kept (csv-parser's IGNORE_ROW policy); *rows = rows kept.
 * Synchronises `stream`. Cells that fail to convert: YQ_ERR_INVALID_ARG with
 * *error filled, every other cell still converted. Dropping rows allocates
 * stream-ordered temporaries (cudaMallocAsync) even with a workspace. */
int yq_csv_parse(const uint8_t* data, uint64_t nbytes, const uint32_t* record_starts, uint32_t records,
                 const int32_t* field_column, int32_t nfields, yq_column* out, int32_t ncols, uint32_t* rows,
                 yq_csv_error* error, void* workspace, size_t workspace_bytes, void* stream);

size_t yq_csv_format_workspace_size(uint32_t rows);
/* CsvWriter::batchToCsv (include/engine/operators/csv_writer.hpp:24-76) on the
 * device, without the header line: each row's cells joined by ',' and ended
 * by '\n'; NULL -> ""; INT32/INT64 -> std::to_chars; FLOAT32 -> std::to_chars
 * (fixed, 4 decimals; inf, -inf, nan, -nan); DATETIME -> quoted gmtime_r +
 * strftime("%Y-%m-%d %H:%M:%S") (data_type_utils.hpp:46-57); TEXT -> quoted
 * bytes up to the slot's first NUL, not escaped. Writes the text to `out`
 * (device) and its length to *bytes; synchronises `stream` to read the
 * length, and returns YQ_ERR_CAPACITY (nothing written, *bytes = the length)
 * when it exceeds `capacity`. Line offsets are 32-bit: YQ_ERR_UNSUPPORTED when
 * rows x the widest possible line reaches 4 GiB. */
int yq_csv_format(const yq_batch* batch, uint8_t* out, uint64_t capacity, uint64_t* bytes, void* workspace,
                  size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- device */
/* Number of SMs of the current device (cached per device). */
int yq_device_sm_count(void);
/* Kernel launches issued by this library on this process (for accounting). */
uint64_t yq_launch_count(void);
/* ---- Program-specialised row kernels.
 * The fused row operators (filter + aggregate / projection, their segmented
 * forms, the star-join aggregate) run an expression program. By default the
 * library compiles, once per distinct program (its instruction words; the
 * constants stay parameters), a kernel whose program is compile-time constant
 * (NVRTC, opened at run time, sm_100a) and launches it instead of the
 * interpreting kernel; the results are the same. yq_jit_enable(0) (or
 * YQ_JIT=0 in the environment) keeps the interpreting kernels; it returns the
 * previous setting. yq_jit_stats reports kernels compiled, compilations that
 * failed (their programs use the interpreting kernel), cache hits, total
 * compile time and the last compiler log. */
int yq_jit_enable(int32_t on);
int yq_jit_stats(int32_t* compiled, int32_t* failed, int32_t* hits, double* compile_ms, char* log,
                 size_t log_bytes);

/* Device timing of the library's own launches: when enabled, every kernel
 * launch records a CUDA event pair on its stream, tagged with the kernel and
 * its algorithmic bytes. yq_profile_read synchronises on the recorded events
 * and writes a JSON object {tag: {launches, ms, units}} (units = bytes);
 * returns the JSON length. */
int yq_profile_enable(int32_t on);
int yq_profile_read(char* out, size_t cap, int32_t reset);

#ifdef __cplusplus
}
#endif
#endif /* YQ_OPS_H */
