// ref_harness.cu — TEST INFRASTRUCTURE ONLY (parity pin).
//
// C entry points around the reference's OWN kernels (its src/kernels/*.cu,
// compiled where they lie by oracle/Makefile with the stand-in headers in
// oracle/ref_stubs/) so tests can run the reference on the same inputs as
// this repository's oracle and kernels. Each function calls the reference's
// launch_* in the same sequence its operators use (cited per function) and
// synchronises before returning. All pointers are device pointers.
//
// Not wrapped: the reference's prefix-sum kernels and everything built on
// them (launch_prefix_sum_mask / launch_prefix_sum, hence FilterOperator's
// compaction and launch_radix_sort). They index shared memory through
// CONFLICT_FREE_OFFSET(n), which expands to n >> (32 + n) >> 10
// (include/kernels/constants.hpp:12), a shift by 32 or more bits; built for
// sm_100a they returned a non-permutation from the radix sort and made an
// illegal memory access in the filter path, so they are not run again.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels/cast_operators_kernel.hpp"
#include "kernels/comparison_operators_kernel.hpp"
#include "kernels/cross_product_kernel.hpp"
#include "kernels/merge_batchs.hpp"
#include "kernels/move_rows_kernel.hpp"
#include "kernels/reduction_kernel.hpp"

using namespace YallaSQL::Kernel;

static int done(cudaStream_t s) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return (int)e;
}

extern "C" {

// Aggregates as AggregateExpression runs them (aggregate.hpp:55-145,
// reduction_kernel.cu:169-185): kind 0 SUM(float)->double, 1 MIN(float),
// 2 MAX(float), 3 SUM(int), 4 MIN(int), 5 MAX(int), 6 COUNT(non-null).
// Initial values follow aggregate.hpp:197-280 (MAX(float) starts at FLT_MIN).
int ref_reduce(const void* x, const char* nulls, uint32_t n, int kind, void* result_host) {
  // reduction_sum_wrap / reduction_count_notnull read isnull[i] unconditionally
  // (reduction_kernel.cu:94, :136): a null-flag array is mandatory.
  if (!nulls || !x) return -2;
  cudaStream_t s = 0;
  void* acc = nullptr;
  cudaMalloc(&acc, 8);
  int rc = 0;
  switch (kind) {
    case 0: {
      double init = 0;
      cudaMemcpy(acc, &init, 8, cudaMemcpyHostToDevice);
      launch_reduction_operators<float, double, SumOperator<double>>((float*)x, (double*)acc, (char*)nulls, n, s, init);
      rc = done(s);
      cudaMemcpy(result_host, acc, 8, cudaMemcpyDeviceToHost);
      break;
    }
    case 1:
    case 2: {
      float init = kind == 1 ? 3.402823466e+38f : 1.175494351e-38f;
      cudaMemcpy(acc, &init, 4, cudaMemcpyHostToDevice);
      if (kind == 1)
        launch_reduction_operators<float, float, MinOperator<float>>((float*)x, (float*)acc, (char*)nulls, n, s, init);
      else
        launch_reduction_operators<float, float, MaxOperator<float>>((float*)x, (float*)acc, (char*)nulls, n, s, init);
      rc = done(s);
      cudaMemcpy(result_host, acc, 4, cudaMemcpyDeviceToHost);
      break;
    }
    case 3:
    case 4:
    case 5: {
      int init = kind == 3 ? 0 : (kind == 4 ? 2147483647 : (-2147483647 - 1));
      cudaMemcpy(acc, &init, 4, cudaMemcpyHostToDevice);
      if (kind == 3) launch_reduction_operators<int, int, SumOperator<int>>((int*)x, (int*)acc, (char*)nulls, n, s, init);
      if (kind == 4) launch_reduction_operators<int, int, MinOperator<int>>((int*)x, (int*)acc, (char*)nulls, n, s, init);
      if (kind == 5) launch_reduction_operators<int, int, MaxOperator<int>>((int*)x, (int*)acc, (char*)nulls, n, s, init);
      rc = done(s);
      cudaMemcpy(result_host, acc, 4, cudaMemcpyDeviceToHost);
      break;
    }
    default: {
      int init = 0;
      cudaMemcpy(acc, &init, 4, cudaMemcpyHostToDevice);
      launch_reduction_count_notnull((char*)nulls, (int*)acc, (char*)nulls, n, s, init);
      rc = done(s);
      cudaMemcpy(result_host, acc, 4, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(acc);
  return rc;
}

// Merge the first k outputs of two sorted float buffers
// (launch_merge_sorted_array_kernel, merge_batchs.cu:144-148).
int ref_merge_f32(const float* A, const float* B, uint32_t m, uint32_t n, uint32_t k, int desc, float* C,
                  uint32_t* idx, uint8_t* from_a, int* last_a) {
  cudaStream_t s = 0;
  if (desc)
    launch_merge_sorted_array_kernel<float, DescSortMergeOp<float>>((float*)A, (float*)B, C, idx, (bool*)from_a,
                                                                    last_a, k, m, n, s);
  else
    launch_merge_sorted_array_kernel<float, AscSortMergeOp<float>>((float*)A, (float*)B, C, idx, (bool*)from_a,
                                                                   last_a, k, m, n, s);
  return done(s);
}

// Equi-join pairs of two int key columns (ComparisonJoinExpression with
// launch_outer_join_operators<int, EQOperator<int>>, comparison_join.hpp:70-236);
// pairs[2k] = left row, pairs[2k+1] = right row, in atomic (unspecified) order.
int ref_join_eq_i32(const int* left, uint32_t L, const int* right, uint32_t R, uint32_t* pairs, int* count) {
  cudaStream_t s = 0;
  cudaMemset(count, 0, 4);
  launch_outer_join_operators<int, EQOperator<int>>((int*)right, (int*)left, pairs, count, L, R, s);
  return done(s);
}

// CrossProductOperator's per-column replication (cross_product_kernel.cu:30-34).
int ref_cross_col_i32(const int* col, const char* nulls, uint32_t L, uint32_t R, int is_left, int* out,
                      char* out_nulls) {
  if (!nulls || !out_nulls) return -2;  // cross_product_kernel copies null bytes (cross_product_kernel.cu:17-22)
  launch_cross_product_col<int>(col, out, nulls, out_nulls, L, R, 0, is_left != 0);
  return done(0);
}

// price * CAST(discount AS FLOAT) as BoundFunc + Cast evaluate it
// (bound_func.hpp:45-167, cast.hpp:23-90).
int ref_mul_cast_f32(const float* price, const int* disc, uint32_t n, float* out) {
  cudaStream_t s = 0;
  float* fd = nullptr;
  cudaMalloc(&fd, n * 4);
  launch_numerical_cast<int, float>((int*)disc, fd, n, s);
  launch_binary_operators<float, MulOperator<float>>(fd, (float*)price, OperandType::VECTOR, OperandType::VECTOR, out,
                                                     n, s);
  int rc = done(s);
  cudaFree(fd);
  return rc;
}

// ------------------------------------------------------------------ timing
// Device time of the reference's own launch sequences on this GPU (CUDA
// events on one stream, one warm call first), for the reference arm of the
// benchmark. Buffers are allocated by the caller outside the timed region;
// the reference's per-batch cudaMallocAsync / host syncs are left out, so the
// figures favour the reference.
}  // extern "C"

template <typename F>
static int time_ms(F fn, int reps, cudaStream_t s, float* ms) {
  fn();
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s);
  for (int r = 0; r < reps; ++r) fn();
  cudaEventRecord(b, s);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  *ms = t / (reps > 0 ? reps : 1);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e == cudaSuccess) e = cudaGetLastError();
  return (int)e;
}

extern "C" {

// The aggregate part of the filter+aggregate query over n rows in the
// reference's batches (AggregateOperator::next per batch, aggregate.hpp:55-145;
// CastExpression + BoundFuncExpression for price * CAST(discount AS FLOAT),
// bound_func.hpp:45-167, cast.hpp:23-90): per batch CAST, MUL,
// reduction_sum_wrap SUM(float -> double), MIN, MAX and COUNT. The WHERE
// compaction is not run (it needs the prefix-sum kernels excluded above), so
// the aggregates see every row. acc: 32 bytes of device memory (SUM double at
// byte 0, MIN and MAX floats at bytes 8 and 12, COUNT int at byte 16).
int ref_time_aggregate(const float* price, const int* disc, const char* nulls, uint32_t n, uint32_t batch,
                       float* fd, float* prod, void* acc, int reps, float* ms) {
  cudaStream_t s;
  cudaStreamCreate(&s);
  auto run = [&]() {
    for (uint32_t o = 0; o < n; o += batch) {
      const uint32_t m = n - o < batch ? n - o : batch;
      launch_numerical_cast<int, float>((int*)disc + o, fd + o, m, s);
      launch_binary_operators<float, MulOperator<float>>(fd + o, (float*)price + o, OperandType::VECTOR,
                                                         OperandType::VECTOR, prod + o, m, s);
      launch_reduction_operators<float, double, SumOperator<double>>(prod + o, (double*)acc, (char*)nulls + o, m, s,
                                                                     0.0);
      launch_reduction_operators<float, float, MinOperator<float>>((float*)price + o, (float*)acc + 2,
                                                                   (char*)nulls + o, m, s, 3.402823466e+38f);
      launch_reduction_operators<float, float, MaxOperator<float>>((float*)price + o, (float*)acc + 3,
                                                                   (char*)nulls + o, m, s, 1.175494351e-38f);
      launch_reduction_count_notnull((char*)nulls + o, (int*)acc + 4, (char*)nulls + o, m, s, 0);
    }
  };
  const int rc = time_ms(run, reps, s, ms);
  cudaStreamDestroy(s);
  return rc;
}

// One merge window of OrderOperator's run merge (merge_two_runs ->
// launch_merge_sorted_array_kernel, order_operator.cpp:117-220,
// merge_batchs.cu:33-77): the first `window` outputs of two sorted float
// buffers of `window` rows each, descending as ORDER BY key DESC.
int ref_time_merge_window(const float* A, const float* B, uint32_t window, float* C, uint32_t* idx, uint8_t* from_a,
                          int* last_a, int reps, float* ms) {
  cudaStream_t s;
  cudaStreamCreate(&s);
  auto run = [&]() {
    launch_merge_sorted_array_kernel<float, DescSortMergeOp<float>>((float*)A, (float*)B, C, idx, (bool*)from_a,
                                                                    last_a, window, window, window, s);
  };
  const int rc = time_ms(run, reps, s, ms);
  cudaStreamDestroy(s);
  return rc;
}

// One fact batch x the dimension table through outer_join_batches<int, EQ>
// (JoinOperator -> ComparisonJoinExpression, comparison_join.hpp:70-236,
// comparison_operators_kernel.cu:6-22). The caller keeps the possible matches
// of a launch within `pairs` (its append is unchecked).
int ref_time_join_batch(const int* fact_key, uint32_t L, const int* dim_key, uint32_t R, uint32_t* pairs, int* count,
                        int reps, float* ms) {
  cudaStream_t s;
  cudaStreamCreate(&s);
  auto run = [&]() {
    cudaMemsetAsync(count, 0, 4, s);
    launch_outer_join_operators<int, EQOperator<int>>((int*)dim_key, (int*)fact_key, pairs, count, L, R, s);
  };
  const int rc = time_ms(run, reps, s, ms);
  cudaStreamDestroy(s);
  return rc;
}

// CrossProductOperator's materialisation of an L x R cross product of two
// int columns, right side in chunks of `chunk` rows (cross_product_operator.hpp:
// 87-125, cross_product_kernel.cu:8-34): per chunk, the left column replicated
// and the right chunk tiled into out_l / out_r (L * chunk rows each).
int ref_time_cross(const int* left, const char* lnulls, uint32_t L, const int* right, const char* rnulls, uint32_t R,
                   uint32_t chunk, int* out_l, char* out_ln, int* out_r, char* out_rn, int reps, float* ms) {
  cudaStream_t s;
  cudaStreamCreate(&s);
  auto run = [&]() {
    for (uint32_t o = 0; o < R; o += chunk) {
      const uint32_t m = R - o < chunk ? R - o : chunk;
      launch_cross_product_col<int>(left, out_l, lnulls, out_ln, L, m, s, true);
      launch_cross_product_col<int>(right + o, out_r, rnulls + o, out_rn, L, m, s, false);
    }
  };
  const int rc = time_ms(run, reps, s, ms);
  cudaStreamDestroy(s);
  return rc;
}

}  // extern "C"
