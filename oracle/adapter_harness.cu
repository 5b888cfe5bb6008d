// adapter_harness.cu — TEST INFRASTRUCTURE ONLY.
//
// C entry points that call the reference's own kernel-layer templates
// (YallaSQL::Kernel::launch_*, declared in the reference's include/kernels/*.hpp)
// as its operators do. Linked with yallasql_b200/adapter/yq_forward.cu, which
// defines those templates by forwarding to libyq_ops.so, so the tests reach
// the library through the reference's own signatures. All pointers are device
// pointers; every function synchronises and returns 0, or -1 when the
// forwarded call threw.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <stdexcept>

#include "kernels/comparison_operators_kernel.hpp"
#include "kernels/prefix_sum.hpp"
#include "kernels/radix_sort_kernel.hpp"

using namespace YallaSQL::Kernel;

namespace {

template <typename F>
int guarded(F f) {
  try {
    f();
  } catch (const std::exception& e) {
    fprintf(stderr, "forwarded call failed: %s\n", e.what());
    return -1;
  }
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

template <typename T>
void compare(const T* lhs, const T* rhs, int rhs_scalar, int op, int isneg, bool* out, unsigned n) {
  cudaStream_t s = 0;
  T* l = const_cast<T*>(lhs);
  T* r = const_cast<T*>(rhs);
  const OperandType tr = rhs_scalar ? OperandType::SCALAR : OperandType::VECTOR;
  const OperandType tl = OperandType::VECTOR;
  switch (op) {  // the reference's functor names: LE "<", LEQ "<=", GE ">", GEQ ">=", EQ, NEQ
    case 0: launch_conditional_operators<T, LEOperator<T>>(r, l, tr, tl, out, n, s, isneg != 0); break;
    case 1: launch_conditional_operators<T, LEQOperator<T>>(r, l, tr, tl, out, n, s, isneg != 0); break;
    case 2: launch_conditional_operators<T, GEOperator<T>>(r, l, tr, tl, out, n, s, isneg != 0); break;
    case 3: launch_conditional_operators<T, GEQOperator<T>>(r, l, tr, tl, out, n, s, isneg != 0); break;
    case 4: launch_conditional_operators<T, EQOperator<T>>(r, l, tr, tl, out, n, s, isneg != 0); break;
    default: launch_conditional_operators<T, NEQOperator<T>>(r, l, tr, tl, out, n, s, isneg != 0); break;
  }
}

// launch_radix_sort as OrderOperator calls it (order_operator.hpp:200-255):
// keys sorted in place, a permutation allocated by the callee.
template <typename Asc, typename Desc, typename T, size_t B>
void radix(T* keys, uint32_t* idx_out, uint32_t n, int desc) {
  uint32_t* idx = nullptr;
  if (desc) launch_radix_sort<Desc, T, B>(keys, idx, n, 0);
  else launch_radix_sort<Asc, T, B>(keys, idx, n, 0);
  cudaMemcpyAsync(idx_out, idx, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, 0);
  cudaFreeAsync(idx, 0);
}

}  // namespace

extern "C" {

int fwd_compare_i32(const int* lhs, const int* rhs, int rhs_scalar, int op, int isneg, uint8_t* out, unsigned n) {
  return guarded([&] { compare<int>(lhs, rhs, rhs_scalar, op, isneg, reinterpret_cast<bool*>(out), n); });
}

int fwd_compare_f32(const float* lhs, const float* rhs, int rhs_scalar, int op, int isneg, uint8_t* out,
                    unsigned n) {
  return guarded([&] { compare<float>(lhs, rhs, rhs_scalar, op, isneg, reinterpret_cast<bool*>(out), n); });
}

int fwd_compare_i64(const int64_t* lhs, const int64_t* rhs, int rhs_scalar, int op, int isneg, uint8_t* out,
                    unsigned n) {
  return guarded([&] { compare<int64_t>(lhs, rhs, rhs_scalar, op, isneg, reinterpret_cast<bool*>(out), n); });
}

int fwd_compare_str(const void* lhs, const void* rhs, int rhs_scalar, int op, int isneg, uint8_t* out, unsigned n) {
  return guarded([&] {
    compare<String>(static_cast<const String*>(lhs), static_cast<const String*>(rhs), rhs_scalar, op, isneg,
                    reinterpret_cast<bool*>(out), n);
  });
}

int fwd_logic(const uint8_t* a, const uint8_t* b, int is_or, uint8_t* out, unsigned n) {
  return guarded([&] {
    cudaStream_t s = 0;
    bool* x = reinterpret_cast<bool*>(const_cast<uint8_t*>(a));
    bool* y = reinterpret_cast<bool*>(const_cast<uint8_t*>(b));
    if (is_or)
      launch_conditional_operators<bool, OROperator>(y, x, OperandType::VECTOR, OperandType::VECTOR,
                                                     reinterpret_cast<bool*>(out), n, s, false);
    else
      launch_conditional_operators<bool, ANDOperator>(y, x, OperandType::VECTOR, OperandType::VECTOR,
                                                      reinterpret_cast<bool*>(out), n, s, false);
  });
}

int fwd_prefix_sum_mask(const uint8_t* mask, uint32_t* out, uint32_t n) {
  return guarded([&] {
    cudaStream_t s = 0;
    launch_prefix_sum_mask(reinterpret_cast<bool*>(const_cast<uint8_t*>(mask)), out, n, s);
  });
}

int fwd_prefix_sum_u32(const uint32_t* in, uint32_t* out, uint32_t n) {
  return guarded([&] {
    cudaStream_t s = 0;
    launch_prefix_sum<uint32_t>(const_cast<uint32_t*>(in), out, n, s);
  });
}

int fwd_radix_sort_u32(uint32_t* keys, uint32_t* idx_out, uint32_t n, int desc) {
  return guarded([&] { radix<AscOp<uint32_t>, DescOp<uint32_t>, uint32_t, BLOCK_DIM>(keys, idx_out, n, desc); });
}

int fwd_radix_sort_u64(uint64_t* keys, uint32_t* idx_out, uint32_t n, int desc) {
  return guarded([&] { radix<AscOp<uint64_t>, DescOp<uint64_t>, uint64_t, BLOCK_DIM>(keys, idx_out, n, desc); });
}

int fwd_radix_sort_str(void* keys, uint32_t* idx_out, uint32_t n, int desc) {
  return guarded([&] {
    radix<AscOpString, DescOpString, String, BLOCK_DIM_STR>(static_cast<String*>(keys), idx_out, n, desc);
  });
}

int fwd_float_to_uint32(const float* in, uint32_t* out, int n) {
  return guarded([&] { launch_float_to_uint32(const_cast<float*>(in), out, n); });
}

int fwd_int_to_uint32(const int* in, uint32_t* out, int n) {
  return guarded([&] { launch_int_to_uint32(const_cast<int*>(in), out, n); });
}

}  // extern "C"
