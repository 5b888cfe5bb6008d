// yq_forward.cu — the reference's kernel-layer templates forwarded to libyq_ops.so.
//
// YallaSQL's operators call YallaSQL::Kernel::launch_* templates declared in
// include/kernels/*.hpp and defined (with explicit instantiations) in
// src/kernels/*.cu. A maintainer keeps those declarations, drops the .cu files
// this file covers, compiles this file in their place and links libyq_ops.so:
// every instantiation the reference defines for these entry points is defined
// here, with the reference's signature, and forwards to the C ABI of
// include/yq_ops.h. Errors become std::runtime_error (the reference exits the
// process on a CUDA error, include/utils/macros.hpp:6-22).
//
// Covered (reference file:line of each declaration):
//   launch_conditional_operators<T, Op>   include/kernels/comparison_operators_kernel.hpp:8
//   launch_prefix_sum_mask                include/kernels/prefix_sum.hpp:26
//   launch_prefix_sum<uint32_t>           include/kernels/prefix_sum.hpp:29
//   launch_radix_sort<Op, T, BlockDim>    include/kernels/radix_sort_kernel.hpp:23
//   launch_{int,float}_to_uint32 and back include/kernels/radix_sort_kernel.hpp:83-89
#include <stdexcept>
#include <string>

#include "yq_ops.h"

#include "kernels/comparison_operators_kernel.hpp"
#include "kernels/prefix_sum.hpp"
#include "kernels/radix_sort_kernel.hpp"

namespace YallaSQL::Kernel {

namespace {

void yq_or_throw(int st, const char* where) {
  if (st != YQ_OK) throw std::runtime_error(std::string(where) + ": " + yq_status_string(st));
}

// The reference's column value types and their yq_type / width.
template <typename T>
struct YqType;
template <>
struct YqType<int> {
  static constexpr int32_t type = YQ_INT32, width = 4;
};
template <>
struct YqType<float> {
  static constexpr int32_t type = YQ_FLOAT32, width = 4;
};
template <>
struct YqType<int64_t> {  // DATETIME: epoch seconds (include/enums/data_type_utils.hpp:24-44)
  static constexpr int32_t type = YQ_DATETIME, width = 8;
};
template <>
struct YqType<String> {  // fixed NUL-padded slot (include/kernels/string_kernel.hpp:6-44)
  static constexpr int32_t type = YQ_TEXT, width = MAX_STR;
};
template <>
struct YqType<bool> {
  static constexpr int32_t type = YQ_BOOL, width = 1;
};

// The reference's comparison functors (comparison_operators_kernel.hpp:24-72):
// LE = "<", LEQ = "<=", GE = ">", GEQ = ">=".
template <typename Op>
struct YqCmp;
template <typename T>
struct YqCmp<LEOperator<T>> {
  static constexpr int32_t cmp = YQ_LT;
};
template <typename T>
struct YqCmp<LEQOperator<T>> {
  static constexpr int32_t cmp = YQ_LE;
};
template <typename T>
struct YqCmp<GEOperator<T>> {
  static constexpr int32_t cmp = YQ_GT;
};
template <typename T>
struct YqCmp<GEQOperator<T>> {
  static constexpr int32_t cmp = YQ_GE;
};
template <typename T>
struct YqCmp<EQOperator<T>> {
  static constexpr int32_t cmp = YQ_EQ;
};
template <typename T>
struct YqCmp<NEQOperator<T>> {
  static constexpr int32_t cmp = YQ_NE;
};

template <typename T>
yq_operand operand(const T* p, OperandType t) {
  return yq_operand{p, YqType<T>::type, YqType<T>::width, t == OperandType::SCALAR ? 1 : 0};
}

}  // namespace

// ------------------------------------------------------------ comparisons
// res[i] = op(lhs[i], rhs[i]), negated when isneg; a SCALAR operand is one
// device value broadcast over the batch.
template <typename T, typename Op>
void launch_conditional_operators(T* __restrict__ d_rhs, T* __restrict__ d_lhs, OperandType t_rhs, OperandType t_lhs,
                                  bool* d_res, unsigned int sz, cudaStream_t& stream, bool isneg) {
  yq_or_throw(yq_compare(operand<T>(d_lhs, t_lhs), operand<T>(d_rhs, t_rhs), YqCmp<Op>::cmp, isneg ? 1 : 0,
                         reinterpret_cast<uint8_t*>(d_res), sz, stream),
              "launch_conditional_operators");
}

// Conjunctions of two masks (ConjuntionExpression, filters/conjunction.hpp:76-113).
template <>
void launch_conditional_operators<bool, ANDOperator>(bool* __restrict__ d_rhs, bool* __restrict__ d_lhs,
                                                     OperandType t_rhs, OperandType t_lhs, bool* d_res,
                                                     unsigned int sz, cudaStream_t& stream, bool isneg) {
  if (isneg) throw std::runtime_error("launch_conditional_operators<bool, ANDOperator>: negation unsupported");
  yq_or_throw(yq_logic(operand<bool>(d_lhs, t_lhs), operand<bool>(d_rhs, t_rhs), 0, reinterpret_cast<uint8_t*>(d_res),
                       sz, stream),
              "launch_conditional_operators<bool, ANDOperator>");
}

template <>
void launch_conditional_operators<bool, OROperator>(bool* __restrict__ d_rhs, bool* __restrict__ d_lhs,
                                                    OperandType t_rhs, OperandType t_lhs, bool* d_res,
                                                    unsigned int sz, cudaStream_t& stream, bool isneg) {
  if (isneg) throw std::runtime_error("launch_conditional_operators<bool, OROperator>: negation unsupported");
  yq_or_throw(yq_logic(operand<bool>(d_lhs, t_lhs), operand<bool>(d_rhs, t_rhs), 1, reinterpret_cast<uint8_t*>(d_res),
                       sz, stream),
              "launch_conditional_operators<bool, OROperator>");
}

// ------------------------------------------------------------ prefix sums
// Inclusive scan of a 0/1 mask: res[i] = number of set flags in [0, i]
// (FilterOperator's 1-based output slots, filter_operator.hpp:31-98).
void launch_prefix_sum_mask(bool* arr, uint32_t* res, const uint32_t sz, cudaStream_t& stream) {
  yq_or_throw(yq_prefix_sum_mask(reinterpret_cast<const uint8_t*>(arr), res, sz, nullptr, 0, stream),
              "launch_prefix_sum_mask");
}

template <typename T>
void launch_prefix_sum(T* arr, T* res, const uint32_t sz, cudaStream_t& stream);

template <>
void launch_prefix_sum<uint32_t>(uint32_t* arr, uint32_t* res, const uint32_t sz, cudaStream_t& stream) {
  yq_or_throw(yq_prefix_sum_u32(arr, res, sz, nullptr, 0, stream), "launch_prefix_sum<uint32_t>");
}

// ------------------------------------------------------------ radix sort
// The reference sorts order-preserving unsigned keys (int_to_uint32 /
// float_to_uint32 output, int64 dates read as uint64, String slots) with a
// stable LSD radix argsort; on return d_input holds the sorted keys and
// d_idxs_in (allocated here, stream-ordered; the caller frees it) the
// permutation (radix_sort_kernel.cu:138-168). Here the keys go through the
// library's stable sort: unsigned keys as signed ones after flipping the top
// bit, String slots as text (compared as unsigned bytes); DESC keeps ties in
// input order as the reference's inverted digits do.
namespace {

template <typename T>
struct SortKey;  // how a reference key type becomes a yq sort column
template <>
struct SortKey<uint32_t> {
  static constexpr int32_t type = YQ_INT32, width = 4;
};
template <>
struct SortKey<uint64_t> {
  static constexpr int32_t type = YQ_INT64, width = 8;
};
template <>
struct SortKey<String> {
  static constexpr int32_t type = YQ_TEXT, width = MAX_STR;
};

template <typename OP, typename T>
void radix_sort(T* d_input, uint32_t*& d_idxs_in, const uint32_t N, cudaStream_t stream, bool desc) {
  d_idxs_in = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&d_idxs_in), (size_t)(N ? N : 1) * sizeof(uint32_t), stream) !=
      cudaSuccess)
    throw std::runtime_error("launch_radix_sort: cudaMallocAsync");
  if (N == 0) return;
  void* keys = d_input;  // the column the library sorts
  void* tmp = nullptr;
  if (cudaMallocAsync(&tmp, (size_t)N * sizeof(T), stream) != cudaSuccess)
    throw std::runtime_error("launch_radix_sort: cudaMallocAsync");
  if (SortKey<T>::type == YQ_INT32 || SortKey<T>::type == YQ_INT64) {
    // unsigned order = signed order of the value with its top bit flipped
    yq_or_throw(yq_key_transform(d_input, SortKey<T>::type, static_cast<uint32_t*>(tmp), N, 1, stream),
                "launch_radix_sort");
    keys = tmp;
  }
  yq_column col{keys, nullptr, SortKey<T>::type, SortKey<T>::width};
  yq_or_throw(yq_sort_indices(&col, N, desc ? 1 : 0, 0, d_idxs_in, nullptr, nullptr, 0, stream), "launch_radix_sort");
  // the sorted keys back into d_input
  yq_column src{d_input, nullptr, SortKey<T>::type, SortKey<T>::width};
  yq_column dst{tmp, nullptr, SortKey<T>::type, SortKey<T>::width};
  yq_or_throw(yq_gather(&src, 1, d_idxs_in, N, &dst, stream), "launch_radix_sort");
  if (cudaMemcpyAsync(d_input, tmp, (size_t)N * sizeof(T), cudaMemcpyDeviceToDevice, stream) != cudaSuccess ||
      cudaFreeAsync(tmp, stream) != cudaSuccess)
    throw std::runtime_error("launch_radix_sort: copy back");
}

}  // namespace

template <typename OP, typename T, size_t BlockDim>
void launch_radix_sort(T* d_input, uint32_t*& d_idxs_in, const uint32_t N, cudaStream_t stream);

template <>
void launch_radix_sort<AscOp<uint32_t>, uint32_t, BLOCK_DIM>(uint32_t* d, uint32_t*& idx, const uint32_t n,
                                                             cudaStream_t s) {
  radix_sort<AscOp<uint32_t>, uint32_t>(d, idx, n, s, false);
}
template <>
void launch_radix_sort<AscOp<uint64_t>, uint64_t, BLOCK_DIM>(uint64_t* d, uint32_t*& idx, const uint32_t n,
                                                             cudaStream_t s) {
  radix_sort<AscOp<uint64_t>, uint64_t>(d, idx, n, s, false);
}
template <>
void launch_radix_sort<AscOpString, String, BLOCK_DIM_STR>(String* d, uint32_t*& idx, const uint32_t n,
                                                           cudaStream_t s) {
  radix_sort<AscOpString, String>(d, idx, n, s, false);
}
template <>
void launch_radix_sort<DescOp<uint32_t>, uint32_t, BLOCK_DIM>(uint32_t* d, uint32_t*& idx, const uint32_t n,
                                                              cudaStream_t s) {
  radix_sort<DescOp<uint32_t>, uint32_t>(d, idx, n, s, true);
}
template <>
void launch_radix_sort<DescOp<uint64_t>, uint64_t, BLOCK_DIM>(uint64_t* d, uint32_t*& idx, const uint32_t n,
                                                              cudaStream_t s) {
  radix_sort<DescOp<uint64_t>, uint64_t>(d, idx, n, s, true);
}
template <>
void launch_radix_sort<DescOpString, String, BLOCK_DIM_STR>(String* d, uint32_t*& idx, const uint32_t n,
                                                            cudaStream_t s) {
  radix_sort<DescOpString, String>(d, idx, n, s, true);
}

// Key transforms BoundRefSortExpression applies before sorting
// (radix_sort_utils.cu:4-53; default stream, as the reference launches them).
void launch_int_to_uint32(int* arr, uint32_t* res, int N) {
  yq_or_throw(yq_key_transform(arr, YQ_INT32, res, (uint32_t)N, 0, nullptr), "launch_int_to_uint32");
}
void launch_uint32_to_int(uint32_t* arr, int* res, int N) {
  yq_or_throw(yq_key_transform(arr, YQ_INT32, reinterpret_cast<uint32_t*>(res), (uint32_t)N, 1, nullptr),
              "launch_uint32_to_int");
}
void launch_float_to_uint32(float* arr, uint32_t* res, int N) {
  yq_or_throw(yq_key_transform(arr, YQ_FLOAT32, res, (uint32_t)N, 0, nullptr), "launch_float_to_uint32");
}
void launch_uint32_to_float(uint32_t* arr, float* res, int N) {
  yq_or_throw(yq_key_transform(arr, YQ_FLOAT32, reinterpret_cast<uint32_t*>(res), (uint32_t)N, 1, nullptr),
              "launch_uint32_to_float");
}

// ------------------------------------------ explicit instantiations
// The instantiations src/kernels/comparison_operators_kernel.cu:169-199 provides.
#define YQ_FWD_CMP(T)                                                                                                 \
  template void launch_conditional_operators<T, LEOperator<T>>(T* __restrict__, T* __restrict__, OperandType,        \
                                                               OperandType, bool*, unsigned int, cudaStream_t&, bool); \
  template void launch_conditional_operators<T, GEOperator<T>>(T* __restrict__, T* __restrict__, OperandType,        \
                                                               OperandType, bool*, unsigned int, cudaStream_t&, bool); \
  template void launch_conditional_operators<T, LEQOperator<T>>(T* __restrict__, T* __restrict__, OperandType,       \
                                                                OperandType, bool*, unsigned int, cudaStream_t&,      \
                                                                bool);                                                \
  template void launch_conditional_operators<T, GEQOperator<T>>(T* __restrict__, T* __restrict__, OperandType,       \
                                                                OperandType, bool*, unsigned int, cudaStream_t&,      \
                                                                bool);                                                \
  template void launch_conditional_operators<T, EQOperator<T>>(T* __restrict__, T* __restrict__, OperandType,        \
                                                               OperandType, bool*, unsigned int, cudaStream_t&, bool); \
  template void launch_conditional_operators<T, NEQOperator<T>>(T* __restrict__, T* __restrict__, OperandType,       \
                                                                OperandType, bool*, unsigned int, cudaStream_t&, bool);
YQ_FWD_CMP(int)
YQ_FWD_CMP(float)
YQ_FWD_CMP(int64_t)
YQ_FWD_CMP(String)
#undef YQ_FWD_CMP

}  // namespace YallaSQL::Kernel
