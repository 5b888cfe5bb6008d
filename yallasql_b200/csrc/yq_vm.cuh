// Register-resident expression machine for the fused row kernels.
//
// A thread evaluates one program over ITEMS consecutive rows at a time. The
// stack (depth 4) is four named slot groups, so every access is static and the
// whole machine stays in registers. The host loader (vm_host.cuh) resolves
// every instruction to one opcode per (operation, value class, comparison or
// arithmetic operator), so the kernel dispatches once per instruction and the
// body that runs is straight-line code for ITEMS rows with no further type or
// operator tests; it also records how many live stack slots each instruction
// has to move, so conjunctions of `column <cmp> constant` terms never touch the
// lower slots. Long, rarely used bodies (integer and float DIV / MOD, float to
// integer casts, text ordering) run out of line so that the common ones keep
// their registers.
//
// Slot encoding (one 64-bit word per row): INT32 and FLOAT32 in the low word
// (the high word is not read), INT64/DATETIME as int64, FLOAT64 bits. A BOOL
// value is a bit mask: v[0] bit k is TRUE for row k. `valid` holds one bit per
// row (0 = NULL or row out of range); a TRUE bit is always also a valid bit.
//
// Column reads come either straight from global memory (`STAGED` = false) or
// from a shared-memory stage that the kernel filled for the current step of
// rows (`STAGED` = true, see yq_stage.cuh).
#pragma once

#include "yq_common.cuh"

namespace yq {

constexpr int ITEMS = 4;  // rows per thread per step (one 16-byte load of a 4-byte column)
constexpr uint32_t kItemsMask = (1u << ITEMS) - 1u;

// Dynamic shared memory of the staged kernels (one declaration for all).
extern __shared__ __align__(128) unsigned char yq_dyn_smem[];

// Loader-side instruction kinds: public yq_opcode values plus the fused forms.
enum : uint8_t {
  OP_COL = YQ_OP_COL,
  OP_CONST = YQ_OP_CONST,
  OP_NULL = YQ_OP_NULL,
  OP_CAST = YQ_OP_CAST,
  OP_ARITH = YQ_OP_ARITH,
  OP_CMP = YQ_OP_CMP,
  OP_CMP_COL_CONST = YQ_OP_CMP_COL_CONST,
  OP_CMP_COL_COL = YQ_OP_CMP_COL_COL,
  OP_AND = YQ_OP_AND,
  OP_OR = YQ_OP_OR,
  OP_NOT = YQ_OP_NOT,
  OP_IS_NULL = YQ_OP_IS_NULL,
  OP_IS_NOT_NULL = YQ_OP_IS_NOT_NULL,
  OP_ARITH_COL = 20,          // top := top <arith a> column b (cast to `type`)
  OP_ARITH_CONST = 21,        // top := top <arith a> constant imm
  OP_AND_CMP_COL_CONST = 22,  // top := top AND (column b <cmp a> constant imm)
  OP_EMIT_PRED = 30,          // selection := top is TRUE; pop
  OP_EMIT_AGG = 31,           // aggregate a absorbs top (update code b); pop
  OP_EMIT_PROJ = 32,          // projection a writes top for selected rows; pop
};

// Value classes of stack slots and columns.
enum : int { TC_I32 = 0, TC_I64 = 1, TC_F32 = 2, TC_F64 = 3, TC_BOOL = 4, TC_TEXT = 5 };

__host__ __device__ inline int type_class(int t) {
  switch (t) {
    case YQ_INT32: return TC_I32;
    case YQ_INT64:
    case YQ_DATETIME: return TC_I64;
    case YQ_FLOAT32: return TC_F32;
    case YQ_FLOAT64: return TC_F64;
    case YQ_BOOL: return TC_BOOL;
    default: return TC_TEXT;
  }
}

// Resolved opcodes (what the kernels dispatch on).
constexpr int R_COL = 0;           // + target class (0..4): push column a, converted from its own class
constexpr int R_CONST = 5;         // + class (0..4): push constant imm
constexpr int R_NULL = 10;         // push NULL
constexpr int R_CAST = 11;         // + from * 5 + to: top := CAST(top)
constexpr int R_ARITH = 36;        // + class * 5 + op (classes I32..F64): top := second <op> top, pop
constexpr int R_ARITH_COL = 56;    // + class * 5 + op: top := top <op> column b (converted)
constexpr int R_ARITH_CONST = 76;  // + class * 5 + op: top := top <op> constant imm
constexpr int R_CMP = 96;          // + class * 6 + cmp (classes I32..BOOL): top := second <cmp> top, pop
constexpr int R_CMP_CC = 126;      // + class * 6 + cmp (classes I32..TEXT): column b <cmp> constant imm
constexpr int R_CMP_CCOL = 162;    // + class * 6 + cmp: column b <cmp> column c
constexpr int R_AND = 198;
constexpr int R_OR = 199;
constexpr int R_NOT = 200;
constexpr int R_IS_NULL = 201;
constexpr int R_IS_NOT_NULL = 202;
constexpr int R_EMIT_PRED = 203;
constexpr int R_EMIT_AGG = 204;   // + aggregate update kind (AK_*): aggregate a absorbs top, pop
constexpr int R_EMIT_PROJ = 217;  // + 0 (one byte), 1 (4 bytes), 2 (8 bytes): projection a, pop
constexpr int R_COUNT = 220;

// Per-row update of an aggregate, with the input's slot class folded in.
enum : int {
  AK_COUNT = 0,
  AK_SUM_I32, AK_SUM_I64, AK_SUM_F32, AK_SUM_F64,
  AK_MIN_I32, AK_MIN_I64, AK_MIN_F32, AK_MIN_F64,
  AK_MAX_I32, AK_MAX_I64, AK_MAX_F32, AK_MAX_F64,
  AK_N
};

// Aggregate state codes (init / combine / read of one aggregate's state).
enum : uint8_t {
  UPD_COUNT_STAR = 0,
  UPD_COUNT = 1,
  UPD_SUM_I = 2,
  UPD_SUM_F = 3,
  UPD_MIN_I = 4,
  UPD_MAX_I = 5,
  UPD_MIN_F = 6,
  UPD_MAX_F = 7
};

// RInsn::flags: bits 0-1 = live stack slots the instruction moves (down for a
// push, up for a pop); RF_AND = a column/constant comparison ANDs its result
// into the top instead of pushing it.
constexpr uint8_t RF_MOVES = 3;
constexpr uint8_t RF_AND = 4;

// Loader-side instruction (public fields plus the fused kinds).
struct Insn {
  uint8_t op, type, a, b;
  int32_t imm;
};

// Resolved instruction.
struct RInsn {
  uint16_t opc;
  uint8_t flags;
  uint8_t a;     // column (COL), aggregate or projection index
  uint8_t b;     // column of ARITH_COL / CMP_CC / CMP_CCOL
  uint8_t c;     // second column of CMP_CCOL
  uint16_t imm;  // constant or text constant index
};

struct DevCol {
  const char* data;
  const uint8_t* nulls;
  int32_t type;
  int32_t tc;      // value class
  int32_t width;
  int32_t vec;     // data is 16-byte aligned (vector loads allowed)
  int32_t nvec;    // nulls is 4-byte aligned
  uint32_t soff;   // staged kernels: byte offset of the column's rows in a stage
  uint32_t snoff;  // staged kernels: byte offset of its null bytes in a stage
};

constexpr int kMaxInsns = 128;

struct VmProgram {
  RInsn code[kMaxInsns];
  int64_t consts[YQ_MAX_CONSTANTS];
  uint32_t text[YQ_MAX_TEXT_CONSTANTS][YQ_MAX_TEXT_WIDTH / 4];  // big-endian words
  int32_t text_words;
  int32_t ncols;
  DevCol cols[YQ_MAX_BATCH_COLUMNS];
};

struct Val {
  uint64_t v[ITEMS];
  uint32_t valid;
};

struct Stack {
  Val s0, s1, s2, s3;
};

// Rows of one step: row k of this thread is tile0 + lr + k. In staged
// kernels the step's rows sit in shared memory at byte offset `stage`.
struct Ctx {
  uint32_t tile0;
  uint32_t lr;
  uint32_t inr;     // rows in range
  uint32_t stage;   // shared-memory offset of the step's stage (staged kernels)
  uint32_t vec_ok;  // tile0 is a multiple of 16 rows (vector loads of aligned columns allowed)
};

// ----------------------------------------------------------- stack moves
__device__ __forceinline__ void push_moves(Stack& S, uint8_t f) {
  const int n = f & RF_MOVES;
  if (n >= 3) S.s3 = S.s2;
  if (n >= 2) S.s2 = S.s1;
  if (n >= 1) S.s1 = S.s0;
}
// After a binary operation wrote its result into s0 (from s1 and s0): the
// slots below the operands move up by one.
__device__ __forceinline__ void binary_moves(Stack& S, uint8_t f) {
  const int n = f & RF_MOVES;
  if (n >= 1) S.s1 = S.s2;
  if (n >= 2) S.s2 = S.s3;
}
// Pop the top.
__device__ __forceinline__ void pop_moves(Stack& S, uint8_t f) {
  const int n = f & RF_MOVES;
  if (n >= 1) S.s0 = S.s1;
  if (n >= 2) S.s1 = S.s2;
  if (n >= 3) S.s2 = S.s3;
}

// ------------------------------------------------------------ slot values
__device__ __forceinline__ int32_t as_i32(uint64_t x) { return (int32_t)(uint32_t)x; }
__device__ __forceinline__ float as_f32(uint64_t x) { return __uint_as_float((uint32_t)x); }
__device__ __forceinline__ int64_t as_i64(uint64_t x) { return (int64_t)x; }
__device__ __forceinline__ double as_f64(uint64_t x) { return __longlong_as_double((long long)x); }
__device__ __forceinline__ uint64_t from_i32(int32_t x) { return (uint64_t)(uint32_t)x; }
__device__ __forceinline__ uint64_t from_f32(float x) { return (uint64_t)__float_as_uint(x); }
__device__ __forceinline__ uint64_t from_i64(int64_t x) { return (uint64_t)x; }
__device__ __forceinline__ uint64_t from_f64(double x) { return (uint64_t)__double_as_longlong(x); }

// Bit k set when byte k of w is non-zero (k < 4).
__device__ __forceinline__ uint32_t nonzero_bytes(uint32_t w) {
  uint32_t t = (w | (w >> 4)) & 0x0f0f0f0fu;
  t = (t | (t >> 2)) & 0x03030303u;
  t = (t | (t >> 1)) & 0x01010101u;
  return (t * 0x01020408u) >> 24;
}

// ------------------------------------------------------------ column reads
template <bool STAGED>
__device__ __forceinline__ uint32_t null_bits(const DevCol& c, const Ctx& X) {
  if (!c.nulls) return 0u;
  if constexpr (STAGED) {
    const uint32_t w = *reinterpret_cast<const uint32_t*>(yq_dyn_smem + X.stage + c.snoff + X.lr);
    return nonzero_bytes(w) & X.inr;
  } else {
    const uint8_t* p = c.nulls + X.tile0 + X.lr;
    if (X.inr == kItemsMask && c.nvec && X.vec_ok) return nonzero_bytes(__ldg(reinterpret_cast<const uint32_t*>(p)));
    uint32_t nb = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
      if (X.inr >> k & 1u) nb |= (uint32_t)(p[k] != 0) << k;
    return nb;
  }
}

// ITEMS values of a column in its own class (BOOL as a mask in v[0]).
template <int T, bool STAGED>
__device__ __forceinline__ void load_raw(const DevCol& c, const Ctx& X, uint64_t (&v)[ITEMS]) {
  if constexpr (T == TC_I32 || T == TC_F32) {
    if constexpr (STAGED) {
      const uint4 q = *reinterpret_cast<const uint4*>(yq_dyn_smem + X.stage + c.soff + X.lr * 4);
      v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
      const char* p = c.data + (size_t)(X.tile0 + X.lr) * 4;
      if (X.inr == kItemsMask && c.vec && X.vec_ok) {
        const uint4 q = ldg_nc_v4(p);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
      } else {
#pragma unroll
        for (int k = 0; k < ITEMS; ++k)
          v[k] = (X.inr >> k & 1u) ? __ldg(reinterpret_cast<const uint32_t*>(p) + k) : 0u;
      }
    }
  } else if constexpr (T == TC_I64 || T == TC_F64) {
    uint4 q0, q1;
    if constexpr (STAGED) {
      const unsigned char* p = yq_dyn_smem + X.stage + c.soff + X.lr * 8;
      q0 = *reinterpret_cast<const uint4*>(p);
      q1 = *reinterpret_cast<const uint4*>(p + 16);
    } else {
      const char* p = c.data + (size_t)(X.tile0 + X.lr) * 8;
      if (X.inr == kItemsMask && c.vec && X.vec_ok) {
        q0 = ldg_nc_v4(p);
        q1 = ldg_nc_v4(p + 16);
      } else {
#pragma unroll
        for (int k = 0; k < ITEMS; ++k)
          v[k] = (X.inr >> k & 1u) ? (uint64_t)__ldg(reinterpret_cast<const unsigned long long*>(p) + k) : 0ull;
        return;
      }
    }
    v[0] = ((uint64_t)q0.y << 32) | q0.x;
    v[1] = ((uint64_t)q0.w << 32) | q0.z;
    v[2] = ((uint64_t)q1.y << 32) | q1.x;
    v[3] = ((uint64_t)q1.w << 32) | q1.z;
  } else if constexpr (T == TC_BOOL) {
    uint32_t w = 0;
    if constexpr (STAGED) {
      w = *reinterpret_cast<const uint32_t*>(yq_dyn_smem + X.stage + c.soff + X.lr);
    } else {
      const uint8_t* p = reinterpret_cast<const uint8_t*>(c.data) + X.tile0 + X.lr;
      if (X.inr == kItemsMask && c.vec && X.vec_ok) {
        w = __ldg(reinterpret_cast<const uint32_t*>(p));
      } else {
#pragma unroll
        for (int k = 0; k < ITEMS; ++k)
          if (X.inr >> k & 1u) w |= (uint32_t)p[k] << (8 * k);
      }
    }
    v[0] = nonzero_bytes(w);
  }
}

// ------------------------------------------------------------------- casts
// One value from class F to class T (both numeric); `ok` false = NULL.
template <int F, int T>
__device__ __forceinline__ uint64_t cast_num(uint64_t x, bool& ok) {
  ok = true;
  if constexpr (F == T) {
    return x;
  } else if constexpr (F == TC_I32 || F == TC_I64) {
    const int64_t v = (F == TC_I32) ? (int64_t)as_i32(x) : as_i64(x);
    if constexpr (T == TC_I32) {
      if (v < INT32_MIN || v > INT32_MAX) { ok = false; return 0; }
      return from_i32((int32_t)v);
    } else if constexpr (T == TC_I64) {
      return from_i64(v);
    } else if constexpr (T == TC_F32) {
      return (F == TC_I32) ? from_f32(__int2float_rn(as_i32(x))) : from_f32(__ll2float_rn(v));
    } else {
      return (F == TC_I32) ? from_f64(__int2double_rn(as_i32(x))) : from_f64(__ll2double_rn(v));
    }
  } else {
    const double v = (F == TC_F32) ? (double)as_f32(x) : as_f64(x);
    if constexpr (T == TC_F32) {
      return from_f32(__double2float_rn(v));
    } else if constexpr (T == TC_F64) {
      return from_f64(v);
    } else if constexpr (T == TC_I32) {
      // Round half to even, NULL when not representable.
      if (!(v >= -2147483648.0 && v < 2147483648.0)) { ok = false; return 0; }
      const double r = rint(v);
      if (r < -2147483648.0 || r > 2147483647.0) { ok = false; return 0; }
      return from_i32((int32_t)r);
    } else {
      if (!(v >= -9223372036854775808.0 && v < 9223372036854775808.0)) { ok = false; return 0; }
      return from_i64((int64_t)rint(v));
    }
  }
}

template <int F>
__device__ __forceinline__ bool num_nonzero(uint64_t x) {
  if constexpr (F == TC_I32) return as_i32(x) != 0;
  else if constexpr (F == TC_I64) return as_i64(x) != 0;
  else if constexpr (F == TC_F32) return as_f32(x) != 0.0f;
  else return as_f64(x) != 0.0;
}

template <int T>
__device__ __forceinline__ uint64_t one_or_zero(bool b) {
  if constexpr (T == TC_F32) return from_f32(b ? 1.0f : 0.0f);
  else if constexpr (T == TC_F64) return from_f64(b ? 1.0 : 0.0);
  else return b ? 1ull : 0ull;
}

// Float -> integer conversions (range checks and rounding) stay out of line.
template <int F, int T>
__device__ __noinline__ Val cast_val_slow(Val x) {
  uint32_t valid = x.valid;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    bool ok;
    x.v[k] = cast_num<F, T>(x.v[k], ok);
    if (!ok) valid &= ~(1u << k);
  }
  x.valid = valid;
  return x;
}

template <int F, int T>
__device__ __forceinline__ void cast_val(Val& x) {
  if constexpr (F == T || F == TC_TEXT || T == TC_TEXT) {
    return;
  } else if constexpr (F == TC_BOOL) {
    const uint32_t m = (uint32_t)x.v[0];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) x.v[k] = one_or_zero<T>(m >> k & 1u);
  } else if constexpr (T == TC_BOOL) {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) m |= (uint32_t)num_nonzero<F>(x.v[k]) << k;
    x.v[0] = m & x.valid;
  } else if constexpr ((F == TC_F32 || F == TC_F64) && (T == TC_I32 || T == TC_I64)) {
    x = cast_val_slow<F, T>(x);
  } else {
    uint32_t valid = x.valid;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      bool ok;
      x.v[k] = cast_num<F, T>(x.v[k], ok);
      if (!ok) valid &= ~(1u << k);
    }
    x.valid = valid;
  }
}

// Column `c` as class T (converted from the column's own class).
template <int T, bool STAGED>
__device__ __forceinline__ void load_as(const DevCol& c, const Ctx& X, Val& out) {
  out.valid = X.inr & ~null_bits<STAGED>(c, X);
  switch (c.tc) {
#define YQ_LOAD_AS(SC)                 \
  case SC:                             \
    load_raw<SC, STAGED>(c, X, out.v); \
    cast_val<SC, T>(out);              \
    break;
    YQ_LOAD_AS(TC_I32) YQ_LOAD_AS(TC_I64) YQ_LOAD_AS(TC_F32) YQ_LOAD_AS(TC_F64) YQ_LOAD_AS(TC_BOOL)
#undef YQ_LOAD_AS
    default: break;
  }
  if constexpr (T == TC_BOOL) out.v[0] &= out.valid;
}

// -------------------------------------------------------------- arithmetic
template <int T, int A>
__device__ __forceinline__ uint64_t arith1(uint64_t a, uint64_t b, bool& ok) {
  ok = true;
  if constexpr (T == TC_I32) {
    const int32_t x = as_i32(a), y = as_i32(b);
    const uint32_t ux = (uint32_t)x, uy = (uint32_t)y;
    if constexpr (A == YQ_ADD) return from_i32((int32_t)(ux + uy));
    else if constexpr (A == YQ_SUB) return from_i32((int32_t)(ux - uy));
    else if constexpr (A == YQ_MUL) return from_i32((int32_t)(ux * uy));
    else if constexpr (A == YQ_DIV) {
      if (y == 0) { ok = false; return 0; }
      if (y == -1) return from_i32((int32_t)(0u - ux));
      return from_i32(x / y);
    } else {
      if (y == 0) { ok = false; return 0; }
      if (y == -1) return 0;
      return from_i32(x % y);
    }
  } else if constexpr (T == TC_I64) {
    const int64_t x = as_i64(a), y = as_i64(b);
    const uint64_t ux = (uint64_t)x, uy = (uint64_t)y;
    if constexpr (A == YQ_ADD) return ux + uy;
    else if constexpr (A == YQ_SUB) return ux - uy;
    else if constexpr (A == YQ_MUL) return ux * uy;
    else if constexpr (A == YQ_DIV) {
      if (y == 0) { ok = false; return 0; }
      if (y == -1) return 0ull - ux;
      return from_i64(x / y);
    } else {
      if (y == 0) { ok = false; return 0; }
      if (y == -1) return 0;
      return from_i64(x % y);
    }
  } else if constexpr (T == TC_F32) {
    const float x = as_f32(a), y = as_f32(b);
    if constexpr (A == YQ_ADD) return from_f32(__fadd_rn(x, y));
    else if constexpr (A == YQ_SUB) return from_f32(__fsub_rn(x, y));
    else if constexpr (A == YQ_MUL) return from_f32(__fmul_rn(x, y));
    else if constexpr (A == YQ_DIV) return from_f32(__fdiv_rn(x, y));
    else return from_f32(fmodf(x, y));
  } else {
    const double x = as_f64(a), y = as_f64(b);
    if constexpr (A == YQ_ADD) return from_f64(__dadd_rn(x, y));
    else if constexpr (A == YQ_SUB) return from_f64(__dsub_rn(x, y));
    else if constexpr (A == YQ_MUL) return from_f64(__dmul_rn(x, y));
    else if constexpr (A == YQ_DIV) return from_f64(__ddiv_rn(x, y));
    else return from_f64(fmod(x, y));
  }
}

// a <A> b for ITEMS rows (valid bits combined; integer DIV/MOD by zero is NULL).
template <int T, int A>
__device__ __forceinline__ Val arith_items(Val a, const Val& b) {
  uint32_t valid = a.valid & b.valid;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    bool ok;
    a.v[k] = arith1<T, A>(a.v[k], b.v[k], ok);
    if (!ok) valid &= ~(1u << k);
  }
  a.valid = valid;
  return a;
}

// DIV and MOD (long instruction sequences) run out of line.
template <int T, int A>
__device__ __noinline__ Val arith_slow(Val a, Val b) {
  return arith_items<T, A>(a, b);
}

template <int T, int A>
__device__ __forceinline__ Val arith_val(const Val& a, const Val& b) {
  if constexpr (A == YQ_DIV || A == YQ_MOD) return arith_slow<T, A>(a, b);
  else return arith_items<T, A>(a, b);
}

// ------------------------------------------------------------- comparisons
template <int R, typename V>
__device__ __forceinline__ bool relop(V x, V y) {
  if constexpr (R == YQ_LT) return x < y;
  else if constexpr (R == YQ_LE) return x <= y;
  else if constexpr (R == YQ_GT) return x > y;
  else if constexpr (R == YQ_GE) return x >= y;
  else if constexpr (R == YQ_EQ) return x == y;
  else return x != y;
}

template <int C, int R>
__device__ __forceinline__ bool rel1(uint64_t a, uint64_t b) {
  if constexpr (C == TC_I32) return relop<R>(as_i32(a), as_i32(b));
  else if constexpr (C == TC_I64) return relop<R>(as_i64(a), as_i64(b));
  else if constexpr (C == TC_F32) return relop<R>(as_f32(a), as_f32(b));
  else return relop<R>(as_f64(a), as_f64(b));
}

// Comparison of two BOOL masks (FALSE < TRUE).
template <int R>
__device__ __forceinline__ uint32_t rel_mask(uint32_t a, uint32_t b) {
  uint32_t m;
  if constexpr (R == YQ_LT) m = ~a & b;
  else if constexpr (R == YQ_LE) m = ~a | b;
  else if constexpr (R == YQ_GT) m = a & ~b;
  else if constexpr (R == YQ_GE) m = a | ~b;
  else if constexpr (R == YQ_EQ) m = ~(a ^ b);
  else m = a ^ b;
  return m & kItemsMask;
}

template <int C, int R>
__device__ __forceinline__ uint32_t rel_items(const uint64_t (&a)[ITEMS], const uint64_t (&b)[ITEMS]) {
  if constexpr (C == TC_BOOL) {
    return rel_mask<R>((uint32_t)a[0], (uint32_t)b[0]);
  } else {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) m |= (uint32_t)rel1<C, R>(a[k], b[k]) << k;
    return m;
  }
}

template <int C, int R>
__device__ __forceinline__ uint32_t rel_items_const(const uint64_t (&a)[ITEMS], uint64_t k0) {
  if constexpr (C == TC_BOOL) {
    return rel_mask<R>((uint32_t)a[0], k0 ? kItemsMask : 0u);
  } else {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) m |= (uint32_t)rel1<C, R>(a[k], k0) << k;
    return m;
  }
}

template <int R>
__device__ __forceinline__ bool sign_rel(int s) {
  if constexpr (R == YQ_LT) return s < 0;
  else if constexpr (R == YQ_LE) return s <= 0;
  else if constexpr (R == YQ_GT) return s > 0;
  else if constexpr (R == YQ_GE) return s >= 0;
  else if constexpr (R == YQ_EQ) return s == 0;
  else return s != 0;
}

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// Pointer to the text slot of this thread's row k (global or stage).
template <bool STAGED>
__device__ __forceinline__ const uint32_t* text_slot(const DevCol& c, const Ctx& X, int k) {
  if constexpr (STAGED)
    return reinterpret_cast<const uint32_t*>(yq_dyn_smem + X.stage + c.soff + (X.lr + k) * (uint32_t)c.width);
  else
    return reinterpret_cast<const uint32_t*>(c.data + (size_t)(X.tile0 + X.lr + k) * c.width);
}

template <bool STAGED>
__device__ __forceinline__ uint32_t text_word(const uint32_t* p, int i) {
  if constexpr (STAGED) return p[i];
  else return __ldg(p + i);
}

// Any slot width, any comparison (word loops, out of line).
template <int R, bool STAGED>
__device__ __noinline__ uint32_t text_cmp_cc_slow(const DevCol& c, const uint32_t* cw, int cwords, Ctx X) {
  const int words = c.width >> 2;
  const int n = words > cwords ? words : cwords;
  uint32_t m = 0;
  for (int k = 0; k < ITEMS; ++k) {
    if (!STAGED && !(X.inr >> k & 1u)) continue;
    const uint32_t* p = text_slot<STAGED>(c, X, k);
    int s = 0;
    for (int i = 0; i < n && s == 0; ++i) {
      const uint32_t a = i < words ? bswap32(text_word<STAGED>(p, i)) : 0u;
      const uint32_t b = i < cwords ? cw[i] : 0u;
      if (a != b) s = a < b ? -1 : 1;
    }
    m |= (uint32_t)sign_rel<R>(s) << k;
  }
  return m;
}

// Text column <R> text constant for ITEMS rows (unsigned bytes, zero padded).
template <int R, bool STAGED>
__device__ __forceinline__ void text_cmp_cc(const VmProgram& P, const DevCol& c, int tidx, const Ctx& X, Val& out) {
  const int words = c.width >> 2, cwords = P.text_words;
  const uint32_t* cw = P.text[tidx];
  out.valid = X.inr & ~null_bits<STAGED>(c, X);
  uint32_t m = 0;
  if ((R == YQ_EQ || R == YQ_NE) && words == 4 && cwords <= 4) {
    // one 16-byte slot against the constant's raw bytes
    const uint32_t r0 = bswap32(cw[0]), r1 = cwords > 1 ? bswap32(cw[1]) : 0u,
                   r2 = cwords > 2 ? bswap32(cw[2]) : 0u, r3 = cwords > 3 ? bswap32(cw[3]) : 0u;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      if (!STAGED && !(X.inr >> k & 1u)) continue;
      const uint32_t* p = text_slot<STAGED>(c, X, k);
      uint4 q;
      if constexpr (STAGED) q = *reinterpret_cast<const uint4*>(p);
      else if (c.vec && X.vec_ok) q = ldg_nc_v4(p);
      else q = make_uint4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3));
      const bool eq = ((q.x ^ r0) | (q.y ^ r1) | (q.z ^ r2) | (q.w ^ r3)) == 0u;
      m |= (uint32_t)(R == YQ_EQ ? eq : !eq) << k;
    }
  } else {
    m = text_cmp_cc_slow<R, STAGED>(c, cw, cwords, X);
  }
  out.v[0] = m & out.valid;
}

template <int R, bool STAGED>
__device__ __noinline__ uint32_t text_cmp_ccol_mask(const DevCol& c, const DevCol& d, Ctx X) {
  const int pw = c.width >> 2, qw = d.width >> 2;
  const int n = pw > qw ? pw : qw;
  uint32_t m = 0;
  for (int k = 0; k < ITEMS; ++k) {
    if (!STAGED && !(X.inr >> k & 1u)) continue;
    const uint32_t* p = text_slot<STAGED>(c, X, k);
    const uint32_t* q = text_slot<STAGED>(d, X, k);
    int s = 0;
    for (int i = 0; i < n && s == 0; ++i) {
      const uint32_t a = i < pw ? bswap32(text_word<STAGED>(p, i)) : 0u;
      const uint32_t b = i < qw ? bswap32(text_word<STAGED>(q, i)) : 0u;
      if (a != b) s = a < b ? -1 : 1;
    }
    m |= (uint32_t)sign_rel<R>(s) << k;
  }
  return m;
}

// ------------------------------------------------------- three-valued logic
__device__ __forceinline__ void and_into(Val& a, uint32_t tb, uint32_t vb) {
  const uint32_t ta = (uint32_t)a.v[0], va = a.valid;
  const uint32_t t = ta & tb;
  const uint32_t f = (va & ~ta) | (vb & ~tb);
  a.v[0] = t;
  a.valid = t | f;
}
__device__ __forceinline__ void or_into(Val& a, uint32_t tb, uint32_t vb) {
  const uint32_t ta = (uint32_t)a.v[0], va = a.valid;
  const uint32_t t = ta | tb;
  const uint32_t f = (va & ~ta) & (vb & ~tb);
  a.v[0] = t;
  a.valid = t | f;
}

// ------------------------------------------------------- aggregate updates
// Per-thread accumulator of one aggregate: count of absorbed values and a
// 64-bit running value (int64 or double bits).
template <int K>
__device__ __forceinline__ void agg_absorb(uint32_t& cnt, uint64_t& acc, const Val& x, uint32_t sel) {
  const uint32_t m = sel & x.valid;
  cnt += __popc(m);
  if constexpr (K == AK_COUNT) {
    return;
  } else if constexpr (K == AK_SUM_I32 || K == AK_SUM_I64) {
    int64_t s = (int64_t)acc;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const int64_t v = (K == AK_SUM_I32) ? (int64_t)as_i32(x.v[k]) : as_i64(x.v[k]);
      s += (m >> k & 1u) ? v : 0;
    }
    acc = (uint64_t)s;
  } else if constexpr (K == AK_SUM_F32 || K == AK_SUM_F64) {
    double s = as_f64(acc);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const double v = (K == AK_SUM_F32) ? (double)as_f32(x.v[k]) : as_f64(x.v[k]);
      if (m >> k & 1u) s += v;
    }
    acc = from_f64(s);
  } else if constexpr (K == AK_MIN_I32 || K == AK_MIN_I64 || K == AK_MAX_I32 || K == AK_MAX_I64) {
    constexpr bool is_min = (K == AK_MIN_I32 || K == AK_MIN_I64);
    constexpr bool is32 = (K == AK_MIN_I32 || K == AK_MAX_I32);
    int64_t s = (int64_t)acc;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const int64_t v = is32 ? (int64_t)as_i32(x.v[k]) : as_i64(x.v[k]);
      if (m >> k & 1u) s = is_min ? (v < s ? v : s) : (v > s ? v : s);
    }
    acc = (uint64_t)s;
  } else {
    constexpr bool is_min = (K == AK_MIN_F32 || K == AK_MIN_F64);
    constexpr bool is32 = (K == AK_MIN_F32 || K == AK_MAX_F32);
    double s = as_f64(acc);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const double v = is32 ? (double)as_f32(x.v[k]) : as_f64(x.v[k]);
      if (m >> k & 1u) s = is_min ? ((v < s) ? v : s) : ((v > s) ? v : s);
    }
    acc = from_f64(s);
  }
}

// ------------------------------------------------------------ the machine
template <int OPC, bool STAGED, typename Emit>
__device__ __forceinline__ void exec(const VmProgram& P, const RInsn& I, const Ctx& X, Stack& S, Emit& E) {
  if constexpr (OPC < R_CONST) {
    constexpr int T = OPC - R_COL;
    push_moves(S, I.flags);
    load_as<T, STAGED>(P.cols[I.a], X, S.s0);
  } else if constexpr (OPC < R_NULL) {
    constexpr int T = OPC - R_CONST;
    push_moves(S, I.flags);
    const uint64_t k0 = (uint64_t)P.consts[I.imm];
    if constexpr (T == TC_BOOL) {
      S.s0.v[0] = k0 ? X.inr : 0u;
    } else {
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) S.s0.v[k] = k0;
    }
    S.s0.valid = X.inr;
  } else if constexpr (OPC == R_NULL) {
    push_moves(S, I.flags);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) S.s0.v[k] = 0;
    S.s0.valid = 0;
  } else if constexpr (OPC < R_ARITH) {
    constexpr int F = (OPC - R_CAST) / 5, T = (OPC - R_CAST) % 5;
    cast_val<F, T>(S.s0);
  } else if constexpr (OPC < R_ARITH_COL) {
    constexpr int T = (OPC - R_ARITH) / 5, A = (OPC - R_ARITH) % 5;
    S.s0 = arith_val<T, A>(S.s1, S.s0);
    binary_moves(S, I.flags);
  } else if constexpr (OPC < R_ARITH_CONST) {
    constexpr int T = (OPC - R_ARITH_COL) / 5, A = (OPC - R_ARITH_COL) % 5;
    Val c;
    load_as<T, STAGED>(P.cols[I.b], X, c);
    S.s0 = arith_val<T, A>(S.s0, c);
  } else if constexpr (OPC < R_CMP) {
    constexpr int T = (OPC - R_ARITH_CONST) / 5, A = (OPC - R_ARITH_CONST) % 5;
    Val c;
    const uint64_t k0 = (uint64_t)P.consts[I.imm];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) c.v[k] = k0;
    c.valid = kItemsMask;
    S.s0 = arith_val<T, A>(S.s0, c);
  } else if constexpr (OPC < R_CMP_CC) {
    constexpr int C = (OPC - R_CMP) / 6, R = (OPC - R_CMP) % 6;
    const uint32_t valid = S.s1.valid & S.s0.valid;
    const uint32_t m = rel_items<C, R>(S.s1.v, S.s0.v);
    S.s0.v[0] = m & valid;
    S.s0.valid = valid;
    binary_moves(S, I.flags);
  } else if constexpr (OPC < R_CMP_CCOL) {
    constexpr int C = (OPC - R_CMP_CC) / 6, R = (OPC - R_CMP_CC) % 6;
    const DevCol& c = P.cols[I.b];
    Val r;
    if constexpr (C == TC_TEXT) {
      text_cmp_cc<R, STAGED>(P, c, I.imm, X, r);
    } else {
      uint64_t v[ITEMS];
      load_raw<C, STAGED>(c, X, v);
      r.valid = X.inr & ~null_bits<STAGED>(c, X);
      r.v[0] = rel_items_const<C, R>(v, (uint64_t)P.consts[I.imm]) & r.valid;
    }
    if (I.flags & RF_AND) {
      and_into(S.s0, (uint32_t)r.v[0], r.valid);
    } else {
      push_moves(S, I.flags);
      S.s0.v[0] = r.v[0];
      S.s0.valid = r.valid;
    }
  } else if constexpr (OPC < R_AND) {
    constexpr int C = (OPC - R_CMP_CCOL) / 6, R = (OPC - R_CMP_CCOL) % 6;
    const DevCol& c = P.cols[I.b];
    const DevCol& d = P.cols[I.c];
    push_moves(S, I.flags);
    const uint32_t valid = X.inr & ~null_bits<STAGED>(c, X) & ~null_bits<STAGED>(d, X);
    if constexpr (C == TC_TEXT) {
      S.s0.v[0] = text_cmp_ccol_mask<R, STAGED>(c, d, X) & valid;
    } else {
      uint64_t a[ITEMS], b[ITEMS];
      load_raw<C, STAGED>(c, X, a);
      load_raw<C, STAGED>(d, X, b);
      S.s0.v[0] = rel_items<C, R>(a, b) & valid;
    }
    S.s0.valid = valid;
  } else if constexpr (OPC == R_AND) {
    and_into(S.s1, (uint32_t)S.s0.v[0], S.s0.valid);
    S.s0.v[0] = S.s1.v[0];
    S.s0.valid = S.s1.valid;
    binary_moves(S, I.flags);
  } else if constexpr (OPC == R_OR) {
    or_into(S.s1, (uint32_t)S.s0.v[0], S.s0.valid);
    S.s0.v[0] = S.s1.v[0];
    S.s0.valid = S.s1.valid;
    binary_moves(S, I.flags);
  } else if constexpr (OPC == R_NOT) {
    S.s0.v[0] = S.s0.valid & ~(uint32_t)S.s0.v[0];
  } else if constexpr (OPC == R_IS_NULL || OPC == R_IS_NOT_NULL) {
    const uint32_t nul = X.inr & ~S.s0.valid;
    S.s0.v[0] = (OPC == R_IS_NULL) ? nul : (X.inr & ~nul);
    S.s0.valid = X.inr;
  } else if constexpr (OPC == R_EMIT_PRED) {
    E.pred((uint32_t)S.s0.v[0]);
    pop_moves(S, I.flags);
  } else if constexpr (OPC < R_EMIT_PROJ) {
    E.template agg<OPC - R_EMIT_AGG>(I.a, S.s0);
    pop_moves(S, I.flags);
  } else if constexpr (OPC < R_COUNT) {
    E.template proj<OPC - R_EMIT_PROJ>(I.a, S.s0);
    pop_moves(S, I.flags);
  }
}

// Run instructions [pc, end) for this thread's ITEMS rows of the step.
template <bool STAGED, typename Emit>
__device__ __forceinline__ void run_vm(const VmProgram& P, int pc, int end, const Ctx& X, Stack& S, Emit& E) {
  for (; pc < end; ++pc) {
    const RInsn I = P.code[pc];
    switch (I.opc) {
#define YQ_X1(n) \
  case (n): exec<(n), STAGED>(P, I, X, S, E); break;
#define YQ_X10(n) YQ_X1(n) YQ_X1(n + 1) YQ_X1(n + 2) YQ_X1(n + 3) YQ_X1(n + 4) YQ_X1(n + 5) YQ_X1(n + 6) YQ_X1(n + 7) \
  YQ_X1(n + 8) YQ_X1(n + 9)
      YQ_X10(0) YQ_X10(10) YQ_X10(20) YQ_X10(30) YQ_X10(40) YQ_X10(50) YQ_X10(60) YQ_X10(70) YQ_X10(80) YQ_X10(90)
      YQ_X10(100) YQ_X10(110) YQ_X10(120) YQ_X10(130) YQ_X10(140) YQ_X10(150) YQ_X10(160) YQ_X10(170) YQ_X10(180)
      YQ_X10(190) YQ_X10(200) YQ_X10(210)
#undef YQ_X10
#undef YQ_X1
      default: break;
    }
  }
}

// Emit hooks that ignore aggregates and projections (selection only).
struct SelEmit {
  uint32_t sel;
  __device__ __forceinline__ void pred(uint32_t bits) { sel &= bits; }
  template <int K>
  __device__ __forceinline__ void agg(int, const Val&) {}
  template <int W>
  __device__ __forceinline__ void proj(int, const Val&) {}
};

// Per-thread aggregate accumulators (static register indices via switch).
struct AggEmit {
  uint32_t sel;
  uint32_t cnt[YQ_MAX_AGGREGATES];
  uint64_t acc[YQ_MAX_AGGREGATES];
  __device__ __forceinline__ void pred(uint32_t bits) { sel &= bits; }
  template <int K>
  __device__ __forceinline__ void agg(int a, const Val& x) {
    switch (a) {
#define YQ_AGG_CASE(i) \
  case i: agg_absorb<K>(cnt[i], acc[i], x, sel); break;
      YQ_AGG_CASE(0) YQ_AGG_CASE(1) YQ_AGG_CASE(2) YQ_AGG_CASE(3)
      YQ_AGG_CASE(4) YQ_AGG_CASE(5) YQ_AGG_CASE(6) YQ_AGG_CASE(7)
#undef YQ_AGG_CASE
      default: break;
    }
  }
  template <int W>
  __device__ __forceinline__ void proj(int, const Val&) {}
};

}  // namespace yq
