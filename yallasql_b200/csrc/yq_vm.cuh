// Register-resident expression machine for the fused row kernels.
//
// A thread evaluates one program over ITEMS consecutive rows at a time. The
// stack (depth 4) is four named slot groups, so every access is static and the
// whole machine stays in registers; the host loader (vm_host.cpp) annotates
// each instruction with whether it must shift the stack, so conjunctions of
// `column <cmp> constant` terms run with no stack traffic at all.
//
// Slot encoding (one 64-bit word per row): INT32 sign-extended, FLOAT32 bits
// in the low word, INT64/DATETIME as int64, FLOAT64 bits, BOOL 0/1. `valid`
// holds one bit per row (0 = NULL or row out of range).
#pragma once

#include "yq_common.cuh"

namespace yq {

constexpr int ITEMS = 4;  // rows per thread per step (one 16-byte load of a 4-byte column)

// Internal opcodes = public yq_opcode values plus the fused forms below.
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
  OP_END = 33
};
// Flag bits in Insn::op's high bits (set by the host loader).
constexpr uint8_t OPF_PUSH = 0x80;      // shift stack down before writing the new top
constexpr uint8_t OPF_POPSHIFT = 0x40;  // after a binary op, slots below the result are live
constexpr uint8_t OP_MASK = 0x3f;

// Aggregate update codes (host picks one per aggregate from kind + type).
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

struct Insn {
  uint8_t op, type, a, b;
  int32_t imm;
};

struct DevCol {
  const char* data;
  const uint8_t* nulls;
  int32_t type;
  int32_t width;
  int32_t vec;   // data is 16-byte aligned (vector loads allowed)
  int32_t nvec;  // nulls is 4-byte aligned
};

constexpr int kMaxInsns = 128;

struct VmProgram {
  Insn code[kMaxInsns];
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

// ------------------------------------------------------------- value access
__device__ __forceinline__ int32_t as_i32(uint64_t x) { return (int32_t)(uint32_t)x; }
__device__ __forceinline__ float as_f32(uint64_t x) { return __uint_as_float((uint32_t)x); }
__device__ __forceinline__ int64_t as_i64(uint64_t x) { return (int64_t)x; }
__device__ __forceinline__ double as_f64(uint64_t x) { return __longlong_as_double((long long)x); }
__device__ __forceinline__ uint64_t from_i32(int32_t x) { return (uint64_t)(int64_t)x; }
__device__ __forceinline__ uint64_t from_f32(float x) { return (uint64_t)__float_as_uint(x); }
__device__ __forceinline__ uint64_t from_i64(int64_t x) { return (uint64_t)x; }
__device__ __forceinline__ uint64_t from_f64(double x) { return (uint64_t)__double_as_longlong(x); }

__device__ __forceinline__ bool is_int_type(int t) {
  return t == YQ_INT32 || t == YQ_INT64 || t == YQ_DATETIME || t == YQ_BOOL;
}

// Load ITEMS values of a fixed-width column starting at row0 into slot form.
// `inr` = in-range bits; `full` = all ITEMS rows in range.
__device__ __forceinline__ void load_col(const DevCol& c, uint32_t row0, uint32_t inr, bool full, Val& out) {
  uint32_t nullbits = 0;
  if (c.nulls) {
    if (full && c.nvec) {
      uint32_t w = *reinterpret_cast<const uint32_t*>(c.nulls + row0);
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) nullbits |= (((w >> (8 * k)) & 0xffu) != 0u) << k;
    } else {
#pragma unroll
      for (int k = 0; k < ITEMS; ++k)
        if (inr & (1u << k)) nullbits |= (c.nulls[row0 + k] != 0) << k;
    }
  }
  out.valid = inr & ~nullbits;
  const int t = c.type;
  if (c.width == 4) {
    uint32_t w[ITEMS];
    if (full && c.vec) {
      uint4 q = ldg_nc_v4(c.data + (size_t)row0 * 4);
      w[0] = q.x; w[1] = q.y; w[2] = q.z; w[3] = q.w;
    } else {
#pragma unroll
      for (int k = 0; k < ITEMS; ++k)
        w[k] = (inr & (1u << k)) ? __ldg(reinterpret_cast<const uint32_t*>(c.data) + row0 + k) : 0u;
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) out.v[k] = (t == YQ_INT32) ? from_i32((int32_t)w[k]) : (uint64_t)w[k];
  } else if (c.width == 8) {
    if (full && c.vec) {
      uint4 q0 = ldg_nc_v4(c.data + (size_t)row0 * 8);
      uint4 q1 = ldg_nc_v4(c.data + (size_t)row0 * 8 + 16);
      out.v[0] = ((uint64_t)q0.y << 32) | q0.x;
      out.v[1] = ((uint64_t)q0.w << 32) | q0.z;
      out.v[2] = ((uint64_t)q1.y << 32) | q1.x;
      out.v[3] = ((uint64_t)q1.w << 32) | q1.z;
    } else {
#pragma unroll
      for (int k = 0; k < ITEMS; ++k)
        out.v[k] = (inr & (1u << k))
                       ? (uint64_t)__ldg(reinterpret_cast<const unsigned long long*>(c.data) + row0 + k)
                       : 0ull;
    }
  } else {  // BOOL (1 byte)
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
      out.v[k] = (inr & (1u << k)) ? (uint64_t)(c.data[row0 + k] != 0) : 0ull;
  }
}

// ------------------------------------------------------------------- casts
__device__ __forceinline__ uint64_t cast_one(uint64_t x, int from, int to, bool& ok) {
  ok = true;
  if (from == to) return x;
  if (from == YQ_DATETIME) from = YQ_INT64;
  if (to == YQ_DATETIME) to = YQ_INT64;
  if (from == to) return x;
  switch (from) {
    case YQ_BOOL:
    case YQ_INT32:
    case YQ_INT64: {
      int64_t v = as_i64(x);  // INT32 and BOOL slots are already sign-extended
      switch (to) {
        case YQ_INT32:
          if (v < INT32_MIN || v > INT32_MAX) { ok = false; return 0; }
          return from_i32((int32_t)v);
        case YQ_INT64: return from_i64(v);
        case YQ_FLOAT32: return from_f32(__ll2float_rn(v));
        case YQ_FLOAT64: return from_f64(__ll2double_rn(v));
        case YQ_BOOL: return (uint64_t)(v != 0);
      }
      break;
    }
    case YQ_FLOAT32:
    case YQ_FLOAT64: {
      double v = (from == YQ_FLOAT32) ? (double)as_f32(x) : as_f64(x);
      switch (to) {
        case YQ_FLOAT32: return from_f32(__double2float_rn(v));
        case YQ_FLOAT64: return from_f64(v);
        case YQ_INT32: {
          // Round half to even, NULL when not representable.
          if (!(v >= -2147483648.0 && v < 2147483648.0)) { ok = false; return 0; }
          double r = rint(v);
          if (r < -2147483648.0 || r > 2147483647.0) { ok = false; return 0; }
          return from_i32((int32_t)r);
        }
        case YQ_INT64: {
          if (!(v >= -9223372036854775808.0 && v < 9223372036854775808.0)) { ok = false; return 0; }
          return from_i64((int64_t)rint(v));
        }
        case YQ_BOOL: return (uint64_t)(v != 0.0);
      }
      break;
    }
  }
  ok = false;
  return 0;
}

__device__ __forceinline__ void cast_val(Val& x, int from, int to) {
  if (from == to) return;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    bool ok;
    x.v[k] = cast_one(x.v[k], from, to, ok);
    if (!ok) x.valid &= ~(1u << k);
  }
}

// -------------------------------------------------------------- arithmetic
__device__ __forceinline__ uint64_t arith_one(uint64_t a, uint64_t b, int op, int t, bool& ok) {
  ok = true;
  switch (t) {
    case YQ_INT32: {
      int32_t x = as_i32(a), y = as_i32(b);
      uint32_t ux = (uint32_t)x, uy = (uint32_t)y;
      switch (op) {
        case YQ_ADD: return from_i32((int32_t)(ux + uy));
        case YQ_SUB: return from_i32((int32_t)(ux - uy));
        case YQ_MUL: return from_i32((int32_t)(ux * uy));
        case YQ_DIV:
          if (y == 0) { ok = false; return 0; }
          if (y == -1) return from_i32((int32_t)(0u - ux));
          return from_i32(x / y);
        case YQ_MOD:
          if (y == 0) { ok = false; return 0; }
          if (y == -1) return 0;
          return from_i32(x % y);
      }
      break;
    }
    case YQ_INT64:
    case YQ_DATETIME: {
      int64_t x = as_i64(a), y = as_i64(b);
      uint64_t ux = (uint64_t)x, uy = (uint64_t)y;
      switch (op) {
        case YQ_ADD: return ux + uy;
        case YQ_SUB: return ux - uy;
        case YQ_MUL: return ux * uy;
        case YQ_DIV:
          if (y == 0) { ok = false; return 0; }
          if (y == -1) return 0ull - ux;
          return from_i64(x / y);
        case YQ_MOD:
          if (y == 0) { ok = false; return 0; }
          if (y == -1) return 0;
          return from_i64(x % y);
      }
      break;
    }
    case YQ_FLOAT32: {
      float x = as_f32(a), y = as_f32(b);
      switch (op) {
        case YQ_ADD: return from_f32(__fadd_rn(x, y));
        case YQ_SUB: return from_f32(__fsub_rn(x, y));
        case YQ_MUL: return from_f32(__fmul_rn(x, y));
        case YQ_DIV: return from_f32(__fdiv_rn(x, y));
        case YQ_MOD: return from_f32(fmodf(x, y));
      }
      break;
    }
    case YQ_FLOAT64: {
      double x = as_f64(a), y = as_f64(b);
      switch (op) {
        case YQ_ADD: return from_f64(__dadd_rn(x, y));
        case YQ_SUB: return from_f64(__dsub_rn(x, y));
        case YQ_MUL: return from_f64(__dmul_rn(x, y));
        case YQ_DIV: return from_f64(__ddiv_rn(x, y));
        case YQ_MOD: return from_f64(fmod(x, y));
      }
      break;
    }
  }
  ok = false;
  return 0;
}

__device__ __forceinline__ void arith_val(Val& a, const Val& b, int op, int t) {
  uint32_t valid = a.valid & b.valid;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    bool ok;
    a.v[k] = arith_one(a.v[k], b.v[k], op, t, ok);
    if (!ok) valid &= ~(1u << k);
  }
  a.valid = valid;
}

// ------------------------------------------------------------- comparisons
template <typename T>
__device__ __forceinline__ bool cmp_t(T x, T y, int op) {
  switch (op) {
    case YQ_LT: return x < y;
    case YQ_LE: return x <= y;
    case YQ_GT: return x > y;
    case YQ_GE: return x >= y;
    case YQ_EQ: return x == y;
    default: return x != y;
  }
}

__device__ __forceinline__ bool cmp_one(uint64_t a, uint64_t b, int op, int t) {
  switch (t) {
    case YQ_INT32:
    case YQ_INT64:
    case YQ_DATETIME:
    case YQ_BOOL: return cmp_t<int64_t>(as_i64(a), as_i64(b), op);
    case YQ_FLOAT32: return cmp_t<float>(as_f32(a), as_f32(b), op);
    default: return cmp_t<double>(as_f64(a), as_f64(b), op);
  }
}

// Result of comparing a with b: -1, 0, 1 mapped through op.
__device__ __forceinline__ bool cmp_sign(int s, int op) {
  switch (op) {
    case YQ_LT: return s < 0;
    case YQ_LE: return s <= 0;
    case YQ_GT: return s > 0;
    case YQ_GE: return s >= 0;
    case YQ_EQ: return s == 0;
    default: return s != 0;
  }
}

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// Lexicographic compare of a text slot (width bytes at p, 4-byte aligned)
// against a constant stored as big-endian words (zero padded).
__device__ __forceinline__ int text_cmp_const(const uint32_t* p, int words, const uint32_t* cw, int cwords) {
  const int n = words > cwords ? words : cwords;
  for (int i = 0; i < n; ++i) {
    uint32_t a = i < words ? bswap32(__ldg(p + i)) : 0u;
    uint32_t b = i < cwords ? cw[i] : 0u;
    if (a != b) return a < b ? -1 : 1;
  }
  return 0;
}

__device__ __forceinline__ int text_cmp_cols(const uint32_t* p, int pw, const uint32_t* q, int qw) {
  const int n = pw > qw ? pw : qw;
  for (int i = 0; i < n; ++i) {
    uint32_t a = i < pw ? bswap32(__ldg(p + i)) : 0u;
    uint32_t b = i < qw ? bswap32(__ldg(q + i)) : 0u;
    if (a != b) return a < b ? -1 : 1;
  }
  return 0;
}

__device__ __forceinline__ uint32_t null_bits(const DevCol& c, uint32_t row0, uint32_t inr) {
  uint32_t nb = 0;
  if (c.nulls) {
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
      if (inr & (1u << k)) nb |= (c.nulls[row0 + k] != 0) << k;
  }
  return nb;
}

// Text column <cmp> text constant for ITEMS rows.
__device__ __forceinline__ void text_cmp_col_const(const VmProgram& P, const DevCol& c, int cidx, int op,
                                                   uint32_t row0, uint32_t inr, Val& out) {
  const int words = c.width >> 2;
  const uint32_t* cw = P.text[cidx];
  out.valid = inr & ~null_bits(c, row0, inr);
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    bool r = false;
    if (inr & (1u << k)) {
      const uint32_t* p = reinterpret_cast<const uint32_t*>(c.data + (size_t)(row0 + k) * c.width);
      if (op == YQ_EQ || op == YQ_NE) {
        bool eq = true;
        const int n = words > P.text_words ? words : P.text_words;
        for (int i = 0; i < n && eq; ++i) {
          uint32_t a = i < words ? bswap32(__ldg(p + i)) : 0u;
          uint32_t b = i < P.text_words ? cw[i] : 0u;
          eq = (a == b);
        }
        r = (op == YQ_EQ) ? eq : !eq;
      } else {
        r = cmp_sign(text_cmp_const(p, words, cw, P.text_words), op);
      }
    }
    out.v[k] = r;
  }
}

__device__ __forceinline__ void text_cmp_col_col(const DevCol& c, const DevCol& d, int op, uint32_t row0,
                                                 uint32_t inr, Val& out) {
  out.valid = inr & ~null_bits(c, row0, inr) & ~null_bits(d, row0, inr);
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    bool r = false;
    if (inr & (1u << k)) {
      const uint32_t* p = reinterpret_cast<const uint32_t*>(c.data + (size_t)(row0 + k) * c.width);
      const uint32_t* q = reinterpret_cast<const uint32_t*>(d.data + (size_t)(row0 + k) * d.width);
      r = cmp_sign(text_cmp_cols(p, c.width >> 2, q, d.width >> 2), op);
    }
    out.v[k] = r;
  }
}

__device__ __forceinline__ void cmp_val(Val& a, const Val& b, int op, int t) {
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) a.v[k] = cmp_one(a.v[k], b.v[k], op, t);
  a.valid &= b.valid;
}

// Three-valued AND / OR on BOOL slots.
__device__ __forceinline__ uint32_t true_bits(const Val& x) {
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) m |= (uint32_t)(x.v[k] & 1u) << k;
  return m & x.valid;
}
__device__ __forceinline__ uint32_t false_bits(const Val& x) {
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) m |= (uint32_t)((x.v[k] & 1u) ^ 1u) << k;
  return m & x.valid;
}
__device__ __forceinline__ void set_bool(Val& x, uint32_t t, uint32_t f) {
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) x.v[k] = (t >> k) & 1u;
  x.valid = t | f;
}
__device__ __forceinline__ void and_val(Val& a, const Val& b) {
  uint32_t f = false_bits(a) | false_bits(b);
  uint32_t t = true_bits(a) & true_bits(b);
  set_bool(a, t, f);
}
__device__ __forceinline__ void or_val(Val& a, const Val& b) {
  uint32_t t = true_bits(a) | true_bits(b);
  uint32_t f = false_bits(a) & false_bits(b);
  set_bool(a, t, f);
}

// Numeric column loaded and converted to `t` (cast-on-load for fused forms).
__device__ __forceinline__ void load_col_as(const DevCol& c, int t, uint32_t row0, uint32_t inr, bool full,
                                            Val& out) {
  load_col(c, row0, inr, full, out);
  cast_val(out, c.type, t);
}

__device__ __forceinline__ void const_val(const VmProgram& P, int idx, uint32_t inr, Val& out) {
  const uint64_t c = (uint64_t)P.consts[idx];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) out.v[k] = c;
  out.valid = inr;
}

// Compare a numeric column against a constant: ITEMS rows -> BOOL slot.
__device__ __forceinline__ void cmp_col_const(const VmProgram& P, const Insn& I, uint32_t row0, uint32_t inr,
                                              bool full, Val& out) {
  const DevCol& c = P.cols[I.b];
  if (c.type == YQ_TEXT) {
    text_cmp_col_const(P, c, I.imm, I.a, row0, inr, out);
    return;
  }
  load_col_as(c, I.type, row0, inr, full, out);
  const uint64_t k0 = (uint64_t)P.consts[I.imm];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) out.v[k] = cmp_one(out.v[k], k0, I.a, I.type);
}

// ------------------------------------------------------------ the machine
// Per-thread accumulators for the fused aggregate kernel.
struct Acc {
  long long cnt;
  long long i;
  double f;
};

__device__ __forceinline__ void acc_init(Acc& a, int upd) {
  a.cnt = 0;
  a.i = (upd == UPD_MIN_I) ? LLONG_MAX : (upd == UPD_MAX_I ? LLONG_MIN : 0);
  a.f = (upd == UPD_MIN_F) ? __longlong_as_double(0x7ff0000000000000ll)
                           : (upd == UPD_MAX_F ? __longlong_as_double((long long)0xfff0000000000000ull) : 0.0);
}

__device__ __forceinline__ void acc_update(Acc& a, int upd, int t, const Val& x, uint32_t sel) {
  if (upd == UPD_COUNT_STAR) {
    a.cnt += __popc(sel);
    return;
  }
  const uint32_t m = sel & x.valid;
  a.cnt += __popc(m);
  if (upd == UPD_COUNT) return;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    if (!(m & (1u << k))) continue;
    switch (upd) {
      case UPD_SUM_I: a.i += as_i64(x.v[k]); break;
      case UPD_MIN_I: a.i = min(a.i, (long long)as_i64(x.v[k])); break;
      case UPD_MAX_I: a.i = max(a.i, (long long)as_i64(x.v[k])); break;
      default: {
        double d = (t == YQ_FLOAT32) ? (double)as_f32(x.v[k]) : as_f64(x.v[k]);
        if (upd == UPD_SUM_F) a.f += d;
        else if (upd == UPD_MIN_F) a.f = (d < a.f) ? d : a.f;
        else a.f = (d > a.f) ? d : a.f;
      }
    }
  }
}

__device__ __forceinline__ void acc_combine(Acc& a, const Acc& b, int upd) {
  a.cnt += b.cnt;
  switch (upd) {
    case UPD_SUM_I: a.i += b.i; break;
    case UPD_MIN_I: a.i = min(a.i, b.i); break;
    case UPD_MAX_I: a.i = max(a.i, b.i); break;
    case UPD_SUM_F: a.f += b.f; break;
    case UPD_MIN_F: a.f = (b.f < a.f) ? b.f : a.f; break;
    case UPD_MAX_F: a.f = (b.f > a.f) ? b.f : a.f; break;
    default: break;
  }
}

__device__ __forceinline__ void acc_shfl_down(Acc& a, int d, int upd) {
  Acc b;
  b.cnt = __shfl_down_sync(0xffffffffu, a.cnt, d);
  b.i = __shfl_down_sync(0xffffffffu, a.i, d);
  b.f = __shfl_down_sync(0xffffffffu, a.f, d);
  acc_combine(a, b, upd);
}

struct Stack {
  Val s0, s1, s2, s3;
};

__device__ __forceinline__ void push(Stack& S, uint8_t flags) {
  if (flags & OPF_PUSH) {
    S.s3 = S.s2;
    S.s2 = S.s1;
    S.s1 = S.s0;
  }
}
// After a binary op wrote its result into s1: move it to s0 and pull up.
__device__ __forceinline__ void pop_binary(Stack& S, uint8_t flags) {
  S.s0 = S.s1;
  if (flags & OPF_POPSHIFT) {
    S.s1 = S.s2;
    S.s2 = S.s3;
  }
}
__device__ __forceinline__ void pop_one(Stack& S, uint8_t flags) {
  if (flags & OPF_POPSHIFT) {
    S.s0 = S.s1;
    S.s1 = S.s2;
    S.s2 = S.s3;
  }
}

// Hook interface for EMIT instructions: the kernel supplies what they do.
// Run instructions [pc, end) for rows row0..row0+ITEMS-1.
template <typename Emit>
__device__ __forceinline__ void run_vm(const VmProgram& P, int pc, int end, uint32_t row0, uint32_t inr, bool full,
                                       Stack& S, Emit& emit) {
  for (; pc < end; ++pc) {
    const Insn I = P.code[pc];
    const uint8_t flags = I.op;
    switch (I.op & OP_MASK) {
      case OP_COL: {
        push(S, flags);
        load_col_as(P.cols[I.a], I.type, row0, inr, full, S.s0);
        break;
      }
      case OP_CONST: {
        push(S, flags);
        const_val(P, I.imm, inr, S.s0);
        break;
      }
      case OP_NULL: {
        push(S, flags);
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) S.s0.v[k] = 0;
        S.s0.valid = 0;
        break;
      }
      case OP_CAST: cast_val(S.s0, I.type, I.a); break;
      case OP_ARITH: {
        arith_val(S.s1, S.s0, I.a, I.type);
        pop_binary(S, flags);
        break;
      }
      case OP_ARITH_COL: {
        Val c;
        load_col_as(P.cols[I.b], I.type, row0, inr, full, c);
        arith_val(S.s0, c, I.a, I.type);
        break;
      }
      case OP_ARITH_CONST: {
        Val c;
        const_val(P, I.imm, inr, c);
        arith_val(S.s0, c, I.a, I.type);
        break;
      }
      case OP_CMP: {
        cmp_val(S.s1, S.s0, I.a, I.type);
        pop_binary(S, flags);
        break;
      }
      case OP_CMP_COL_CONST: {
        push(S, flags);
        cmp_col_const(P, I, row0, inr, full, S.s0);
        break;
      }
      case OP_AND_CMP_COL_CONST: {
        Val c;
        cmp_col_const(P, I, row0, inr, full, c);
        and_val(S.s0, c);
        break;
      }
      case OP_CMP_COL_COL: {
        push(S, flags);
        const DevCol& c = P.cols[I.b];
        if (c.type == YQ_TEXT) {
          text_cmp_col_col(c, P.cols[I.imm], I.a, row0, inr, S.s0);
        } else {
          Val d;
          load_col_as(c, I.type, row0, inr, full, S.s0);
          load_col_as(P.cols[I.imm], I.type, row0, inr, full, d);
          cmp_val(S.s0, d, I.a, I.type);
        }
        break;
      }
      case OP_AND: {
        and_val(S.s1, S.s0);
        pop_binary(S, flags);
        break;
      }
      case OP_OR: {
        or_val(S.s1, S.s0);
        pop_binary(S, flags);
        break;
      }
      case OP_NOT: {
        uint32_t t = true_bits(S.s0), f = false_bits(S.s0);
        set_bool(S.s0, f, t);
        break;
      }
      case OP_IS_NULL:
      case OP_IS_NOT_NULL: {
        uint32_t nul = inr & ~S.s0.valid;
        uint32_t t = ((I.op & OP_MASK) == OP_IS_NULL) ? nul : (inr & ~nul);
        set_bool(S.s0, t, inr & ~t);
        break;
      }
      case OP_EMIT_PRED: {
        emit.pred(true_bits(S.s0));
        pop_one(S, flags);
        break;
      }
      case OP_EMIT_AGG: {
        emit.agg(I.a, I.b, I.type, S.s0);
        pop_one(S, flags);
        break;
      }
      case OP_EMIT_PROJ: {
        emit.proj(I.a, S.s0);
        pop_one(S, flags);
        break;
      }
      default: break;
    }
  }
}

}  // namespace yq
