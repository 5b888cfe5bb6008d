// Host-side loader for expression programs: validates a client's postfix
// program against the batch schema, applies peephole fusions, and resolves
// each instruction into the kernels' opcode for its operation, value class and
// operator, with the stack moves it needs (see yq_vm.cuh).
#pragma once

#include <string.h>
#include "yq_vm.cuh"

namespace yq {

struct ProgramBuilder {
  VmProgram P;
  Insn code[kMaxInsns];  // loader form; resolved into P.code by finalize()
  int len = 0;
  int nconsts = 0;
  int ntext = 0;
  uint32_t used_cols = 0;    // bit c: column c is read by the program (after finalize)
  int remap[kMaxInsns + 1];  // after finalize: loader index -> resolved index

  ProgramBuilder() {
    memset(&P, 0, sizeof(P));
    memset(code, 0, sizeof(code));
  }

  int set_columns(const yq_column* cols, int ncols) {
    if (ncols < 0 || ncols > YQ_MAX_BATCH_COLUMNS || (ncols > 0 && !cols)) return YQ_ERR_INVALID_ARG;
    P.ncols = ncols;
    for (int i = 0; i < ncols; ++i) {
      const yq_column& c = cols[i];
      if (!valid_column(c)) return YQ_ERR_INVALID_ARG;
      DevCol& d = P.cols[i];
      d.data = static_cast<const char*>(c.data);
      d.nulls = c.nulls;
      d.type = c.type;
      d.tc = type_class(c.type);
      d.width = c.width;
      d.vec = ((reinterpret_cast<uintptr_t>(c.data) & 15u) == 0);
      d.nvec = ((reinterpret_cast<uintptr_t>(c.nulls) & 3u) == 0);
      d.soff = d.snoff = 0;
    }
    return YQ_OK;
  }

  static bool valid_column(const yq_column& c) {
    switch (c.type) {
      case YQ_INT32:
      case YQ_FLOAT32: return c.width == 4;
      case YQ_INT64:
      case YQ_DATETIME:
      case YQ_FLOAT64: return c.width == 8;
      case YQ_BOOL: return c.width == 1;
      case YQ_TEXT: return c.width >= 4 && c.width <= YQ_MAX_TEXT_WIDTH && (c.width % 4) == 0;
      default: return false;
    }
  }

  int set_constants(const yq_constants* k) {
    if (!k) return YQ_OK;
    if (k->count < 0 || k->count > YQ_MAX_CONSTANTS || (k->count > 0 && !k->values)) return YQ_ERR_INVALID_ARG;
    for (int i = 0; i < k->count; ++i) P.consts[i] = k->values[i];
    nconsts = k->count;
    if (k->text_count < 0 || k->text_count > YQ_MAX_TEXT_CONSTANTS) return YQ_ERR_INVALID_ARG;
    if (k->text_count > 0) {
      if (!k->text || k->text_width <= 0 || k->text_width > YQ_MAX_TEXT_WIDTH) return YQ_ERR_INVALID_ARG;
      const int words = (k->text_width + 3) / 4;
      P.text_words = words;
      for (int s = 0; s < k->text_count; ++s) {
        const unsigned char* src = reinterpret_cast<const unsigned char*>(k->text) + (size_t)s * k->text_width;
        for (int w = 0; w < words; ++w) {
          uint32_t v = 0;
          for (int b = 0; b < 4; ++b) {
            int idx = w * 4 + b;
            v = (v << 8) | (idx < k->text_width ? src[idx] : 0u);
          }
          P.text[s][w] = v;
        }
      }
      ntext = k->text_count;
    }
    return YQ_OK;
  }

  static bool numeric(int t) {
    return t == YQ_INT32 || t == YQ_FLOAT32 || t == YQ_INT64 || t == YQ_DATETIME || t == YQ_FLOAT64;
  }
  static bool loadable(int t) { return numeric(t) || t == YQ_BOOL; }
  static bool castable(int from, int to) { return loadable(from) && loadable(to); }

  int col_type(int c) const { return (c >= 0 && c < P.ncols) ? P.cols[c].type : -1; }

  // Append one client program; on success `result_type` is the type left on
  // the stack (exactly one value).
  int append(const yq_program* prog, int& result_type) {
    if (!prog || prog->len <= 0 || !prog->code) return YQ_ERR_INVALID_ARG;
    int types[8];
    int depth = 0;
    const int start = len;
    for (int i = 0; i < prog->len; ++i) {
      Insn I;
      I.op = prog->code[i].op;
      I.type = prog->code[i].type;
      I.a = prog->code[i].a;
      I.b = prog->code[i].b;
      I.imm = prog->code[i].imm;
      int pushes = 0, pops = 0, out_t = -1;
      switch (I.op) {
        case OP_COL: {
          int ct = col_type(I.a);
          if (ct < 0 || !castable(ct, I.type)) return YQ_ERR_INVALID_ARG;
          pushes = 1; out_t = I.type;
          break;
        }
        case OP_CONST:
          if (I.imm < 0 || I.imm >= nconsts || !loadable(I.type)) return YQ_ERR_INVALID_ARG;
          pushes = 1; out_t = I.type;
          break;
        case OP_NULL:
          if (!loadable(I.type)) return YQ_ERR_INVALID_ARG;
          pushes = 1; out_t = I.type;
          break;
        case OP_CAST:
          if (depth < 1 || types[depth - 1] != I.type || !castable(I.type, I.a)) return YQ_ERR_INVALID_ARG;
          pops = 1; pushes = 1; out_t = I.a;
          break;
        case OP_ARITH:
          if (depth < 2 || types[depth - 1] != I.type || types[depth - 2] != I.type || !numeric(I.type) || I.a > YQ_MOD)
            return YQ_ERR_INVALID_ARG;
          pops = 2; pushes = 1; out_t = I.type;
          break;
        case OP_ARITH_COL: {
          int ct = col_type(I.b);
          if (depth < 1 || types[depth - 1] != I.type || !numeric(I.type) || ct < 0 || !castable(ct, I.type) || I.a > YQ_MOD)
            return YQ_ERR_INVALID_ARG;
          pops = 1; pushes = 1; out_t = I.type;
          break;
        }
        case OP_ARITH_CONST:
          if (depth < 1 || types[depth - 1] != I.type || !numeric(I.type) || I.imm < 0 || I.imm >= nconsts || I.a > YQ_MOD)
            return YQ_ERR_INVALID_ARG;
          pops = 1; pushes = 1; out_t = I.type;
          break;
        case OP_CMP:
          if (depth < 2 || types[depth - 1] != I.type || types[depth - 2] != I.type || !loadable(I.type) || I.a > YQ_NE)
            return YQ_ERR_INVALID_ARG;
          pops = 2; pushes = 1; out_t = YQ_BOOL;
          break;
        case OP_CMP_COL_CONST:
        case OP_AND_CMP_COL_CONST: {
          int ct = col_type(I.b);
          if (ct < 0 || I.a > YQ_NE) return YQ_ERR_INVALID_ARG;
          if (ct == YQ_TEXT) {
            if (I.imm < 0 || I.imm >= ntext) return YQ_ERR_INVALID_ARG;
            I.type = YQ_TEXT;
          } else if (!castable(ct, I.type) || I.imm < 0 || I.imm >= nconsts) {
            return YQ_ERR_INVALID_ARG;
          }
          if (I.op == OP_AND_CMP_COL_CONST) {
            if (depth < 1 || types[depth - 1] != YQ_BOOL) return YQ_ERR_INVALID_ARG;
            pops = 1;
          }
          pushes = 1; out_t = YQ_BOOL;
          break;
        }
        case OP_CMP_COL_COL: {
          int ct = col_type(I.b), dt = col_type(I.imm);
          if (ct < 0 || dt < 0 || I.a > YQ_NE) return YQ_ERR_INVALID_ARG;
          if ((ct == YQ_TEXT) != (dt == YQ_TEXT)) return YQ_ERR_INVALID_ARG;
          if (ct == YQ_TEXT) I.type = YQ_TEXT;
          else if (!castable(ct, I.type) || !castable(dt, I.type)) return YQ_ERR_INVALID_ARG;
          pushes = 1; out_t = YQ_BOOL;
          break;
        }
        case OP_AND:
        case OP_OR:
          if (depth < 2 || types[depth - 1] != YQ_BOOL || types[depth - 2] != YQ_BOOL) return YQ_ERR_INVALID_ARG;
          pops = 2; pushes = 1; out_t = YQ_BOOL;
          break;
        case OP_NOT:
          if (depth < 1 || types[depth - 1] != YQ_BOOL) return YQ_ERR_INVALID_ARG;
          pops = 1; pushes = 1; out_t = YQ_BOOL;
          break;
        case OP_IS_NULL:
        case OP_IS_NOT_NULL:
          if (depth < 1) return YQ_ERR_INVALID_ARG;
          pops = 1; pushes = 1; out_t = YQ_BOOL;
          break;
        default: return YQ_ERR_INVALID_ARG;
      }
      depth -= pops;
      if (depth + pushes > 4) return YQ_ERR_UNSUPPORTED;  // deeper than the register stack
      for (int p = 0; p < pushes; ++p) types[depth++] = out_t;
      if (len >= kMaxInsns - 1) return YQ_ERR_UNSUPPORTED;
      code[len++] = I;
      peephole(start);
    }
    if (depth != 1) return YQ_ERR_INVALID_ARG;
    result_type = types[0];
    return YQ_OK;
  }

  // Fuse the last instructions of the current program where possible.
  void peephole(int start) {
    for (;;) {
      if (len - start >= 2) {
        Insn& x = code[len - 2];
        Insn& y = code[len - 1];
        // COL c ; CAST c.type->t   =>  COL c as t (only from the column's own type)
        if (x.op == OP_COL && y.op == OP_CAST && x.type == y.type && x.type == col_type(x.a)) {
          x.type = y.a;
          --len;
          continue;
        }
      }
      if (len - start >= 3) {
        Insn& x = code[len - 3];
        Insn& y = code[len - 2];
        Insn& z = code[len - 1];
        // <bool> ; CMP_COL_CONST ; AND  =>  <bool> ; AND_CMP_COL_CONST
        if (y.op == OP_CMP_COL_CONST && z.op == OP_AND && produces_value(x)) {
          y.op = OP_AND_CMP_COL_CONST;
          --len;
          continue;
        }
        // <v> ; COL c ; ARITH op  =>  <v> ; ARITH_COL op c
        if (y.op == OP_COL && z.op == OP_ARITH && z.type == y.type && produces_value(x)) {
          Insn f;
          f.op = OP_ARITH_COL;
          f.type = z.type;
          f.a = z.a;
          f.b = y.a;
          f.imm = 0;
          y = f;
          --len;
          continue;
        }
        // <v> ; CONST k ; ARITH op  =>  <v> ; ARITH_CONST op k
        if (y.op == OP_CONST && z.op == OP_ARITH && z.type == y.type && produces_value(x)) {
          Insn f;
          f.op = OP_ARITH_CONST;
          f.type = z.type;
          f.a = z.a;
          f.b = 0;
          f.imm = y.imm;
          y = f;
          --len;
          continue;
        }
      }
      break;
    }
  }
  // True when x leaves a value on the stack that the next instruction's
  // fused form may consume (any non-emit instruction).
  static bool produces_value(const Insn& x) {
    return x.op != OP_EMIT_PRED && x.op != OP_EMIT_AGG && x.op != OP_EMIT_PROJ;
  }

  int emit(uint8_t op, uint8_t a, uint8_t b, uint8_t type) {
    if (len >= kMaxInsns) return YQ_ERR_UNSUPPORTED;
    Insn I;
    I.op = op; I.a = a; I.b = b; I.type = type; I.imm = 0;
    code[len++] = I;
    return YQ_OK;
  }

  static int agg_kind(int upd, int cls) {
    switch (upd) {
      case UPD_SUM_I: return cls == TC_I32 ? AK_SUM_I32 : AK_SUM_I64;
      case UPD_SUM_F: return cls == TC_F32 ? AK_SUM_F32 : AK_SUM_F64;
      case UPD_MIN_I: return cls == TC_I32 ? AK_MIN_I32 : AK_MIN_I64;
      case UPD_MAX_I: return cls == TC_I32 ? AK_MAX_I32 : AK_MAX_I64;
      case UPD_MIN_F: return cls == TC_F32 ? AK_MIN_F32 : AK_MIN_F64;
      case UPD_MAX_F: return cls == TC_F32 ? AK_MAX_F32 : AK_MAX_F64;
      default: return AK_COUNT;
    }
  }

  static Insn mk(uint8_t op, uint8_t type, uint8_t a, uint8_t b, int32_t imm) {
    Insn I;
    I.op = op; I.type = type; I.a = a; I.b = b; I.imm = imm;
    return I;
  }

  // Resolve the loader form into P.code. A fused comparison whose column is
  // not already of the comparison's class runs as its plain sequence, and a
  // BOOL aggregate input is widened to INT64 first. Resolved programs end up
  // in P.code[0, len); `remap` maps loader positions (such as the end of a
  // predicate) to resolved ones and `used_cols` lists the columns read.
  int finalize() {
    Insn x[kMaxInsns];
    int m = 0;
    auto put = [&](const Insn& I) {
      if (m >= kMaxInsns) return false;
      x[m++] = I;
      return true;
    };
    for (int i = 0; i < len; ++i) {
      const Insn& I = code[i];
      remap[i] = m;
      bool ok = true;
      if ((I.op == OP_CMP_COL_CONST || I.op == OP_AND_CMP_COL_CONST) && I.type != YQ_TEXT &&
          P.cols[I.b].tc != type_class(I.type)) {
        ok = put(mk(OP_COL, I.type, I.b, 0, 0)) && put(mk(OP_CONST, I.type, 0, 0, I.imm)) &&
             put(mk(OP_CMP, I.type, I.a, 0, 0)) && (I.op == OP_CMP_COL_CONST || put(mk(OP_AND, YQ_BOOL, 0, 0, 0)));
      } else if (I.op == OP_CMP_COL_COL && I.type != YQ_TEXT &&
                 (P.cols[I.b].tc != type_class(I.type) || P.cols[I.imm].tc != type_class(I.type))) {
        ok = put(mk(OP_COL, I.type, I.b, 0, 0)) && put(mk(OP_COL, I.type, (uint8_t)I.imm, 0, 0)) &&
             put(mk(OP_CMP, I.type, I.a, 0, 0));
      } else if (I.op == OP_EMIT_AGG && I.type == YQ_BOOL && I.b != UPD_COUNT && I.b != UPD_COUNT_STAR) {
        ok = put(mk(OP_CAST, YQ_BOOL, YQ_INT64, 0, 0)) && put(mk(OP_EMIT_AGG, YQ_INT64, I.a, I.b, 0));
      } else {
        ok = put(I);
      }
      if (!ok) return YQ_ERR_UNSUPPORTED;
    }
    remap[len] = m;
    int depth = 0;
    used_cols = 0;
    for (int i = 0; i < m; ++i) {
      const Insn& I = x[i];
      RInsn R;
      memset(&R, 0, sizeof(R));
      int pushes = 0, pops = 0;
      const int tc = type_class(I.type);
      switch (I.op) {
        case OP_COL:
          R.opc = (uint16_t)(R_COL + tc);
          R.a = I.a;
          used_cols |= 1u << I.a;
          pushes = 1;
          break;
        case OP_CONST:
          R.opc = (uint16_t)(R_CONST + tc);
          R.imm = (uint16_t)I.imm;
          pushes = 1;
          break;
        case OP_NULL:
          R.opc = R_NULL;
          pushes = 1;
          break;
        case OP_CAST:
          R.opc = (uint16_t)(R_CAST + tc * 5 + type_class(I.a));
          break;
        case OP_ARITH:
          R.opc = (uint16_t)(R_ARITH + tc * 5 + I.a);
          pops = 2;
          break;
        case OP_ARITH_COL:
          R.opc = (uint16_t)(R_ARITH_COL + tc * 5 + I.a);
          R.b = I.b;
          used_cols |= 1u << I.b;
          break;
        case OP_ARITH_CONST:
          R.opc = (uint16_t)(R_ARITH_CONST + tc * 5 + I.a);
          R.imm = (uint16_t)I.imm;
          break;
        case OP_CMP:
          R.opc = (uint16_t)(R_CMP + tc * 6 + I.a);
          pops = 2;
          break;
        case OP_CMP_COL_CONST:
        case OP_AND_CMP_COL_CONST:
          R.opc = (uint16_t)(R_CMP_CC + tc * 6 + I.a);
          R.b = I.b;
          R.imm = (uint16_t)I.imm;
          used_cols |= 1u << I.b;
          if (I.op == OP_AND_CMP_COL_CONST) R.flags |= RF_AND;
          else pushes = 1;
          break;
        case OP_CMP_COL_COL:
          R.opc = (uint16_t)(R_CMP_CCOL + tc * 6 + I.a);
          R.b = I.b;
          R.c = (uint8_t)I.imm;
          used_cols |= (1u << I.b) | (1u << I.imm);
          pushes = 1;
          break;
        case OP_AND: R.opc = R_AND; pops = 2; break;
        case OP_OR: R.opc = R_OR; pops = 2; break;
        case OP_NOT: R.opc = R_NOT; break;
        case OP_IS_NULL: R.opc = R_IS_NULL; break;
        case OP_IS_NOT_NULL: R.opc = R_IS_NOT_NULL; break;
        case OP_EMIT_PRED: R.opc = R_EMIT_PRED; pops = 1; break;
        case OP_EMIT_AGG:
          R.opc = (uint16_t)(R_EMIT_AGG + agg_kind(I.b, tc));
          R.a = I.a;
          pops = 1;
          break;
        case OP_EMIT_PROJ: {
          const int w = tc == TC_BOOL ? 0 : ((tc == TC_I32 || tc == TC_F32) ? 1 : 2);
          R.opc = (uint16_t)(R_EMIT_PROJ + w);
          R.a = I.a;
          pops = 1;
          break;
        }
        default: return YQ_ERR_INVALID_ARG;
      }
      if (pushes) {
        if (depth >= 4) return YQ_ERR_UNSUPPORTED;
        R.flags |= (uint8_t)(depth < 3 ? depth : 3);
        ++depth;
      } else if (pops == 2) {
        if (depth < 2) return YQ_ERR_INVALID_ARG;
        R.flags |= (uint8_t)(depth - 2);
        --depth;
      } else if (pops == 1) {
        if (depth < 1) return YQ_ERR_INVALID_ARG;
        R.flags |= (uint8_t)(depth - 1 < 3 ? depth - 1 : 3);
        --depth;
      }
      P.code[i] = R;
    }
    len = m;
    return YQ_OK;
  }
};

}  // namespace yq
