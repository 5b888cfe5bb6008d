// CSV scan: tokenizer state machine and field conversions (host + device).
//
// What the reference does per row (src/engine/operators/get_operator.cpp:66-101):
// the vendored csv-parser (vendor/csv-parser/csv.hpp:7063-7140, default
// format) splits the text into records and fields, and each projected field
// becomes a value by
//   INT      std::stoi   (strtol base 10, then an int range check)
//   FLOAT    std::stof   (strtof; errno == ERANGE throws)
//   DATETIME strptime("%Y-%m-%d %H:%M:%S") + timegm, 0 when strptime fails
//            (include/enums/data_type_utils.hpp:24-44)
//   STRING   String::set: the bytes up to the first NUL, at most slot-1 of
//            them, NUL padded (include/kernels/string_kernel.hpp:16-31)
// and an empty field is NULL with the sentinel INT_MIN / FLT_MIN / 0 / "".
//
// Everything here is written from those semantics and checked against the C
// library the reference links (tests/test_csv_cpu.py fuzzes these functions,
// compiled for the host, against glibc's strtof/strtol/strptime/timegm).
// The same header compiles as plain C++ (no nvcc) for those checks.
#pragma once

#if defined(__CUDACC__)
#define YQ_CSV_HD __host__ __device__ inline
#define YQ_CSV_COLD __host__ __device__ __noinline__  // rare paths stay out of the hot loops
#else
#define YQ_CSV_HD inline
#define YQ_CSV_COLD inline __attribute__((noinline))
#endif

#include <stdint.h>

namespace yq {
namespace csv {

// ------------------------------------------------------------- tokenizer
// Character classes and states of the record/field state machine. It restates
// csv-parser's default parse loop (csv.hpp:7063-7140): ',' delimits fields;
// '\r' and '\n' end a record, and a run of them ends ONE record (blank lines
// vanish); a '"' that opens a field starts quoted mode; inside quoted mode
// "" is an escaped quote, a quote before a delimiter or newline closes the
// field, and a lone quote before anything else is kept as a literal; a quote
// inside an unquoted field is a literal.
enum : uint32_t { C_OTHER = 0, C_QUOTE = 1, C_DELIM = 2, C_NL = 3 };
enum : uint32_t { S_FIELD = 0, S_UNQ = 1, S_QUO = 2, S_QQ = 3, S_REC = 4 };
constexpr int NSTATES = 5;
constexpr int NMAPS = 48;  // state maps reachable by composing the four class maps

YQ_CSV_HD constexpr uint32_t char_class(uint32_t c) {
  return c == '"' ? C_QUOTE : c == ',' ? C_DELIM : (c == '\n' || c == '\r') ? C_NL : C_OTHER;
}

// next state for (class, state): 15 bits per class (3 per state) in one word.
// rows: OTHER, QUOTE, DELIM, NL; within a row: FIELD, UNQ, QUO, QQ, REC
constexpr uint64_t row15(uint32_t f, uint32_t u, uint32_t q, uint32_t qq, uint32_t r) {
  return (uint64_t)(f | u << 3 | q << 6 | qq << 9 | r << 12);
}
constexpr uint64_t STEP_WORD = row15(S_UNQ, S_UNQ, S_QUO, S_QUO, S_UNQ) |
                               row15(S_QUO, S_UNQ, S_QQ, S_QUO, S_QUO) << 15 |
                               row15(S_FIELD, S_FIELD, S_QUO, S_FIELD, S_FIELD) << 30 |
                               row15(S_REC, S_REC, S_QUO, S_REC, S_REC) << 45;
YQ_CSV_HD constexpr uint32_t step(uint32_t cls, uint32_t s) {
  return (uint32_t)(STEP_WORD >> (15 * cls + 3 * s)) & 7u;
}

// A byte begins a record when the machine is at a record start and the byte
// is not a newline (the first record starts at byte 0 in state S_REC).
YQ_CSV_HD constexpr bool starts_record(uint32_t cls, uint32_t s) { return s == S_REC && cls != C_NL; }

// The monoid of state maps, enumerated at compile time: map m sends start
// state s to state (map_word[m] >> 3s) & 7. step[4m + c] describes map m
// followed by one byte of class c: bits 0-5 hold the resulting map's index,
// and byte s of (step >> 8) is 1 when that byte starts a record for start
// state s. Map 0 is the identity.
struct Tables {
  uint64_t step[NMAPS * 4];
  uint32_t map_word[NMAPS];
  int count;
};

constexpr Tables make_tables() {
  Tables t{};
  uint32_t id = 0;
  for (uint32_t s = 0; s < NSTATES; ++s) id |= s << (3 * s);
  t.map_word[0] = id;
  int n = 1;
  for (int i = 0; i < n; ++i) {
    for (uint32_t c = 0; c < 4; ++c) {
      uint32_t m = 0;
      uint64_t inc = 0;
      for (uint32_t s = 0; s < NSTATES; ++s) {
        uint32_t st = (t.map_word[i] >> (3 * s)) & 7u;
        m |= step(c, st) << (3 * s);
        if (starts_record(c, st)) inc |= 1ull << (8 * s);
      }
      int j = 0;
      while (j < n && t.map_word[j] != m) ++j;
      if (j == n) {
        if (n == NMAPS) { t.count = -1; return t; }
        t.map_word[n++] = m;
      }
      t.step[4 * i + c] = (uint64_t)j | inc << 8;
    }
  }
  t.count = n;
  return t;
}

// ------------------------------------------------------- chunk summaries
// A byte range's effect on the tokenizer: the state map and, per start state,
// how many records start inside the range.
struct Summary {
  uint32_t map;
  uint32_t c[NSTATES];
};

// 0xff in each byte of w equal to the same byte of pat.
YQ_CSV_HD uint32_t eq4(uint32_t w, uint32_t pat) {
#if defined(__CUDA_ARCH__)
  return __vcmpeq4(w, pat);
#else
  uint32_t r = 0;
  for (int b = 0; b < 4; ++b)
    if (((w >> (8 * b)) & 0xffu) == ((pat >> (8 * b)) & 0xffu)) r |= 0xffu << (8 * b);
  return r;
#endif
}

// One bit per byte (bit b = byte b) of a 0x00/0xff byte mask.
YQ_CSV_HD uint32_t byte_bits(uint32_t m) { return ((((m >> 7) & 0x01010101u) * 0x01020408u) >> 24) & 0xfu; }

YQ_CSV_HD int popc64(uint64_t x) {
#if defined(__CUDA_ARCH__)
  return __popcll(x);
#else
  return __builtin_popcountll(x);
#endif
}

// Class of each byte of a word, 2 bits at the bottom of each byte.
YQ_CSV_HD uint32_t classes4(uint32_t w) {
  const uint32_t q = eq4(w, 0x22222222u), d = eq4(w, 0x2c2c2c2cu);
  const uint32_t n = eq4(w, 0x0a0a0a0au) | eq4(w, 0x0d0d0d0du);
  return (q & 0x01010101u) | (d & 0x02020202u) | (n & 0x03030303u);
}

// Quote-free 64-byte chunks (most chunks of numeric text): newline bitmask
// and the first and last byte classes decide everything. With no quote, a
// start state outside quotes ends in the state the last byte sets, QUO stays
// QUO, and QQ leaves quotes unless its first byte is ordinary; records start
// at the non-newline bytes that follow a newline, plus byte 0 from REC.
struct Chunk64 {
  uint64_t nl;      // bit b: byte b is '\n' or '\r'
  bool quotes;      // any '"' in the chunk
  uint32_t c0, cl;  // classes of the first and last byte
};

YQ_CSV_HD Chunk64 scan64(const uint32_t* w) {
  Chunk64 k;
  uint32_t anyq = 0;
  k.nl = 0;
  for (int i = 0; i < 16; ++i) {
    anyq |= eq4(w[i], 0x22222222u);
    k.nl |= (uint64_t)byte_bits(eq4(w[i], 0x0a0a0a0au) | eq4(w[i], 0x0d0d0d0du)) << (4 * i);
  }
  k.quotes = anyq != 0;
  k.c0 = char_class(w[0] & 0xffu);
  k.cl = char_class(w[15] >> 24);
  return k;
}

YQ_CSV_HD Summary summary_quote_free(const Chunk64& k) {
  const uint32_t e = k.cl == C_NL ? S_REC : k.cl == C_DELIM ? S_FIELD : S_UNQ;
  const uint32_t cnt = (uint32_t)popc64(~k.nl & (k.nl << 1));
  const bool qq_stays = k.c0 == C_OTHER;
  Summary s;
  s.map = e | e << 3 | S_QUO << 6 | (qq_stays ? S_QUO : e) << 9 | e << 12;
  s.c[S_FIELD] = cnt;
  s.c[S_UNQ] = cnt;
  s.c[S_QUO] = 0;
  s.c[S_QQ] = qq_stays ? 0 : cnt;
  s.c[S_REC] = cnt + (k.c0 != C_NL ? 1u : 0u);
  return s;
}

// Record starts of a quote-free chunk entered in `state`, as a bitmask.
YQ_CSV_HD uint64_t starts_quote_free(const Chunk64& k, uint32_t state) {
  if (state == S_QUO || (state == S_QQ && k.c0 == C_OTHER)) return 0;
  uint64_t m = ~k.nl & (k.nl << 1);
  if (state == S_REC && k.c0 != C_NL) m |= 1;
  return m;
}

// Summary of 64 bytes (16 little-endian words) by the map table: one lookup
// per byte, one per word of four ordinary bytes (the "other" class map is
// idempotent and starts at most one record).
YQ_CSV_HD Summary summary_by_table(const uint32_t* w, const uint64_t* step_tab, const uint32_t* map_word) {
  uint32_t id = 0;
  uint64_t cnt = 0;
  for (int i = 0; i < 16; ++i) {
    const uint32_t c4 = classes4(w[i]);
    if (c4 == 0) {
      const uint64_t e = step_tab[id * 4 + C_OTHER];
      id = (uint32_t)e & 63u;
      cnt += e >> 8;
    } else {
      for (int b = 0; b < 4; ++b) {
        const uint64_t e = step_tab[id * 4 + ((c4 >> (8 * b)) & 3u)];
        id = (uint32_t)e & 63u;
        cnt += e >> 8;
      }
    }
  }
  Summary s;
  s.map = map_word[id];
  for (int k = 0; k < NSTATES; ++k) s.c[k] = (uint32_t)(cnt >> (8 * k)) & 0xffu;
  return s;
}

// ------------------------------------------------------------ field views
// A field's value as the reference's std::string sees it, viewed through the
// raw bytes: reads stop at `len` and, like the C functions behind the reference
// (which read the std::string through c_str()), at a NUL byte. In a quoted
// field the first '"' of the content also ends every numeric/date conversion,
// which is exactly where those conversions stop on the unescaped text too.
struct View {
  const uint8_t* p;
  uint32_t len;
  YQ_CSV_HD uint32_t at(uint32_t i) const { return i < len ? (uint32_t)p[i] : 0u; }
};

YQ_CSV_HD bool is_space(uint32_t c) { return c == ' ' || (c >= 9 && c <= 13); }
YQ_CSV_HD bool is_digit(uint32_t c) { return c - '0' < 10u; }
YQ_CSV_HD uint32_t lower(uint32_t c) { return (c - 'A' < 26u) ? c + 32 : c; }

enum : int32_t { CONV_OK = 0, CONV_INVALID = 1, CONV_RANGE = 2 };
constexpr int32_t INT32_MIN_ = -2147483647 - 1;

// ------------------------------------------------------------------ stoi
// std::stoi(s) = strtol(s, &end, 10) on a 64-bit long: leading white space,
// an optional sign, decimal digits; no digit -> invalid_argument; a value
// outside long, or outside int, -> out_of_range.
YQ_CSV_HD int32_t parse_int32(View v, int32_t* out) {
  uint32_t i = 0;
  while (is_space(v.at(i))) ++i;
  bool neg = false;
  if (v.at(i) == '+' || v.at(i) == '-') { neg = v.at(i) == '-'; ++i; }
  if (!is_digit(v.at(i))) { *out = 0; return CONV_INVALID; }
  uint64_t mag = 0;
  bool big = false;
  for (; is_digit(v.at(i)); ++i) {
    if (!big) {
      mag = mag * 10 + (v.at(i) - '0');
      if (mag > 0x80000000ull) big = true;
    }
  }
  if (big || (!neg && mag > 0x7fffffffull)) { *out = 0; return CONV_RANGE; }
  *out = neg ? (int32_t)(0u - (uint32_t)mag) : (int32_t)mag;
  return CONV_OK;
}

// ----------------------------------------------------------------- bignum
// Small fixed-size unsigned integer for the exact comparisons of the float
// conversion's rare path (32-bit limbs, little endian).
constexpr int BIG_LIMBS = 40;
struct Big {
  uint32_t w[BIG_LIMBS];
  int n;
  YQ_CSV_HD void set(uint64_t v) {
    n = 0;
    while (v) { w[n++] = (uint32_t)v; v >>= 32; }
  }
  YQ_CSV_HD void mul_add(uint32_t m, uint32_t a) {
    uint64_t carry = a;
    for (int i = 0; i < n; ++i) {
      uint64_t t = (uint64_t)w[i] * m + carry;
      w[i] = (uint32_t)t;
      carry = t >> 32;
    }
    if (carry && n < BIG_LIMBS) w[n++] = (uint32_t)carry;
  }
  YQ_CSV_HD void mul_pow5(int k) {
    while (k >= 13) { mul_add(1220703125u, 0); k -= 13; }  // 5^13
    uint32_t m = 1;
    while (k-- > 0) m *= 5;
    if (m != 1) mul_add(m, 0);
  }
  YQ_CSV_HD void shl(int bits) {
    if (n == 0 || bits <= 0) return;
    int limbs = bits >> 5, b = bits & 31;
    int nn = n + limbs + 1;
    if (nn > BIG_LIMBS) nn = BIG_LIMBS;
    for (int i = nn - 1; i >= 0; --i) {
      int src = i - limbs;
      uint32_t hi = (src >= 0 && src < n) ? w[src] : 0u;
      uint32_t lo = (src - 1 >= 0 && src - 1 < n) ? w[src - 1] : 0u;
      w[i] = b ? (hi << b) | (lo >> (32 - b)) : hi;
    }
    n = nn;
    while (n > 0 && w[n - 1] == 0) --n;
  }
};

YQ_CSV_HD int big_cmp(const Big& a, const Big& b) {
  if (a.n != b.n) return a.n < b.n ? -1 : 1;
  for (int i = a.n - 1; i >= 0; --i)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
  return 0;
}

// Significant decimal digits of a number, kept for exact comparisons.
constexpr int MAX_SIG_DIGITS = 120;

// The decimal value: the digits at dig[0..nd) (already without leading zeros),
// times 10^exp10, plus `sticky` (nonzero digits beyond the kept ones).
struct Decimal {
  const uint8_t* base;   // the field bytes
  uint32_t int_begin;    // first digit of the significand (may be a leading zero)
  uint32_t int_end;      // end of the integer digits
  uint32_t frac_begin;   // first fraction digit (== frac_end when none)
  uint32_t frac_end;
  int64_t exp10;         // the written exponent (after 'e')
};

// Compare the decimal (exactly) with m * 2^e. Returns -1, 0, 1.
YQ_CSV_HD int cmp_decimal(const Decimal& d, uint64_t m, int e) {
  // Collect up to MAX_SIG_DIGITS significant digits into a bignum.
  Big a;
  a.n = 0;
  int kept = 0;
  bool sticky = false, started = false;
  int64_t q = d.exp10;  // value = digits * 10^q, q adjusted per fraction digit kept
  for (int part = 0; part < 2; ++part) {
    uint32_t b = part ? d.frac_begin : d.int_begin, en = part ? d.frac_end : d.int_end;
    for (uint32_t i = b; i < en; ++i) {
      uint32_t c = d.base[i] - '0';
      if (!started && c == 0) { if (part) --q; continue; }
      started = true;
      if (kept < MAX_SIG_DIGITS) {
        a.mul_add(10, c);
        ++kept;
        if (part) --q;
      } else {
        if (c) sticky = true;
        if (!part) ++q;
      }
    }
  }
  Big bm;
  bm.set(m);
  if (a.n == 0) return bm.n == 0 ? 0 : -1;
  // digits * 10^q vs m * 2^e  ->  digits * 5^q * 2^q vs m * 2^e
  int64_t ea = q, eb = e;
  if (q >= 0) a.mul_pow5((int)q); else bm.mul_pow5((int)-q);
  if (ea >= eb) a.shl((int)(ea - eb)); else bm.shl((int)(eb - ea));
  int c = big_cmp(a, bm);
  if (c == 0 && sticky) c = 1;
  return c;
}

// float32 pieces: f = sig * 2^e with sig < 2^24.
YQ_CSV_HD void float_parts(uint32_t bits, uint64_t* sig, int* e) {
  uint32_t ex = (bits >> 23) & 0xff, man = bits & 0x7fffff;
  if (ex == 0) { *sig = man; *e = -149; }
  else { *sig = man | 0x800000u; *e = (int)ex - 150; }
}

YQ_CSV_HD float bits_float(uint32_t b) {
  union { uint32_t u; float f; } x;
  x.u = b;
  return x.f;
}
YQ_CSV_HD uint32_t float_bits(float f) {
  union { uint32_t u; float f; } x;
  x.f = f;
  return x.u;
}

// Exact powers of ten representable in double.
YQ_CSV_HD double pow10_exact(int k) {
  double r = 1.0;
  double b = 10.0;
  while (k) { if (k & 1) r *= b; b *= b; k >>= 1; }  // exact for k <= 22
  return r;
}

// Round a positive decimal to float32 exactly (round to nearest, ties to
// even) and report ERANGE as glibc's strtof does: overflow, or a result that
// is tiny (below 2^-126 after rounding to 24 bits) and inexact.
// `approx` is a double within a relative 1e-12 of the value (or a clamp).
YQ_CSV_COLD int32_t round_decimal(const Decimal& d, double approx, uint32_t* out_bits) {
  const uint32_t FMAX = 0x7f7fffffu;
  uint32_t f;
  if (!(approx < 3.4028234663852886e38)) f = FMAX;
  else {
    float g = (float)approx;
    f = float_bits(g);
    if (f > FMAX) f = FMAX;
  }
  uint64_t s;
  int e;
  // above the midpoint to the next float?
  float_parts(f, &s, &e);
  int c = cmp_decimal(d, 2 * s + 1, e - 1);
  if (c > 0 || (c == 0 && (f & 1))) {
    ++f;  // FMAX + 1 is +inf
  } else if (f > 0) {
    // below the midpoint to the previous float?
    uint64_t ls;
    int le;
    if ((f & 0x7fffff) == 0 && (f >> 23) > 1) { ls = 4 * s - 1; le = e - 2; }
    else { ls = 2 * s - 1; le = e - 1; }
    c = cmp_decimal(d, ls, le);
    if (c < 0 || (c == 0 && (f & 1))) --f;
  }
  *out_bits = f;
  if (f >= 0x7f800000u) return CONV_RANGE;
  if (f <= 0x00800000u) {
    // tiny: below 2^-126 - 2^-151 (the value rounds below 2^-126 at 24 bits)
    int tiny = cmp_decimal(d, (1ull << 25) - 1, -151) < 0;
    if (tiny) {
      uint64_t fs;
      int fe;
      float_parts(f, &fs, &fe);
      if (cmp_decimal(d, fs, fe) != 0) return CONV_RANGE;
    }
  }
  return CONV_OK;
}

// Round m * 2^e (m > 0, exact) to float32 bits; sticky = nonzero bits below m.
YQ_CSV_COLD int32_t round_binary(uint64_t m, int64_t e, bool sticky, uint32_t* out_bits) {
  // normalise m to have bit 63 set
  int lz = 0;
  while (!(m >> 63)) { m <<= 1; ++lz; }
  e -= lz;
  // value = m * 2^e, m in [2^63, 2^64): binary exponent of the leading bit
  int64_t lead = e + 63;
  // tininess after rounding to 24 bits with an unbounded exponent
  uint64_t keep24 = m >> 40, rem24 = m & ((1ull << 40) - 1);
  bool half24 = rem24 >> 39, rest24 = (rem24 & ((1ull << 39) - 1)) || sticky;
  uint64_t r24 = keep24 + (half24 && (rest24 || (keep24 & 1)));
  int64_t lead24 = lead + (r24 >> 24 ? 1 : 0);
  bool tiny = lead24 < -126;
  if (lead24 > 127) { *out_bits = 0x7f800000u; return CONV_RANGE; }
  // bits kept: normal 24, subnormal fewer
  int64_t shift = 40;  // bits dropped from m
  if (lead < -126) shift += (-126 - lead);
  uint64_t keep, rem;
  bool half, rest;
  if (shift >= 64) {
    keep = 0;
    half = shift == 64 ? (m >> 63) != 0 : false;
    rest = (shift == 64 ? (m << 1) != 0 : true) || sticky;
  } else {
    keep = m >> shift;
    rem = m & ((1ull << shift) - 1);
    half = (rem >> (shift - 1)) & 1;
    rest = (rem & ((1ull << (shift - 1)) - 1)) || sticky;
  }
  bool inexact = half || rest;
  keep += half && (rest || (keep & 1));
  uint32_t bits;
  if (lead < -126) {
    bits = (uint32_t)keep;  // subnormal (or rounds up to 0x00800000 = FLT_MIN)
  } else {
    int64_t ex = lead + 127;
    if (keep >> 24) { keep >>= 1; ++ex; }
    if (ex >= 255) { *out_bits = 0x7f800000u; return CONV_RANGE; }
    bits = (uint32_t)(ex << 23) | (uint32_t)(keep & 0x7fffff);
  }
  *out_bits = bits;
  return (tiny && inexact) ? CONV_RANGE : CONV_OK;
}

YQ_CSV_HD uint32_t hex_val(uint32_t c) {
  if (c - '0' < 10u) return c - '0';
  c = lower(c);
  if (c - 'a' < 6u) return c - 'a' + 10;
  return 16;
}

// std::stof(s): strtof semantics on the field (white space, sign, decimal or
// hexadecimal significand with optional exponent, inf/infinity, nan and
// nan(n-char-sequence)); CONV_INVALID when nothing converts, CONV_RANGE when
// strtof sets ERANGE (std::stof throws in both cases).
YQ_CSV_HD int32_t parse_float32(View v, float* out) {
  uint32_t i = 0;
  while (is_space(v.at(i))) ++i;
  uint32_t sign = 0;
  if (v.at(i) == '+' || v.at(i) == '-') { sign = v.at(i) == '-' ? 0x80000000u : 0u; ++i; }
  uint32_t bits = 0;
  int32_t st = CONV_OK;
  uint32_t c0 = lower(v.at(i));
  if (c0 == 'i') {
    if (lower(v.at(i + 1)) == 'n' && lower(v.at(i + 2)) == 'f') {
      *out = bits_float(sign | 0x7f800000u);
      return CONV_OK;
    }
    *out = 0.0f;
    return CONV_INVALID;
  }
  if (c0 == 'n') {
    if (lower(v.at(i + 1)) == 'a' && lower(v.at(i + 2)) == 'n') {
      uint32_t nan = 0x7fc00000u;
      uint32_t j = i + 3;
      if (v.at(j) == '(') {
        uint32_t k = j + 1;
        while (true) {
          uint32_t c = v.at(k);
          if (is_digit(c) || lower(c) - 'a' < 26u || c == '_') ++k;
          else break;
        }
        if (v.at(k) == ')') {
          // payload = strtoull(sequence, base 0), used when it spans the sequence
          uint32_t p = j + 1;
          uint64_t val = 0;
          bool ovf = false;
          uint32_t base = 10;
          if (v.at(p) == '0' && lower(v.at(p + 1)) == 'x' && hex_val(v.at(p + 2)) < 16) { base = 16; p += 2; }
          else if (v.at(p) == '0') base = 8;
          uint32_t q = p;
          while (q < k) {
            uint32_t dv = base == 16 ? hex_val(v.at(q)) : v.at(q) - '0';
            if (dv >= base) break;
            if (val > (~0ull - dv) / base) ovf = true;
            val = val * base + dv;
            ++q;
          }
          if (q == k && k > j + 1) {
            if (ovf) val = ~0ull;
            nan = 0x7fc00000u | (uint32_t)(val & 0x3fffff);
          }
        }
      }
      *out = bits_float(sign | nan);
      return CONV_OK;
    }
    *out = 0.0f;
    return CONV_INVALID;
  }
  if (v.at(i) == '0' && lower(v.at(i + 1)) == 'x' &&
      (hex_val(v.at(i + 2)) < 16 || (v.at(i + 2) == '.' && hex_val(v.at(i + 3)) < 16))) {
    uint32_t j = i + 2;
    uint64_t m = 0;
    int64_t e = 0;
    bool sticky = false;
    int used = 0;  // significant hex digits in m
    for (; hex_val(v.at(j)) < 16; ++j) {
      uint32_t h = hex_val(v.at(j));
      if (used == 0 && h == 0) continue;
      if (used < 16) { m = m << 4 | h; ++used; }
      else { e += 4; if (h) sticky = true; }
    }
    if (v.at(j) == '.') {
      ++j;
      for (; hex_val(v.at(j)) < 16; ++j) {
        uint32_t h = hex_val(v.at(j));
        if (used == 0 && h == 0) { e -= 4; continue; }
        if (used < 16) { m = m << 4 | h; ++used; e -= 4; }
        else if (h) sticky = true;
      }
    }
    if (lower(v.at(j)) == 'p') {
      uint32_t k = j + 1;
      bool eneg = false;
      if (v.at(k) == '+' || v.at(k) == '-') { eneg = v.at(k) == '-'; ++k; }
      if (is_digit(v.at(k))) {
        int64_t x = 0;
        for (; is_digit(v.at(k)); ++k)
          if (x < 100000000) x = x * 10 + (v.at(k) - '0');
        e += eneg ? -x : x;
      }
    }
    if (m == 0) bits = 0;
    else st = round_binary(m, e, sticky, &bits);
    *out = bits_float(sign | bits);
    return st;
  }
  // decimal
  Decimal d;
  d.base = v.p;
  d.int_begin = i;
  uint32_t j = i;
  while (is_digit(v.at(j))) ++j;
  d.int_end = j;
  d.frac_begin = d.frac_end = j;
  if (v.at(j) == '.') {
    d.frac_begin = j + 1;
    uint32_t k = j + 1;
    while (is_digit(v.at(k))) ++k;
    d.frac_end = k;
    j = k;
  }
  if (d.int_end == d.int_begin && d.frac_end == d.frac_begin) { *out = 0.0f; return CONV_INVALID; }
  d.exp10 = 0;
  if (lower(v.at(j)) == 'e') {
    uint32_t k = j + 1;
    bool eneg = false;
    if (v.at(k) == '+' || v.at(k) == '-') { eneg = v.at(k) == '-'; ++k; }
    if (is_digit(v.at(k))) {
      int64_t x = 0;
      for (; is_digit(v.at(k)); ++k)
        if (x < 100000000) x = x * 10 + (v.at(k) - '0');
      d.exp10 = eneg ? -x : x;
    }
  }
  // first 19 significant digits, the decimal position of the leading digit
  uint64_t w = 0;
  int nd = 0;           // significant digits read into w
  int64_t lead = 0;     // value in [10^lead, 10^(lead+1))
  bool more = false;    // nonzero significant digits beyond w
  bool started = false;
  int64_t pos = (int64_t)(d.int_end - d.int_begin) - 1;  // power of ten of the current digit
  for (int part = 0; part < 2; ++part) {
    uint32_t b = part ? d.frac_begin : d.int_begin, en = part ? d.frac_end : d.int_end;
    for (uint32_t k = b; k < en; ++k, --pos) {
      uint32_t c = v.p[k] - '0';
      if (!started) {
        if (c == 0) continue;
        started = true;
        lead = pos;
      }
      if (nd < 19) { w = w * 10 + c; ++nd; }
      else if (c) more = true;
    }
  }
  if (!started) { *out = bits_float(sign); return CONV_OK; }  // zero
  lead += d.exp10;
  if (lead >= 39) { *out = bits_float(sign | 0x7f800000u); return CONV_RANGE; }
  if (lead <= -47) { *out = bits_float(sign); return CONV_RANGE; }
  int64_t q = lead - (nd - 1);  // value ~= w * 10^q
  // fast path: exact w, one correctly rounded double operation, a float
  // result comfortably inside the normal range and not a float midpoint
  if (!more && w < (1ull << 53) && q >= -22 && q <= 22 && lead > -36 && lead < 37) {
    double dv = q >= 0 ? (double)w * pow10_exact((int)q) : (double)w / pow10_exact((int)-q);
    union { double d; uint64_t u; } x;
    x.d = dv;
    uint32_t low = (uint32_t)(x.u & ((1ull << 29) - 1));
    if (low != (1u << 28)) {
      *out = bits_float(sign | float_bits((float)dv));
      return CONV_OK;
    }
  }
  double approx;
  {
    double dw = (double)w;
    int64_t k = q;
    double p = 1.0;
    while (k > 22) { p *= 1e22; k -= 22; }
    while (k < -22) { p /= 1e22; k += 22; }
    approx = k >= 0 ? dw * p * pow10_exact((int)k) : dw * p / pow10_exact((int)-k);
  }
  st = round_decimal(d, approx, &bits);
  *out = bits_float(sign | bits);
  return st;
}

// -------------------------------------------------------------- datetime
// days from 1970-01-01 to y-m-d in the proleptic Gregorian calendar (the
// civil-day count of H. Hinnant's "chrono-compatible low-level date
// algorithms"); m in 1..12, d may exceed the month (timegm normalises it).
YQ_CSV_HD int64_t days_from_civil(int64_t y, int64_t m, int64_t d) {
  y -= m <= 2;
  int64_t era = (y >= 0 ? y : y - 399) / 400;
  int64_t yoe = y - era * 400;
  int64_t doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
  int64_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + doe - 719468;
}

// strptime's numeric field: white space, then at least one digit, reading
// while fewer than `n` digits are read and val*10 <= hi; then lo <= val <= hi.
YQ_CSV_HD bool get_num(View v, uint32_t* i, int lo, int hi, int n, int* out) {
  uint32_t k = *i;
  while (is_space(v.at(k))) ++k;
  if (!is_digit(v.at(k))) return false;
  int val = 0, cnt = 0;
  do {
    val = val * 10 + (int)(v.at(k) - '0');
    ++k;
    ++cnt;
  } while (cnt < n && val * 10 <= hi && is_digit(v.at(k)));
  if (val < lo || val > hi) return false;
  *i = k;
  *out = val;
  return true;
}

// getDateTime (include/enums/data_type_utils.hpp:24-44): strptime with
// "%Y-%m-%d %H:%M:%S" then timegm; 0 when strptime fails. Trailing bytes
// after the seconds are ignored, as strptime's return value is.
YQ_CSV_HD int64_t parse_datetime(View v) {
  uint32_t i = 0;
  int Y, M, D, h, m, s;
  if (!get_num(v, &i, 0, 9999, 4, &Y)) return 0;
  if (v.at(i) != '-') return 0;
  ++i;
  if (!get_num(v, &i, 1, 12, 2, &M)) return 0;
  if (v.at(i) != '-') return 0;
  ++i;
  if (!get_num(v, &i, 1, 31, 2, &D)) return 0;
  while (is_space(v.at(i))) ++i;  // ' ' in the format: any white space, or none
  if (!get_num(v, &i, 0, 23, 2, &h)) return 0;
  if (v.at(i) != ':') return 0;
  ++i;
  if (!get_num(v, &i, 0, 59, 2, &m)) return 0;
  if (v.at(i) != ':') return 0;
  ++i;
  if (!get_num(v, &i, 0, 61, 2, &s)) return 0;
  return days_from_civil(Y, M, D) * 86400 + h * 3600 + m * 60 + s;
}

// ------------------------------------------------------------- records
// Output description of one CSV field: the output column it feeds (or -1),
// its type and slot width.
struct FieldOut {
  int32_t column;
  int32_t type;   // YQ_INT32, YQ_FLOAT32, YQ_DATETIME, YQ_TEXT
  int32_t width;  // bytes per value in the output column
};

// Walks one record field by field, from its first byte (a record start) to
// the newline that ends it or to `len`: the state machine above, taken one
// field at a time. A field that opens with '"' is quoted: inside it, "" is an
// escaped quote, a quote before ',' or a newline (or the end) closes it, and a
// quote before anything else is kept. An unquoted field runs to the first ','
// or newline (a quote in it is an ordinary byte).
struct FieldCursor {
  const uint8_t* rec;
  uint32_t len;
  uint32_t i;
  bool done;

  YQ_CSV_HD void init(const uint8_t* r, uint32_t l) {
    rec = r;
    len = l;
    i = 0;
    done = false;
  }
  // The next field's content (without its quotes); false once the record has
  // no more fields.
  YQ_CSV_HD bool next(View* v, bool* escapes) {
    if (done) return false;
    *escapes = false;
    if (i < len && rec[i] == '"') {
      const uint32_t begin = ++i;
      for (;;) {
        if (i >= len) {  // the text ends inside the quotes
          *v = View{rec + begin, i - begin};
          done = true;
          return true;
        }
        if (rec[i] != '"') { ++i; continue; }
        if (i + 1 >= len) {  // closing quote at the end of the text
          *v = View{rec + begin, i - begin};
          done = true;
          return true;
        }
        const uint32_t d = rec[i + 1];
        if (d == ',') {
          *v = View{rec + begin, i - begin};
          i += 2;
          return true;
        }
        if (d == '\n' || d == '\r') {
          *v = View{rec + begin, i - begin};
          done = true;
          return true;
        }
        if (d == '"') { *escapes = true; i += 2; continue; }
        ++i;  // a lone quote stays in the field
      }
    }
    const uint32_t begin = i;
    for (; i < len; ++i) {
      const uint32_t c = rec[i];
      if (c == ',') {
        *v = View{rec + begin, i - begin};
        ++i;
        return true;
      }
      if (c == '\n' || c == '\r') break;
    }
    *v = View{rec + begin, i - begin};
    done = true;
    return true;
  }
  YQ_CSV_HD bool more() const { return !done; }
};

// ------------------------------------------------------ typed fast paths
// One pass over an unquoted field in its common written form: find its end
// and convert it together. Each returns false, with the cursor unmoved, when
// the field is in any other form (quoted, empty, signs or spaces where the
// general conversion decides, too many digits, a float needing exact
// rounding, a date outside the canonical layout...); the caller then takes
// the general path (next() + parse_*), which is exact for every input.

// Consumes the terminator at rec[j] (',', newline or the end), if it is one.
YQ_CSV_HD bool FieldCursor_end(FieldCursor& c, uint32_t j) {
  if (j >= c.len) { c.i = j; c.done = true; return true; }
  const uint32_t t = c.rec[j];
  if (t == ',') { c.i = j + 1; return true; }
  if (t == '\n' || t == '\r') { c.i = j; c.done = true; return true; }
  return false;
}

// [+-]digits (at most 9) then a terminator.
YQ_CSV_HD bool fast_int32(FieldCursor& c, int32_t* out) {
  if (c.done) return false;
  uint32_t j = c.i;
  bool neg = false;
  if (j < c.len && (c.rec[j] == '-' || c.rec[j] == '+')) { neg = c.rec[j] == '-'; ++j; }
  uint32_t v = 0, nd = 0;
  while (j < c.len && (uint32_t)c.rec[j] - '0' < 10u && nd < 10) { v = v * 10 + (c.rec[j] - '0'); ++j; ++nd; }
  if (nd == 0 || nd > 9) return false;
  if (!FieldCursor_end(c, j)) return false;
  *out = neg ? (int32_t)(0u - v) : (int32_t)v;
  return true;
}

// [+-]digits[.digits] (at most 19 significant digits) then a terminator, when
// one double operation on exact operands rounds it exactly (the parse_float32
// fast path's conditions).
YQ_CSV_HD bool fast_float32(FieldCursor& c, float* out) {
  if (c.done) return false;
  uint32_t j = c.i;
  uint32_t sign = 0;
  if (j < c.len && (c.rec[j] == '-' || c.rec[j] == '+')) { sign = c.rec[j] == '-' ? 0x80000000u : 0u; ++j; }
  uint64_t w = 0;
  int nd = 0, frac = 0, digits = 0;
  bool dot = false;
  for (; j < c.len; ++j) {
    const uint32_t ch = c.rec[j];
    if (ch - '0' < 10u) {
      ++digits;
      if (w == 0 && ch == '0') { if (dot) ++frac; continue; }
      if (nd == 19) return false;
      w = w * 10 + (ch - '0');
      ++nd;
      if (dot) ++frac;
    } else if (ch == '.' && !dot) {
      dot = true;
    } else {
      break;
    }
  }
  if (digits == 0) return false;
  if (j < c.len && (c.rec[j] == 'e' || c.rec[j] == 'E')) return false;
  const uint32_t j_end = j;
  if (w == 0) {
    if (!FieldCursor_end(c, j_end)) return false;
    *out = bits_float(sign);
    return true;
  }
  const int q = -frac;                     // value = w * 10^q
  const int lead = nd - 1 + q;             // decimal position of the leading digit
  if (w >= (1ull << 53) || q < -22 || lead <= -36 || lead >= 37) return false;
  const double dv = (double)w / pow10_exact(-q);
  union { double d; uint64_t u; } x;
  x.d = dv;
  if ((uint32_t)(x.u & ((1ull << 29) - 1)) == (1u << 28)) return false;  // a float midpoint
  if (!FieldCursor_end(c, j_end)) return false;
  *out = bits_float(sign | float_bits((float)dv));
  return true;
}

// "YYYY-MM-DD HH:MM:SS" exactly, each part a value strptime's field rule
// accepts with that many digits, then a terminator.
YQ_CSV_HD bool fast_datetime(FieldCursor& c, int64_t* out) {
  if (c.done || c.i + 19 > c.len) return false;
  const uint8_t* p = c.rec + c.i;
  const uint8_t sep[6] = {'-', '-', ' ', ':', ':', 0};
  const int at[5] = {4, 7, 10, 13, 16};
  for (int k = 0; k < 5; ++k)
    if (p[at[k]] != sep[k]) return false;
  const int dpos[14] = {0, 1, 2, 3, 5, 6, 8, 9, 11, 12, 14, 15, 17, 18};
  for (int k = 0; k < 14; ++k)
    if ((uint32_t)p[dpos[k]] - '0' >= 10u) return false;
  const int Y = (p[0] - '0') * 1000 + (p[1] - '0') * 100 + (p[2] - '0') * 10 + (p[3] - '0');
  const int M0 = p[5] - '0', D0 = p[8] - '0', h0 = p[11] - '0', m0 = p[14] - '0', s0 = p[17] - '0';
  // a two-digit field is read as two digits only when its first digit * 10 <= the maximum
  if (M0 > 1 || D0 > 3 || h0 > 2 || m0 > 5 || s0 > 6) return false;
  const int M = M0 * 10 + (p[6] - '0'), D = D0 * 10 + (p[9] - '0'), h = h0 * 10 + (p[12] - '0');
  const int mi = m0 * 10 + (p[15] - '0'), se = s0 * 10 + (p[18] - '0');
  if (M < 1 || M > 12 || D < 1 || D > 31 || h > 23 || mi > 59 || se > 61) return false;
  if (!FieldCursor_end(c, c.i + 19)) return false;
  *out = days_from_civil(Y, M, D) * 86400 + h * 3600 + mi * 60 + se;
  return true;
}

// An unquoted text field copied while it is scanned (String::set: up to the
// first NUL, at most width-1 bytes, NUL padded).
template <class Store>
YQ_CSV_HD bool fast_text(FieldCursor& c, uint32_t width, Store& store) {
  if (c.done || (c.i < c.len && c.rec[c.i] == '"')) return false;
  uint32_t j = c.i, o = 0, word = 0;
  bool stop = false;
  for (; j < c.len; ++j) {
    const uint32_t ch = c.rec[j];
    if (ch == ',' || ch == '\n' || ch == '\r') break;
    if (stop) continue;
    if (ch == 0 || o >= width - 1) { stop = true; continue; }
    word |= ch << (8 * (o & 3));
    ++o;
    if ((o & 3) == 0) { store(o / 4 - 1, word); word = 0; }
  }
  for (; o < width; ++o)
    if ((o & 3) == 3) { store(o / 4, word); word = 0; }
  FieldCursor_end(c, j);
  return true;
}

// Every field of one record into its output through `emit` (fields in
// order; types uniform across a warp). desc(f) gives {projected, type,
// width}. Returns the field count check: true when the record has exactly
// nfields fields. Conversion failures go to *bad / *first_bad (key: field << 2
// | kind, the smallest field first).
template <class Desc, class Emit>
YQ_CSV_HD bool convert_record(const uint8_t* rec, uint32_t len, int nfields, const Desc& desc, Emit& emit,
                              uint32_t* bad, uint32_t* first_bad) {
  FieldCursor cur;
  cur.init(rec, len);
  for (int f = 0; f < nfields; ++f) {
    const FieldOut d = desc(f);
    View v;
    bool esc;
    if (d.column < 0) {
      if (!cur.next(&v, &esc)) return false;
      continue;
    }
    switch (d.type) {
      case 0: {
        int32_t x;
        if (fast_int32(cur, &x)) { emit.i32(f, x, false); continue; }
        break;
      }
      case 1: {
        float x;
        if (fast_float32(cur, &x)) { emit.f32(f, x, false); continue; }
        break;
      }
      case 2: {
        int64_t x;
        if (fast_datetime(cur, &x)) { emit.i64(f, x, false); continue; }
        break;
      }
      default: {
        auto store = [&emit, f](uint32_t k, uint32_t w) { emit.word(f, k, w); };
        if (cur.i < cur.len && cur.rec[cur.i] != ',' && cur.rec[cur.i] != '\n' && cur.rec[cur.i] != '\r' &&
            fast_text(cur, (uint32_t)d.width, store)) {
          emit.null(f, false);
          continue;
        }
        break;
      }
    }
    if (!cur.next(&v, &esc)) return false;  // fewer fields than the header
    const bool empty = v.len == 0;
    int32_t st = CONV_OK;
    switch (d.type) {
      case 0: {
        int32_t x = INT32_MIN_;
        if (!empty) st = parse_int32(v, &x);
        emit.i32(f, st == CONV_OK ? x : 0, empty);
        break;
      }
      case 1: {
        float x = bits_float(0x00800000u);  // FLT_MIN, the reference's NULL sentinel
        if (!empty) st = parse_float32(v, &x);
        emit.f32(f, st == CONV_OK ? x : 0.0f, empty);
        break;
      }
      case 2:
        emit.i64(f, empty ? 0 : parse_datetime(v), empty);
        break;
      default: {
        auto store = [&emit, f](uint32_t k, uint32_t w) { emit.word(f, k, w); };
        copy_text(v, esc, (uint32_t)d.width, store);
        emit.null(f, empty);
        break;
      }
    }
    if (st != CONV_OK) {
      ++*bad;
      const uint32_t key = (uint32_t)f << 2 | (uint32_t)st;
      if (key < *first_bad) *first_bad = key;
    }
  }
  return !cur.more();  // more fields than the header when the record goes on
}

// Calls sink(field_index, content_view, has_escapes) for every field of the
// record; returns the field count.
template <class Sink>
YQ_CSV_HD uint32_t walk_record(const uint8_t* rec, uint32_t len, Sink& sink) {
  FieldCursor cur;
  cur.init(rec, len);
  View v;
  bool esc;
  uint32_t n = 0;
  while (cur.next(&v, &esc)) sink(n++, v, esc);
  return n;
}

// Copies a field's text into a slot of `width` bytes as String::set does:
// the bytes up to the first NUL, at most width-1, NUL padded. A quoted field
// that held an escaped "" is un-escaped the way csv-parser's CSVRow::get_field
// does it (csv.hpp:7775-7792): of all the quotes in the field, the 1st, 3rd,
// 5th ... are kept and the others dropped, whether adjacent or not.
template <class Store>
YQ_CSV_HD void copy_text(View v, bool escapes, uint32_t width, Store& store) {
  uint32_t o = 0, word = 0;
  bool prev_quote = false;
  for (uint32_t i = 0; i < v.len; ++i) {
    uint32_t c = v.p[i];
    if (escapes && c == '"') {
      if (prev_quote) { prev_quote = false; continue; }
      prev_quote = true;
    }
    if (c == 0 || o >= width - 1) break;
    word |= c << (8 * (o & 3));
    ++o;
    if ((o & 3) == 0) { store(o / 4 - 1, word); word = 0; }
  }
  // flush the partial word and the NUL padding
  for (; o < width; ++o) {
    if ((o & 3) == 3) { store(o / 4, word); word = 0; }
  }
}

// ---------------------------------------------------------------- writer
// Cell text as CsvWriter::batchToCsv writes it
// (include/engine/operators/csv_writer.hpp:42-73): INT by std::to_chars,
// FLOAT by std::to_chars(..., chars_format::fixed, 4), DATETIME quoted as
// gmtime_r + strftime("%Y-%m-%d %H:%M:%S") (data_type_utils.hpp:46-57), STRING
// quoted as stored (up to its NUL, no escaping), NULL as "". `Out` provides
// put(c) (append a byte), put_at(k, c) (the byte k places after the current
// end, before a skip(n) that moves the end past it) and skip(n).

template <class Out>
YQ_CSV_HD void put_u64(Out& o, uint64_t v) {
  uint32_t n = 1;
  for (uint64_t t = v; t >= 10; t /= 10) ++n;
  for (uint32_t k = n; k-- > 0; v /= 10) o.put_at(k, (uint32_t)('0' + v % 10));
  o.skip(n);
}

template <class Out>
YQ_CSV_HD void put_i64(Out& o, int64_t v) {
  if (v < 0) {
    o.put('-');
    put_u64(o, 0ull - (uint64_t)v);
  } else {
    put_u64(o, (uint64_t)v);
  }
}

template <class Out>
YQ_CSV_HD void put_2(Out& o, uint32_t v) {
  o.put('0' + v / 10);
  o.put('0' + v % 10);
}

// Decimal digits of a value below 2^128 held as four 32-bit limbs.
template <class Out>
YQ_CSV_COLD void put_u128(Out& o, uint32_t l0, uint32_t l1, uint32_t l2, uint32_t l3) {
  uint32_t lim[4] = {l0, l1, l2, l3};
  uint32_t chunk[5];  // base 10^9, least significant first
  int nc = 0;
  do {
    uint64_t rem = 0;
    for (int i = 3; i >= 0; --i) {
      const uint64_t cur = rem << 32 | lim[i];
      lim[i] = (uint32_t)(cur / 1000000000u);
      rem = cur % 1000000000u;
    }
    chunk[nc++] = (uint32_t)rem;
  } while ((lim[0] | lim[1] | lim[2] | lim[3]) && nc < 5);
  put_u64(o, chunk[nc - 1]);
  for (int c = nc - 2; c >= 0; --c) {
    uint32_t v = chunk[c];
    for (int k = 8; k >= 0; --k, v /= 10) o.put_at((uint32_t)k, '0' + v % 10);
    o.skip(9);
  }
}

// std::to_chars(float, fixed, 4): the exact binary value rounded to four
// decimals, ties to even; "inf", "-inf", "nan", "-nan".
template <class Out>
YQ_CSV_HD void put_fixed4(Out& o, float x) {
  const uint32_t b = float_bits(x);
  const uint32_t ex = (b >> 23) & 0xffu, man = b & 0x7fffffu;
  if (b >> 31) o.put('-');
  if (ex == 0xff) {
    if (man) { o.put('n'); o.put('a'); o.put('n'); }
    else { o.put('i'); o.put('n'); o.put('f'); }
    return;
  }
  const uint64_t m = ex ? (man | 0x800000u) : man;
  const int e = ex ? (int)ex - 150 : -149;
  if (e >= 0) {  // an integer m * 2^e < 2^128
    const int w = e >> 5, sh = e & 31;
    uint32_t lim[5] = {0, 0, 0, 0, 0};
    const uint64_t v = m << sh;  // < 2^56
    lim[w] = (uint32_t)v;
    lim[w + 1] = (uint32_t)(v >> 32);
    put_u128(o, lim[0], lim[1], lim[2], lim[3]);
    o.put('.'); o.put('0'); o.put('0'); o.put('0'); o.put('0');
    return;
  }
  const int k = -e;                  // 1..149
  const uint64_t t = m * 10000u;     // < 2^38
  uint64_t q = 0;
  if (k < 64) {
    q = t >> k;
    const uint64_t r = t & ((1ull << k) - 1), half = 1ull << (k - 1);
    if (r > half || (r == half && (q & 1))) ++q;
  }
  put_u64(o, q / 10000);
  uint32_t f = (uint32_t)(q % 10000);
  o.put('.');
  o.put('0' + f / 1000);
  o.put('0' + f / 100 % 10);
  o.put('0' + f / 10 % 10);
  o.put('0' + f % 10);
}

// y-m-d from days since 1970-01-01 (proleptic Gregorian; the inverse of
// days_from_civil, H. Hinnant's civil_from_days).
YQ_CSV_HD void civil_from_days(int64_t z, int64_t* y, uint32_t* m, uint32_t* d) {
  z += 719468;
  const int64_t era = (z >= 0 ? z : z - 146096) / 146097;
  const uint64_t doe = (uint64_t)(z - era * 146097);
  const uint64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  const uint64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const uint64_t mp = (5 * doy + 2) / 153;
  *d = (uint32_t)(doy - (153 * mp + 2) / 5 + 1);
  *m = (uint32_t)(mp < 10 ? mp + 3 : mp - 9);
  *y = (int64_t)yoe + era * 400 + (*m <= 2);
}

// gmtime_r + strftime("%Y-%m-%d %H:%M:%S"): the year unpadded, with its sign.
template <class Out>
YQ_CSV_HD void put_datetime(Out& o, int64_t secs) {
  int64_t days = secs / 86400, rem = secs % 86400;
  if (rem < 0) { rem += 86400; --days; }
  int64_t y;
  uint32_t mo, d;
  civil_from_days(days, &y, &mo, &d);
  put_i64(o, y);
  o.put('-');
  put_2(o, mo);
  o.put('-');
  put_2(o, d);
  o.put(' ');
  put_2(o, (uint32_t)(rem / 3600));
  o.put(':');
  put_2(o, (uint32_t)(rem / 60 % 60));
  o.put(':');
  put_2(o, (uint32_t)(rem % 60));
}

// One cell. type: YQ_INT32 0, YQ_FLOAT32 1, YQ_DATETIME 2, YQ_TEXT 3, YQ_INT64 4.
template <class Out>
YQ_CSV_HD void put_cell(Out& o, const void* data, const uint8_t* nulls, int32_t type, int32_t width, uint64_t row) {
  if (nulls && nulls[row]) {
    o.put('"');
    o.put('"');
    return;
  }
  switch (type) {
    case 0: put_i64(o, static_cast<const int32_t*>(data)[row]); break;
    case 1: put_fixed4(o, static_cast<const float*>(data)[row]); break;
    case 2:
      o.put('"');
      put_datetime(o, static_cast<const int64_t*>(data)[row]);
      o.put('"');
      break;
    case 4: put_i64(o, static_cast<const int64_t*>(data)[row]); break;
    default: {
      const uint8_t* t = static_cast<const uint8_t*>(data) + row * (uint64_t)width;
      o.put('"');
      for (int32_t i = 0; i < width && t[i]; ++i) o.put(t[i]);
      o.put('"');
      break;
    }
  }
}

// Output that only counts bytes.
struct CountOut {
  uint32_t n = 0;
  YQ_CSV_HD void put(uint32_t) { ++n; }
  YQ_CSV_HD void put_at(uint32_t, uint32_t) {}
  YQ_CSV_HD void skip(uint32_t k) { n += k; }
};

// Output into a byte buffer.
struct BufOut {
  uint8_t* p;
  YQ_CSV_HD void put(uint32_t c) { *p++ = (uint8_t)c; }
  YQ_CSV_HD void put_at(uint32_t k, uint32_t c) { p[k] = (uint8_t)c; }
  YQ_CSV_HD void skip(uint32_t k) { p += k; }
};

}  // namespace csv
}  // namespace yq
