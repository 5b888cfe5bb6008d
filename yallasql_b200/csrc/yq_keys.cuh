// Order-preserving key words shared by the radix sort and the merge path.
// A key of KW 32-bit words compares as an unsigned integer, word KW-1 most
// significant: signed integers are biased, floats sign-flipped (-0.0 == +0.0,
// NaN canonicalised above +inf), text slots read as big-endian words, DESC
// inverts the value words, and an optional top word orders NULLs.
#pragma once

#include "yq_common.cuh"

namespace yq {

struct KeySrc {
  const char* data;
  const uint8_t* nulls;
  const uint32_t* in_perm;  // multi-key sorts: this key's row for element e is in_perm[e]
  int32_t type;
  int32_t width;
  int32_t vwords;       // value words in the key (excluding the null word)
  int32_t desc;
  int32_t nulls_first;
  int32_t null_word;    // 1: word `vwords` is the null flag
  uint32_t* lossy;      // optional: the histogram sets it when a value would not survive the key words
};

// A value whose key words decode to a different bit pattern: -0.0, a NaN
// other than the canonical one, a bool byte other than 0/1.
__device__ __forceinline__ bool key_value_lossy(int type, const char* p) {
  if (type == YQ_FLOAT32) {
    const uint32_t b = *reinterpret_cast<const uint32_t*>(p);
    return b == 0x80000000u || (((b & 0x7f800000u) == 0x7f800000u) && (b & 0x007fffffu) && b != 0x7fc00000u);
  }
  if (type == YQ_FLOAT64) {
    const unsigned long long b = *reinterpret_cast<const unsigned long long*>(p);
    return b == 0x8000000000000000ull ||
           (((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull) && (b & 0x000fffffffffffffull) &&
            b != 0x7ff8000000000000ull);
  }
  if (type == YQ_BOOL) return (uint8_t)*p > 1u;
  return false;
}

__device__ __forceinline__ uint32_t bswap(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// Key words of the value stored at `p` (generic pointer: global or shared).
template <int KW>
__device__ __forceinline__ void make_key_ptr(const KeySrc& s, const char* p, bool is_null, uint32_t (&k)[KW]) {
#pragma unroll
  for (int j = 0; j < KW; ++j) k[j] = 0u;
  if (!is_null) {
    switch (s.type) {
      case YQ_INT32: k[0] = *reinterpret_cast<const uint32_t*>(p) ^ 0x80000000u; break;
      case YQ_FLOAT32: {
        uint32_t b = *reinterpret_cast<const uint32_t*>(p);
        if ((b & 0x7fffffffu) == 0u) b = 0u;                                               // -0.0 ties +0.0
        else if ((b & 0x7f800000u) == 0x7f800000u && (b & 0x007fffffu)) b = 0x7fc00000u;  // NaN above +inf
        k[0] = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        break;
      }
      case YQ_INT64:
      case YQ_DATETIME: {
        const uint2 v = *reinterpret_cast<const uint2*>(p);
        k[0] = v.x;
        if (KW > 1) k[KW > 1 ? 1 : 0] = v.y ^ 0x80000000u;
        break;
      }
      case YQ_FLOAT64: {
        unsigned long long b = *reinterpret_cast<const unsigned long long*>(p);
        if ((b & 0x7fffffffffffffffull) == 0ull) b = 0ull;
        else if ((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull && (b & 0x000fffffffffffffull))
          b = 0x7ff8000000000000ull;
        b = (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
        k[0] = (uint32_t)b;
        if (KW > 1) k[KW > 1 ? 1 : 0] = (uint32_t)(b >> 32);
        break;
      }
      case YQ_BOOL: k[0] = (uint32_t)(*p != 0); break;
      default: {  // TEXT: first vwords words of the slot as a big-endian integer
        const uint32_t* w = reinterpret_cast<const uint32_t*>(p);
#pragma unroll
        for (int j = 0; j < KW; ++j)
          if (j < s.vwords) k[j] = bswap(w[s.vwords - 1 - j]);
        break;
      }
    }
    if (s.desc) {
#pragma unroll
      for (int j = 0; j < KW; ++j)
        if (j < s.vwords) k[j] = ~k[j];
    }
  }
  if (s.null_word) {
    const uint32_t nv = s.nulls_first ? (is_null ? 0u : 1u) : (is_null ? 1u : 0u);
#pragma unroll
    for (int j = 0; j < KW; ++j)
      if (j == s.vwords) k[j] = nv;
  }
}

template <int KW>
__device__ __forceinline__ void make_key(const KeySrc& s, uint32_t row, uint32_t (&k)[KW]) {
  const bool is_null = s.nulls && s.nulls[row];
  make_key_ptr<KW>(s, s.data + (size_t)row * s.width, is_null, k);
}

// a <= b on KW-word unsigned keys (most significant word last).
template <int KW>
__device__ __forceinline__ bool key_le(const uint32_t (&a)[KW], const uint32_t (&b)[KW]) {
#pragma unroll
  for (int j = KW - 1; j >= 0; --j)
    if (a[j] != b[j]) return a[j] < b[j];
  return true;
}

}  // namespace yq
