// Test infrastructure: the device CSV scan's tokenizer and field conversions
// (yallasql_b200/csrc/yq_csv.cuh) compiled for the host with g++, so the CPU
// suite checks them against glibc and the reference's csv-parser without a GPU.
// hs_csv_scan follows the kernels' structure: record starts from 64-byte chunk
// summaries composed in order (the state-map tables, with the same
// four-ordinary-bytes shortcut), then one walk per record.
#include "../yallasql_b200/csrc/yq_csv.cuh"

#include <cfloat>
#include <climits>
#include <cstring>
#include <vector>

using namespace yq::csv;

namespace {

constexpr Tables kT = make_tables();
static_assert(kT.count == NMAPS, "tables");

// Summary of a chunk as the kernels make it: full 64-byte chunks through the
// quote-free shortcut or the map table, shorter ones byte by byte.
Summary chunk_summary(const uint8_t* p, uint64_t n) {
  if (n == 64) {
    uint32_t w[16];
    std::memcpy(w, p, 64);
    const Chunk64 k = scan64(w);
    if (!k.quotes) return summary_quote_free(k);
    return summary_by_table(w, kT.step, kT.map_word);
  }
  uint32_t id = 0;
  uint64_t cnt = 0;
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t e = kT.step[id * 4 + char_class(p[i])];
    id = (uint32_t)(e & 63);
    cnt += e >> 8;
  }
  Summary s;
  s.map = kT.map_word[id];
  for (int k = 0; k < NSTATES; ++k) s.c[k] = (cnt >> (8 * k)) & 0xff;
  return s;
}

}  // namespace

extern "C" {

// kind 0: stoi -> out (int32), 1: stof -> out (float bits), 2: datetime -> out.
void hs_convert(int kind, const uint8_t* buf, const uint64_t* offs, uint64_t n, int64_t* out, int32_t* status) {
  for (uint64_t i = 0; i < n; ++i) {
    View v{buf + offs[i], (uint32_t)(offs[i + 1] - offs[i])};
    if (kind == 0) {
      int32_t x;
      status[i] = parse_int32(v, &x);
      out[i] = x;
    } else if (kind == 1) {
      float x;
      status[i] = parse_float32(v, &x);
      out[i] = float_bits(x);
    } else {
      status[i] = 0;
      out[i] = parse_datetime(v);
    }
  }
}

// Record starts two ways: the plain state machine, and chunk summaries
// composed in order. Returns the count, or -1 when the two disagree.
int64_t hs_record_starts(const uint8_t* text, uint64_t n, uint32_t* starts, uint64_t cap) {
  std::vector<uint32_t> a;
  uint32_t st = S_REC;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t cls = char_class(text[i]);
    if (starts_record(cls, st)) a.push_back((uint32_t)i);
    st = step(cls, st);
  }
  uint64_t total = 0;
  uint32_t state = S_REC;
  std::vector<uint32_t> b;  // record starts as the emit kernel finds them, chunk by chunk
  for (uint64_t lo = 0; lo < n; lo += 64) {
    uint64_t len = n - lo < 64 ? n - lo : 64;
    Summary s = chunk_summary(text + lo, len);
    if (len == 64) {
      uint32_t w[16];
      std::memcpy(w, text + lo, 64);
      const Chunk64 k = scan64(w);
      if (!k.quotes) {
        for (uint64_t m = starts_quote_free(k, state); m; m &= m - 1) b.push_back((uint32_t)(lo + __builtin_ctzll(m)));
      } else {
        uint32_t st2 = state;
        for (uint64_t i = 0; i < 64; ++i) {
          uint32_t cls = char_class(text[lo + i]);
          if (starts_record(cls, st2)) b.push_back((uint32_t)(lo + i));
          st2 = step(cls, st2);
        }
      }
    } else {
      uint32_t st2 = state;
      for (uint64_t i = 0; i < len; ++i) {
        uint32_t cls = char_class(text[lo + i]);
        if (starts_record(cls, st2)) b.push_back((uint32_t)(lo + i));
        st2 = step(cls, st2);
      }
    }
    total += s.c[state];
    state = (s.map >> (3 * state)) & 7;
  }
  if (b != a) return -1;
  if (total != a.size()) return -1;
  for (uint64_t k = 0; k < a.size() && k < cap; ++k) starts[k] = a[k];
  return (int64_t)a.size();
}

// The device scan on the host: the same record split and the same
// per-record routine (convert_record) as k_csv_parse.
struct HostEmit {
  void** data;
  unsigned char** nulls;
  const int* width;
  uint64_t row;
  void i32(int f, int32_t x, bool n) { static_cast<int32_t*>(data[f])[row] = x; nulls[f][row] = n; }
  void f32(int f, float x, bool n) { static_cast<float*>(data[f])[row] = x; nulls[f][row] = n; }
  void i64(int f, int64_t x, bool n) { static_cast<int64_t*>(data[f])[row] = x; nulls[f][row] = n; }
  void word(int f, uint32_t k, uint32_t w) {
    std::memcpy(static_cast<char*>(data[f]) + row * (uint64_t)width[f] + 4 * k, &w, 4);
  }
  void null(int f, bool n) { nulls[f][row] = n; }
};

int64_t hs_csv_scan(const uint8_t* text, uint64_t n, int nfields, const int* field_type, const int* field_width,
                    void** out_data, unsigned char** out_nulls, uint64_t capacity, uint64_t* bad,
                    int64_t* first_bad_row, int* first_bad_field, int* first_bad_kind) {
  std::vector<uint32_t> starts(n + 1);
  int64_t nrec = hs_record_starts(text, n, starts.data(), n + 1);
  if (nrec < 0) return -2;
  *bad = 0;
  *first_bad_row = -1;
  *first_bad_field = -1;
  *first_bad_kind = 0;
  // records convert into scratch rows (like the kernel, which writes every
  // record's row and drops the short/long ones afterwards)
  std::vector<std::vector<uint8_t>> vals(nfields), nul(nfields);
  std::vector<void*> vp(nfields);
  std::vector<unsigned char*> np(nfields);
  std::vector<int> width(nfields);
  for (int f = 0; f < nfields; ++f) {
    const int ty = field_type[f];
    width[f] = ty == 3 ? field_width[f] : ty == 2 ? 8 : 4;
    vals[f].assign((size_t)(nrec + 1) * width[f], 0xee);
    nul[f].assign((size_t)nrec + 1, 7);
    vp[f] = vals[f].data();
    np[f] = nul[f].data();
  }
  auto desc = [&](int f) { return FieldOut{field_type[f] < 0 ? -1 : 0, field_type[f], field_width[f]}; };
  uint64_t rows = 0;
  for (int64_t r = 0; r < nrec; ++r) {
    const uint64_t st = starts[r], en = r + 1 < nrec ? starts[r + 1] : n;
    HostEmit emit{vp.data(), np.data(), width.data(), (uint64_t)r};
    uint32_t b = 0, first = ~0u;
    if (!convert_record(text + st, (uint32_t)(en - st), nfields, desc, emit, &b, &first)) continue;
    if (rows >= capacity) return -1;
    for (int f = 0; f < nfields; ++f) {
      if (field_type[f] < 0) continue;
      std::memcpy(static_cast<char*>(out_data[f]) + rows * width[f], vals[f].data() + r * width[f], width[f]);
      out_nulls[f][rows] = nul[f][r];
    }
    if (b) {
      if (*bad == 0) { *first_bad_row = (int64_t)rows; *first_bad_field = (int)(first >> 2); *first_bad_kind = (int)(first & 3); }
      *bad += b;
    }
    ++rows;
  }
  return (int64_t)rows;
}

}  // extern "C"

extern "C" {
// The writer's cell formatting on the host: kind 0 int32, 1 float32 (bits),
// 2 datetime, 4 int64. Each cell's text goes to out[i*64 ...], its length to len[i].
void hs_format(int kind, const int64_t* vals, uint64_t n, char* out, int32_t* len) {
  for (uint64_t i = 0; i < n; ++i) {
    int32_t i32 = (int32_t)vals[i];
    uint32_t fb = (uint32_t)vals[i];
    float f;
    std::memcpy(&f, &fb, 4);
    const void* data = kind == 0 ? (const void*)&i32 : kind == 1 ? (const void*)&f : (const void*)&vals[i];
    BufOut o{reinterpret_cast<uint8_t*>(out + i * 64)};
    put_cell(o, data, nullptr, kind, 0, 0);
    CountOut c;
    put_cell(c, data, nullptr, kind, 0, 0);
    len[i] = (int32_t)(o.p - reinterpret_cast<uint8_t*>(out + i * 64));
    if ((uint32_t)len[i] != c.n) len[i] = -1;  // the counting pass must agree with the writing pass
  }
}
}

#include <charconv>
extern "C" {
// std::to_chars(float, fixed, 4): the reference writer's own float routine.
int32_t hs_to_chars_fixed4(uint32_t bits, char* out) {
  float f;
  std::memcpy(&f, &bits, 4);
  auto r = std::to_chars(out, out + 64, f, std::chars_format::fixed, 4);
  return (int32_t)(r.ptr - out);
}
}
