// CSV scan on the device: record index + typed field conversion.
//
// Replaces the per-row host loop of GetOperator::next
// (src/engine/operators/get_operator.cpp:56-109: csv-parser read_row, then
// std::stoi / std::stof / getDateTime / String::set per projected field, then
// a synchronous cudaMemcpy per column in storeBuffer, :125-148).
//
// Pipeline over CSV text resident in HBM (the header line removed):
//   k_csv_tiles     each 16 KiB tile -> the state map of the tokenizer over it
//                   and its record-start counts per start state (64 bytes a
//                   thread, one shared-memory table lookup per byte, a word of
//                   four ordinary bytes in one lookup)
//   k_csv_tile_scan one block composes the tile maps in order: the tokenizer
//                   state and the first record index at every tile
//   k_csv_emit      each tile again, now from its known state: byte offset of
//                   every record start
//   k_csv_parse     128 records a block: their bytes staged into shared memory
//                   with 16-byte loads; one thread per record, the lanes of a
//                   warp on the same field at a time, so each conversion runs
//                   converged
// Rows whose field count differs from the header's are dropped afterwards
// (csv-parser's default VariableColumnPolicy::IGNORE_ROW), by a stable
// compaction that only runs when there are such rows.
#include "yq_common.cuh"
#include "yq_csv.cuh"

using namespace yq;
using namespace yq::csv;

namespace {

constexpr Tables kHostTables = make_tables();
static_assert(kHostTables.count == NMAPS, "tokenizer map enumeration");
__constant__ Tables kTab = make_tables();

constexpr int kTileThreads = 256;
constexpr int kBytesPerThread = 64;
constexpr uint64_t kTileBytes = (uint64_t)kTileThreads * kBytesPerThread;  // 16 KiB
constexpr int kScanThreads = 1024;
constexpr int kParseThreads = 128;
constexpr uint32_t kSpanCap = 16 * 1024;  // staged bytes per parse block (128 B a record on average)
constexpr uint32_t kIdentityMap = 0u | 1u << 3 | 2u << 6 | 3u << 9 | 4u << 12;

using Summ = Summary;

__device__ __forceinline__ uint32_t map_at(uint32_t map, uint32_t s) { return (map >> (3 * s)) & 7u; }

// a followed by b
__device__ __forceinline__ Summ compose(const Summ& a, const Summ& b) {
  Summ r;
  r.map = 0;
#pragma unroll
  for (uint32_t s = 0; s < NSTATES; ++s) {
    uint32_t m = map_at(a.map, s);
    r.map |= map_at(b.map, m) << (3 * s);
    uint32_t bc = b.c[0];
#pragma unroll
    for (uint32_t k = 1; k < NSTATES; ++k) bc = (m == k) ? b.c[k] : bc;
    r.c[s] = a.c[s] + bc;
  }
  return r;
}

__device__ __forceinline__ Summ identity_summ() {
  Summ r;
  r.map = kIdentityMap;
#pragma unroll
  for (int s = 0; s < NSTATES; ++s) r.c[s] = 0;
  return r;
}

__device__ __forceinline__ Summ shfl_up_summ(const Summ& x, int d) {
  Summ r;
  r.map = __shfl_up_sync(0xffffffffu, x.map, d);
#pragma unroll
  for (int s = 0; s < NSTATES; ++s) r.c[s] = __shfl_up_sync(0xffffffffu, x.c[s], d);
  return r;
}

// Exclusive scan of the block's summaries in thread order (composition is
// associative, not commutative). `warp_tot` holds blockDim/32 entries.
template <int kThreads>
__device__ Summ block_exclusive(const Summ& mine, Summ* warp_tot, Summ* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kThreads / 32;
  Summ inc = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Summ o = shfl_up_summ(inc, d);
    if (lane >= d) inc = compose(o, inc);
  }
  Summ excl = shfl_up_summ(inc, 1);
  if (lane == 0) excl = identity_summ();
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    Summ t = lane < kWarps ? warp_tot[lane] : identity_summ();
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      Summ o = shfl_up_summ(t, d);
      if (lane >= d) t = compose(o, t);
    }
    Summ e = shfl_up_summ(t, 1);
    if (lane == 0) e = identity_summ();
    if (lane < kWarps) warp_tot[lane] = e;
    if (lane == kWarps - 1 && total) *total = t;
  }
  __syncthreads();
  Summ r = compose(warp_tot[warp], excl);
  __syncthreads();  // warp_tot is reused by the caller's next scan
  return r;
}

__device__ __forceinline__ void load_tables(uint64_t* s_step, uint32_t* s_mapw) {
  for (int i = threadIdx.x; i < NMAPS * 4; i += blockDim.x) s_step[i] = kTab.step[i];
  for (int i = threadIdx.x; i < NMAPS; i += blockDim.x) s_mapw[i] = kTab.map_word[i];
  __syncthreads();
}

__device__ __forceinline__ void load64(const uint8_t* p, uint32_t* w) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const uint4 x = __ldg(q + v);
    w[4 * v] = x.x;
    w[4 * v + 1] = x.y;
    w[4 * v + 2] = x.z;
    w[4 * v + 3] = x.w;
  }
}

// Summary of this thread's 64 bytes of the tile.
__device__ Summ thread_summary(const uint8_t* data, uint64_t nbytes, uint64_t lo, bool aligned,
                               const uint64_t* s_step, const uint32_t* s_mapw) {
  if (aligned && lo + kBytesPerThread <= nbytes) {
    uint32_t w[16];
    load64(data + lo, w);
    const Chunk64 k = scan64(w);
    if (!k.quotes) return summary_quote_free(k);
    return summary_by_table(w, s_step, s_mapw);
  }
  const uint64_t hi = lo + kBytesPerThread < nbytes ? lo + kBytesPerThread : nbytes;
  uint32_t id = 0;
  uint64_t cnt = 0;
  for (uint64_t i = lo; i < hi; ++i) {
    const uint64_t e = s_step[id * 4 + char_class(data[i])];
    id = (uint32_t)e & 63u;
    cnt += e >> 8;
  }
  Summ r;
  r.map = s_mapw[id];
#pragma unroll
  for (int st = 0; st < NSTATES; ++st) r.c[st] = (uint32_t)(cnt >> (8 * st)) & 0xffu;
  return r;
}

__global__ void __launch_bounds__(kTileThreads) k_csv_tiles(const uint8_t* __restrict__ data, uint64_t nbytes,
                                                            int aligned, uint32_t* __restrict__ tile_map,
                                                            uint32_t* __restrict__ tile_cnt) {
  __shared__ uint64_t s_step[NMAPS * 4];
  __shared__ uint32_t s_mapw[NMAPS];
  __shared__ Summ s_warp[kTileThreads / 32];
  __shared__ Summ s_total;
  load_tables(s_step, s_mapw);
  const uint64_t tile = blockIdx.x;
  const uint64_t lo = tile * kTileBytes + (uint64_t)threadIdx.x * kBytesPerThread;
  Summ mine = lo < nbytes ? thread_summary(data, nbytes, lo, aligned != 0, s_step, s_mapw) : identity_summ();
  block_exclusive<kTileThreads>(mine, s_warp, &s_total);
  // the total is written by warp 0 before the scan's second barrier
  if (threadIdx.x == 0) {
    tile_map[tile] = s_total.map;
#pragma unroll
    for (int s = 0; s < NSTATES; ++s) tile_cnt[tile * NSTATES + s] = s_total.c[s];
  }
}

// One block: the state at the start of every tile and the index of its first
// record. tile_start[t] = state << 32 | first record index. records[0] = total.
__global__ void __launch_bounds__(kScanThreads) k_csv_tile_scan(const uint32_t* __restrict__ tile_map,
                                                                const uint32_t* __restrict__ tile_cnt,
                                                                uint32_t ntiles,
                                                                unsigned long long* __restrict__ tile_start,
                                                                unsigned long long* __restrict__ records) {
  __shared__ Summ s_warp[kScanThreads / 32];
  const uint32_t per = (ntiles + kScanThreads - 1) / kScanThreads;
  const uint32_t t0 = threadIdx.x * per;
  const uint32_t t1 = t0 + per < ntiles ? t0 + per : ntiles;
  Summ mine = identity_summ();
  for (uint32_t t = t0; t < t1; ++t) {
    Summ x;
    x.map = tile_map[t];
#pragma unroll
    for (int s = 0; s < NSTATES; ++s) x.c[s] = tile_cnt[(size_t)t * NSTATES + s];
    mine = compose(mine, x);
  }
  Summ excl = block_exclusive<kScanThreads>(mine, s_warp, nullptr);
  uint32_t state = map_at(excl.map, S_REC);
  unsigned long long base = excl.c[S_REC];
  for (uint32_t t = t0; t < t1; ++t) {
    tile_start[t] = (unsigned long long)state << 32 | base;
    base += tile_cnt[(size_t)t * NSTATES + state];
    state = map_at(tile_map[t], state);
  }
  if (t1 == ntiles && t0 < t1) records[0] = base;
  if (ntiles == 0 && threadIdx.x == 0) records[0] = 0;
}

__global__ void __launch_bounds__(kTileThreads) k_csv_emit(const uint8_t* __restrict__ data, uint64_t nbytes,
                                                           int aligned,
                                                           const unsigned long long* __restrict__ tile_start,
                                                           uint32_t* __restrict__ starts) {
  __shared__ uint64_t s_step[NMAPS * 4];
  __shared__ uint32_t s_mapw[NMAPS];
  __shared__ Summ s_warp[kTileThreads / 32];
  load_tables(s_step, s_mapw);
  const uint64_t tile = blockIdx.x;
  const uint64_t lo = tile * kTileBytes + (uint64_t)threadIdx.x * kBytesPerThread;
  Summ mine = lo < nbytes ? thread_summary(data, nbytes, lo, aligned != 0, s_step, s_mapw) : identity_summ();
  Summ excl = block_exclusive<kTileThreads>(mine, s_warp, nullptr);
  if (lo >= nbytes) return;
  const unsigned long long ts = tile_start[tile];
  const uint32_t tstate = (uint32_t)(ts >> 32);
  uint32_t state = map_at(excl.map, tstate);
  uint32_t idx = (uint32_t)ts + excl.c[tstate];
  const uint64_t hi = lo + kBytesPerThread < nbytes ? lo + kBytesPerThread : nbytes;
  if (aligned && hi - lo == kBytesPerThread) {
    uint32_t w[16];
    load64(data + lo, w);  // a second read of the same 64 bytes: an L1 hit
    const Chunk64 k = scan64(w);
    if (!k.quotes) {
      for (uint64_t m = starts_quote_free(k, state); m; m &= m - 1) starts[idx++] = (uint32_t)(lo + __ffsll(m) - 1);
      return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const uint32_t c4 = classes4(w[j]);
      const uint32_t off = (uint32_t)(lo + 4 * j);
      if (c4 == 0) {
        if (state == S_REC) starts[idx++] = off;
        state = step(C_OTHER, state);
      } else {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const uint32_t cls = (c4 >> (8 * b)) & 3u;
          if (starts_record(cls, state)) starts[idx++] = off + b;
          state = step(cls, state);
        }
      }
    }
  } else {
    for (uint64_t i = lo; i < hi; ++i) {
      const uint32_t cls = char_class(data[i]);
      if (starts_record(cls, state)) starts[idx++] = (uint32_t)i;
      state = step(cls, state);
    }
  }
}

// ------------------------------------------------------------------ parse
struct FieldDesc {
  void* data;      // output column (nullptr: field not projected)
  uint8_t* nulls;  // output null bytes
  int32_t type;
  int32_t width;
};

struct ParseParams {
  const uint8_t* data;
  uint64_t nbytes;
  const uint32_t* starts;
  uint32_t nrec;
  int32_t nfields;
  int32_t aligned;
  uint8_t* valid;                   // per record: field count matches
  unsigned long long* counters;     // [0] invalid rows, [1] bad cells, [2] first bad cell key
  FieldDesc f[YQ_CSV_MAX_FIELDS];
};

// Output of one record's cells into row `row` of the projected columns.
struct DevEmit {
  const ParseParams* P;
  uint32_t row;
  __device__ __forceinline__ void i32(int f, int32_t x, bool null) {
    static_cast<int32_t*>(P->f[f].data)[row] = x;
    P->f[f].nulls[row] = null;
  }
  __device__ __forceinline__ void f32(int f, float x, bool null) {
    static_cast<float*>(P->f[f].data)[row] = x;
    P->f[f].nulls[row] = null;
  }
  __device__ __forceinline__ void i64(int f, int64_t x, bool null) {
    static_cast<long long*>(P->f[f].data)[row] = x;
    P->f[f].nulls[row] = null;
  }
  __device__ __forceinline__ void word(int f, uint32_t k, uint32_t w) {
    reinterpret_cast<uint32_t*>(static_cast<char*>(P->f[f].data) + (size_t)row * P->f[f].width)[k] = w;
  }
  __device__ __forceinline__ void null(int f, bool null) { P->f[f].nulls[row] = null; }
};

struct DevDesc {
  const ParseParams* P;
  __device__ __forceinline__ FieldOut operator()(int f) const {
    const FieldDesc& d = P->f[f];
    return FieldOut{d.data ? 0 : -1, d.type, d.width};
  }
};

// One thread per record, fields in lockstep: every lane of a warp takes field
// f of its own record at the same time with the same field type, so the
// conversions run converged (convert_record: typed one-pass fast paths, the
// exact general path for every other form).
__global__ void __launch_bounds__(kParseThreads) k_csv_parse(const __grid_constant__ ParseParams P) {
  extern __shared__ __align__(16) uint8_t s_span[];
  const uint32_t r0 = blockIdx.x * kParseThreads;
  const uint32_t rend = r0 + kParseThreads < P.nrec ? r0 + kParseThreads : P.nrec;
  const uint64_t b0 = P.starts[r0];
  const uint64_t b1 = rend < P.nrec ? P.starts[rend] : P.nbytes;
  const uint64_t a0 = b0 & ~15ull;
  const bool staged = b1 - a0 <= kSpanCap;
  if (staged) {
    const uint64_t nchunks = (b1 - a0 + 15) / 16;
    for (uint64_t k = threadIdx.x; k < nchunks; k += kParseThreads) {
      const uint64_t g = a0 + k * 16;
      if (P.aligned && g + 16 <= P.nbytes) {
        *reinterpret_cast<uint4*>(s_span + k * 16) = __ldg(reinterpret_cast<const uint4*>(P.data + g));
      } else {
        for (int j = 0; j < 16; ++j) s_span[k * 16 + j] = g + j < P.nbytes ? P.data[g + j] : 0;
      }
    }
  }
  __syncthreads();
  const uint32_t r = r0 + threadIdx.x;
  if (r >= rend) return;
  const uint64_t st = P.starts[r];
  const uint64_t en = r + 1 < P.nrec ? P.starts[r + 1] : P.nbytes;
  DevEmit emit{&P, r};
  uint32_t bad = 0, first = ~0u;
  const bool ok = convert_record(staged ? s_span + (st - a0) : P.data + st, (uint32_t)(en - st), P.nfields,
                                 DevDesc{&P}, emit, &bad, &first);
  P.valid[r] = ok ? 1 : 0;
  if (!ok) {
    atomicAdd(&P.counters[0], 1ull);
  } else if (bad) {
    atomicAdd(&P.counters[1], (unsigned long long)bad);
    atomicMin(&P.counters[2], (unsigned long long)r << 12 | first);
  }
}

// Stable compaction of one column by the valid flags: pos = inclusive scan.
__global__ void k_csv_compact(const uint8_t* __restrict__ src, const uint8_t* __restrict__ src_nulls,
                              uint32_t width, const uint8_t* __restrict__ valid, const uint32_t* __restrict__ pos,
                              uint32_t n, uint8_t* __restrict__ dst, uint8_t* __restrict__ dst_nulls) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!valid[i]) continue;
    const uint32_t o = pos[i] - 1;
    for (uint32_t b = 0; b < width; b += 4)
      *reinterpret_cast<uint32_t*>(dst + (size_t)o * width + b) =
          *reinterpret_cast<const uint32_t*>(src + (size_t)i * width + b);
    dst_nulls[o] = src_nulls[i];
  }
}

// ------------------------------------------------------------------ writer
constexpr int kFmtThreads = 128;
constexpr uint32_t kFmtSpan = 24 * 1024;  // staged output bytes per write block

struct FmtCol {
  const void* data;
  const uint8_t* nulls;
  int32_t type;
  int32_t width;
};

struct FmtParams {
  FmtCol c[YQ_CSV_MAX_FIELDS];
  int32_t ncols;
  uint32_t rows;
  uint32_t* len;        // bytes of each row's line
  const uint32_t* end;  // inclusive scan of len: where each line ends
  uint8_t* out;
  int32_t out_aligned4;  // `out` is 4-byte aligned: the copy-out may use word stores
};

// One row's line, columns in lockstep across the warp (one cell type at a time).
template <class Out>
__device__ __forceinline__ void format_row(const FmtParams& P, uint32_t r, Out& o) {
  for (int c = 0; c < P.ncols; ++c) {
    if (c) o.put(',');
    const FmtCol& fc = P.c[c];
    put_cell(o, fc.data, fc.nulls, fc.type, fc.width, r);
  }
  o.put('\n');
}

__global__ void __launch_bounds__(256) k_csv_format_len(const __grid_constant__ FmtParams P) {
  const uint32_t r = blockIdx.x * 256 + threadIdx.x;
  if (r >= P.rows) return;
  CountOut o;
  format_row(P, r, o);
  P.len[r] = o.n;
}

// 128 lines a block, written into shared memory and copied out with 4-byte
// stores (the block's first and last partial words byte by byte: they share
// a word with the neighbouring blocks' lines).
__global__ void __launch_bounds__(kFmtThreads) k_csv_format_write(const __grid_constant__ FmtParams P) {
  extern __shared__ __align__(16) uint8_t s_out[];
  const uint32_t r0 = blockIdx.x * kFmtThreads;
  const uint32_t rend = r0 + kFmtThreads < P.rows ? r0 + kFmtThreads : P.rows;
  const uint32_t base = r0 ? P.end[r0 - 1] : 0u, stop = P.end[rend - 1];
  const uint32_t abase = base & ~3u;  // s_out[i] holds output byte abase + i
  const bool staged = stop - abase <= kFmtSpan;
  const uint32_t r = r0 + threadIdx.x;
  if (r < rend) {
    const uint32_t off = P.end[r] - P.len[r];
    BufOut o{staged ? s_out + (off - abase) : P.out + off};
    format_row(P, r, o);
  }
  if (!staged) return;
  __syncthreads();
  const uint32_t w0 = (base + 3) & ~3u, w1 = stop & ~3u;  // whole words inside [base, stop)
  if (w0 >= w1 || !P.out_aligned4) {
    for (uint32_t i = base + threadIdx.x; i < stop; i += kFmtThreads) P.out[i] = s_out[i - abase];
    return;
  }
  for (uint32_t i = base + threadIdx.x; i < w0; i += kFmtThreads) P.out[i] = s_out[i - abase];
  for (uint32_t i = w1 + threadIdx.x; i < stop; i += kFmtThreads) P.out[i] = s_out[i - abase];
  for (uint32_t i = w0 + 4 * threadIdx.x; i < w1; i += 4 * kFmtThreads)
    *reinterpret_cast<uint32_t*>(P.out + i) = *reinterpret_cast<const uint32_t*>(s_out + (i - abase));
}

int fmt_max_cell(int32_t type, int32_t width) {
  switch (type) {
    case YQ_INT32: return 11;
    case YQ_INT64: return 20;
    case YQ_FLOAT32: return 46;   // sign, 39 integer digits, '.', 4 decimals
    case YQ_DATETIME: return 29;  // quotes, signed 11-digit year, "-MM-DD HH:MM:SS"
    case YQ_TEXT: return width + 2;
    default: return -1;
  }
}

uint32_t csv_tiles(uint64_t nbytes) { return (uint32_t)((nbytes + kTileBytes - 1) / kTileBytes); }

int value_width(int32_t type) {
  switch (type) {
    case YQ_INT32:
    case YQ_FLOAT32: return 4;
    case YQ_DATETIME: return 8;
    default: return 0;
  }
}

}  // namespace

extern "C" {

size_t yq_csv_index_workspace_size(uint64_t nbytes) {
  const size_t nt = csv_tiles(nbytes) + 1;
  WsSize w;
  w.add<uint32_t>(nt);
  w.add<uint32_t>(nt * NSTATES);
  w.add<unsigned long long>(nt);
  w.add<unsigned long long>(2);
  return w.total();
}

int yq_csv_index(const uint8_t* data, uint64_t nbytes, uint32_t* record_starts, uint64_t capacity,
                 uint64_t* records, void* workspace, size_t workspace_bytes, void* stream) {
  if (!records || (nbytes && !data)) return YQ_ERR_INVALID_ARG;
  if (nbytes >= (1ull << 32)) return YQ_ERR_UNSUPPORTED;  // record offsets are 32-bit
  *records = 0;
  if (nbytes == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  const uint32_t nt = csv_tiles(nbytes);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_csv_index_workspace_size(nbytes), s));
  uint32_t* tile_map = ws.take<uint32_t>((size_t)nt + 1);
  uint32_t* tile_cnt = ws.take<uint32_t>(((size_t)nt + 1) * NSTATES);
  unsigned long long* tile_start = ws.take<unsigned long long>((size_t)nt + 1);
  unsigned long long* total = ws.take<unsigned long long>(2);
  const int aligned = (reinterpret_cast<uintptr_t>(data) & 15) == 0;
  {
    ProfScope ps("csv_tiles", s, (double)nbytes);
    k_csv_tiles<<<nt, kTileThreads, 0, s>>>(data, nbytes, aligned, tile_map, tile_cnt);
    YQ_CHECK_LAUNCH();
  }
  {
    ProfScope ps("csv_tile_scan", s, (double)nt * 32.0);
    k_csv_tile_scan<<<1, kScanThreads, 0, s>>>(tile_map, tile_cnt, nt, tile_start, total);
    YQ_CHECK_LAUNCH();
  }
  unsigned long long h = 0;
  YQ_TRY(d2h_sync(&h, total, sizeof(h), s));
  *records = h;
  if (h > capacity) return YQ_ERR_CAPACITY;
  if (!record_starts) return h ? YQ_ERR_INVALID_ARG : YQ_OK;
  {
    ProfScope ps("csv_emit", s, (double)nbytes + 4.0 * (double)h);
    k_csv_emit<<<nt, kTileThreads, 0, s>>>(data, nbytes, aligned, tile_start, record_starts);
    YQ_CHECK_LAUNCH();
  }
  return YQ_OK;
}

size_t yq_csv_parse_workspace_size(uint32_t records) {
  WsSize w;
  w.add<uint8_t>((size_t)records + 16);
  w.add<unsigned long long>(4);
  w.add<uint32_t>((size_t)records + 1);
  w.used += yq_prefix_sum_workspace_size(records);
  return w.total();
}

int yq_csv_parse(const uint8_t* data, uint64_t nbytes, const uint32_t* record_starts, uint32_t records,
                 const int32_t* field_column, int32_t nfields, yq_column* out, int32_t ncols, uint32_t* rows,
                 yq_csv_error* error, void* workspace, size_t workspace_bytes, void* stream) {
  if (!rows || !field_column || !out || nfields <= 0 || nfields > YQ_CSV_MAX_FIELDS || ncols < 0 ||
      (records && (!data || !record_starts)) || nbytes >= (1ull << 32))
    return YQ_ERR_INVALID_ARG;
  ParseParams P;
  P.data = data;
  P.nbytes = nbytes;
  P.starts = record_starts;
  P.nrec = records;
  P.nfields = nfields;
  P.aligned = (reinterpret_cast<uintptr_t>(data) & 15) == 0;
  uint8_t seen[YQ_MAX_BATCH_COLUMNS * 4] = {0};
  for (int f = 0; f < nfields; ++f) {
    const int c = field_column[f];
    P.f[f] = FieldDesc{nullptr, nullptr, 0, 0};
    if (c < 0) continue;
    if (c >= ncols || c >= (int)sizeof(seen) || seen[c]) return YQ_ERR_INVALID_ARG;
    seen[c] = 1;
    const yq_column& oc = out[c];
    if (records && (!oc.data || !oc.nulls)) return YQ_ERR_INVALID_ARG;  // nothing is written for 0 records
    if (oc.type == YQ_TEXT) {
      if (oc.width < 4 || oc.width > YQ_MAX_TEXT_WIDTH || oc.width % 4) return YQ_ERR_INVALID_ARG;
    } else if (value_width(oc.type) == 0 || oc.width != value_width(oc.type)) {
      return YQ_ERR_UNSUPPORTED;
    }
    P.f[f] = FieldDesc{oc.data, const_cast<uint8_t*>(oc.nulls), oc.type, oc.width};
  }
  for (int f = nfields; f < YQ_CSV_MAX_FIELDS; ++f) P.f[f] = FieldDesc{nullptr, nullptr, 0, 0};
  if (error) *error = yq_csv_error{0, 0, -1, 0};
  *rows = 0;
  if (records == 0) return YQ_OK;
  cudaStream_t s = as_stream(stream);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_csv_parse_workspace_size(records), s));
  P.valid = ws.take<uint8_t>((size_t)records + 16);
  P.counters = ws.take<unsigned long long>(4);
  uint32_t* pos = ws.take<uint32_t>((size_t)records + 1);
  void* scan_ws = ws.take<uint8_t>(yq_prefix_sum_workspace_size(records));
  const unsigned long long init[4] = {0, 0, ~0ull, 0};
  YQ_TRY(h2d_async(P.counters, init, sizeof(init), s));
  YQ_TRY(kernel_allow_smem((const void*)k_csv_parse, kSpanCap + 16));
  double out_bytes = 1.0;  // valid flag
  for (int f = 0; f < nfields; ++f)
    if (P.f[f].data) out_bytes += P.f[f].width + 1.0;
  {
    ProfScope ps("csv_parse", s, (double)nbytes + out_bytes * records);
    k_csv_parse<<<ceil_div<uint32_t>(records, kParseThreads), kParseThreads, kSpanCap + 16, s>>>(P);
    YQ_CHECK_LAUNCH();
  }
  unsigned long long h[3];
  YQ_TRY(d2h_sync(h, P.counters, sizeof(h), s));
  const unsigned long long invalid = h[0];
  if (invalid) {
    // rare path: drop the rows with a different field count, keeping order
    YQ_TRY(yq_prefix_sum_mask(P.valid, pos, records, scan_ws, yq_prefix_sum_workspace_size(records), stream));
    for (int f = 0; f < nfields; ++f) {
      const FieldDesc& fd = P.f[f];
      if (!fd.data) continue;
      const size_t bytes = (size_t)records * fd.width;
      void* tmp = nullptr;
      cudaError_t e = cudaMallocAsync(&tmp, bytes + records, s);
      if (e != cudaSuccess) { set_cuda_error(e); return YQ_ERR_ALLOC; }
      uint8_t* tmp_nulls = static_cast<uint8_t*>(tmp) + bytes;
      YQ_TRY_CUDA(cudaMemcpyAsync(tmp, fd.data, bytes, cudaMemcpyDeviceToDevice, s));
      YQ_TRY_CUDA(cudaMemcpyAsync(tmp_nulls, fd.nulls, records, cudaMemcpyDeviceToDevice, s));
      k_csv_compact<<<ceil_div<uint32_t>(records, 256) < 4096 ? ceil_div<uint32_t>(records, 256) : 4096, 256, 0,
                      s>>>(static_cast<const uint8_t*>(tmp), tmp_nulls, (uint32_t)fd.width, P.valid, pos, records,
                           static_cast<uint8_t*>(fd.data), fd.nulls);
      YQ_CHECK_LAUNCH();
      YQ_TRY_CUDA(cudaFreeAsync(tmp, s));
    }
  }
  *rows = (uint32_t)(records - invalid);
  if (h[1]) {
    if (error) {
      uint32_t first = (uint32_t)(h[2] >> 12);  // record index of the first bad cell
      if (invalid) {                           // -> its output row once dropped rows are gone
        uint32_t p = 0;
        YQ_TRY(d2h_sync(&p, pos + first, sizeof(p), s));
        first = p - 1;
      }
      *error = yq_csv_error{h[1], first, (int32_t)((h[2] >> 2) & 1023), (int32_t)(h[2] & 3)};
    }
    return YQ_ERR_INVALID_ARG;
  }
  return YQ_OK;
}

size_t yq_csv_format_workspace_size(uint32_t rows) {
  WsSize w;
  w.add<uint32_t>((size_t)rows + 1);
  w.add<uint32_t>((size_t)rows + 1);
  w.used += yq_prefix_sum_workspace_size(rows);
  return w.total();
}

int yq_csv_format(const yq_batch* batch, uint8_t* out, uint64_t capacity, uint64_t* bytes, void* workspace,
                  size_t workspace_bytes, void* stream) {
  if (!batch || !bytes || batch->ncols <= 0 || batch->ncols > YQ_CSV_MAX_FIELDS || !batch->columns)
    return YQ_ERR_INVALID_ARG;
  *bytes = 0;
  const uint32_t rows = batch->rows;
  FmtParams P;
  uint64_t max_line = 0;
  for (int c = 0; c < batch->ncols; ++c) {
    const yq_column& col = batch->columns[c];
    const int mc = fmt_max_cell(col.type, col.width);
    if (mc < 0) return YQ_ERR_UNSUPPORTED;
    if ((col.type == YQ_TEXT && (col.width < 1 || col.width > YQ_MAX_TEXT_WIDTH)) ||
        (col.type != YQ_TEXT && col.width != (col.type == YQ_INT32 || col.type == YQ_FLOAT32 ? 4 : 8)))
      return YQ_ERR_INVALID_ARG;
    if (rows && !col.data) return YQ_ERR_INVALID_ARG;
    P.c[c] = FmtCol{col.data, col.nulls, col.type, col.width};
    max_line += (uint64_t)mc + 1;
  }
  if (rows == 0) return YQ_OK;
  if ((uint64_t)rows * max_line >= (1ull << 32)) return YQ_ERR_UNSUPPORTED;  // 32-bit line offsets
  cudaStream_t s = as_stream(stream);
  Workspace ws;
  YQ_TRY(ws.acquire(workspace, workspace_bytes, yq_csv_format_workspace_size(rows), s));
  P.ncols = batch->ncols;
  P.rows = rows;
  P.len = ws.take<uint32_t>((size_t)rows + 1);
  uint32_t* end = ws.take<uint32_t>((size_t)rows + 1);
  void* scan_ws = ws.take<uint8_t>(yq_prefix_sum_workspace_size(rows));
  P.end = end;
  P.out = out;
  P.out_aligned4 = (reinterpret_cast<uintptr_t>(out) & 3) == 0;
  {
    ProfScope ps("csv_format_len", s, 0.0);
    k_csv_format_len<<<ceil_div<uint32_t>(rows, 256), 256, 0, s>>>(P);
    YQ_CHECK_LAUNCH();
  }
  YQ_TRY(yq_prefix_sum_u32(P.len, end, rows, scan_ws, yq_prefix_sum_workspace_size(rows), stream));
  uint32_t total = 0;
  YQ_TRY(d2h_sync(&total, end + rows - 1, sizeof(total), s));
  *bytes = total;
  if (total > capacity) return YQ_ERR_CAPACITY;
  if (!out) return YQ_ERR_INVALID_ARG;
  YQ_TRY(kernel_allow_smem((const void*)k_csv_format_write, kFmtSpan + 16));
  double in_bytes = 0;
  for (int c = 0; c < batch->ncols; ++c)
    in_bytes += (double)rows * (batch->columns[c].width + (batch->columns[c].nulls ? 1 : 0));
  {
    ProfScope ps("csv_format_write", s, in_bytes + (double)total);
    k_csv_format_write<<<ceil_div<uint32_t>(rows, kFmtThreads), kFmtThreads, kFmtSpan + 16, s>>>(P);
    YQ_CHECK_LAUNCH();
  }
  return YQ_OK;
}

}  // extern "C"
