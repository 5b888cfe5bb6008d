/*
 * oracle.c — CPU restatement of YallaSQL's per-batch operators.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker and the timed CPU
 * baseline; the product (libyq_ops.so, libyq_engine.so) never links or calls
 * it. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load liboracle.so.
 *
 * Semantics follow the reference where it is well defined and DuckDB where
 * the two differ (the reference plans with DuckDB and is compared against it):
 *  - ORDER BY: stable; ties keep input order; DESC reverses the key order
 *    only (radix_sort_kernel.hpp:38-43 inverts digits, which keeps ties
 *    stable); floats order with -0.0 == +0.0 and NaN above +inf (DuckDB's
 *    sort-key encoding; the reference's float_to_uint32,
 *    radix_sort_utils.cu:20-27, orders -0.0 before +0.0); int64/dates order
 *    as signed values (the reference sorts them as uint64,
 *    order_operator.hpp:226-232); NULL keys last unless nulls_first.
 *  - merging sorted runs: ties take the earlier run (merge_batchs.cu:61), so a
 *    stable sort of runs followed by pairwise merges equals one stable sort.
 *  - nested-loop join: every (l, r) with all conditions true
 *    (comparison_operators_kernel.cu:6-22); the reference emits pairs in
 *    atomic order, this oracle in (l, r) order; compare as multisets.
 *  - aggregates: FP64 accumulation of float sums (reduction_kernel.cu:79-121
 *    accumulates SUM(float) in double), exact int64 integer sums.
 */
#define _GNU_SOURCE  /* strptime, timegm (the CSV scan restatement) */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { T_INT32 = 0, T_FLOAT32 = 1, T_DATETIME = 2, T_TEXT = 3, T_INT64 = 4, T_FLOAT64 = 5, T_BOOL = 6 };
enum { C_LT = 0, C_LE = 1, C_GT = 2, C_GE = 3, C_EQ = 4, C_NE = 5 };

/* ------------------------------------------------------------ sort keys */
/* Total order of one float: -0.0 == +0.0, every NaN equal and above +inf. */
static int cmp_f64(double a, double b) {
  int na = isnan(a), nb = isnan(b);
  if (na || nb) return na - nb;
  return (a > b) - (a < b);
}

typedef struct {
  int type, width, desc, nulls_first;
  const char* data;
  const uint8_t* nulls;
} key_t_;

static int cmp_rows(const key_t_* k, uint32_t x, uint32_t y) {
  int nx = k->nulls ? k->nulls[x] != 0 : 0;
  int ny = k->nulls ? k->nulls[y] != 0 : 0;
  if (nx || ny) {
    if (nx && ny) return 0;
    int r = nx ? 1 : -1; /* nulls last */
    return k->nulls_first ? -r : r;
  }
  int c;
  switch (k->type) {
    case T_INT32: {
      int32_t a = ((const int32_t*)k->data)[x], b = ((const int32_t*)k->data)[y];
      c = (a > b) - (a < b);
      break;
    }
    case T_INT64:
    case T_DATETIME: {
      int64_t a = ((const int64_t*)k->data)[x], b = ((const int64_t*)k->data)[y];
      c = (a > b) - (a < b);
      break;
    }
    case T_FLOAT32: c = cmp_f64(((const float*)k->data)[x], ((const float*)k->data)[y]); break;
    case T_FLOAT64: c = cmp_f64(((const double*)k->data)[x], ((const double*)k->data)[y]); break;
    case T_BOOL: c = (k->data[x] != 0) - (k->data[y] != 0); break;
    default: {
      /* fixed NUL-padded slot: unsigned bytes (strcmp_device, string_kernel.hpp:48-57) */
      c = memcmp(k->data + (size_t)x * k->width, k->data + (size_t)y * k->width, (size_t)k->width);
      c = (c > 0) - (c < 0);
    }
  }
  return k->desc ? -c : c;
}

/* Stable bottom-up merge sort of idx[0..n) by key (ties keep order). */
static void merge_sort(const key_t_* k, uint32_t* idx, uint32_t* tmp, uint32_t n) {
  const uint32_t run0 = 32;
  for (uint32_t s = 0; s < n; s += run0) { /* insertion sort small runs */
    uint32_t e = s + run0 < n ? s + run0 : n;
    for (uint32_t i = s + 1; i < e; ++i) {
      uint32_t v = idx[i], j = i;
      while (j > s && cmp_rows(k, idx[j - 1], v) > 0) { idx[j] = idx[j - 1]; --j; }
      idx[j] = v;
    }
  }
  uint32_t* a = idx;
  uint32_t* b = tmp;
  for (uint32_t w = run0; w < n; w *= 2) {
    for (uint32_t lo = 0; lo < n; lo += 2 * w) {
      uint32_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
      uint32_t i = lo, j = mid, o = lo;
      while (i < mid && j < hi) b[o++] = (cmp_rows(k, a[j], a[i]) < 0) ? a[j++] : a[i++];
      while (i < mid) b[o++] = a[i++];
      while (j < hi) b[o++] = a[j++];
    }
    uint32_t* t = a; a = b; b = t;
  }
  if (a != idx) memcpy(idx, a, (size_t)n * sizeof(uint32_t));
}

/* Stable merge of two sorted ranges (ties take the left range first). */
static void merge_two(const key_t_* k, const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, uint32_t* out) {
  uint32_t i = 0, j = 0, o = 0;
  while (i < na && j < nb) out[o++] = (cmp_rows(k, b[j], a[i]) < 0) ? b[j++] : a[i++];
  while (i < na) out[o++] = a[i++];
  while (j < nb) out[o++] = b[j++];
}

typedef struct {
  const key_t_* k;
  uint32_t *idx, *tmp;
  uint32_t n;
} sort_job;

static void* sort_worker(void* p) {
  sort_job* j = (sort_job*)p;
  merge_sort(j->k, j->idx, j->tmp, j->n);
  return NULL;
}

typedef struct {
  const key_t_* k;
  const uint32_t *a, *b;
  uint32_t na, nb;
  uint32_t* out;
} merge_job;

static void* merge_worker(void* p) {
  merge_job* j = (merge_job*)p;
  merge_two(j->k, j->a, j->na, j->b, j->nb, j->out);
  return NULL;
}

/* Sort idx[0..n) stably with up to `threads` threads: chunk sorts, then a
 * parallel tree of pairwise stable merges (left chunk first on ties). */
static int parallel_sort(const key_t_* k, uint32_t* idx, uint32_t n, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 64) threads = 64;
  if (n < 65536) threads = 1;
  uint32_t* tmp = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
  if (!tmp) return -1;
  uint32_t bounds[65];
  for (int t = 0; t <= threads; ++t) bounds[t] = (uint32_t)((uint64_t)n * t / threads);
  pthread_t th[64];
  sort_job sj[64];
  for (int t = 0; t < threads; ++t) {
    sj[t].k = k; sj[t].idx = idx + bounds[t]; sj[t].tmp = tmp + bounds[t]; sj[t].n = bounds[t + 1] - bounds[t];
    pthread_create(&th[t], NULL, sort_worker, &sj[t]);
  }
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  int runs = threads;
  uint32_t* src = idx;
  uint32_t* dst = tmp;
  while (runs > 1) {
    merge_job mj[64];
    int nm = 0, nr = 0;
    uint32_t nb[65];
    nb[0] = 0;
    for (int r = 0; r < runs; r += 2) {
      if (r + 1 < runs) {
        mj[nm].k = k; mj[nm].a = src + bounds[r]; mj[nm].na = bounds[r + 1] - bounds[r];
        mj[nm].b = src + bounds[r + 1]; mj[nm].nb = bounds[r + 2] - bounds[r + 1]; mj[nm].out = dst + bounds[r];
        pthread_create(&th[nm], NULL, merge_worker, &mj[nm]);
        ++nm;
        nb[++nr] = bounds[r + 2];
      } else {
        memcpy(dst + bounds[r], src + bounds[r], (size_t)(bounds[r + 1] - bounds[r]) * sizeof(uint32_t));
        nb[++nr] = bounds[r + 1];
      }
    }
    for (int m = 0; m < nm; ++m) pthread_join(th[m], NULL);
    for (int r = 0; r <= nr; ++r) bounds[r] = nb[r];
    runs = nr;
    uint32_t* t = src; src = dst; dst = t;
  }
  if (src != idx) memcpy(idx, src, (size_t)n * sizeof(uint32_t));
  free(tmp);
  return 0;
}

/* ORDER BY permutation of one key within each segment [seg[s], seg[s+1]);
 * `in_perm` (may be NULL) is the order produced by less significant keys:
 * the result is a stable re-sort of that order. out_perm holds row ids. */
int orc_sort_perm(int type, const void* data, const uint8_t* nulls, int width, uint32_t n, int desc, int nulls_first,
                  const uint32_t* seg, int nseg, const uint32_t* in_perm, uint32_t* out_perm, int threads) {
  key_t_ k = {type, width, desc, nulls_first, (const char*)data, nulls};
  for (uint32_t i = 0; i < n; ++i) out_perm[i] = in_perm ? in_perm[i] : i;
  if (!seg || nseg <= 1) return parallel_sort(&k, out_perm, n, threads);
  for (int s = 0; s < nseg; ++s) {
    uint32_t a = seg[s], b = seg[s + 1];
    if (b > a && parallel_sort(&k, out_perm + a, b - a, threads) != 0) return -1;
  }
  return 0;
}

/* --------------------------------------------------------------- joins */
typedef struct {
  const void* data;
  const uint8_t* nulls;
  int type, width;
} orc_col;

static int cmp_cells(const orc_col* a, uint32_t x, const orc_col* b, uint32_t y) {
  switch (a->type) {
    case T_INT32: {
      int32_t u = ((const int32_t*)a->data)[x], v = ((const int32_t*)b->data)[y];
      return (u > v) - (u < v);
    }
    case T_INT64:
    case T_DATETIME: {
      int64_t u = ((const int64_t*)a->data)[x], v = ((const int64_t*)b->data)[y];
      return (u > v) - (u < v);
    }
    case T_FLOAT32: {
      float u = ((const float*)a->data)[x], v = ((const float*)b->data)[y];
      return (u > v) - (u < v);
    }
    case T_FLOAT64: {
      double u = ((const double*)a->data)[x], v = ((const double*)b->data)[y];
      return (u > v) - (u < v);
    }
    default: {
      int w = a->width < b->width ? a->width : b->width;
      int c = memcmp((const char*)a->data + (size_t)x * a->width, (const char*)b->data + (size_t)y * b->width, w);
      if (c == 0 && a->width != b->width) {
        const unsigned char* p = (const unsigned char*)(a->width > b->width ? a->data : b->data);
        int wide = a->width > b->width ? a->width : b->width;
        uint32_t row = a->width > b->width ? x : y;
        for (int i = w; i < wide && !c; ++i) c = p[(size_t)row * wide + i] ? (a->width > b->width ? 1 : -1) : 0;
      }
      return (c > 0) - (c < 0);
    }
  }
}

static int cmp_holds(int c, int op) {
  switch (op) {
    case C_LT: return c < 0;
    case C_LE: return c <= 0;
    case C_GT: return c > 0;
    case C_GE: return c >= 0;
    case C_EQ: return c == 0;
    default: return c != 0;
  }
}

/* Inner join: pairs (l, r) with every condition lcol[cl] <op> rcol[cr] true and
 * no NULL operand, in (l, r) order. Returns the pair count (writes at most cap). */
uint64_t orc_join_pairs(const orc_col* lcols, const orc_col* rcols, const int* conds, int ncond, uint32_t L,
                        uint32_t R, uint32_t* out_l, uint32_t* out_r, uint64_t cap) {
  uint64_t cnt = 0;
  for (uint32_t l = 0; l < L; ++l) {
    for (uint32_t r = 0; r < R; ++r) {
      int ok = 1;
      for (int c = 0; c < ncond && ok; ++c) {
        const orc_col* a = &lcols[conds[3 * c]];
        const orc_col* b = &rcols[conds[3 * c + 1]];
        if ((a->nulls && a->nulls[l]) || (b->nulls && b->nulls[r])) ok = 0;
        else ok = cmp_holds(cmp_cells(a, l, b, r), conds[3 * c + 2]);
      }
      if (ok) {
        if (cnt < cap) { out_l[cnt] = l; out_r[cnt] = r; }
        ++cnt;
      }
    }
  }
  return cnt;
}

/* ------------------------------------------------- timed CPU baselines */
typedef struct {
  const float* price;
  const int32_t *qty, *disc;
  const uint8_t* cat;
  const uint8_t* excluded;
  int cat_width;
  uint32_t lo, hi;
  double sum;
  int64_t count;
  float mn, mx;
} sales_job;

static void* sales_worker(void* p) {
  sales_job* j = (sales_job*)p;
  double s = 0;
  int64_t c = 0;
  float mn = INFINITY, mx = -INFINITY;
  for (uint32_t i = j->lo; i < j->hi; ++i) {
    int32_t d = j->disc[i];
    if (d < 1 || d > 3 || j->qty[i] >= 25) continue;
    if (memcmp(j->cat + (size_t)i * j->cat_width, j->excluded, (size_t)j->cat_width) == 0) continue;
    float pr = j->price[i];
    s += (double)(pr * (float)d);
    ++c;
    if (pr < mn) mn = pr;
    if (pr > mx) mx = pr;
  }
  j->sum = s; j->count = c; j->mn = mn; j->mx = mx;
  return NULL;
}

/* SUM(price*discount), COUNT(*), MIN(price), MAX(price) WHERE discount BETWEEN 1
 * AND 3 AND qty < 25 AND category <> excluded — per-thread FP64 partials. */
void orc_sales_query(const float* price, const int32_t* qty, const int32_t* disc, const uint8_t* cat, int cat_width,
                     const uint8_t* excluded, uint32_t n, int threads, double* out_sum, int64_t* out_count,
                     float* out_min, float* out_max) {
  if (threads < 1) threads = 1;
  if (threads > 64) threads = 64;
  pthread_t th[64];
  sales_job js[64];
  for (int t = 0; t < threads; ++t) {
    sales_job* j = &js[t];
    j->price = price; j->qty = qty; j->disc = disc; j->cat = cat; j->excluded = excluded; j->cat_width = cat_width;
    j->lo = (uint32_t)((uint64_t)n * t / threads); j->hi = (uint32_t)((uint64_t)n * (t + 1) / threads);
    pthread_create(&th[t], NULL, sales_worker, j);
  }
  double s = 0; int64_t c = 0; float mn = INFINITY, mx = -INFINITY;
  for (int t = 0; t < threads; ++t) {
    pthread_join(th[t], NULL);
    s += js[t].sum; c += js[t].count;
    if (js[t].mn < mn) mn = js[t].mn;
    if (js[t].mx > mx) mx = js[t].mx;
  }
  *out_sum = s; *out_count = c; *out_min = mn; *out_max = mx;
}

typedef struct {
  const int32_t *datekey, *qty, *disc;
  const float* price;
  const uint8_t* dim_ok; /* per datekey: dimension row passes its filter */
  int32_t dim_n;
  uint32_t lo, hi;
  double sum;
  int64_t count;
} star_job;

static void* star_worker(void* p) {
  star_job* j = (star_job*)p;
  double s = 0;
  int64_t c = 0;
  for (uint32_t i = j->lo; i < j->hi; ++i) {
    int32_t d = j->disc[i];
    if (d < 1 || d > 3 || j->qty[i] >= 25) continue;
    int32_t k = j->datekey[i];
    if (k < 0 || k >= j->dim_n || !j->dim_ok[k]) continue;
    s += (double)(j->price[i] * (float)d);
    ++c;
  }
  j->sum = s; j->count = c;
  return NULL;
}

/* Star join + aggregate: SUM(extendedprice*discount) over fact JOIN date ON
 * datekey WHERE year = Y AND discount BETWEEN 1 AND 3 AND quantity < 25.
 * The date dimension is keyed 0..dim_n-1; dim_ok marks rows passing year = Y. */
void orc_star_query(const int32_t* datekey, const int32_t* qty, const int32_t* disc, const float* price, uint32_t n,
                    const uint8_t* dim_ok, int32_t dim_n, int threads, double* out_sum, int64_t* out_count) {
  if (threads < 1) threads = 1;
  if (threads > 64) threads = 64;
  pthread_t th[64];
  star_job js[64];
  for (int t = 0; t < threads; ++t) {
    star_job* j = &js[t];
    j->datekey = datekey; j->qty = qty; j->disc = disc; j->price = price; j->dim_ok = dim_ok; j->dim_n = dim_n;
    j->lo = (uint32_t)((uint64_t)n * t / threads); j->hi = (uint32_t)((uint64_t)n * (t + 1) / threads);
    pthread_create(&th[t], NULL, star_worker, j);
  }
  double s = 0; int64_t c = 0;
  for (int t = 0; t < threads; ++t) {
    pthread_join(th[t], NULL);
    s += js[t].sum; c += js[t].count;
  }
  *out_sum = s; *out_count = c;
}

/* Cross product with predicate x[l] < y[r]: writes (x, y) in (l, r) order and
 * returns the pair count (at most cap written). */
uint64_t orc_cross_lt(const int32_t* x, uint32_t nx, const int32_t* y, uint32_t ny, int32_t* out_x, int32_t* out_y,
                      uint64_t cap) {
  uint64_t c = 0;
  for (uint32_t l = 0; l < nx; ++l)
    for (uint32_t r = 0; r < ny; ++r)
      if (x[l] < y[r]) {
        if (c < cap) { out_x[c] = x[l]; out_y[c] = y[r]; }
        ++c;
      }
  return c;
}

/* Gather every column by a permutation (move_one_col, move_rows_kernel.cu:52-70). */
void orc_gather(const void* src, void* dst, int width, const uint32_t* perm, uint32_t n) {
  const char* s = (const char*)src;
  char* d = (char*)dst;
  for (uint32_t i = 0; i < n; ++i) memcpy(d + (size_t)i * width, s + (size_t)perm[i] * width, (size_t)width);
}

/* ------------------------------------------------------------------ CSV scan
 * Restates the reference's CSV path for the device CSV scan's parity tests:
 * csv-parser's default parse loop (vendor/csv-parser/csv.hpp:7063-7140 and
 * end_feed, :6985-7003) over the text after the header line, rows whose field
 * count differs from the header's dropped (VariableColumnPolicy::IGNORE_ROW,
 * csv.hpp CSVReader::read_row), then GetOperator::next's conversions
 * (src/engine/operators/get_operator.cpp:66-101): strtol + int range check
 * (std::stoi), strtof + ERANGE check (std::stof), strptime("%Y-%m-%d
 * %H:%M:%S") + timegm (include/enums/data_type_utils.hpp:24-44), and a
 * NUL-padded copy of at most width-1 bytes (string_kernel.hpp:16-31). */
#include <errno.h>
#include <limits.h>
#include <float.h>
#include <stdio.h>
#include <time.h>

typedef struct {
  const int* type;
  const int* width;
  void** data;
  unsigned char** nulls;
  int nfields;
  uint64_t capacity;
  uint64_t rows;
  uint64_t bad;
  int64_t bad_row;
  int bad_field, bad_kind;
  int overflow;
  int has_dq; /* the current field held an escaped "" */
  /* fields of the current row: contents back to back in buf */
  char* buf;
  size_t len, cap;
  size_t* fstart;
  int nf, fcap;
} csv_state;

static void csv_append(csv_state* S, char c) {
  if (S->len + 1 >= S->cap) {
    S->cap = S->cap ? 2 * S->cap : 4096;
    S->buf = (char*)realloc(S->buf, S->cap);
  }
  S->buf[S->len++] = c;
}

static void csv_push_field(csv_state* S, size_t* field_start) {
  if (S->has_dq) {
    /* csv-parser's un-escaping (csv.hpp:7775-7792): of the field's quotes,
     * keep the 1st, 3rd, ... and drop the others */
    size_t o = *field_start;
    int prev = 0;
    for (size_t i = *field_start; i < S->len; ++i) {
      if (S->buf[i] == '"') {
        if (prev) { prev = 0; continue; }
        prev = 1;
      }
      S->buf[o++] = S->buf[i];
    }
    S->len = o;
    S->has_dq = 0;
  }
  if (S->nf + 2 > S->fcap) {
    S->fcap = S->fcap ? 2 * S->fcap : 64;
    S->fstart = (size_t*)realloc(S->fstart, sizeof(size_t) * (S->fcap + 1));
  }
  S->fstart[S->nf++] = *field_start;
  csv_append(S, 0); /* each field NUL terminated in buf, like c_str() */
  *field_start = S->len;
}

static void csv_convert_row(csv_state* S) {
  const uint64_t r = S->rows;
  if (S->nf != S->nfields) return; /* IGNORE_ROW */
  if (r >= S->capacity) { S->overflow = 1; return; }
  for (int f = 0; f < S->nfields; ++f) {
    const int ty = S->type[f];
    if (ty < 0) continue;
    const char* v = S->buf + S->fstart[f];
    /* the field's std::string length: up to the next field (embedded NULs count) */
    size_t vlen = (f + 1 < S->nf ? S->fstart[f + 1] : S->len) - S->fstart[f] - 1;
    S->nulls[f][r] = vlen == 0;
    int kind = 0;
    if (ty == 0) {
      int32_t x = INT_MIN;
      if (vlen) {
        char* end;
        errno = 0;
        long l = strtol(v, &end, 10);
        if (end == v) { x = 0; kind = 1; }
        else if (errno == ERANGE || l < INT_MIN || l > INT_MAX) { x = 0; kind = 2; }
        else x = (int32_t)l;
      }
      ((int32_t*)S->data[f])[r] = x;
    } else if (ty == 1) {
      float x = FLT_MIN;
      if (vlen) {
        char* end;
        errno = 0;
        x = strtof(v, &end);
        if (end == v) { x = 0; kind = 1; }
        else if (errno == ERANGE) { x = 0; kind = 2; }
      }
      ((float*)S->data[f])[r] = x;
    } else if (ty == 2) {
      int64_t x = 0;
      if (vlen) {
        struct tm t;
        memset(&t, 0, sizeof t);
        if (strptime(v, "%Y-%m-%d %H:%M:%S", &t) != NULL) x = (int64_t)timegm(&t);
      }
      ((int64_t*)S->data[f])[r] = x;
    } else {
      const int w = S->width[f];
      char* slot = (char*)S->data[f] + r * (uint64_t)w;
      memset(slot, 0, w);
      for (int i = 0; i < w - 1 && v[i]; ++i) slot[i] = v[i];
    }
    if (kind) {
      if (S->bad == 0) { S->bad_row = (int64_t)r; S->bad_field = f; S->bad_kind = kind; }
      ++S->bad;
    }
  }
  ++S->rows;
}

static void csv_push_row(csv_state* S) {
  csv_convert_row(S);
  S->nf = 0;
  S->len = 0;
}

/* text: the CSV body (after the header line). Returns rows kept; -1 on overflow. */
int64_t orc_csv_scan(const char* text, uint64_t n, int nfields, const int* field_type, const int* field_width,
                     void** out_data, unsigned char** out_nulls, uint64_t capacity, uint64_t* bad_cells,
                     int64_t* first_bad_row, int* first_bad_field, int* first_bad_kind) {
  csv_state S;
  memset(&S, 0, sizeof S);
  S.type = field_type;
  S.width = field_width;
  S.data = out_data;
  S.nulls = out_nulls;
  S.nfields = nfields;
  S.capacity = capacity;
  S.bad_row = -1;
  S.bad_field = -1;
  size_t field_start = 0;
  int quoted = 0;
  uint64_t pos = 0;
  /* newlines at the start belong to the header line's newline run */
  while (pos < n && (text[pos] == '\r' || text[pos] == '\n')) ++pos;
  while (pos < n) {
    const char c = text[pos];
    if (!quoted) {
      if (c == ',') { csv_push_field(&S, &field_start); ++pos; }
      else if (c == '\r' || c == '\n') {
        ++pos;
        while (pos < n && (text[pos] == '\r' || text[pos] == '\n')) ++pos;
        csv_push_field(&S, &field_start);
        csv_push_row(&S);
        field_start = 0;
      } else if (c == '"' && S.len == field_start) { quoted = 1; ++pos; }  /* opens only an empty field */
      else { csv_append(&S, c); ++pos; }
    } else if (c == '"') {
      if (pos + 1 == n) { quoted = 0; ++pos; }                        /* closing quote at the end */
      else {
        const char d = text[pos + 1];
        if (d == ',' || d == '\r' || d == '\n') { quoted = 0; ++pos; } /* closes the field */
        else if (d == '"') { csv_append(&S, '"'); csv_append(&S, '"'); S.has_dq = 1; pos += 2; } /* "" */
        else { csv_append(&S, '"'); ++pos; }                           /* a lone quote stays */
      }
    } else { csv_append(&S, c); ++pos; }
  }
  /* end of data: the last field is pushed when it has bytes or the text ends
   * in a delimiter or a quote; the row when it has fields */
  if (S.len > field_start || (n && (text[n - 1] == ',' || text[n - 1] == '"'))) csv_push_field(&S, &field_start);
  if (S.nf) csv_push_row(&S);
  free(S.buf);
  free(S.fstart);
  *bad_cells = S.bad;
  *first_bad_row = S.bad_row;
  *first_bad_field = S.bad_field;
  *first_bad_kind = S.bad_kind;
  return S.overflow ? -1 : (int64_t)S.rows;
}

/* glibc conversions, one per string (strings back to back, offs[n+1]):
 * kind 0 std::stoi, 1 std::stof (out = float bits), 2 strptime + timegm.
 * status: 0 ok, 1 nothing converts, 2 out of range (where the std:: calls throw). */
void orc_convert_batch(int kind, const char* buf, const uint64_t* offs, uint64_t n, int64_t* out, int32_t* status) {
  char tmp[4096];
  for (uint64_t i = 0; i < n; ++i) {
    size_t len = offs[i + 1] - offs[i];
    if (len >= sizeof tmp) len = sizeof tmp - 1;
    memcpy(tmp, buf + offs[i], len);
    tmp[len] = 0;
    status[i] = 0;
    char* end;
    if (kind == 0) {
      errno = 0;
      long l = strtol(tmp, &end, 10);
      if (end == tmp) { status[i] = 1; out[i] = 0; }
      else if (errno == ERANGE || l < INT_MIN || l > INT_MAX) { status[i] = 2; out[i] = 0; }
      else out[i] = l;
    } else if (kind == 1) {
      errno = 0;
      float f = strtof(tmp, &end);
      uint32_t b;
      memcpy(&b, &f, 4);
      out[i] = b;
      if (end == tmp) status[i] = 1;
      else if (errno == ERANGE) status[i] = 2;
    } else {
      struct tm t;
      memset(&t, 0, sizeof t);
      out[i] = strptime(tmp, "%Y-%m-%d %H:%M:%S", &t) != NULL ? (int64_t)timegm(&t) : 0;
    }
  }
}

/* ---------------------------------------------------------------- CSV writer
 * Restates CsvWriter::batchToCsv's row loop (include/engine/operators/
 * csv_writer.hpp:42-76) without the header line: cells joined by ',', rows
 * ended by '\n'; NULL -> ""; STRING -> "value" (up to its NUL, no escaping);
 * INT -> decimal (std::to_chars); FLOAT -> std::to_chars(fixed, 4), which
 * formats like printf("%.4f") of the exact value; DATETIME -> "..." from
 * gmtime_r + strftime("%Y-%m-%d %H:%M:%S") into 26 bytes (data_type_utils.hpp:46-57).
 * type: 0 INT32, 1 FLOAT32, 2 DATETIME, 3 TEXT (slot `width`), 4 INT64.
 * Returns the bytes written, or the bytes needed when above `cap`. */
static size_t orc_cell(char* o, int type, const void* data, const unsigned char* nulls, int width, uint64_t r) {
  if (nulls && nulls[r]) { memcpy(o, "\"\"", 2); return 2; }
  if (type == 0) return (size_t)sprintf(o, "%d", ((const int32_t*)data)[r]);
  if (type == 4) return (size_t)sprintf(o, "%lld", (long long)((const int64_t*)data)[r]);
  if (type == 1) return (size_t)sprintf(o, "%.4f", (double)((const float*)data)[r]);
  if (type == 2) {
    time_t t = (time_t)((const int64_t*)data)[r];
    struct tm tm;
    char buf[26];
    size_t n = 0;
    o[n++] = '"';
    if (gmtime_r(&t, &tm)) {
      size_t k = strftime(buf, 26, "%Y-%m-%d %H:%M:%S", &tm);
      memcpy(o + n, buf, k);
      n += k;
    }
    o[n++] = '"';
    return n;
  }
  const char* s = (const char*)data + r * (uint64_t)width;
  size_t n = 0;
  o[n++] = '"';
  for (int i = 0; i < width && s[i]; ++i) o[n++] = s[i];
  o[n++] = '"';
  return n;
}

uint64_t orc_csv_format(int ncols, const int* types, const int* widths, const void** data,
                        const unsigned char** nulls, uint64_t rows, char* out, uint64_t cap) {
  char cell[512];
  uint64_t n = 0;
  for (uint64_t r = 0; r < rows; ++r) {
    for (int c = 0; c < ncols; ++c) {
      size_t k = orc_cell(cell, types[c], data[c], nulls ? nulls[c] : NULL, widths[c], r);
      if (c + 1 < ncols) cell[k++] = ',';
      else cell[k++] = '\n';
      if (n + k <= cap) memcpy(out + n, cell, k);
      n += k;
    }
  }
  return n;
}
