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
