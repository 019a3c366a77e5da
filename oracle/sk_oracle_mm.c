/*
 * sk_oracle_mm.c -- Matrix Market reading and writing, restated in plain C
 * for the CPU oracle.  TEST INFRASTRUCTURE ONLY: the product never links it.
 *
 * Follows, sequentially and line by line:
 *   parse_banner            sparkit/data/matrix_market.cpp:28-87
 *   read_matrix_market<T>   sparkit/data/matrix_market.hpp:45-115 (getline
 *                           per line, istream >> for every number, which is
 *                           strtoll / strtod / strtof on the token)
 *   Coordinate_matrix       Coordinate_matrix.hpp:36-41 (a map keyed by
 *                           (row, column): the last duplicate wins)
 *   to_compressed_row       conversions.hpp:45 (entries sorted by row, column)
 *   write_matrix_market     sparkit/data/matrix_market.hpp:119-150
 * The reference leaves malformed, missing or out-of-range entry lines
 * undefined; here they are errors, as in the library.
 */
#include <ctype.h>
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sk_oracle.h"

static int sko_mm_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

/* the next line of [*p, end) without its '\n' (getline) */
static int sko_mm_getline(const char** p, const char* end, const char** b, const char** e) {
  if (*p >= end) return 0;
  const char* q = memchr(*p, '\n', (size_t)(end - *p));
  *b = *p;
  *e = q ? q : end;
  *p = q ? q + 1 : end;
  return 1;
}

/* the i-th whitespace-separated word of [b, e), lower-cased, into w */
static void sko_mm_word(const char* b, const char* e, int i, char* w, size_t cap) {
  int k = -1;
  w[0] = 0;
  while (b < e) {
    while (b < e && sko_mm_space(*b)) ++b;
    const char* s = b;
    while (b < e && !sko_mm_space(*b)) ++b;
    if (b > s && ++k == i) {
      size_t n = (size_t)(b - s) < cap - 1 ? (size_t)(b - s) : cap - 1;
      for (size_t j = 0; j < n; ++j) w[j] = (char)tolower((unsigned char)s[j]);
      w[n] = 0;
      return;
    }
  }
}

/* istream >> long long on [*p, e): whitespace, then strtoll's number */
static int sko_mm_int(const char** p, const char* e, long long* v) {
  char buf[64];
  while (*p < e && sko_mm_space(**p)) ++*p;
  size_t n = 0;
  while (*p + n < e && !sko_mm_space((*p)[n]) && n < sizeof(buf) - 1) ++n;
  memcpy(buf, *p, n);
  buf[n] = 0;
  char* end = NULL;
  *v = strtoll(buf, &end, 10);
  if (end == buf) return 0;
  *p += (size_t)(end - buf);
  return 1;
}

/* istream >> double / float: strtod / strtof on the token; as libstdc++'s
 * num_get does, an overflow gives the largest finite value of that sign and
 * an underflow strtod's (or strtof's) zero or subnormal */
static int sko_mm_real(const char** p, const char* e, int f32, double* v) {
  char buf[128];
  while (*p < e && sko_mm_space(**p)) ++*p;
  size_t n = 0;
  while (*p + n < e && !sko_mm_space((*p)[n]) && n < sizeof(buf) - 1) ++n;
  memcpy(buf, *p, n);
  buf[n] = 0;
  char* end = NULL;
  if (f32)
    *v = (double)strtof(buf, &end);
  else
    *v = strtod(buf, &end);
  if (end == buf) return 0;
  if (isinf(*v)) *v = copysign(f32 ? (double)FLT_MAX : DBL_MAX, *v);
  *p += (size_t)(end - buf);
  return 1;
}

typedef struct {
  int64_t row, col, seq;
  double v;
} sko_mm_entry;

static int sko_mm_cmp(const void* a, const void* b) {
  const sko_mm_entry* x = (const sko_mm_entry*)a;
  const sko_mm_entry* y = (const sko_mm_entry*)b;
  if (x->row != y->row) return x->row < y->row ? -1 : 1;
  if (x->col != y->col) return x->col < y->col ? -1 : 1;
  return x->seq < y->seq ? -1 : (x->seq > y->seq);
}

static int sko_mm_fail(sko_mm_csr* out, const char* msg) {
  snprintf(out->err, sizeof(out->err), "%s", msg);
  return 1;
}

static int sko_mm_read(const char* text, int64_t len, int f32, sko_mm_csr* out) {
  memset(out, 0, sizeof(*out));
  const char* p = text;
  const char* end = text + len;
  const char *b, *e;
  if (!sko_mm_getline(&p, end, &b, &e)) return sko_mm_fail(out, "matrix market: unexpected end of input");
  char w[64];
  sko_mm_word(b, e, 0, w, sizeof(w));
  if (strcmp(w, "%%matrixmarket") != 0) return sko_mm_fail(out, "matrix market: invalid banner header");
  sko_mm_word(b, e, 2, w, sizeof(w));
  int array = 0;
  if (strcmp(w, "array") == 0)
    array = 1;
  else if (strcmp(w, "coordinate") != 0)
    return sko_mm_fail(out, "matrix market: unknown format");
  sko_mm_word(b, e, 3, w, sizeof(w));
  int pattern = 0, complex_ = 0;
  if (strcmp(w, "pattern") == 0)
    pattern = 1;
  else if (strcmp(w, "complex") == 0)
    complex_ = 1;
  else if (strcmp(w, "real") != 0 && strcmp(w, "integer") != 0)
    return sko_mm_fail(out, "matrix market: unknown field");
  sko_mm_word(b, e, 4, w, sizeof(w));
  int symmetric = 0;
  if (strcmp(w, "symmetric") == 0)
    symmetric = 1;
  else if (strcmp(w, "general") != 0 && strcmp(w, "skew-symmetric") != 0 && strcmp(w, "hermitian") != 0)
    return sko_mm_fail(out, "matrix market: unknown symmetry");
  if (array) return sko_mm_fail(out, "matrix market: only coordinate format is supported");
  if (complex_) return sko_mm_fail(out, "matrix market: complex field is not yet supported");
  int found = 0;
  while (sko_mm_getline(&p, end, &b, &e))
    if (e > b && *b != '%') {
      found = 1;
      break;
    }
  if (!found) return sko_mm_fail(out, "matrix market: missing size line");
  long long rows = 0, cols = 0, nnz = 0;
  {
    const char* q = b;
    if (sko_mm_int(&q, e, &rows) && sko_mm_int(&q, e, &cols)) sko_mm_int(&q, e, &nnz);
  }
  if (rows <= 1 || cols <= 1) return sko_mm_fail(out, "invalid matrix shape");
  if (nnz < 0) return sko_mm_fail(out, "matrix market: negative entry count");
  sko_mm_entry* ent = (sko_mm_entry*)malloc((size_t)(2 * nnz + 1) * sizeof(sko_mm_entry));
  int64_t m = 0;
  for (long long k = 0; k < nnz; ++k) {
    if (!sko_mm_getline(&p, end, &b, &e)) {
      free(ent);
      return sko_mm_fail(out, "matrix market: unexpected end of input");
    }
    const char* q = b;
    long long r = 0, c = 0;
    double v = 1.0;
    int ok = sko_mm_int(&q, e, &r) && sko_mm_int(&q, e, &c) && (pattern || sko_mm_real(&q, e, f32, &v));
    if (!ok || r < 1 || r > rows || c < 1 || c > cols) {
      free(ent);
      return sko_mm_fail(out, "matrix market: bad entry line");
    }
    ent[m] = (sko_mm_entry){r - 1, c - 1, m, v};
    ++m;
    if (symmetric && r != c) {
      ent[m] = (sko_mm_entry){c - 1, r - 1, m, v};
      ++m;
    }
  }
  qsort(ent, (size_t)m, sizeof(sko_mm_entry), sko_mm_cmp);
  out->nrow = rows;
  out->ncol = cols;
  out->row_ptr = (int64_t*)calloc((size_t)rows + 1, sizeof(int64_t));
  out->col_ind = (int64_t*)malloc((size_t)(m + 1) * sizeof(int64_t));
  out->values = malloc((size_t)(m + 1) * (f32 ? sizeof(float) : sizeof(double)));
  int64_t u = 0;
  for (int64_t i = 0; i < m; ++i) {
    if (i + 1 < m && ent[i + 1].row == ent[i].row && ent[i + 1].col == ent[i].col) continue; /* last wins */
    out->col_ind[u] = ent[i].col;
    if (f32)
      ((float*)out->values)[u] = (float)ent[i].v;
    else
      ((double*)out->values)[u] = ent[i].v;
    out->row_ptr[ent[i].row + 1] += 1;
    ++u;
  }
  for (long long r = 0; r < rows; ++r) out->row_ptr[r + 1] += out->row_ptr[r];
  out->nnz = u;
  free(ent);
  return 0;
}

int sko_mm_read_f64(const char* text, int64_t len, sko_mm_csr* out) { return sko_mm_read(text, len, 0, out); }
int sko_mm_read_f32(const char* text, int64_t len, sko_mm_csr* out) { return sko_mm_read(text, len, 1, out); }

void sko_mm_free(sko_mm_csr* m) {
  free(m->row_ptr);
  free(m->col_ind);
  free(m->values);
  m->row_ptr = NULL;
  m->col_ind = NULL;
  m->values = NULL;
}

/* write_matrix_market into a malloc'd string (sko_free) */
static char* sko_mm_write(int64_t nrow, int64_t ncol, const int64_t* rp, const int64_t* ci, const void* v, int f32,
                          int64_t* len) {
  size_t cap = 128 + (size_t)rp[nrow] * 64, n = 0;
  char* s = (char*)malloc(cap);
  n += (size_t)snprintf(s + n, cap - n, "%%%%MatrixMarket matrix coordinate real general\n%lld %lld %lld\n",
                        (long long)nrow, (long long)ncol, (long long)rp[nrow]);
  for (int64_t r = 0; r < nrow; ++r)
    for (int64_t j = rp[r]; j < rp[r + 1]; ++j) {
      double x = f32 ? (double)((const float*)v)[j] : ((const double*)v)[j];
      n += (size_t)snprintf(s + n, cap - n, "%lld %lld %g\n", (long long)(r + 1), (long long)(ci[j] + 1), x);
    }
  *len = (int64_t)n;
  return s;
}

char* sko_mm_write_f64(int64_t nrow, int64_t ncol, const int64_t* rp, const int64_t* ci, const double* v,
                       int64_t* len) {
  return sko_mm_write(nrow, ncol, rp, ci, v, 0, len);
}

char* sko_mm_write_f32(int64_t nrow, int64_t ncol, const int64_t* rp, const int64_t* ci, const float* v,
                       int64_t* len) {
  return sko_mm_write(nrow, ncol, rp, ci, v, 1, len);
}

void sko_free(void* p) { free(p); }
