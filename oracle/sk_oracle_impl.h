/*
 * sk_oracle_impl.h -- body of the CPU oracle, instantiated once per value
 * type by sk_oracle.c (T = double with suffix _f64, T = float with suffix
 * _f32).  TEST INFRASTRUCTURE ONLY: the product never links this file.
 *
 * Every routine restates, in plain C, the sequential algorithm of the
 * sparkit reference (file:line cited per function) with the same operation
 * order, so that a build with -ffp-contract=off reproduces the reference's
 * rounding bit for bit.
 */
#ifndef SKO_T
#error "define SKO_T and SKO_SFX before including sk_oracle_impl.h"
#endif

#define SKO_CAT2(a, b) a##b
#define SKO_CAT(a, b) SKO_CAT2(a, b)
#define SKO_FN(name) SKO_CAT(name, SKO_SFX)

/* ------------------------------------------------------------------ */
/* SpMV kernels                                                        */
/* ------------------------------------------------------------------ */

/* CSR: y_i = sum_j vals[j] * x[col[j]], accumulated from 0 in storage
 * order.  Follows sparkit/data/sparse_blas.hpp:19-35. */
void SKO_FN(sko_csr_spmv_)(int64_t nrow, const int64_t* row_ptr,
                           const int64_t* col_ind, const SKO_T* vals,
                           const SKO_T* x, SKO_T* y) {
  for (int64_t i = 0; i < nrow; ++i) {
    SKO_T sum = 0;
    for (int64_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j)
      sum += vals[j] * x[col_ind[j]];
    y[i] = sum;
  }
}

/* ELLPACK, row-major nrow x width, stop at the first -1 sentinel.
 * Follows sparkit/data/spmv.hpp:119-140. */
void SKO_FN(sko_ell_spmv_)(int64_t nrow, int64_t width,
                           const int64_t* col_ind, const SKO_T* vals,
                           const SKO_T* x, SKO_T* y) {
  for (int64_t i = 0; i < nrow; ++i) y[i] = 0;
  if (width == 0) return;
  for (int64_t i = 0; i < nrow; ++i) {
    SKO_T sum = 0;
    int64_t base = i * width;
    for (int64_t k = 0; k < width; ++k) {
      int64_t col = col_ind[base + k];
      if (col == -1) break;
      sum += vals[base + k] * x[col];
    }
    y[i] = sum;
  }
}

/* Jagged diagonal: for each diagonal k, for i < width_k,
 * y[perm[i]] += vals * x[col].  Follows sparkit/data/spmv.hpp:182-200. */
void SKO_FN(sko_jad_spmv_)(int64_t nrow, int64_t njd, const int64_t* perm,
                           const int64_t* jdiag, const int64_t* col_ind,
                           const SKO_T* vals, const SKO_T* x, SKO_T* y) {
  for (int64_t i = 0; i < nrow; ++i) y[i] = 0;
  for (int64_t k = 0; k < njd; ++k) {
    int64_t width = jdiag[k + 1] - jdiag[k];
    for (int64_t i = 0; i < width; ++i) {
      int64_t idx = jdiag[k] + i;
      y[perm[i]] += vals[idx] * x[col_ind[idx]];
    }
  }
}

/* Block sparse row with dense row-major br x bc blocks.  The block-row
 * loop bound is nrow / br (truncating), as in the reference.
 * Follows sparkit/data/spmv.hpp:148-174. */
void SKO_FN(sko_bsr_spmv_)(int64_t nrow, int64_t br, int64_t bc,
                           const int64_t* row_ptr, const int64_t* col_ind,
                           const SKO_T* vals, const SKO_T* x, SKO_T* y) {
  for (int64_t i = 0; i < nrow; ++i) y[i] = 0;
  int64_t nbr = nrow / br;
  for (int64_t I = 0; I < nbr; ++I) {
    for (int64_t bj = row_ptr[I]; bj < row_ptr[I + 1]; ++bj) {
      int64_t J = col_ind[bj];
      int64_t base = bj * br * bc;
      for (int64_t r = 0; r < br; ++r) {
        SKO_T sum = 0;
        for (int64_t c = 0; c < bc; ++c)
          sum += vals[base + r * bc + c] * x[J * bc + c];
        y[I * br + r] += sum;
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* Operator / preconditioner dispatch                                  */
/* ------------------------------------------------------------------ */

static void SKO_FN(sko_apply_op_)(const sko_operator* op, const SKO_T* in,
                                  SKO_T* out) {
  const SKO_T* v = (const SKO_T*)op->vals;
  switch (op->format) {
    case SKO_CSR:
      SKO_FN(sko_csr_spmv_)(op->nrow, op->row_ptr, op->col_ind, v, in, out);
      break;
    case SKO_ELL:
      SKO_FN(sko_ell_spmv_)(op->nrow, op->width, op->col_ind, v, in, out);
      break;
    case SKO_JAD:
      SKO_FN(sko_jad_spmv_)(op->nrow, op->width, op->perm, op->row_ptr,
                            op->col_ind, v, in, out);
      break;
    case SKO_BSR:
      SKO_FN(sko_bsr_spmv_)(op->nrow, op->block_rows, op->block_cols,
                            op->row_ptr, op->col_ind, v, in, out);
      break;
  }
}

/* Diagonal by binary search per row; absent diagonal gives 0.
 * Follows sparkit/data/unary.hpp:20-39. */
void SKO_FN(sko_extract_diagonal_)(int64_t nrow, int64_t ncol,
                                   const int64_t* row_ptr,
                                   const int64_t* col_ind, const SKO_T* vals,
                                   SKO_T* d) {
  int64_t len = nrow < ncol ? nrow : ncol;
  for (int64_t i = 0; i < len; ++i) {
    int64_t lo = row_ptr[i], hi = row_ptr[i + 1];
    while (lo < hi) { /* lower_bound */
      int64_t mid = lo + (hi - lo) / 2;
      if (col_ind[mid] < i) lo = mid + 1; else hi = mid;
    }
    d[i] = (lo < row_ptr[i + 1] && col_ind[lo] == i) ? vals[lo] : (SKO_T)0;
  }
}

/* Jacobi set-up: inverse diagonal, error on an exact zero.
 * Follows sparkit/data/jacobi.hpp:27-35.  Returns 0, or -1 on a zero. */
int SKO_FN(sko_jacobi_)(int64_t nrow, int64_t ncol, const int64_t* row_ptr,
                        const int64_t* col_ind, const SKO_T* vals,
                        SKO_T* inv_d) {
  SKO_FN(sko_extract_diagonal_)(nrow, ncol, row_ptr, col_ind, vals, inv_d);
  int64_t len = nrow < ncol ? nrow : ncol;
  for (int64_t i = 0; i < len; ++i) {
    if (inv_d[i] == (SKO_T)0) return -1;
    inv_d[i] = (SKO_T)1 / inv_d[i];
  }
  return 0;
}

/* Chebyshev coefficients of 1/lambda on [lmin, lmax] from
 * N = max(d+1, 64) cosine-sampled nodes; c_0 halved.
 * Follows sparkit/data/chebyshev_preconditioner.hpp:46-84. */
void SKO_FN(sko_chebyshev_coeffs_)(SKO_T lmin, SKO_T lmax, int64_t degree,
                                   SKO_T* coeffs) {
  int64_t d = degree;
  int64_t N = d + 1 > 64 ? d + 1 : 64;
  SKO_T center = (lmax + lmin) / (SKO_T)2;
  SKO_T half_width = (lmax - lmin) / (SKO_T)2;
  const SKO_T pi = (SKO_T)SKO_PI;
  for (int64_t k = 0; k <= d; ++k) {
    SKO_T ck = 0;
    for (int64_t j = 0; j < N; ++j) {
      SKO_T tj = SKO_COS(pi * ((SKO_T)j + (SKO_T)0.5) / (SKO_T)N);
      SKO_T lj = center + half_width * tj;
      SKO_T fj = (SKO_T)1 / lj;
      SKO_T cos_k = SKO_COS(pi * (SKO_T)k * ((SKO_T)j + (SKO_T)0.5) / (SKO_T)N);
      ck += fj * cos_k;
    }
    coeffs[k] = (SKO_T)2 * ck / (SKO_T)N;
  }
  coeffs[0] *= (SKO_T)0.5;
}

/* Clenshaw evaluation of z = p(A) r with Abar = (2A - (lmax+lmin)I) /
 * (lmax-lmin).  `work` holds 3*n scratch values.
 * Follows sparkit/data/chebyshev_preconditioner.hpp:98-169. */
static void SKO_FN(sko_chebyshev_apply_op_)(const sko_operator* A,
                                            const SKO_T* coeffs, SKO_T lmin,
                                            SKO_T lmax, int64_t d,
                                            const SKO_T* r, SKO_T* z,
                                            SKO_T* work) {
  int64_t n = A->nrow;
  SKO_T sum = lmax + lmin;
  SKO_T diff = lmax - lmin;
  if (d == 0 || diff == (SKO_T)0) {
    for (int64_t i = 0; i < n; ++i) z[i] = coeffs[0] * r[i];
    return;
  }
  SKO_T* b_prev = work;
  SKO_T* b_curr = work + n;
  SKO_T* av = work + 2 * n;
  for (int64_t i = 0; i < n; ++i) b_prev[i] = 0;
  for (int64_t i = 0; i < n; ++i) b_curr[i] = coeffs[d] * r[i];
  for (int64_t k = d - 1; k >= 1; --k) {
    SKO_FN(sko_apply_op_)(A, b_curr, av);
    for (int64_t i = 0; i < n; ++i) {
      SKO_T abar = ((SKO_T)2 * av[i] - sum * b_curr[i]) / diff;
      SKO_T b_new = coeffs[k] * r[i] + (SKO_T)2 * abar - b_prev[i];
      b_prev[i] = b_curr[i];
      b_curr[i] = b_new;
    }
  }
  SKO_FN(sko_apply_op_)(A, b_curr, av);
  for (int64_t i = 0; i < n; ++i) {
    SKO_T abar = ((SKO_T)2 * av[i] - sum * b_curr[i]) / diff;
    z[i] = coeffs[0] * r[i] + abar - b_prev[i];
  }
}

void SKO_FN(sko_chebyshev_apply_)(const sko_operator* A, const SKO_T* coeffs,
                                  SKO_T lmin, SKO_T lmax, int64_t d,
                                  const SKO_T* r, SKO_T* z) {
  SKO_T* work = (SKO_T*)malloc(sizeof(SKO_T) * 3 * (size_t)(A->nrow + 1));
  SKO_FN(sko_chebyshev_apply_op_)(A, coeffs, lmin, lmax, d, r, z, work);
  free(work);
}

static void SKO_FN(sko_apply_prec_)(const sko_precond* M, const sko_operator* A,
                                    const SKO_T* in, SKO_T* out, int64_t n,
                                    SKO_T* work) {
  if (M == NULL || M->kind == SKO_PREC_IDENTITY) {
    memcpy(out, in, sizeof(SKO_T) * (size_t)n);
  } else if (M->kind == SKO_PREC_JACOBI) {
    /* sparkit/data/jacobi.hpp:44-51 */
    const SKO_T* inv_d = (const SKO_T*)M->inv_diag;
    for (int64_t i = 0; i < n; ++i) out[i] = inv_d[i] * in[i];
  } else {
    const sko_operator* Ap = M->op ? M->op : A;
    SKO_FN(sko_chebyshev_apply_op_)(Ap, (const SKO_T*)M->coeffs,
                                    (SKO_T)M->lambda_min, (SKO_T)M->lambda_max,
                                    M->degree, in, out, work);
  }
}

/* std::inner_product(a, a+n, b, T{0}): sequential, as every solver of the
 * reference sums its dot products.  With sko_set_dot_order(1) the sum is
 * instead taken in 256-element sequential chunks whose partial sums are then
 * added in order -- a different association of the same products, used only
 * to measure how sensitive a solver's iteration count is to the summation
 * order (the GPU sums in a fixed tree by default).  Order 2 sums from the
 * last element down; order 3 sums the rounded products accurately
 * (double-double) and rounds once. */
static SKO_T SKO_FN(sko_dot_)(const SKO_T* a, const SKO_T* b, int64_t n) {
  if (sko_dot_order == 3) {
    /* the same rounded products summed in double-double (two-sum of each
     * addition, Knuth; accurate to about 2^-104 of the sum's magnitude) and
     * rounded once: the accurately summed dot product */
    double hi = 0.0, lo = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const double p = (double)(a[i] * b[i]);
      const double s = hi + p;
      const double bp = s - hi;
      lo += (hi - (s - bp)) + (p - bp);
      hi = s;
    }
    return (SKO_T)(hi + lo);
  }
  if (sko_dot_order == 2) {
    SKO_T s = 0;
    for (int64_t i = n; i > 0; --i) s += a[i - 1] * b[i - 1];
    return s;
  }
  if (sko_dot_order == 1) {
    SKO_T total = 0;
    for (int64_t c = 0; c < n; c += 256) {
      SKO_T part = 0;
      int64_t e = c + 256 < n ? c + 256 : n;
      for (int64_t i = c; i < e; ++i) part += a[i] * b[i];
      total += part;
    }
    return total;
  }
  SKO_T s = 0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* ------------------------------------------------------------------ */
/* Conjugate gradient (dual preconditioned)                            */
/* Follows sparkit/data/conjugate_gradient.hpp:122-312.                */
/* ------------------------------------------------------------------ */
void SKO_FN(sko_cg_)(const sko_operator* A, const sko_precond* left,
                     const sko_precond* right, const SKO_T* b, SKO_T* x,
                     const sko_cg_config* cfg, sko_summary* out,
                     double* history) {
  int64_t n = A->nrow;
  size_t bytes = sizeof(SKO_T) * (size_t)(n + 1);
  SKO_T* ax = (SKO_T*)calloc(1, bytes);
  SKO_T* r = (SKO_T*)calloc(1, bytes);
  SKO_T* z = (SKO_T*)calloc(1, bytes);
  SKO_T* hatp = (SKO_T*)calloc(1, bytes);
  SKO_T* p = (SKO_T*)calloc(1, bytes);
  SKO_T* q = (SKO_T*)calloc(1, bytes);
  SKO_T* work = (SKO_T*)calloc(3, bytes);
  out->residual_norm = 0;
  out->computed_iterations = 0;
  out->converged = 0;
  out->status = 0;
  SKO_T rz = 0;
  SKO_T bnorm = SKO_SQRT(SKO_FN(sko_dot_)(b, b, n)); /* :194 */
  if (bnorm == (SKO_T)0) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    out->converged = 1;
    goto done;
  }
  for (int64_t k = 0; k < cfg->max_iterations; ++k) { /* :200-205 */
    if (k % cfg->restart_iterations == 0) {            /* :210, :217-230 */
      SKO_FN(sko_apply_op_)(A, x, ax);
      for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
      SKO_FN(sko_apply_prec_)(left, A, r, z, n, work);
      rz = SKO_FN(sko_dot_)(r, z, n);
      memcpy(p, z, sizeof(SKO_T) * (size_t)n);
    }
    SKO_FN(sko_apply_prec_)(right, A, p, hatp, n, work); /* :233-239 */
    SKO_FN(sko_apply_op_)(A, hatp, q);
    SKO_T pq = SKO_FN(sko_dot_)(p, q, n);
    SKO_T alpha = rz / pq;
    for (int64_t i = 0; i < n; ++i) x[i] = alpha * hatp[i] + x[i]; /* :242 */
    for (int64_t i = 0; i < n; ++i) r[i] = r[i] - alpha * q[i];    /* :252 */
    out->computed_iterations += 1;
    SKO_T rn = SKO_SQRT(SKO_FN(sko_dot_)(r, r, n)); /* :261-276 */
    out->residual_norm = (double)rn;
    out->converged = (rn / bnorm < (SKO_T)cfg->tolerance);
    if (history && cfg->collect_residuals) history[k] = (double)rn;
    if (out->converged) break;
    SKO_FN(sko_apply_prec_)(left, A, r, z, n, work); /* :279-292 */
    SKO_T rz_new = SKO_FN(sko_dot_)(r, z, n);
    SKO_T beta = rz_new / rz;
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rz = rz_new;
  }
done:
  free(ax); free(r); free(z); free(hatp); free(p); free(q); free(work);
}

/* ------------------------------------------------------------------ */
/* BiCGSTAB with left and right preconditioning                        */
/* Follows sparkit/data/bicgstab.hpp:93-361.  One divergence: a zero   */
/* rho (bicgstab.hpp:204) returns without consuming budget and loops   */
/* forever in the reference; here it ends the solve with status        */
/* SKO_BREAKDOWN so that a test can never hang.                        */
/* ------------------------------------------------------------------ */
void SKO_FN(sko_bicgstab_)(const sko_operator* A, const sko_precond* left,
                           const sko_precond* right, const SKO_T* b, SKO_T* x,
                           const sko_krylov_config* cfg, sko_summary* out,
                           double* history) {
  int64_t n = A->nrow;
  size_t bytes = sizeof(SKO_T) * (size_t)(n + 1);
  SKO_T* r = (SKO_T*)calloc(1, bytes);
  SKO_T* r_hat = (SKO_T*)calloc(1, bytes);
  SKO_T* p = (SKO_T*)calloc(1, bytes);
  SKO_T* v = (SKO_T*)calloc(1, bytes);
  SKO_T* s = (SKO_T*)calloc(1, bytes);
  SKO_T* t = (SKO_T*)calloc(1, bytes);
  SKO_T* p_hat = (SKO_T*)calloc(1, bytes);
  SKO_T* s_hat = (SKO_T*)calloc(1, bytes);
  SKO_T* tmp = (SKO_T*)calloc(1, bytes);
  SKO_T* work = (SKO_T*)calloc(3, bytes);
  int64_t nhist = 0;
  out->residual_norm = 0;
  out->computed_iterations = 0;
  out->converged = 0;
  out->status = 0;
  SKO_T bnorm = SKO_SQRT(SKO_FN(sko_dot_)(b, b, n)); /* :160 */
  if (bnorm == (SKO_T)0) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    out->converged = 1;
    goto done;
  }
  SKO_FN(sko_apply_op_)(A, x, tmp); /* :186-194 */
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
  memcpy(r_hat, r, sizeof(SKO_T) * (size_t)n);
  SKO_T rho = 1, alpha = 1, omega = 1;
  while (out->computed_iterations < cfg->max_iterations && !out->converged) {
    SKO_T rho_new = SKO_FN(sko_dot_)(r_hat, r, n); /* :203 */
    if (rho_new == (SKO_T)0) { out->status = SKO_BREAKDOWN; break; }
    SKO_T beta = (rho_new / rho) * (alpha / omega);
    for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    SKO_FN(sko_apply_prec_)(left, A, p, tmp, n, work);
    SKO_FN(sko_apply_prec_)(right, A, tmp, p_hat, n, work);
    SKO_FN(sko_apply_op_)(A, p_hat, v);
    out->computed_iterations += 1;
    alpha = rho_new / SKO_FN(sko_dot_)(r_hat, v, n);
    for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
    SKO_T s_norm = SKO_SQRT(SKO_FN(sko_dot_)(s, s, n)); /* :261-268 */
    out->residual_norm = (double)s_norm;
    if (history && cfg->collect_residuals) history[nhist++] = (double)s_norm;
    if (s_norm / bnorm < (SKO_T)cfg->tolerance) {
      for (int64_t i = 0; i < n; ++i) x[i] += alpha * p_hat[i];
      out->converged = 1;
      break;
    }
    SKO_FN(sko_apply_prec_)(left, A, s, tmp, n, work);
    SKO_FN(sko_apply_prec_)(right, A, tmp, s_hat, n, work);
    SKO_FN(sko_apply_op_)(A, s_hat, t);
    out->computed_iterations += 1;
    SKO_T tt = SKO_FN(sko_dot_)(t, t, n); /* :293-297 */
    omega = (tt == (SKO_T)0) ? (SKO_T)0 : SKO_FN(sko_dot_)(t, s, n) / tt;
    if (omega == (SKO_T)0) continue; /* :223 */
    for (int64_t i = 0; i < n; ++i)
      x[i] += alpha * p_hat[i] + omega * s_hat[i];
    for (int64_t i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
    rho = rho_new;
    SKO_T r_norm = SKO_SQRT(SKO_FN(sko_dot_)(r, r, n)); /* :316-324 */
    out->residual_norm = (double)r_norm;
    if (history && cfg->collect_residuals) history[nhist++] = (double)r_norm;
    if (r_norm / bnorm < (SKO_T)cfg->tolerance) out->converged = 1;
  }
done:
  out->history_length = nhist;
  free(r); free(r_hat); free(p); free(v); free(s); free(t);
  free(p_hat); free(s_hat); free(tmp); free(work);
}

/* ------------------------------------------------------------------ */
/* Flexible GMRES(m), modified Gram-Schmidt, Givens rotations          */
/* Follows sparkit/data/fgmres.hpp:96-428.  One divergence: a zero     */
/* initial residual norm (fgmres.hpp:217-218 divides by it) is treated */
/* as convergence of the current iterate.                              */
/* ------------------------------------------------------------------ */
void SKO_FN(sko_fgmres_)(const sko_operator* A, const sko_precond* M,
                         const SKO_T* b, SKO_T* x,
                         const sko_fgmres_config* cfg, sko_summary* out,
                         double* history) {
  int64_t n = A->nrow;
  int64_t m = cfg->restart_dimension;
  size_t vb = sizeof(SKO_T) * (size_t)(n + 1);
  SKO_T* V = (SKO_T*)calloc((size_t)(m + 1), vb);
  SKO_T* Z = (SKO_T*)calloc((size_t)(m > 0 ? m : 1), vb);
  SKO_T* H = (SKO_T*)calloc((size_t)((m + 1) * m + 1), sizeof(SKO_T));
  SKO_T* cs = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  SKO_T* sn = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  SKO_T* g = (SKO_T*)calloc((size_t)(m + 2), sizeof(SKO_T));
  SKO_T* y = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  SKO_T* w = (SKO_T*)calloc(1, vb);
  SKO_T* work = (SKO_T*)calloc(3, vb);
  int64_t nhist = 0;
  int64_t um1 = m + 1;
  out->residual_norm = 0;
  out->computed_iterations = 0;
  out->converged = 0;
  out->status = 0;
  SKO_T bnorm = SKO_SQRT(SKO_FN(sko_dot_)(b, b, n)); /* :168 */
  if (bnorm == (SKO_T)0) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    out->converged = 1;
    goto done;
  }
  while (out->computed_iterations < cfg->max_iterations && !out->converged) {
    /* compute_initial_residual :207-224 */
    SKO_FN(sko_apply_op_)(A, x, w);
    for (int64_t i = 0; i < n; ++i) V[i] = b[i] - w[i];
    SKO_T beta = SKO_SQRT(SKO_FN(sko_dot_)(V, V, n));
    if (beta == (SKO_T)0) {
      out->residual_norm = 0;
      out->converged = 1;
      break;
    }
    {
      SKO_T f = (SKO_T)1 / beta;
      for (int64_t i = 0; i < n; ++i) V[i] *= f;
    }
    for (int64_t i = 0; i <= m; ++i) g[i] = 0;
    g[0] = beta;
    memset(Z, 0, vb * (size_t)m);
    memset(H, 0, sizeof(SKO_T) * (size_t)((m + 1) * m)); /* :227-231 */
    memset(cs, 0, sizeof(SKO_T) * (size_t)m);
    memset(sn, 0, sizeof(SKO_T) * (size_t)m);
    int64_t left = cfg->max_iterations - out->computed_iterations;
    int64_t m_eff = m < left ? m : left; /* :241-244 */
    int64_t j_final = 0;
    for (int64_t j = 0; j < m_eff; ++j) {
      SKO_T* Vj = V + j * (n + 1);
      SKO_T* Vj1 = V + (j + 1) * (n + 1);
      SKO_T* Zj = Z + j * (n + 1);
      /* arnoldi_step :247-256 */
      SKO_FN(sko_apply_prec_)(M, A, Vj, Zj, n, work);
      SKO_FN(sko_apply_op_)(A, Zj, w);
      memcpy(Vj1, w, sizeof(SKO_T) * (size_t)n);
      for (int64_t i = 0; i <= j; ++i) { /* orthogonalize :259-273 */
        SKO_T* Vi = V + i * (n + 1);
        SKO_T h = SKO_FN(sko_dot_)(Vi, Vj1, n);
        H[i + j * um1] = h;
        for (int64_t k = 0; k < n; ++k) Vj1[k] -= h * Vi[k];
      }
      SKO_T hn = SKO_SQRT(SKO_FN(sko_dot_)(Vj1, Vj1, n)); /* :276-284 */
      H[j + 1 + j * um1] = hn;
      if (hn > (SKO_T)0) {
        SKO_T f = (SKO_T)1 / hn;
        for (int64_t k = 0; k < n; ++k) Vj1[k] *= f;
      }
      /* apply_givens_rotations :287-337 */
      for (int64_t i = 0; i < j; ++i) {
        SKO_T temp = cs[i] * H[i + j * um1] + sn[i] * H[i + 1 + j * um1];
        H[i + 1 + j * um1] = -sn[i] * H[i + j * um1] + cs[i] * H[i + 1 + j * um1];
        H[i + j * um1] = temp;
      }
      {
        SKO_T a = H[j + j * um1];
        SKO_T bb = H[j + 1 + j * um1];
        if (bb == (SKO_T)0) { cs[j] = 1; sn[j] = 0; }
        else if (a == (SKO_T)0) { cs[j] = 0; sn[j] = 1; }
        else {
          SKO_T rr = SKO_SQRT(a * a + bb * bb);
          cs[j] = a / rr;
          sn[j] = bb / rr;
        }
      }
      H[j + j * um1] = cs[j] * H[j + j * um1] + sn[j] * H[j + 1 + j * um1];
      H[j + 1 + j * um1] = 0;
      {
        SKO_T temp = cs[j] * g[j] + sn[j] * g[j + 1];
        g[j + 1] = -sn[j] * g[j] + cs[j] * g[j + 1];
        g[j] = temp;
      }
      out->computed_iterations += 1;
      j_final = j;
      SKO_T absres = SKO_FABS(g[j + 1]); /* :340-356 */
      out->residual_norm = (double)absres;
      if (history && cfg->collect_residuals) history[nhist++] = (double)absres;
      if (absres / bnorm < (SKO_T)cfg->tolerance) {
        out->converged = 1;
        break;
      }
    }
    /* form_solution :359-394 */
    int64_t nj = j_final + 1;
    for (int64_t ii = nj; ii > 0; --ii) {
      int64_t i = ii - 1;
      y[i] = g[i];
      for (int64_t k = i + 1; k < nj; ++k) y[i] -= H[i + k * um1] * y[k];
      y[i] /= H[i + i * um1];
    }
    for (int64_t i = 0; i < n; ++i) {
      SKO_T sum = 0;
      for (int64_t k = 0; k < nj; ++k) sum += Z[k * (n + 1) + i] * y[k];
      x[i] += sum;
    }
  }
done:
  out->history_length = nhist;
  free(V); free(Z); free(H); free(cs); free(sn); free(g); free(y);
  free(w); free(work);
}

/* ------------------------------------------------------------------ */
/* Restarted GMRES(m) with left and right preconditioning              */
/* Follows sparkit/data/gmres.hpp:106-396: M_L on the initial residual  */
/* and on A z_j, M_R on v_j (z_j kept for the update), normalisation by */
/* division (:230, :278), convergence on |g_{j+1}| / ||b|| (:202).      */
/* One divergence, as for FGMRES: a zero initial residual norm (the     */
/* reference divides by it) is treated as convergence.                  */
/* ------------------------------------------------------------------ */
void SKO_FN(sko_gmres_)(const sko_operator* A, const sko_precond* ML,
                        const sko_precond* MR, const SKO_T* b, SKO_T* x,
                        const sko_fgmres_config* cfg, sko_summary* out,
                        double* history) {
  int64_t n = A->nrow;
  int64_t m = cfg->restart_dimension;
  size_t vb = sizeof(SKO_T) * (size_t)(n + 1);
  SKO_T* V = (SKO_T*)calloc((size_t)(m + 1), vb);
  SKO_T* Z = (SKO_T*)calloc((size_t)(m > 0 ? m : 1), vb);
  SKO_T* H = (SKO_T*)calloc((size_t)((m + 1) * m + 1), sizeof(SKO_T));
  SKO_T* cs = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  SKO_T* sn = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  SKO_T* g = (SKO_T*)calloc((size_t)(m + 2), sizeof(SKO_T));
  SKO_T* y = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  SKO_T* w = (SKO_T*)calloc(1, vb);
  SKO_T* r0 = (SKO_T*)calloc(1, vb);
  SKO_T* work = (SKO_T*)calloc(3, vb);
  int64_t nhist = 0;
  int64_t um1 = m + 1;
  out->residual_norm = 0;
  out->computed_iterations = 0;
  out->converged = 0;
  out->status = 0;
  SKO_T bnorm = SKO_SQRT(SKO_FN(sko_dot_)(b, b, n)); /* :165 */
  if (bnorm == (SKO_T)0) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    out->converged = 1;
    goto done;
  }
  while (out->computed_iterations < cfg->max_iterations && !out->converged) {
    /* compute_initial_residual :212-241 */
    SKO_FN(sko_apply_op_)(A, x, w);
    for (int64_t i = 0; i < n; ++i) r0[i] = b[i] - w[i];
    SKO_FN(sko_apply_prec_)(ML, A, r0, V, n, work);
    SKO_T beta = SKO_SQRT(SKO_FN(sko_dot_)(V, V, n));
    if (beta == (SKO_T)0) {
      out->residual_norm = 0;
      out->converged = 1;
      break;
    }
    for (int64_t i = 0; i < n; ++i) V[i] /= beta;
    for (int64_t i = 0; i <= m; ++i) g[i] = 0;
    g[0] = beta;
    memset(Z, 0, vb * (size_t)m);
    memset(H, 0, sizeof(SKO_T) * (size_t)((m + 1) * m)); /* :182-184 */
    memset(cs, 0, sizeof(SKO_T) * (size_t)m);
    memset(sn, 0, sizeof(SKO_T) * (size_t)m);
    int64_t left = cfg->max_iterations - out->computed_iterations;
    int64_t m_eff = m < left ? m : left; /* :186-187 */
    int64_t j_final = 0;
    for (int64_t j = 0; j < m_eff; ++j) {
      SKO_T* Vj = V + j * (n + 1);
      SKO_T* Vj1 = V + (j + 1) * (n + 1);
      SKO_T* Zj = Z + j * (n + 1);
      /* arnoldi_step :244-281 */
      SKO_FN(sko_apply_prec_)(MR, A, Vj, Zj, n, work);
      SKO_FN(sko_apply_op_)(A, Zj, w);
      SKO_FN(sko_apply_prec_)(ML, A, w, Vj1, n, work);
      for (int64_t i = 0; i <= j; ++i) {
        SKO_T* Vi = V + i * (n + 1);
        SKO_T h = SKO_FN(sko_dot_)(Vi, Vj1, n);
        H[i + j * um1] = h;
        for (int64_t k = 0; k < n; ++k) Vj1[k] -= h * Vi[k];
      }
      SKO_T hn = SKO_SQRT(SKO_FN(sko_dot_)(Vj1, Vj1, n));
      H[j + 1 + j * um1] = hn;
      if (hn > (SKO_T)0)
        for (int64_t k = 0; k < n; ++k) Vj1[k] /= hn;
      /* apply_givens_rotations :284-310, generate_givens :312-326 */
      for (int64_t i = 0; i < j; ++i) {
        SKO_T temp = cs[i] * H[i + j * um1] + sn[i] * H[i + 1 + j * um1];
        H[i + 1 + j * um1] = -sn[i] * H[i + j * um1] + cs[i] * H[i + 1 + j * um1];
        H[i + j * um1] = temp;
      }
      {
        SKO_T a = H[j + j * um1];
        SKO_T bb = H[j + 1 + j * um1];
        if (bb == (SKO_T)0) { cs[j] = 1; sn[j] = 0; }
        else if (a == (SKO_T)0) { cs[j] = 0; sn[j] = 1; }
        else {
          SKO_T rr = SKO_SQRT(a * a + bb * bb);
          cs[j] = a / rr;
          sn[j] = bb / rr;
        }
      }
      H[j + j * um1] = cs[j] * H[j + j * um1] + sn[j] * H[j + 1 + j * um1];
      H[j + 1 + j * um1] = 0;
      {
        SKO_T temp = cs[j] * g[j] + sn[j] * g[j + 1];
        g[j + 1] = -sn[j] * g[j] + cs[j] * g[j + 1];
        g[j] = temp;
      }
      out->computed_iterations += 1;
      j_final = j;
      SKO_T absres = SKO_FABS(g[j + 1]); /* :195-205 */
      out->residual_norm = (double)absres;
      if (history && cfg->collect_residuals) history[nhist++] = (double)absres;
      if (absres / bnorm < (SKO_T)cfg->tolerance) {
        out->converged = 1;
        break;
      }
    }
    /* form_solution :329-355 */
    int64_t nj = j_final + 1;
    for (int64_t ii = nj; ii > 0; --ii) {
      int64_t i = ii - 1;
      y[i] = g[i];
      for (int64_t k = i + 1; k < nj; ++k) y[i] -= H[i + k * um1] * y[k];
      y[i] /= H[i + i * um1];
    }
    for (int64_t i = 0; i < n; ++i) {
      SKO_T sum = 0;
      for (int64_t k = 0; k < nj; ++k) sum += Z[k * (n + 1) + i] * y[k];
      x[i] += sum;
    }
  }
done:
  out->history_length = nhist;
  free(V); free(Z); free(H); free(cs); free(sn); free(g); free(y);
  free(w); free(r0); free(work);
}

/* ------------------------------------------------------------------ */
/* Conjugate gradient squared with left and right preconditioning      */
/* Follows sparkit/data/cgs.hpp:106-395 step for step (two matrix-     */
/* vector products per step, counted as two iterations; rho_new == 0   */
/* leaves the directions as they are, as the reference does).          */
/* ------------------------------------------------------------------ */
void SKO_FN(sko_cgs_)(const sko_operator* A, const sko_precond* ML,
                      const sko_precond* MR, const SKO_T* b, SKO_T* x,
                      const sko_krylov_config* cfg, sko_summary* out,
                      double* history) {
  int64_t n = A->nrow;
  size_t vb = sizeof(SKO_T) * (size_t)(n + 1);
  SKO_T* r = (SKO_T*)calloc(1, vb);
  SKO_T* r_hat = (SKO_T*)calloc(1, vb);
  SKO_T* p = (SKO_T*)calloc(1, vb);
  SKO_T* u = (SKO_T*)calloc(1, vb);
  SKO_T* q = (SKO_T*)calloc(1, vb);
  SKO_T* q_hat = (SKO_T*)calloc(1, vb);
  SKO_T* u_hat = (SKO_T*)calloc(1, vb);
  SKO_T* p_hat = (SKO_T*)calloc(1, vb);
  SKO_T* tmp = (SKO_T*)calloc(1, vb);
  SKO_T* work = (SKO_T*)calloc(3, vb);
  int64_t nhist = 0;
  out->residual_norm = 0;
  out->computed_iterations = 0;
  out->converged = 0;
  out->status = 0;
  SKO_T bnorm = SKO_SQRT(SKO_FN(sko_dot_)(b, b, n)); /* :168 */
  if (bnorm == (SKO_T)0) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    out->converged = 1;
    goto done;
  }
  SKO_FN(sko_apply_op_)(A, x, tmp); /* compute_initial_residual :191-198 */
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
  memcpy(r_hat, r, vb); /* :201-209 */
  memcpy(p, r, vb);
  memcpy(u, r, vb);
  SKO_T rho = SKO_FN(sko_dot_)(r_hat, r, n);
  while (out->computed_iterations < cfg->max_iterations && !out->converged) {
    /* cgs_step :212-232 */
    SKO_FN(sko_apply_prec_)(ML, A, p, tmp, n, work); /* compute_q_hat :235-239 */
    SKO_FN(sko_apply_prec_)(MR, A, tmp, p_hat, n, work);
    SKO_FN(sko_apply_op_)(A, p_hat, q_hat);
    SKO_T alpha = rho / SKO_FN(sko_dot_)(r_hat, q_hat, n); /* :242-244 */
    for (int64_t i = 0; i < n; ++i) q[i] = u[i] - alpha * q_hat[i]; /* :247-252 */
    for (int64_t i = 0; i < n; ++i) u_hat[i] = u[i] + q[i];          /* :255-260 */
    SKO_FN(sko_apply_prec_)(ML, A, u_hat, tmp, n, work);             /* :263-266 */
    SKO_FN(sko_apply_prec_)(MR, A, tmp, p_hat, n, work);
    for (int64_t i = 0; i < n; ++i) x[i] += alpha * p_hat[i];        /* :269-275 */
    SKO_FN(sko_apply_op_)(A, p_hat, tmp);                            /* :278-284 */
    for (int64_t i = 0; i < n; ++i) r[i] -= alpha * tmp[i];
    out->computed_iterations += 2;
    SKO_T r_norm = SKO_SQRT(SKO_FN(sko_dot_)(r, r, n)); /* check_convergence :287-298 */
    out->residual_norm = (double)r_norm;
    if (history && cfg->collect_residuals) history[nhist++] = (double)r_norm;
    if (r_norm / bnorm < (SKO_T)cfg->tolerance) {
      out->converged = 1;
      break;
    }
    SKO_T rho_new = SKO_FN(sko_dot_)(r_hat, r, n);
    if (rho_new == (SKO_T)0) continue;
    SKO_T beta = rho_new / rho;
    for (int64_t i = 0; i < n; ++i) u[i] = r[i] + beta * q[i]; /* :301-309 */
    for (int64_t i = 0; i < n; ++i) p[i] = u[i] + beta * (q[i] + beta * p[i]);
    rho = rho_new;
  }
done:
  out->history_length = nhist;
  free(r); free(r_hat); free(p); free(u); free(q); free(q_hat); free(u_hat);
  free(p_hat); free(tmp); free(work);
}

/* ------------------------------------------------------------------ */
/* MINRES with left and right preconditioning                          */
/* Follows sparkit/data/minres.hpp:106-418 step for step, including    */
/* its two exits: rho == 0 in apply_givens_rotations (:265-286) marks  */
/* convergence but the step still updates x with the previous step's   */
/* rho, delta and phi before check_convergence (:300-309) decides      */
/* again; beta_new == 0 skips rotate_state (:311-325), so the next step */
/* repeats on the same Lanczos vectors.                                 */
/* ------------------------------------------------------------------ */
void SKO_FN(sko_minres_)(const sko_operator* A, const sko_precond* ML,
                         const sko_precond* MR, const SKO_T* b, SKO_T* x,
                         const sko_krylov_config* cfg, sko_summary* out,
                         double* history) {
  int64_t n = A->nrow;
  size_t vb = sizeof(SKO_T) * (size_t)(n + 1);
  SKO_T* v_prev = (SKO_T*)calloc(1, vb);
  SKO_T* v = (SKO_T*)calloc(1, vb);
  SKO_T* z = (SKO_T*)calloc(1, vb);
  SKO_T* w = (SKO_T*)calloc(1, vb);
  SKO_T* tmp = (SKO_T*)calloc(1, vb);
  SKO_T* d_prev = (SKO_T*)calloc(1, vb);
  SKO_T* d = (SKO_T*)calloc(1, vb);
  SKO_T* work = (SKO_T*)calloc(3, vb);
  int64_t nhist = 0;
  SKO_T beta = 0, alpha = 0, epsilon = 0, delta = 0, rho = 0, phi = 0, phi_bar = 0;
  SKO_T cs_prev = 0, sn_prev = 0, cs = 0, sn = 0, cs_new = 0, sn_new = 0;
  out->residual_norm = 0;
  out->computed_iterations = 0;
  out->converged = 0;
  out->status = 0;
  SKO_T bnorm = SKO_SQRT(SKO_FN(sko_dot_)(b, b, n)); /* :170 */
  if (bnorm == (SKO_T)0) {
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    out->converged = 1;
    goto done;
  }
  /* compute_initial_residual :184-217 */
  SKO_FN(sko_apply_op_)(A, x, w);
  for (int64_t i = 0; i < n; ++i) v[i] = b[i] - w[i];
  SKO_FN(sko_apply_prec_)(ML, A, v, tmp, n, work);
  SKO_FN(sko_apply_prec_)(MR, A, tmp, z, n, work);
  beta = SKO_SQRT(SKO_FN(sko_dot_)(v, z, n));
  if (beta == (SKO_T)0) {
    out->converged = 1;
    goto done;
  }
  {
    SKO_T inv_beta = (SKO_T)1 / beta;
    for (int64_t i = 0; i < n; ++i) v[i] = v[i] * inv_beta;
    for (int64_t i = 0; i < n; ++i) z[i] = z[i] * inv_beta;
  }
  phi_bar = beta;
  cs_prev = 1; sn_prev = 0; cs = 1; sn = 0;
  while (out->computed_iterations < cfg->max_iterations && !out->converged) {
    /* minres_step :225-234; lanczos_step :237-247 */
    SKO_FN(sko_apply_op_)(A, z, w);
    alpha = SKO_FN(sko_dot_)(z, w, n);
    for (int64_t i = 0; i < n; ++i) w[i] -= alpha * v[i] + beta * v_prev[i];
    /* precondition_lanczos :250-262 */
    SKO_FN(sko_apply_prec_)(ML, A, w, tmp, n, work);
    SKO_FN(sko_apply_prec_)(MR, A, tmp, v_prev, n, work);
    SKO_T beta_new = SKO_SQRT(SKO_FN(sko_dot_)(w, v_prev, n));
    /* apply_givens_rotations :265-286 */
    epsilon = sn_prev * beta;
    {
      SKO_T delta_1 = cs_prev * beta;
      SKO_T delta_l = cs * delta_1 + sn * alpha;
      SKO_T rho_bar = -sn * delta_1 + cs * alpha;
      SKO_T rho_l = SKO_SQRT(rho_bar * rho_bar + beta_new * beta_new);
      if (rho_l == (SKO_T)0) {
        out->converged = 1;
      } else {
        cs_new = rho_bar / rho_l;
        sn_new = beta_new / rho_l;
        phi = cs_new * phi_bar;
        phi_bar = -sn_new * phi_bar;
        rho = rho_l;
        delta = delta_l;
      }
    }
    /* update_solution :288-297 */
    for (int64_t i = 0; i < n; ++i) {
      SKO_T d_old = d[i];
      d_prev[i] = (z[i] - delta * d[i] - epsilon * d_prev[i]) / rho;
      d[i] = d_prev[i];
      d_prev[i] = d_old;
      x[i] += phi * d[i];
    }
    {
      SKO_T res = SKO_FABS(phi_bar); /* check_convergence :300-309 */
      out->residual_norm = (double)res;
      out->converged = res / bnorm < (SKO_T)cfg->tolerance;
      if (history && cfg->collect_residuals) history[nhist++] = (double)res;
    }
    out->computed_iterations += 1;
    if (out->converged || beta_new == (SKO_T)0) continue;
    {
      SKO_T inv_beta_new = (SKO_T)1 / beta_new; /* rotate_state :311-325 */
      for (int64_t i = 0; i < n; ++i) {
        SKO_T v_old = v[i];
        z[i] = v_prev[i] * inv_beta_new;
        v_prev[i] = v_old;
        v[i] = w[i] * inv_beta_new;
      }
      cs_prev = cs; sn_prev = sn; cs = cs_new; sn = sn_new;
      beta = beta_new;
    }
  }
done:
  out->history_length = nhist;
  free(v_prev); free(v); free(z); free(w); free(tmp); free(d_prev); free(d);
  free(work);
}

#undef SKO_FN
#undef SKO_CAT
#undef SKO_CAT2
