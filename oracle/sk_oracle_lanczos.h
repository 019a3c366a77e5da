/*
 * sk_oracle_lanczos.h -- implicitly restarted Lanczos and the eigenvalue
 * estimates built on it, restated in plain C for the CPU oracle.
 * Instantiated per value type by sk_oracle.c after sk_oracle_impl.h (it uses
 * that file's operator application and dot product).  TEST INFRASTRUCTURE
 * ONLY: the product never links this file.
 *
 * Follows, with the reference's operation order:
 *   tridiagonal_eigen           sparkit/data/dense_tridiagonal_eigen.hpp:58-193
 *   LanczosSolver / lanczos     sparkit/data/lanczos.hpp:64-503
 *   estimate_spectral_radius    sparkit/data/conditioning.hpp:112-126
 *   estimate_eigenvalue_bounds  sparkit/data/conditioning.hpp:132-168
 */
#define SKO_CAT2(a, b) a##b
#define SKO_CAT(a, b) SKO_CAT2(a, b)
#define SKO_FN(name) SKO_CAT(name, SKO_SFX)

/* Symmetric tridiagonal eigensolver, implicit QR with Wilkinson shift
 * (dense_tridiagonal_eigen.hpp:58-193).  d[n] and e[n-1] are overwritten;
 * on return d holds the eigenvalues (unsorted).  Q (n*n, may be NULL)
 * receives the eigenvectors: Q[k*n + i] = component i of eigenvector k. */
void SKO_FN(sko_tridiagonal_eigen_)(int64_t n, SKO_T* d, SKO_T* e, SKO_T tol, int64_t max_iterations,
                                    SKO_T* Q) {
  if (n == 0) return;
  if (Q) {
    for (int64_t i = 0; i < n * n; ++i) Q[i] = 0;
    for (int64_t i = 0; i < n; ++i) Q[i * n + i] = 1;
  }
  int64_t hi = n - 1;
  int64_t total = 0;
  while (hi > 0 && total < max_iterations * n) {
    SKO_T tol_hi = tol * (SKO_FABS(d[hi - 1]) + SKO_FABS(d[hi]));
    if (tol_hi == 0) tol_hi = tol;
    if (SKO_FABS(e[hi - 1]) <= tol_hi) {
      --hi;
      continue;
    }
    int64_t lo = hi - 1;
    while (lo > 0) {
      SKO_T tol_lo = tol * (SKO_FABS(d[lo - 1]) + SKO_FABS(d[lo]));
      if (tol_lo == 0) tol_lo = tol;
      if (SKO_FABS(e[lo - 1]) <= tol_lo) break;
      --lo;
    }
    /* Wilkinson shift (:97-109) */
    SKO_T delta = (d[hi - 1] - d[hi]) / (SKO_T)2;
    SKO_T e_him1 = e[hi - 1];
    SKO_T shift;
    if (delta == 0) {
      shift = d[hi] - SKO_FABS(e_him1);
    } else {
      SKO_T sign_d = delta > 0 ? (SKO_T)1 : (SKO_T)-1;
      shift = d[hi] - e_him1 * e_him1 / (delta + sign_d * SKO_SQRT(delta * delta + e_him1 * e_him1));
    }
    /* bulge chase (:112-164) */
    SKO_T x = d[lo] - shift;
    SKO_T z = e[lo];
    for (int64_t k = lo; k < hi; ++k) {
      SKO_T cs, sn;
      SKO_T r = SKO_SQRT(x * x + z * z);
      if (r == 0) {
        cs = 1;
        sn = 0;
      } else {
        cs = x / r;
        sn = z / r;
      }
      if (k > lo) e[k - 1] = r;
      SKO_T d_k = d[k], d_k1 = d[k + 1], e_k = e[k];
      d[k] = cs * cs * d_k + (SKO_T)2 * cs * sn * e_k + sn * sn * d_k1;
      d[k + 1] = sn * sn * d_k - (SKO_T)2 * cs * sn * e_k + cs * cs * d_k1;
      /* the first form of e[k] (:137) is overwritten at once (:140) */
      e[k] = cs * (d_k1 - d_k) * sn + (cs * cs - sn * sn) * e_k;
      if (k + 1 < hi) {
        SKO_T e_k1 = e[k + 1];
        z = sn * e_k1;
        e[k + 1] = cs * e_k1;
        x = e[k];
      }
      if (Q) {
        for (int64_t i = 0; i < n; ++i) {
          SKO_T q_ik = Q[k * n + i], q_ik1 = Q[(k + 1) * n + i];
          Q[k * n + i] = cs * q_ik + sn * q_ik1;
          Q[(k + 1) * n + i] = -sn * q_ik + cs * q_ik1;
        }
      }
    }
    ++total;
  }
}

/* The Lanczos state (lanczos.hpp:86-101). */
typedef struct {
  const sko_operator* A;
  int64_t n, m, nev;
  SKO_T tol;
  int64_t max_restarts;
  int target;
  int collect;
  SKO_T* V;     /* (m + 1) x n */
  SKO_T* alpha; /* m */
  SKO_T* beta;  /* m + 1 */
  SKO_T* w;     /* n */
  SKO_T* tri_d; /* m: Ritz values */
  SKO_T* tri_e;
  SKO_T* tri_Q; /* m x m */
  int64_t* wanted;
  SKO_T* residual_norms;
  double* restart_residuals;
  int64_t n_restart_res;
  int64_t converged_count;
  int64_t computed_restarts;
} SKO_FN(sko_lz_);

static SKO_T SKO_FN(sko_lz_norm_)(const SKO_T* v, int64_t n) { return SKO_SQRT(SKO_FN(sko_dot_)(v, v, n)); }

static void SKO_FN(sko_lz_normalize_)(SKO_T* v, int64_t n) {
  SKO_T nv = SKO_FN(sko_lz_norm_)(v, n);
  if (nv > 0)
    for (int64_t i = 0; i < n; ++i) v[i] /= nv;
}

/* lanczos.hpp:194-205: the two-pass modified Gram-Schmidt */
static void SKO_FN(sko_lz_reorth_)(SKO_FN(sko_lz_) * L, int64_t j) {
  for (int pass = 0; pass < 2; ++pass)
    for (int64_t k = 0; k <= j; ++k) {
      const SKO_T* vk = L->V + k * L->n;
      SKO_T h = SKO_FN(sko_dot_)(vk, L->w, L->n);
      for (int64_t i = 0; i < L->n; ++i) L->w[i] -= h * vk[i];
    }
}

/* lanczos.hpp:207-222 */
static void SKO_FN(sko_lz_random_restart_)(SKO_FN(sko_lz_) * L, int64_t j) {
  sko_mt19937 g;
  sko_mt_seed(&g, (uint32_t)(j + 137));
  SKO_T* v = L->V + (j + 1) * L->n;
  for (int64_t i = 0; i < L->n; ++i) v[i] = SKO_UNIFORM(&g);
  for (int64_t k = 0; k <= j; ++k) {
    const SKO_T* vk = L->V + k * L->n;
    SKO_T h = SKO_FN(sko_dot_)(vk, v, L->n);
    for (int64_t i = 0; i < L->n; ++i) v[i] -= h * vk[i];
  }
  SKO_FN(sko_lz_normalize_)(v, L->n);
}

/* lanczos.hpp:158-191 */
static void SKO_FN(sko_lz_steps_)(SKO_FN(sko_lz_) * L, int64_t start, int64_t stop) {
  const int64_t n = L->n;
  for (int64_t j = start; j < stop; ++j) {
    SKO_T* vj = L->V + j * n;
    SKO_FN(sko_apply_op_)(L->A, vj, L->w);
    L->alpha[j] = SKO_FN(sko_dot_)(vj, L->w, n);
    for (int64_t i = 0; i < n; ++i) L->w[i] -= L->alpha[j] * vj[i];
    if (j > 0) {
      const SKO_T* vjm1 = L->V + (j - 1) * n;
      for (int64_t i = 0; i < n; ++i) L->w[i] -= L->beta[j] * vjm1[i];
    }
    SKO_FN(sko_lz_reorth_)(L, j);
    SKO_T beta_next = SKO_FN(sko_lz_norm_)(L->w, n);
    L->beta[j + 1] = beta_next;
    if (beta_next > 0) {
      SKO_T* vj1 = L->V + (j + 1) * n;
      for (int64_t i = 0; i < n; ++i) vj1[i] = L->w[i] / beta_next;
    } else {
      SKO_FN(sko_lz_random_restart_)(L, j);
    }
  }
}

/* lanczos.hpp:141-151 */
static void SKO_FN(sko_lz_eig_)(SKO_FN(sko_lz_) * L) {
  const int64_t m = L->m;
  for (int64_t i = 0; i < m; ++i) L->tri_d[i] = L->alpha[i];
  for (int64_t i = 0; i + 1 < m; ++i) L->tri_e[i] = L->beta[i + 1];
  SKO_FN(sko_tridiagonal_eigen_)(m, L->tri_d, L->tri_e, (SKO_T)1e-15, m * 30, L->tri_Q);
}

/* Eigen_target order (eigen_target.hpp:13-20): a comes before b */
static int SKO_FN(sko_lz_before_)(int target, SKO_T a, SKO_T b) {
  switch (target) {
    case 0: return SKO_FABS(a) > SKO_FABS(b);  /* largest_magnitude */
    case 1: return SKO_FABS(a) < SKO_FABS(b);  /* smallest_magnitude */
    case 2: case 4: return a > b;              /* largest_algebraic / _real */
    default: return a < b;                     /* smallest_algebraic / _real */
  }
}

/* lanczos.hpp:225-269: the indices sorted by the target, first nev kept.
 * The reference sorts with std::sort, whose order among equal keys is
 * unspecified; this sort is stable (equal Ritz values keep index order). */
static void SKO_FN(sko_lz_select_)(SKO_FN(sko_lz_) * L) {
  const int64_t m = L->m;
  int64_t* order = (int64_t*)malloc((size_t)(m > 0 ? m : 1) * sizeof(int64_t));
  for (int64_t i = 0; i < m; ++i) order[i] = i;
  for (int64_t i = 1; i < m; ++i) {
    int64_t v = order[i], k = i;
    while (k > 0 && SKO_FN(sko_lz_before_)(L->target, L->tri_d[v], L->tri_d[order[k - 1]])) {
      order[k] = order[k - 1];
      --k;
    }
    order[k] = v;
  }
  for (int64_t i = 0; i < L->nev; ++i) L->wanted[i] = order[i];
  free(order);
}

/* lanczos.hpp:153-177 */
static int SKO_FN(sko_lz_converged_)(SKO_FN(sko_lz_) * L) {
  int all = 1;
  L->converged_count = 0;
  SKO_T beta_m = L->beta[L->m];
  for (int64_t w = 0; w < L->nev; ++w) {
    int64_t idx = L->wanted[w];
    SKO_T abs_res = SKO_FABS(beta_m * L->tri_Q[idx * L->m + (L->m - 1)]);
    SKO_T abs_theta = SKO_FABS(L->tri_d[idx]);
    SKO_T floor_ = (SKO_T)1e-20;
    SKO_T threshold = L->tol * (abs_theta > floor_ ? abs_theta : floor_);
    L->residual_norms[w] = abs_res;
    if (abs_res <= threshold)
      ++L->converged_count;
    else
      all = 0;
  }
  if (L->collect) {
    SKO_T mx = 0;
    for (int64_t w = 0; w < L->nev; ++w) mx = L->residual_norms[w] > mx ? L->residual_norms[w] : mx;
    L->restart_residuals[L->n_restart_res++] = (double)mx;
  }
  return all;
}

/* lanczos.hpp:373-434: one implicit QR step with shift mu on the
 * tridiagonal, the basis and the last row of Q */
static void SKO_FN(sko_lz_qr_step_)(SKO_FN(sko_lz_) * L, SKO_T mu, SKO_T* q_row) {
  const int64_t m = L->m, n = L->n;
  SKO_T* alpha = L->alpha;
  SKO_T* beta = L->beta;
  SKO_T x = alpha[0] - mu;
  SKO_T z = beta[1];
  for (int64_t k = 0; k < m - 1; ++k) {
    SKO_T cs, sn;
    SKO_T r = SKO_SQRT(x * x + z * z);
    if (r == 0) {
      cs = 1;
      sn = 0;
    } else {
      cs = x / r;
      sn = z / r;
    }
    if (k > 0) beta[k] = r;
    SKO_T a_k = alpha[k], a_k1 = alpha[k + 1], b_k1 = beta[k + 1];
    alpha[k] = cs * cs * a_k + (SKO_T)2 * cs * sn * b_k1 + sn * sn * a_k1;
    alpha[k + 1] = sn * sn * a_k - (SKO_T)2 * cs * sn * b_k1 + cs * cs * a_k1;
    beta[k + 1] = cs * sn * (a_k1 - a_k) + (cs * cs - sn * sn) * b_k1;
    if (k + 2 < m) {
      SKO_T b_k2 = beta[k + 2];
      x = beta[k + 1];
      z = sn * b_k2;
      beta[k + 2] = cs * b_k2;
    }
    SKO_T* vk = L->V + k * n;
    SKO_T* vk1 = L->V + (k + 1) * n;
    for (int64_t i = 0; i < n; ++i) {
      SKO_T v_k = vk[i], v_k1 = vk1[i];
      vk[i] = cs * v_k + sn * v_k1;
      vk1[i] = -sn * v_k + cs * v_k1;
    }
    SKO_T q_k = q_row[k], q_k1 = q_row[k + 1];
    q_row[k] = cs * q_k + sn * q_k1;
    q_row[k + 1] = -sn * q_k + cs * q_k1;
  }
}

/* lanczos.hpp:314-369 */
static void SKO_FN(sko_lz_restart_)(SKO_FN(sko_lz_) * L) {
  const int64_t m = L->m, n = L->n, nev = L->nev;
  SKO_T beta_m_saved = L->beta[m];
  SKO_T* v_mp1 = (SKO_T*)malloc((size_t)n * sizeof(SKO_T) + 8);
  memcpy(v_mp1, L->V + m * n, (size_t)n * sizeof(SKO_T));
  SKO_T* q_row = (SKO_T*)calloc((size_t)m, sizeof(SKO_T));
  q_row[m - 1] = 1;
  for (int64_t u = 0; u < m; ++u) {  /* unwanted, ascending (:273-283) */
    int is_wanted = 0;
    for (int64_t w = 0; w < nev; ++w) is_wanted |= (L->wanted[w] == u);
    if (!is_wanted) SKO_FN(sko_lz_qr_step_)(L, L->tri_d[u], q_row);
  }
  SKO_T sigma_k = L->beta[nev];
  SKO_T tau = beta_m_saved * q_row[nev - 1];
  SKO_T* vk = L->V + nev * n;
  for (int64_t i = 0; i < n; ++i) vk[i] = sigma_k * vk[i] + tau * v_mp1[i];
  SKO_T beta_new = SKO_FN(sko_lz_norm_)(vk, n);
  if (beta_new > 0)
    for (int64_t i = 0; i < n; ++i) vk[i] /= beta_new;
  L->beta[nev] = beta_new;
  free(q_row);
  free(v_mp1);
  SKO_FN(sko_lz_steps_)(L, nev, m);
}

/* lanczos.hpp:437-461: Ritz values, and vectors when asked */
static void SKO_FN(sko_lz_extract_)(SKO_FN(sko_lz_) * L, SKO_T* eigenvalues, SKO_T* eigenvectors) {
  const int64_t n = L->n, m = L->m;
  for (int64_t w = 0; w < L->nev; ++w) {
    int64_t idx = L->wanted[w];
    eigenvalues[w] = L->tri_d[idx];
    if (!eigenvectors) continue;
    SKO_T* x = eigenvectors + w * n;
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    for (int64_t j = 0; j < m; ++j) {
      SKO_T coeff = L->tri_Q[idx * m + j];
      const SKO_T* vj = L->V + j * n;
      for (int64_t i = 0; i < n; ++i) x[i] += coeff * vj[i];
    }
    SKO_FN(sko_lz_normalize_)(x, n);
  }
}

/* lanczos(n, cfg, op) (lanczos.hpp:64-139, :495-503).  eigenvalues and
 * residual_norms hold min(num_eigenvalues, m) values, eigenvectors (may be
 * NULL) as many n-vectors, restart_residuals (collect only) up to
 * max_restarts values. */
void SKO_FN(sko_lanczos_)(const sko_operator* A, const sko_lanczos_config* cfg, SKO_T* eigenvalues,
                          SKO_T* eigenvectors, SKO_T* residual_norms, double* restart_residuals,
                          sko_lanczos_result* out) {
  SKO_FN(sko_lz_) L;
  memset(&L, 0, sizeof(L));
  L.A = A;
  L.n = A->nrow;
  L.m = cfg->krylov_dimension;
  L.nev = cfg->num_eigenvalues;
  if (L.m > L.n) L.m = L.n;
  if (L.nev > L.m) L.nev = L.m;
  L.tol = (SKO_T)cfg->tolerance;
  L.max_restarts = cfg->max_restarts;
  L.target = cfg->target;
  L.collect = cfg->collect_residuals;
  const int64_t n = L.n, m = L.m;
  L.V = (SKO_T*)calloc((size_t)((m + 1) * n + 1), sizeof(SKO_T));
  L.alpha = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  L.beta = (SKO_T*)calloc((size_t)(m + 2), sizeof(SKO_T));
  L.w = (SKO_T*)calloc((size_t)(n + 1), sizeof(SKO_T));
  L.tri_d = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  L.tri_e = (SKO_T*)calloc((size_t)(m + 1), sizeof(SKO_T));
  L.tri_Q = (SKO_T*)calloc((size_t)(m * m + 1), sizeof(SKO_T));
  L.wanted = (int64_t*)calloc((size_t)(L.nev + 1), sizeof(int64_t));
  L.residual_norms = residual_norms;
  L.restart_residuals = restart_residuals;
  /* init (:104-121): random unit start vector */
  sko_mt19937 g;
  sko_mt_seed(&g, 42u);
  for (int64_t i = 0; i < n; ++i) L.V[i] = SKO_UNIFORM(&g);
  SKO_FN(sko_lz_normalize_)(L.V, n);
  /* run (:123-139) */
  SKO_FN(sko_lz_steps_)(&L, 0, m);
  int done = 0;
  for (int64_t r = 0; r < L.max_restarts && !done; ++r) {
    L.computed_restarts = r + 1;
    SKO_FN(sko_lz_eig_)(&L);
    SKO_FN(sko_lz_select_)(&L);
    if (SKO_FN(sko_lz_converged_)(&L) || L.nev == m) {
      SKO_FN(sko_lz_extract_)(&L, eigenvalues, eigenvectors);
      out->converged = 1;
      done = 1;
    } else {
      SKO_FN(sko_lz_restart_)(&L);
    }
  }
  if (!done) {
    SKO_FN(sko_lz_eig_)(&L);
    SKO_FN(sko_lz_select_)(&L);
    SKO_FN(sko_lz_extract_)(&L, eigenvalues, eigenvectors);
    out->converged = 0;
  }
  out->count = L.nev;
  out->computed_restarts = L.computed_restarts;
  out->converged_count = L.converged_count;
  out->restart_residuals_count = L.n_restart_res;
  /* residual_norms are those of the last convergence check (none when
   * max_restarts is 0) */
  out->residual_count = L.max_restarts > 0 ? L.nev : 0;
  free(L.V);
  free(L.alpha);
  free(L.beta);
  free(L.w);
  free(L.tri_d);
  free(L.tri_e);
  free(L.tri_Q);
  free(L.wanted);
}

/* estimate_spectral_radius (conditioning.hpp:112-126) */
SKO_T SKO_FN(sko_spectral_radius_)(const sko_operator* A, int64_t num_iter) {
  int64_t m = A->nrow < num_iter + 1 ? A->nrow : num_iter + 1;
  sko_lanczos_config cfg = {1, m, 1e-10, 10, 0, 0};
  SKO_T ev[1] = {0}, res[1] = {0};
  sko_lanczos_result r;
  memset(&r, 0, sizeof(r));
  SKO_FN(sko_lanczos_)(A, &cfg, ev, NULL, res, NULL, &r);
  if (r.count == 0) return 0;
  return SKO_FABS(ev[0]);
}

/* estimate_eigenvalue_bounds (conditioning.hpp:132-168): out[0] = lambda_min,
 * out[1] = lambda_max (0 when a pass returns no eigenvalue). */
void SKO_FN(sko_eigenvalue_bounds_)(const sko_operator* A, int64_t num_iter, SKO_T* out) {
  int64_t m = A->nrow < num_iter + 1 ? A->nrow : num_iter + 1;
  sko_lanczos_config cmax = {1, m, 1e-10, 10, 2, 0};
  sko_lanczos_config cmin = {1, m, 1e-10, 10, 3, 0};
  SKO_T ev[1] = {0}, res[1] = {0};
  sko_lanczos_result r;
  memset(&r, 0, sizeof(r));
  SKO_FN(sko_lanczos_)(A, &cmax, ev, NULL, res, NULL, &r);
  SKO_T lmax = r.count ? ev[0] : 0;
  memset(&r, 0, sizeof(r));
  ev[0] = 0;
  SKO_FN(sko_lanczos_)(A, &cmin, ev, NULL, res, NULL, &r);
  SKO_T lmin = r.count ? ev[0] : 0;
  out[0] = lmin;
  out[1] = lmax;
}

#undef SKO_FN
#undef SKO_CAT
#undef SKO_CAT2
