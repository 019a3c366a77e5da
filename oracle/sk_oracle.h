/*
 * sk_oracle.h -- CPU oracle for the sparkit preconditioned-Krylov hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the sparkit
 * reference's sequential algorithms (SpMV over CSR / ELLPACK / jagged
 * diagonal / BSR, Jacobi and Chebyshev preconditioners, CG, BiCGSTAB,
 * FGMRES, GMRES, CGS, MINRES, the Lanczos eigenvalue estimates and the
 * Matrix Market reader and writer), used
 * by the tests, the smoke check and the CPU-baseline leg of the benchmark
 * to check the CUDA library.  The product never links it.
 *
 * Parity pinning: tests/test_oracle.py checks every routine here against
 * the known-answer vectors of the reference's own Catch2 tests
 * (tests/golden/) and, bit for bit, against the reference itself compiled
 * from its sources into oracle/_ref (see oracle/build_ref.sh).
 */
#ifndef SK_ORACLE_H
#define SK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { SKO_CSR = 0, SKO_ELL = 1, SKO_JAD = 2, SKO_BSR = 3 };
enum { SKO_PREC_IDENTITY = 0, SKO_PREC_JACOBI = 1, SKO_PREC_CHEBYSHEV = 2 };
enum { SKO_BREAKDOWN = 4 };

/* A matrix in one of the reference's storage layouts (int64 indices, as
 * sparkit's size_type = std::ptrdiff_t).
 *   CSR: row_ptr[nrow+1], col_ind[nnz]
 *   ELL: col_ind[nrow*width] row-major, -1 padding; width = max nnz/row
 *   JAD: perm[nrow], row_ptr = jdiag[width+1], width = number of jagged
 *        diagonals, col_ind in jagged-diagonal order
 *   BSR: row_ptr[nbr+1] over block rows, col_ind[nblocks] block columns,
 *        vals = nblocks dense row-major block_rows x block_cols blocks */
typedef struct {
  int32_t format;
  int64_t nrow, ncol;
  int64_t width;
  int64_t block_rows, block_cols;
  const int64_t* row_ptr;
  const int64_t* col_ind;
  const int64_t* perm;
  const void* vals;
} sko_operator;

typedef struct {
  int32_t kind;
  const void* inv_diag;          /* Jacobi: inverse diagonal */
  const void* coeffs;            /* Chebyshev: degree+1 coefficients */
  double lambda_min, lambda_max; /* Chebyshev interval */
  int64_t degree;
  const sko_operator* op;        /* Chebyshev: matrix (NULL = solver's A) */
} sko_precond;

/* CGConfig, sparkit/data/conjugate_gradient.hpp:48-74 */
typedef struct {
  double tolerance;
  int64_t restart_iterations;
  int64_t max_iterations;
  int32_t collect_residuals;
} sko_cg_config;

/* Bicgstab_config, sparkit/data/bicgstab.hpp:25-42; Cgs_config
 * (cgs.hpp:25-42) and Minres_config (minres.hpp:25-45) have the same fields */
typedef struct {
  double tolerance;
  int64_t max_iterations;
  int32_t collect_residuals;
} sko_krylov_config;

/* Fgmres_config, sparkit/data/fgmres.hpp:25-47; Gmres_config
 * (gmres.hpp:25-47) has the same fields */
typedef struct {
  double tolerance;
  int64_t restart_dimension;
  int64_t max_iterations;
  int32_t collect_residuals;
} sko_fgmres_config;

/* CGSummary / Bicgstab_summary / Fgmres_summary, minus the vector (which
 * goes to the caller's history buffer). */
typedef struct {
  double residual_norm;
  int64_t computed_iterations;
  int32_t converged;
  int32_t status;
  int64_t history_length;
} sko_summary;

#define SKO_DECLARE(T, S)                                                     \
  void sko_csr_spmv_##S(int64_t, const int64_t*, const int64_t*, const T*,    \
                        const T*, T*);                                        \
  void sko_ell_spmv_##S(int64_t, int64_t, const int64_t*, const T*, const T*, \
                        T*);                                                  \
  void sko_jad_spmv_##S(int64_t, int64_t, const int64_t*, const int64_t*,     \
                        const int64_t*, const T*, const T*, T*);              \
  void sko_bsr_spmv_##S(int64_t, int64_t, int64_t, const int64_t*,            \
                        const int64_t*, const T*, const T*, T*);              \
  void sko_extract_diagonal_##S(int64_t, int64_t, const int64_t*,             \
                                const int64_t*, const T*, T*);                \
  int sko_jacobi_##S(int64_t, int64_t, const int64_t*, const int64_t*,        \
                     const T*, T*);                                           \
  void sko_chebyshev_coeffs_##S(T, T, int64_t, T*);                           \
  void sko_chebyshev_apply_##S(const sko_operator*, const T*, T, T, int64_t,  \
                               const T*, T*);                                 \
  void sko_cg_##S(const sko_operator*, const sko_precond*,                    \
                  const sko_precond*, const T*, T*, const sko_cg_config*,     \
                  sko_summary*, double*);                                     \
  void sko_bicgstab_##S(const sko_operator*, const sko_precond*,              \
                        const sko_precond*, const T*, T*,                     \
                        const sko_krylov_config*, sko_summary*, double*);     \
  void sko_fgmres_##S(const sko_operator*, const sko_precond*, const T*, T*,  \
                      const sko_fgmres_config*, sko_summary*, double*);       \
  void sko_gmres_##S(const sko_operator*, const sko_precond*,                 \
                     const sko_precond*, const T*, T*,                        \
                     const sko_fgmres_config*, sko_summary*, double*);        \
  void sko_cgs_##S(const sko_operator*, const sko_precond*,                   \
                   const sko_precond*, const T*, T*,                          \
                   const sko_krylov_config*, sko_summary*, double*);          \
  void sko_minres_##S(const sko_operator*, const sko_precond*,                \
                      const sko_precond*, const T*, T*,                       \
                      const sko_krylov_config*, sko_summary*, double*);       \
  void sko_tridiagonal_eigen_##S(int64_t, T*, T*, T, int64_t, T*);            \
  void sko_lanczos_##S(const sko_operator*, const sko_lanczos_config*, T*,    \
                       T*, T*, double*, sko_lanczos_result*);                 \
  T sko_spectral_radius_##S(const sko_operator*, int64_t);                    \
  void sko_eigenvalue_bounds_##S(const sko_operator*, int64_t, T*);

/* Lanczos_config<T> (lanczos.hpp:25-33); target in Eigen_target order
 * (eigen_target.hpp:13-20: largest_magnitude, smallest_magnitude,
 * largest_algebraic, smallest_algebraic, largest_real, smallest_real). */
typedef struct {
  int64_t num_eigenvalues;
  int64_t krylov_dimension;
  double tolerance;
  int64_t max_restarts;
  int32_t target;
  int32_t collect_residuals;
} sko_lanczos_config;

/* The scalars of Lanczos_result<T> (lanczos.hpp:39-47). */
typedef struct {
  int64_t count;                   /* eigenvalues returned */
  int64_t computed_restarts;
  int64_t converged_count;
  int64_t residual_count;          /* residual_norms written */
  int64_t restart_residuals_count; /* restart_residuals written */
  int32_t converged;
} sko_lanczos_result;

/* A CSR matrix read from Matrix Market text (sk_oracle_mm.c); the arrays
 * are malloc'd (sko_mm_free); err holds the reason when reading fails. */
typedef struct {
  int64_t nrow, ncol, nnz;
  int64_t* row_ptr;
  int64_t* col_ind;
  void* values;
  char err[256];
} sko_mm_csr;

int sko_mm_read_f64(const char* text, int64_t len, sko_mm_csr* out);
int sko_mm_read_f32(const char* text, int64_t len, sko_mm_csr* out);
void sko_mm_free(sko_mm_csr* m);
char* sko_mm_write_f64(int64_t nrow, int64_t ncol, const int64_t* rp, const int64_t* ci, const double* v,
                       int64_t* len);
char* sko_mm_write_f32(int64_t nrow, int64_t ncol, const int64_t* rp, const int64_t* ci, const float* v,
                       int64_t* len);
void sko_free(void* p);

/* Summation order of the solvers' dot products: 0 = the reference's
 * sequential order (default), 1 = 256-element chunks added in order,
 * 2 = sequential from the last element (sensitivity studies). */
void sko_set_dot_order(int mode);

SKO_DECLARE(double, f64)
SKO_DECLARE(float, f32)

/* Learned preconditioner network (sk_oracle_net.c).  coef holds, per
 * sample, six planes of H*W floats: diagonal, west, east, south, north
 * coefficients and the inverse diagonal. */
int64_t skon_param_count(void);
void skon_features(int B, int H, int W, const double* r, const float* coef, int round_bf16, double* xin,
                   double* scale);
void skon_apply(int H, int W, const float* params, const double* v, const float* coef, int round_bf16,
                double* z, double* y_out);
double skon_loss_grad(int B, int H, int W, const float* params, const double* r, const double* e,
                      const float* coef, double mu, int round_bf16, double* grad, double* y_out);
void skon_adam(int64_t n, float* p, float* m, float* v, const float* g, float lr, float b1, float b2,
               float eps, int64_t t);

#ifdef __cplusplus
}
#endif
#endif
