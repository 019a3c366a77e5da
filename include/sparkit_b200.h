/*
 * sparkit_b200.h -- C ABI of the B200 (sm_100a) preconditioned-Krylov path.
 *
 * The sparkit reference is a C++20 template library with no C ABI of its
 * own: its hot path is reached through C++ overloads and templates
 * (namespace sparkit::data::detail).  Each entry point below states which
 * reference interface it replaces (file:line within the sparkit project).
 *
 * Conventions
 *  - Every call returns sk_status; SK_OK is 0.  sk_last_error() gives a
 *    message for the calling thread's most recent failure.
 *  - Index arrays coming from the reference are int64 (sparkit's size_type
 *    is std::ptrdiff_t, sparkit/data/import.hpp:19).  The device keeps int32
 *    indices; a value outside int32 fails with SK_INDEX_OVERFLOW.
 *  - "host" pointers are ordinary CPU memory, borrowed for the call.
 *    "dev" pointers are device memory of the current CUDA device.
 *  - sk_stream is a cudaStream_t; NULL means the library's own stream of
 *    the matrix handle.  Calls on one handle are not reentrant; calls on
 *    different handles may run on different threads.
 *  - Value arrays are double (SK_F64) or float (SK_F32), as the handle's
 *    dtype says.
 */
#ifndef SPARKIT_B200_H
#define SPARKIT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SK_API __attribute__((visibility("default")))
#else
#define SK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SK_OK = 0,
  SK_INVALID_ARG = 1,     /* bad size, null pointer, format mismatch */
  SK_INDEX_OVERFLOW = 2,  /* an index does not fit the device's int32 */
  SK_OUT_OF_MEMORY = 3,
  SK_BREAKDOWN = 4,       /* Krylov breakdown (zero rho or <r_hat, v>) */
  SK_NOT_CONVERGED = 5,   /* reserved; solvers report it in sk_summary */
  SK_TIMEOUT = 6,         /* a bounded device wait gave up */
  SK_CUDA_ERROR = 7,
  SK_ZERO_DIAGONAL = 8,   /* jacobi set-up met an exact zero diagonal */
  SK_NOT_SUPPORTED = 9,
  SK_NO_DEVICE = 10
} sk_status;

typedef enum { SK_F64 = 0, SK_F32 = 1 } sk_dtype;
typedef enum { SK_CSR = 0, SK_ELL = 1, SK_JAD = 2, SK_BSR = 3 } sk_format;

typedef struct sk_matrix_s* sk_matrix;
typedef struct sk_precond_s* sk_precond;
typedef void* sk_stream;

/* ---------------------------------------------------------------- */
/* Library                                                           */
/* ---------------------------------------------------------------- */

/* Version string of this library. */
SK_API const char* sk_version(void);
/* Message of the calling thread's most recent failed call. */
SK_API const char* sk_last_error(void);
/* Number of CUDA devices visible (0 on a machine without a GPU). */
SK_API sk_status sk_device_count(int* count);
/* Count of this library's kernel launches since load (for accounting). */
SK_API sk_status sk_launch_count(int64_t* count);

/* Summation order of the solvers' dot products and norms (process-wide,
 * read at the start of each solve).  SK_SUM_TREE (the default) sums each
 * one in a fixed, deterministic tree over the grid: repeatable bit for bit,
 * and fast.  SK_SUM_SEQUENTIAL sums the terms one after another in element
 * order, in the value type, as std::inner_product does in every solver of
 * the reference (conjugate_gradient.hpp:194-282, bicgstab.hpp:328-335,
 * fgmres.hpp:266,400, cgs.hpp:313-320, minres.hpp:170-259,
 * gmres.hpp:165-272); with the products and
 * element-wise updates already in the reference's arithmetic order, a
 * solve then reproduces the reference's iterates.  It is for validation:
 * one warp adds each sum's n terms in turn, which costs n dependent
 * additions per dot product.  The mixed-precision, batched and Lanczos
 * paths keep the tree order. */
enum { SK_SUM_TREE = 0, SK_SUM_SEQUENTIAL = 1 };
SK_API sk_status sk_set_summation_order(int32_t order);
SK_API sk_status sk_get_summation_order(int32_t* order);

/* No reference counterpart: a setting for tests of the timeout path.  The
 * persistent kernels (the mixed solver's inner CG, the GMRES / FGMRES
 * Arnoldi step) wait at grid barriers, and every wait is bounded in time:
 * when it runs out the kernel returns and the call reports SK_TIMEOUT.
 * limit_ns sets that bound for launches made after this call (0 restores
 * the default of 2 s; at most 10 s).  unmeetable != 0 makes every barrier
 * of those launches wait for one arrival more than the grid makes, so that
 * the first wait runs out on an ordinary, correct solve.  Process-wide;
 * sk_debug_set_wait(0, 0) restores the defaults. */
SK_API sk_status sk_debug_set_wait(uint64_t limit_ns, int32_t unmeetable);

/* Device memory helpers, so that a C/C++ caller needs no CUDA headers. */
SK_API sk_status sk_device_alloc(void** dev, size_t bytes);
SK_API sk_status sk_device_free(void* dev);
SK_API sk_status sk_memcpy_h2d(void* dev, const void* host, size_t bytes, sk_stream s);
SK_API sk_status sk_memcpy_d2h(void* host, const void* dev, size_t bytes, sk_stream s);
SK_API sk_status sk_stream_synchronize(sk_stream s);

/* ---------------------------------------------------------------- */
/* Matrix handles (upload once, device resident)                     */
/* ---------------------------------------------------------------- */

/* Compressed_row_matrix<T> (sparkit/data/Compressed_row_matrix.hpp:20-132):
 * row_ptr[nrow+1], col_ind[nnz] sorted within each row, values[nnz]. */
SK_API sk_status sk_csr_create(sk_matrix* out, int64_t nrow, int64_t ncol,
                        const int64_t* row_ptr, const int64_t* col_ind,
                        const void* values, sk_dtype dtype);

/* Ellpack_matrix<T> (sparkit/data/Ellpack_matrix.hpp:20-122): row-major
 * nrow x width col_ind padded with -1 (Ellpack_sparsity_Impl.cpp:33-36),
 * values with the same layout.  width = max_nnz_per_row(). */
SK_API sk_status sk_ell_create(sk_matrix* out, int64_t nrow, int64_t ncol,
                        int64_t width, const int64_t* col_ind,
                        const void* values, sk_dtype dtype);

/* Jagged_diagonal_matrix<T> (sparkit/data/Jagged_diagonal_matrix.hpp:20-144):
 * perm[nrow], jdiag[njd+1], col_ind[nnz] and values[nnz] in
 * jagged-diagonal order (Jagged_diagonal_sparsity_Impl.cpp:11-93).  perm
 * may be NULL when njd == 0 (the reference's empty JAD holds no perm). */
SK_API sk_status sk_jad_create(sk_matrix* out, int64_t nrow, int64_t ncol,
                        int64_t njd, const int64_t* perm, const int64_t* jdiag,
                        const int64_t* col_ind, const void* values,
                        sk_dtype dtype);

/* Block_sparse_row_matrix<T> (sparkit/data/Block_sparse_row_matrix.hpp:21-150):
 * row_ptr over ceil(nrow/block_rows) block rows, col_ind[nblocks] block
 * columns, values = nblocks dense row-major block_rows x block_cols blocks. */
SK_API sk_status sk_bsr_create(sk_matrix* out, int64_t nrow, int64_t ncol,
                        int64_t block_rows, int64_t block_cols,
                        const int64_t* row_ptr, const int64_t* col_ind,
                        const void* values, sk_dtype dtype);

/* Conversions built on the device from a CSR handle (its dtype kept; the
 * CSR col_ind sorted within each row, as every reference CSR is).  The new
 * handle holds exactly what sk_ell_create / sk_jad_create / sk_bsr_create
 * would build from the reference's conversion of the same matrix.
 *   to_ellpack(Compressed_row_matrix<T>)          conversions.hpp:427-467
 *   to_jagged_diagonal(Compressed_row_matrix<T>)  conversions.hpp:641-691
 *     (rows by decreasing length, ties by row index:
 *      Jagged_diagonal_sparsity_Impl.cpp:41-47)
 *   to_block_sparse_row(csr, block_rows, block_cols) conversions.hpp:524-577 */
SK_API sk_status sk_ell_from_csr(sk_matrix* out, sk_matrix csr);
SK_API sk_status sk_jad_from_csr(sk_matrix* out, sk_matrix csr);
SK_API sk_status sk_bsr_from_csr(sk_matrix* out, sk_matrix csr,
                          int64_t block_rows, int64_t block_cols);
/* Device time in ms of the kernels that built a handle on the device (the
 * conversions above; host allocations between them not counted; the BSR
 * sliced product copy not counted); 0 for handles uploaded from the host. */
SK_API sk_status sk_matrix_build_ms(sk_matrix A, double* ms);

/* The reference's accessors row_ptr() / col_ind() / values() / perm() /
 * jdiag() (Compressed_row_matrix.hpp, Ellpack_matrix.hpp,
 * Jagged_diagonal_matrix.hpp, Block_sparse_row_matrix.hpp) as host copies
 * of a handle, sized by sk_matrix_info:
 *   CSR  row_ptr[nrow+1], col_ind[nnz], values[nnz]
 *   ELL  col_ind[nrow*width] row-major with -1 past each row, values alike
 *   JAD  perm[nrow] (written only when width > 0: an empty reference JAD
 *        holds none), jdiag[width+1], col_ind[nnz], values[nnz]
 *   BSR  row_ptr[ceil(nrow/block_rows)+1], col_ind[width],
 *        values[width*block_rows*block_cols] */
SK_API sk_status sk_csr_export(sk_matrix A, int64_t* row_ptr, int64_t* col_ind, void* values);
SK_API sk_status sk_ell_export(sk_matrix A, int64_t* col_ind, void* values);
SK_API sk_status sk_jad_export(sk_matrix A, int64_t* perm, int64_t* jdiag,
                        int64_t* col_ind, void* values);
SK_API sk_status sk_bsr_export(sk_matrix A, int64_t* row_ptr, int64_t* col_ind, void* values);

/* read_matrix_market<T>(path) followed by to_compressed_row
 * (sparkit/data/matrix_market.hpp:45-115, matrix_market.cpp:28-87,
 * Coordinate_matrix.hpp:36-41) into a device CSR handle of dtype.  As the
 * reference: a case-insensitive banner; coordinate format only; real,
 * integer and pattern fields (pattern entries are 1); comment and empty
 * lines skipped before the size line; exactly nnz entry lines with 1-based
 * indices; a symmetric file's off-diagonal entries mirrored (skew-symmetric
 * and hermitian files read as stored); the last of duplicate entries kept;
 * a side of 1 or less rejected ("invalid matrix shape").  Unlike the
 * reference, a malformed or out-of-range entry line, or fewer than nnz of
 * them, is an error.  The entry lines are parsed by `threads` host threads
 * (0: all cores); mirroring, sorting, de-duplication and the row pointers
 * run on the device.  Errors: SK_INVALID_ARG with the reason in
 * sk_last_error(). */
SK_API sk_status sk_matrix_market_read(sk_matrix* out, const char* path, sk_dtype dtype,
                                int32_t threads);
SK_API sk_status sk_matrix_market_read_buffer(sk_matrix* out, const char* text, int64_t length,
                                       sk_dtype dtype, int32_t threads);

/* write_matrix_market(path, A) (matrix_market.hpp:119-150) of a CSR handle:
 * the banner "%%MatrixMarket matrix coordinate real general", the size line
 * and one "row col value" line per entry.  precision 0 prints values as the
 * reference's ostream does (6 significant digits); 17 round-trips FP64. */
SK_API sk_status sk_matrix_market_write(sk_matrix A, const char* path, int32_t precision,
                                 int32_t threads);

SK_API sk_status sk_matrix_destroy(sk_matrix A);

/* info[0..7] = format, dtype, nrow, ncol, nnz (stored entries), width
 * (ELL width / JAD diagonal count / BSR block count), device bytes held,
 * algorithmic bytes of one FP SpMV (the roofline byte model). */
SK_API sk_status sk_matrix_info(sk_matrix A, int64_t info[8]);

/* The device layout the product of a handle runs on (chosen at upload; the
 * values agree whichever it is):
 *   SK_LAYOUT_NATIVE    the handle's own format (CSR: row tiles);
 *   SK_LAYOUT_SELL      SELL-32 copy (CSR rows of at most 64 entries; 2x2
 *                       and 3x3 BSR);
 *   SK_LAYOUT_DIAGONALS diagonal copy (sk_matrix_add_diagonals);
 *   SK_LAYOUT_SPLIT     CSR split by row length (skewed rows);
 *   SK_LAYOUT_PANELS    CSR column panels (sk_matrix_add_panels: x staged
 *                       panel by panel in shared memory, every row summed
 *                       in column order). */
enum { SK_LAYOUT_NATIVE = 0, SK_LAYOUT_SELL = 1, SK_LAYOUT_DIAGONALS = 2, SK_LAYOUT_SPLIT = 3,
       SK_LAYOUT_PANELS = 4 };
SK_API sk_status sk_matrix_layout(sk_matrix A, int32_t* layout);

/* Adds an FP32 copy of the values of an FP64 CSR handle (indices shared),
 * used by the mixed-precision solver and the FP32 SpMV. */
SK_API sk_status sk_matrix_add_f32_values(sk_matrix A);

/* Adds a diagonal copy of a CSR handle whose entries lie on at most 16
 * diagonals c - r (a stencil in natural order) with every row's columns in
 * ascending order: the values of each 32-row slice stored diagonal by
 * diagonal, and a mask of the entries each row stores.  The later products
 * on the handle (sk_spmv, sk_spmv_host, the solvers' steps, the per-step
 * FP32 inner solve of the mixed solver) read it instead of the CSR arrays:
 * no column indices and no gathered x, and each row summed over its stored
 * entries in its CSR order, so the results keep their bits.  The persistent
 * FP32 inner solve of the mixed solver reads it too, at two CTAs per SM
 * (its dot products then sum in another order than over SELL-32).
 * No reference counterpart: a device layout of Compressed_row_matrix
 * (Compressed_row_matrix.hpp:20-132), as the SELL-32 copy is.  *built is 1
 * when the handle has the copy, 0 when its pattern does not qualify (more
 * than 16 diagonals, planes more than half empty, or a row whose columns
 * do not ascend); the handle is unchanged then. */
SK_API sk_status sk_matrix_add_diagonals(sk_matrix A, int* built);

/* Adds the column-panel copy of a CSR handle whose product is not already
 * summed in the reference's order (a handle without SELL-32 or diagonal
 * copy: rows longer than 64 entries).  The later products (sk_spmv,
 * sk_spmv_host, the solvers' steps) then sum every row, of any length,
 * entry after entry from 0 in ascending column order, as
 * sparse_blas.hpp:25-28 does, so they equal the reference's bit for bit:
 * each CTA walks column panels of x staged in shared memory with a running
 * sum per row of its block, and the matrix stream arrives by bulk copies.
 * It costs 10 (FP64) or 6 (FP32) bytes per entry beside the CSR arrays.
 * On the Zipf-row matrix of the sweep it runs at 0.79x the speed of the
 * default split product, which sums rows longer than 32 entries in a
 * fixed tree.  *built is 1 when the handle has the copy, 0 when it does
 * not qualify (SELL-32 or diagonal copy present, a row whose columns do
 * not ascend, or rows too many for a block's running sums); the handle is
 * unchanged then. */
SK_API sk_status sk_matrix_add_panels(sk_matrix A, int* built);

/* ---------------------------------------------------------------- */
/* SpMV: y = A x                                                     */
/* ---------------------------------------------------------------- */

/* multiply(A, x) on device vectors, in the handle's dtype.  Replaces
 * multiply(Compressed_row_matrix const&, span)  sparse_blas.hpp:19-35,
 * multiply(Ellpack_matrix const&, span)         spmv.hpp:119-140,
 * multiply(Block_sparse_row_matrix const&, span) spmv.hpp:148-174,
 * multiply(Jagged_diagonal_matrix const&, span) spmv.hpp:182-200. */
SK_API sk_status sk_spmv(sk_matrix A, const void* x_dev, void* y_dev, sk_stream s);

/* Same product with the FP32 value copy (sk_matrix_add_f32_values) on
 * float vectors. */
SK_API sk_status sk_spmv_f32(sk_matrix A, const float* x_dev, float* y_dev,
                      sk_stream s);

/* The drop-in form of multiply(A, span<T const>) -> std::vector<T>: x is
 * a host array of ncol values, y a host array of nrow values.  Copies x in,
 * runs the product and copies y out (synchronous).  A CSR product with at
 * least 8 MiB of y is pipelined in row chunks: each chunk's product starts
 * once the prefix of x its columns reach is on the device, and its rows of
 * y are copied out while later pieces of x still arrive (page-locked host
 * buffers let the two copy directions overlap).  The result is the same as
 * sk_spmv's, bit for bit. */
SK_API sk_status sk_spmv_host(sk_matrix A, const void* x_host, void* y_host);

/* ---------------------------------------------------------------- */
/* BLAS-1 on device vectors (deterministic reductions)                */
/* ---------------------------------------------------------------- */

/* std::inner_product(a, a+n, b, 0) as used by every solver
 * (e.g. conjugate_gradient.hpp:227, bicgstab.hpp:327-329). result is a host
 * double; the call synchronizes on s. */
SK_API sk_status sk_dot(sk_dtype dtype, int64_t n, const void* a_dev,
                 const void* b_dev, double* result, sk_stream s);
/* sqrt(<a, a>), e.g. bicgstab.hpp:333-336, fgmres.hpp:398-401. */
SK_API sk_status sk_nrm2(sk_dtype dtype, int64_t n, const void* a_dev,
                  double* result, sk_stream s);
/* y = alpha * x + y (conjugate_gradient.hpp:243-248 order). */
SK_API sk_status sk_axpy(sk_dtype dtype, int64_t n, double alpha, const void* x_dev,
                  void* y_dev, sk_stream s);
/* y = x + beta * y (conjugate_gradient.hpp:285-290 order). */
SK_API sk_status sk_xpay(sk_dtype dtype, int64_t n, const void* x_dev, double beta,
                  void* y_dev, sk_stream s);

/* ---------------------------------------------------------------- */
/* Preconditioners                                                   */
/* ---------------------------------------------------------------- */

/* jacobi(A) (sparkit/data/jacobi.hpp:27-35) on a CSR handle: inverse
 * diagonal kept on the device.  An exact zero diagonal entry fails with
 * SK_ZERO_DIAGONAL (the reference throws std::invalid_argument). */
SK_API sk_status sk_jacobi_create(sk_precond* out, sk_matrix A);

/* chebyshev_preconditioner(A, lmin, lmax, degree)
 * (sparkit/data/chebyshev_preconditioner.hpp:46-84) on a CSR handle.
 * The coefficients are computed on the host as the reference does. */
SK_API sk_status sk_chebyshev_create(sk_precond* out, sk_matrix A, double lambda_min,
                              double lambda_max, int64_t degree);

/* ---------------------------------------------------------------- */
/* Eigenvalue estimates (symmetric matrices)                         */
/* ---------------------------------------------------------------- */

/* Eigen_target (sparkit/data/eigen_target.hpp:13-20). */
typedef enum {
  SK_LARGEST_MAGNITUDE = 0,
  SK_SMALLEST_MAGNITUDE = 1,
  SK_LARGEST_ALGEBRAIC = 2,
  SK_SMALLEST_ALGEBRAIC = 3,
  SK_LARGEST_REAL = 4,
  SK_SMALLEST_REAL = 5
} sk_eigen_target;

/* Lanczos_config<T> (sparkit/data/lanczos.hpp:25-33); target is an
 * sk_eigen_target. */
typedef struct {
  int64_t num_eigenvalues;
  int64_t krylov_dimension;
  double tolerance;
  int64_t max_restarts;
  int32_t target;
  int32_t collect_residuals;
} sk_lanczos_config;

/* The scalars of Lanczos_result<T> (lanczos.hpp:39-47): count eigenvalues
 * (min(num_eigenvalues, krylov_dimension, n)), residual_count residual
 * norms of the last convergence test (0 when max_restarts is 0),
 * restart_residuals_count entries of restart_residuals (collect only). */
typedef struct {
  int64_t count;
  int64_t computed_restarts;
  int64_t converged_count;
  int64_t residual_count;
  int64_t restart_residuals_count;
  int32_t converged;
  int32_t status;
} sk_lanczos_summary;

/* lanczos(n, cfg, op) with op = multiply(A) (lanczos.hpp:495-503), A square
 * and symmetric, any format.  Host outputs: eigenvalues[count],
 * residual_norms[count] and restart_residuals[max_restarts] (each may be
 * NULL).  eigenvectors_dev (may be NULL): count device vectors of nrow
 * entries of A's dtype, one after another.  The n-length work runs on the
 * device; the tridiagonal eigensolve and restart arithmetic on the host.
 * The reorthogonalisation is the reference's modified Gram-Schmidt. */
SK_API sk_status sk_lanczos(sk_matrix A, const sk_lanczos_config* cfg, double* eigenvalues,
                     double* residual_norms, double* restart_residuals,
                     void* eigenvectors_dev, sk_lanczos_summary* out, sk_stream stream);

/* estimate_spectral_radius(n, multiply(A), num_iter) (conditioning.hpp:112-126;
 * the reference's default num_iter is 20).  This and sk_eigenvalue_bounds
 * reorthogonalise by block Gram-Schmidt (the same to rounding for the one
 * extreme eigenvalue they estimate). */
SK_API sk_status sk_spectral_radius(sk_matrix A, int64_t num_iter, double* rho);

/* estimate_eigenvalue_bounds(n, multiply(A), num_iter)
 * (conditioning.hpp:132-168; default num_iter 30): two Lanczos passes,
 * largest and smallest algebraic. */
SK_API sk_status sk_eigenvalue_bounds(sk_matrix A, int64_t num_iter, double* lambda_min,
                               double* lambda_max);

/* chebyshev_preconditioner(A, lambda_min, lambda_max, degree) with the
 * bounds from sk_eigenvalue_bounds(A, num_iter); bounds (may be NULL)
 * receives them. */
SK_API sk_status sk_chebyshev_create_auto(sk_precond* out, sk_matrix A, int64_t degree,
                                   int64_t num_iter, double bounds[2]);

/* z = M^{-1} r on device vectors: jacobi_apply (jacobi.hpp:44-51) or
 * chebyshev_preconditioner_apply (chebyshev_preconditioner.hpp:98-169).
 * A NULL precond is the identity (a copy). */
SK_API sk_status sk_precond_apply(sk_precond M, int64_t n, const void* r_dev,
                           void* z_dev, sk_stream s);

/* Copies the preconditioner's parameters to the host: the inverse
 * diagonal (Jacobi, n values) or the degree+1 coefficients (Chebyshev). */
SK_API sk_status sk_precond_values(sk_precond M, void* host_out, int64_t capacity,
                            int64_t* count);

SK_API sk_status sk_precond_destroy(sk_precond M);

/* No reference counterpart: an addition of this library.  The Chebyshev
 * apply z = p(A) r of sk_precond_apply, for callers that cannot allocate
 * device memory when they apply the preconditioner (a callback inside
 * another solver library's loop, where that library reserved all device
 * memory up front).  It takes the parameters of
 * sk_chebyshev_create directly and keeps its two work vectors in a static
 * device array instead of allocating them: A is a square CSR handle of at
 * most 1,048,576 rows (larger ones fail with SK_INVALID_ARG), degree is at
 * most 64, and every GPU that runs it holds that 16 MiB array until the
 * process exits.  Calls share the array, so calls that overlap on the GPU
 * race; serialize them.  Every call looks the array's device address up;
 * the first call on a device may load the module to do so and should come
 * before any stream capture.  Results are identical to
 * sk_precond_apply with a preconditioner from sk_chebyshev_create. */
SK_API sk_status sk_chebyshev_apply_noalloc(sk_matrix A, double lambda_min,
                                            double lambda_max, int64_t degree,
                                            const void* r_dev, void* z_dev,
                                            sk_stream s);

/* ---------------------------------------------------------------- */
/* Solvers                                                           */
/* ---------------------------------------------------------------- */

/* CGConfig<T>, sparkit/data/conjugate_gradient.hpp:48-74 */
typedef struct {
  double tolerance;
  int64_t restart_iterations;
  int64_t max_iterations;
  int32_t collect_residuals;
} sk_cg_config;

/* Bicgstab_config<T>, sparkit/data/bicgstab.hpp:25-42 */
typedef struct {
  double tolerance;
  int64_t max_iterations;
  int32_t collect_residuals;
} sk_bicgstab_config;

/* Fgmres_config<T>, sparkit/data/fgmres.hpp:25-47 */
typedef struct {
  double tolerance;
  int64_t restart_dimension;
  int64_t max_iterations;
  int32_t collect_residuals;
} sk_fgmres_config;

/* Cgs_config<T> (sparkit/data/cgs.hpp:25-42) and Minres_config<T>
 * (minres.hpp:25-45): tolerance, max_iterations, collect_residuals */
typedef struct {
  double tolerance;
  int64_t max_iterations;
  int32_t collect_residuals;
} sk_cgs_config;
typedef sk_cgs_config sk_minres_config;

/* Gmres_config<T>, sparkit/data/gmres.hpp:25-47 (the same fields) */
typedef struct {
  double tolerance;
  int64_t restart_dimension;
  int64_t max_iterations;
  int32_t collect_residuals;
} sk_gmres_config;

/* CGSummary / Bicgstab_summary / Fgmres_summary
 * (conjugate_gradient.hpp:27-40, bicgstab.hpp:50-63, fgmres.hpp:55-68).
 * The per-iteration residual norms go to the caller's history buffer
 * (capacity max_iterations); history_length says how many were written.
 * status is SK_OK, or SK_BREAKDOWN when a Krylov breakdown ended the solve
 * (the reference would loop or divide by zero there). */
typedef struct {
  double residual_norm;
  int64_t computed_iterations;
  int32_t converged;
  int32_t status;
  int64_t history_length;
} sk_summary;

/* conjugate_gradient(b, x, cfg, op, left, right)
 * (sparkit/data/conjugate_gradient.hpp:339-366) with op = multiply(A, .)
 * and left / right = a preconditioner handle or NULL (identity).  b and x
 * are device vectors in the handle's dtype; x holds the initial guess and
 * receives the solution.  history_host may be NULL. */
SK_API sk_status sk_cg_solve(sk_matrix A, sk_precond left, sk_precond right,
                      const void* b_dev, void* x_dev, const sk_cg_config* cfg,
                      sk_summary* out, double* history_host, sk_stream s);

/* bicgstab(b, x, cfg, op, left, right) (sparkit/data/bicgstab.hpp:383-410). */
SK_API sk_status sk_bicgstab_solve(sk_matrix A, sk_precond left, sk_precond right,
                            const void* b_dev, void* x_dev,
                            const sk_bicgstab_config* cfg, sk_summary* out,
                            double* history_host, sk_stream s);

/* fgmres(b, x, cfg, op, preconditioner) (sparkit/data/fgmres.hpp:452-470). */
SK_API sk_status sk_fgmres_solve(sk_matrix A, sk_precond M, const void* b_dev,
                          void* x_dev, const sk_fgmres_config* cfg,
                          sk_summary* out, double* history_host, sk_stream s);

/* gmres(b, x, cfg, op, left, right) (sparkit/data/gmres.hpp:400-429):
 * restarted GMRES(m) with M_L = left and M_R = right (NULL: identity).
 * Convergence on |g_{j+1}| / ||b|| as in the reference (the residual of
 * the left-preconditioned system over the unpreconditioned ||b||). */
SK_API sk_status sk_gmres_solve(sk_matrix A, sk_precond left, sk_precond right,
                                const void* b_dev, void* x_dev,
                                const sk_gmres_config* cfg, sk_summary* out,
                                double* history_host, sk_stream s);

/* cgs(b, x, cfg, op, left, right) (sparkit/data/cgs.hpp:374-395):
 * conjugate gradient squared; each step spends two matrix-vector products
 * and counts as two iterations, as in the reference. */
SK_API sk_status sk_cgs_solve(sk_matrix A, sk_precond left, sk_precond right,
                              const void* b_dev, void* x_dev, const sk_cgs_config* cfg,
                              sk_summary* out, double* history_host, sk_stream s);

/* minres(b, x, cfg, op, left, right) (sparkit/data/minres.hpp:397-418):
 * preconditioned MINRES with M = M_R M_L, for symmetric A (and SPD M);
 * convergence on the recurrence's |phi_bar| / ||b||. */
SK_API sk_status sk_minres_solve(sk_matrix A, sk_precond left, sk_precond right,
                                 const void* b_dev, void* x_dev,
                                 const sk_minres_config* cfg, sk_summary* out,
                                 double* history_host, sk_stream s);

/* Mixed precision (no reference counterpart; the reference solves in one
 * value type): FP64 iterative refinement around conjugate_gradient
 * (conjugate_gradient.hpp:347) instantiated for float.  Each outer step
 * forms r = b - A x in FP64, stops when ||r|| / ||b|| < tolerance, solves
 * A d = r / ||r|| in FP32 with (Jacobi-preconditioned when jacobi != 0) CG
 * to inner_tolerance on the FP32 copy of the values, and adds ||r|| d to x
 * in FP64.  A is an FP64 CSR handle; b and x are FP64 device vectors. */
typedef struct {
  double tolerance;        /* outer, on the true FP64 residual */
  double inner_tolerance;  /* FP32 CG relative tolerance */
  int64_t max_outer;
  int64_t max_inner;
  int32_t collect_residuals;  /* true residual norm per outer step */
  int32_t adaptive_last_step; /* tighten the inner tolerance of a step to
                                 half the remaining factor tol ||b|| / ||r||
                                 when that is below inner_tolerance */
  int32_t l2_window;          /* keep the FP32 inner vectors resident in L2
                                 (a persisting access-policy window on the
                                 handle's stream, this process only) */
  int32_t inner_kernel;       /* 0: each inner solve is one persistent
                                 cooperative launch when the handle has its
                                 SELL-32 copy (else per-step kernels);
                                 1: one kernel per CG step */
} sk_mixed_config;

typedef struct {
  double residual_norm;      /* true FP64 ||b - A x|| at exit */
  int64_t outer_iterations;
  int64_t inner_iterations;  /* FP32 CG iterations summed */
  int32_t converged;
  int32_t status;
  double setup_ms;           /* host wall time: FP32 copies, Jacobi, ||b|| */
  double inner_ms;           /* host wall time in the FP32 inner solves */
  double outer_ms;           /* host wall time in the FP64 residual / update */
  int32_t inner_kernel;      /* 0: persistent launch, 1: per-step kernels */
} sk_mixed_summary;

SK_API sk_status sk_mixed_cg_solve(sk_matrix A, int32_t jacobi,
                                   const double* b_dev, double* x_dev,
                                   const sk_mixed_config* cfg,
                                   sk_mixed_summary* out, double* history_host,
                                   sk_stream s);

/* Mixed-precision FGMRES(m) (no reference counterpart as a whole; the inner
 * solve is fgmres.hpp:96-428 in FP32): FP64 iterative refinement around an
 * FP32 FGMRES(m) inner solve.  FP64 stays in the outer residual b - A x,
 * the solution update and the inner Hessenberg least-squares problem
 * (Givens rotations, back substitution); the basis vectors, the products
 * (the handle's FP32 value copy, made on first use) and the Gram-Schmidt
 * sums are FP32.  M: NULL, Jacobi, Chebyshev (applied in FP32) or a
 * two-level preconditioner (applied in FP64); the learned network is
 * refused.  b and x are FP64 device vectors of an FP64 CSR handle. */
typedef struct {
  double tolerance;          /* outer, on the true FP64 residual */
  double inner_tolerance;    /* FP32 FGMRES relative tolerance on |g| */
  int64_t restart_dimension; /* m */
  int64_t max_outer;
  int64_t max_inner;         /* FP32 FGMRES iterations per outer step */
  int32_t collect_residuals; /* true residual norm per outer step */
  int32_t adaptive_last_step;
} sk_mixed_fgmres_config;

SK_API sk_status sk_mixed_fgmres_solve(sk_matrix A, sk_precond M, const double* b_dev,
                                       double* x_dev, const sk_mixed_fgmres_config* cfg,
                                       sk_mixed_summary* out, double* history_host,
                                       sk_stream s);

/* ---------------------------------------------------------------- */
/* Batched solves (no reference counterpart: the reference solves one */
/* system per call; the comparison is a loop of the plain solver)     */
/* ---------------------------------------------------------------- */

typedef struct sk_batch_s* sk_batch;

/* nsys independent SPD systems as the diagonal blocks of one CSR matrix
 * (FP32 values): system s owns rows [sys_offsets[s], sys_offsets[s+1]) and
 * every column index of those rows lies in the same range. */
SK_API sk_status sk_batch_create(sk_batch* out, int64_t nsys,
                                 const int64_t* sys_offsets,
                                 const int64_t* row_ptr,
                                 const int64_t* col_ind, const float* values);
SK_API sk_status sk_batch_destroy(sk_batch B);

typedef struct {
  double tolerance;          /* FP64 true relative residual per system */
  double inner_tolerance;    /* FP32 Jacobi-CG relative tolerance */
  int64_t max_outer;
  int64_t max_inner;
  int32_t adaptive_last_step;
  int32_t lanes_per_row;     /* 1, 2, 4 or 8 (from sk_batched_autotune) */
  int32_t threads_per_cta;   /* 256, 512 or 1024 */
} sk_batch_config;

/* Device arrays of nsys entries each, written by the solve. */
typedef struct {
  int32_t* inner_iterations;
  int32_t* outer_iterations;
  double* relative_residual;
  int32_t* converged;
} sk_batch_results;

/* Solves every system in one persistent launch (FP32 Jacobi-CG inside FP64
 * iterative refinement, conjugate_gradient.hpp:122-312 per system), one CTA
 * per system at a time taken from a longest-first queue.  The launch is
 * captured into a CUDA graph and replayed while the pointers and settings
 * stay the same.  b and x are FP64 device vectors over all rows; x holds the
 * initial guesses and receives the solutions. */
SK_API sk_status sk_batched_cg_solve(sk_batch B, const double* b_dev,
                                     double* x_dev, const sk_batch_config* cfg,
                                     sk_batch_results* res, sk_stream s);

/* Times every (lanes_per_row, threads_per_cta) variant on the `sample`
 * largest systems and returns the fastest; ms_out (may be NULL) receives
 * sk_batched_variant_count() timings.  x is overwritten with zeros. */
SK_API sk_status sk_batched_autotune(sk_batch B, const double* b_dev,
                                     double* x_dev, const sk_batch_config* cfg,
                                     sk_batch_results* res, int64_t sample,
                                     int32_t* lanes_per_row,
                                     int32_t* threads_per_cta, double* ms_out);
SK_API int32_t sk_batched_variant_count(void);

/* ---------------------------------------------------------------- */
/* Learned variable preconditioner for FGMRES (no reference           */
/* counterpart: fgmres, sparkit/data/fgmres.hpp:452-470, accepts any   */
/* callable as its variable preconditioner; this is one such callable */
/* with the training that produces it)                                */
/* ---------------------------------------------------------------- */

/* A convolutional encoder-decoder over the 2-D grid of a 5-point matrix:
 * nine 3x3 convolutions over four levels (16, 32, 64, 64 channels), BF16
 * weights and activations, FP32 accumulation and FP32 master weights.
 * It maps a residual to an approximation of the error.  Created with
 * seeded He-initialised weights. */
typedef struct sk_net_s* sk_net;
SK_API sk_status sk_net_create(sk_net* out, uint64_t seed);
SK_API sk_status sk_net_destroy(sk_net N);
SK_API int64_t sk_net_param_count(void);
/* Flat FP32 parameters, layer by layer: W[cout][9][cin] (tap 3 ky + kx
 * reads pixel (y + ky - 1, x + kx - 1)) then b[cout]. */
SK_API sk_status sk_net_get_params(sk_net N, float* host, int64_t capacity);
SK_API sk_status sk_net_set_params(sk_net N, const float* host, int64_t count);
/* Test hook: run the convolutions on mma.sync instead of tcgen05 (the two
 * must agree; the tests compare them). */
SK_API sk_status sk_net_set_legacy_mma(sk_net N, int32_t on);
/* SK_TIMEOUT when a network kernel gave up a bounded wait (then clears). */
SK_API sk_status sk_net_status(sk_net N);

/* Training set of (residual, error) pairs on an nx x ny grid, stored FP32
 * on the device, each tied to an instance (the coefficient planes of its
 * matrix). */
typedef struct sk_pairs_s* sk_pairs;
SK_API sk_status sk_pairs_create(sk_pairs* out, int64_t nx, int64_t ny, int64_t capacity,
                                 int32_t max_instances);
SK_API sk_status sk_pairs_destroy(sk_pairs D);
SK_API sk_status sk_pairs_count(sk_pairs D, int64_t* count);
/* Registers the FP64 CSR 5-point matrix A of an nx x ny grid (row y*nx+x). */
SK_API sk_status sk_pairs_add_instance(sk_pairs D, sk_matrix A, int32_t* instance);
SK_API sk_status sk_pairs_add(sk_pairs D, int32_t instance, const double* r_dev,
                              const double* e_dev, sk_stream s);
/* Runs the plain Jacobi-FGMRES(restart) on A x = b from x = 0 one restart
 * cycle at a time and adds (b - A x, xstar - x) after every cycle, for at
 * most `cycles` cycles; xstar is the exact solution (b = A xstar). */
SK_API sk_status sk_learned_harvest(sk_pairs D, int32_t instance, sk_matrix A, const double* b_dev,
                                    const double* xstar_dev, int64_t restart, int64_t cycles,
                                    int64_t* added);

/* Adam on the loss
 *   mean_b |A (y_b - e_b / s_b)|^2 / |r_b / s_b|^2 + mu |y_b - e_b / s_b|^2 / |e_b / s_b|^2
 * (y_b the network's output for pair b, s_b the RMS of D^-1 r_b), batches
 * drawn uniformly with the seed, learning rate cosine-decayed from lr to
 * lr * lr_final_ratio. */
typedef struct {
  int64_t steps;
  int32_t batch;
  float lr;
  float lr_final_ratio;
  float beta1, beta2, eps;
  double mu;
  uint64_t seed;
} sk_train_config;

typedef struct {
  double first_loss, last_loss;
  double ms;  /* host wall time of the whole training */
  int64_t steps;
} sk_train_summary;

SK_API sk_status sk_net_train(sk_net N, sk_pairs D, const sk_train_config* cfg,
                              sk_train_summary* out, double* loss_history);
/* Loss of one batch and its gradient (FP32, sk_net_param_count() values)
 * without an update: the gradient check of the tests. */
SK_API sk_status sk_net_loss_grad(sk_net N, sk_pairs D, const int32_t* pairs_host, int32_t batch,
                                  double mu, double* loss, float* grad_host, int64_t capacity);

/* The network as a preconditioner of the FP64 CSR 5-point matrix A on an
 * nx x ny grid: z = s net(D^-1 r / s, off-diagonals / diagonal) with
 * s = rms(D^-1 r).  Applied by sk_precond_apply and by FGMRES. */
SK_API sk_status sk_learned_create(sk_precond* out, sk_matrix A, sk_net net, int64_t nx,
                                   int64_t ny);
/* The six coefficient planes (d, w, e, s, n, 1/d; FP32, 6 n values). */
SK_API sk_status sk_learned_planes(sk_precond M, float* host, int64_t capacity);

/* No reference counterpart (fgmres.hpp:96-428 accepts any callable as its
 * variable preconditioner): a two-level preconditioner for the FP64 CSR
 * matrix A on an nx x ny grid, with P piecewise constant over agg x agg
 * aggregates of cells (agg divides nx and ny, at most 4096 aggregates) and
 * Ac = P^T A P the Galerkin coarse operator, inverted at set-up (banded LU
 * without pivoting; a zero pivot fails with SK_INVALID_ARG).
 *   default:        z = S(r); z += P Ac^-1 P^T (r - A z)
 *                   [SK_TWOLEVEL_POST_SMOOTH: z += S(r - A z)]
 *   COARSE_FIRST:   z = P Ac^-1 P^T r; z += S(r - A z)
 * S is `smoother` (Jacobi, Chebyshev or learned, FP64, not owned: destroy
 * it after this one) or NULL (the coarse correction alone).  Applied by
 * sk_precond_apply and by the FGMRES calls. */
#define SK_TWOLEVEL_POST_SMOOTH 1
#define SK_TWOLEVEL_COARSE_FIRST 2
SK_API sk_status sk_twolevel_create(sk_precond* out, sk_matrix A, sk_precond smoother,
                                    int64_t nx, int64_t ny, int64_t agg, int32_t flags);

/* fgmres with M as the variable preconditioner and a fallback: after a
 * restart cycle whose final residual estimate is above stall_ratio times
 * its starting residual, the remaining cycles use `fallback` (Jacobi or
 * Chebyshev).  *switched_at (may be NULL) receives the first cycle run with
 * the fallback, or -1. */
SK_API sk_status sk_fgmres_fallback_solve(sk_matrix A, sk_precond M, sk_precond fallback,
                                          const double* b_dev, double* x_dev,
                                          const sk_fgmres_config* cfg, double stall_ratio,
                                          sk_summary* out, double* history_host,
                                          int64_t* switched_at, sk_stream s);

/* Host-buffer forms of the three solvers (b and x in host memory, copied
 * in and out inside the call): the drop-in boundary of the C++ overloads. */
SK_API sk_status sk_cg_solve_host(sk_matrix A, sk_precond left, sk_precond right,
                           const void* b_host, void* x_host,
                           const sk_cg_config* cfg, sk_summary* out,
                           double* history_host);
SK_API sk_status sk_bicgstab_solve_host(sk_matrix A, sk_precond left,
                                 sk_precond right, const void* b_host,
                                 void* x_host, const sk_bicgstab_config* cfg,
                                 sk_summary* out, double* history_host);
SK_API sk_status sk_fgmres_solve_host(sk_matrix A, sk_precond M, const void* b_host,
                               void* x_host, const sk_fgmres_config* cfg,
                               sk_summary* out, double* history_host);
SK_API sk_status sk_cgs_solve_host(sk_matrix A, sk_precond left, sk_precond right,
                                   const void* b_host, void* x_host, const sk_cgs_config* cfg,
                                   sk_summary* out, double* history_host);
SK_API sk_status sk_minres_solve_host(sk_matrix A, sk_precond left, sk_precond right,
                                      const void* b_host, void* x_host,
                                      const sk_minres_config* cfg, sk_summary* out,
                                      double* history_host);
SK_API sk_status sk_gmres_solve_host(sk_matrix A, sk_precond left, sk_precond right,
                                     const void* b_host, void* x_host,
                                     const sk_gmres_config* cfg, sk_summary* out,
                                     double* history_host);

#ifdef __cplusplus
}
#endif
#endif /* SPARKIT_B200_H */
