// sk_mixed.cuh -- the FP32 inner conjugate-gradient solve of the
// mixed-precision solver as one persistent cooperative launch.
#pragma once

#include "sk_internal.cuh"

namespace sk {

struct InnerResult {
  long long iterations = 0;
  int converged = 0;
  double rnorm = 0;  // FP32 recursive residual norm at exit
};

// Whether the handle can run the persistent inner solve on a device that
// can co-schedule the grid (cooperative launch).  Unscaled: a CSR handle
// with its SELL-32 copy and FP32 values or its FP32 diagonal copy.
// Scaled: after inner_sym_prepare succeeded.
bool inner_persistent_ok(sk_matrix A, bool scaled);

// Forms, once per handle, the symmetrically scaled FP32 copy S = D^-1/2 A
// D^-1/2 (without its unit diagonal) and 1 / sqrt(a_ii).  S is stored as
// diagonal planes when the pattern has at most 16 diagonals whose planes
// are at most half empty (whether or not the handle keeps its own diagonal
// copy), else as SELL-32 (rows of at most 255 off-diagonal entries, at
// most a quarter of padding).  *ok is false when S cannot be formed (an
// FP32 handle, a diagonal entry absent or not positive, neither layout).
sk_status inner_sym_prepare(sk_matrix A, cudaStream_t st, bool* ok);

// 1 / sqrt(a_ii) (FP64, n values) after inner_sym_prepare succeeded.
const double* inner_sym_isq(sk_matrix A);

// Scratch of the persistent solve: the grid-barrier words and the
// per-CTA reduction slots.
size_t inner_persistent_scratch(sk_matrix A);

// CG in FP32 until ||r|| / ||r0|| < tol on the recursive residual of
// A d = r0 or max_iters (conjugate_gradient.hpp:122-312 with
// restart_iterations = max_iters: the true residual only at k = 0).
// scaled: the Jacobi-preconditioned solve, run as CG on S y = r (r holds
// D^-1/2 r0 on entry, d receives y; the caller scales both); otherwise
// unpreconditioned CG on A.  r holds the final residual on exit; p and q
// are work vectors of n floats (16-byte aligned); scratch holds
// inner_persistent_scratch(A) bytes.  Synchronous.
sk_status inner_cg_persistent(sk_matrix A, bool scaled, float* r, float* d, float* p, float* q, void* scratch,
                              double tol, long long max_iters, cudaStream_t st, InnerResult* out);

// Plain FP64 CG (Jacobi or identity left preconditioner, identity right,
// the true residual at k = 0 only) as one cooperative launch: for FP64 CSR
// handles with SELL-32 of at most kCg64MaxRows rows, on a device that can
// co-schedule the grid, outside the sequential summation order.
constexpr long long kCg64MaxRows = 262144;
bool cg64_persistent_ok(sk_matrix A);

// Runs the whole solve: sc holds bnorm, tol and max_iters on entry and
// iters, converged, done, rnorm, rz, alpha, beta and hist_len on exit; r,
// p0, p1, q are work vectors of n values; invd is the Jacobi inverse diagonal
// or null; hist receives one residual norm per step when not null; scratch
// holds inner_persistent_scratch(A) bytes.  Synchronous; SK_TIMEOUT when a
// grid barrier wait runs out.
sk_status cg64_persistent(sk_matrix A, const double* b, double* x, double* r, double* p0, double* p1, double* q,
                          const double* invd, double* hist, Scalars* sc, void* scratch, cudaStream_t st);

// Plain FP64 BiCGSTAB (identity or Jacobi on either side) as one
// cooperative launch, under the same conditions as cg64_persistent_ok.
bool bi64_persistent_ok(sk_matrix A);

// Runs the whole solve: sc holds bnorm, tol and max_iters on entry and
// iters, converged, status, done, rnorm, rho, rho_new, alpha, omega and
// hist_len on exit; vec holds ten work vectors of n values (r, r_hat, two
// p, two v, p_hat, s, s_hat, t); invl / invr are the Jacobi inverse
// diagonals or null; hist receives one norm per half step when not null;
// scratch holds inner_persistent_scratch(A) bytes.  Synchronous;
// SK_TIMEOUT when a grid barrier wait runs out.
sk_status bi64_persistent(sk_matrix A, const double* b, double* x, double* const* vec, const double* invl,
                          const double* invr, double* hist, Scalars* sc, void* scratch, cudaStream_t st);

// Plain FP64 CGS (identity or Jacobi on either side) as one cooperative
// launch, under the same conditions as cg64_persistent_ok.
bool cgs64_persistent_ok(sk_matrix A);

// Runs the whole solve: sc holds bnorm, tol and max_iters on entry and
// iters, converged, done, rnorm, rho, alpha, beta, skip and hist_len on
// exit; vec holds seven work vectors of n values (r, r_hat, two p, u, q,
// q_hat); invl / invr are the Jacobi inverse diagonals or null; hist
// receives one norm per step when not null; scratch holds
// inner_persistent_scratch(A) bytes.  Synchronous; SK_TIMEOUT when a grid
// barrier wait runs out.
sk_status cgs64_persistent(sk_matrix A, const double* b, double* x, double* const* vec, const double* invl,
                           const double* invr, double* hist, Scalars* sc, void* scratch, cudaStream_t st);

// Plain FP64 MINRES (identity or Jacobi on either side) as one
// cooperative launch, under the same conditions as cg64_persistent_ok.
bool min64_persistent_ok(sk_matrix A);

// Runs the whole solve: sc holds bnorm, tol and max_iters on entry and
// iters, converged, done, rnorm and hist_len on exit; vec holds seven work
// vectors of n values (v, v_prev, z, w, q, d, d_prev); invl / invr are the
// Jacobi inverse diagonals or null; hist receives one norm per step when
// not null; scratch holds inner_persistent_scratch(A) bytes.  Synchronous;
// SK_TIMEOUT when a grid barrier wait runs out.
sk_status min64_persistent(sk_matrix A, const double* b, double* x, double* const* vec, const double* invl,
                           const double* invr, double* hist, Scalars* sc, void* scratch, cudaStream_t st);

}  // namespace sk
