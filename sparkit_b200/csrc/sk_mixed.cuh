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

// Whether the handle can run the persistent inner solve: a CSR handle with
// its SELL-32 copy and FP32 values, and a device that can co-schedule the
// grid (cooperative launch).
bool inner_persistent_ok(sk_matrix A);

// Scratch of the persistent solve: the grid-barrier words and the
// per-CTA reduction slots.
size_t inner_persistent_scratch(sk_matrix A);

// Solves A d = r0 from d = 0 with Jacobi (inv_d != null) or unpreconditioned
// CG in FP32, the reference iteration (conjugate_gradient.hpp:122-312 with
// restart_iterations = max_iters: the true residual only at k = 0), until
// ||r|| / ||r0|| < tol on the recursive residual or max_iters.  r holds r0 on
// entry and the final residual on exit; p and q are work vectors of n
// floats; scratch holds inner_persistent_scratch(A) bytes.  Synchronous.
sk_status inner_cg_persistent(sk_matrix A, const float* inv_d, float* r, float* d, float* p, float* q,
                              void* scratch, double tol, long long max_iters, cudaStream_t st,
                              InnerResult* out);

}  // namespace sk
