// sk_twolevel.cuh -- the two-level grid preconditioner (smoother plus an
// aggregation coarse-grid correction) used by the preconditioner dispatch.
#pragma once

#include "sk_internal.cuh"

namespace sk {

void precond_apply_dispatch(const sk_precond_s* M, sk_dtype dt, i64 n, const void* r, void* z,
                            RedWs ws, const Scalars* sc, cudaStream_t st);

// Whether S can serve as the smoother (FP64 Jacobi, Chebyshev or learned).
bool twolevel_smoother_ok(const sk_precond_s* S);
// z = M^-1 r for a two-level preconditioner (kind 4); kernels only.
void twolevel_apply(const sk_precond_s* M, const double* r, double* z, RedWs ws, const Scalars* sc,
                    cudaStream_t st);
// Frees the coarse inverse and the work vectors (not the smoother).
void twolevel_release(sk_precond_s* M);

}  // namespace sk
