// sk_learned.cuh -- entry points of the learned preconditioner used by the
// preconditioner dispatch (sk_ops.cu) and the FGMRES driver.
#pragma once

#include "sk_internal.cuh"

namespace sk {

// z = s * net(features(v)) for an FP64 vector on the precond's grid.
sk_status learned_apply(const sk_precond_s* M, const double* v, double* z, cudaStream_t st);
// The same with z += s * net(...) when `add`, and with the scale s = rms(v /
// d) already in learned_scale_slot(M) when `scale_ready` (a fused reduction
// of the kernel that produced v wrote it).
sk_status learned_apply_ex(const sk_precond_s* M, const double* v, double* z, cudaStream_t st, bool add,
                           bool scale_ready);
// Where an apply on M's grid reads the scale s (one double); null when the
// network's workspace cannot be set up.
double* learned_scale_slot(const sk_precond_s* M);
// Allocates everything an apply on M's grid needs and sets the kernels'
// attributes, so that applies can then be captured into a CUDA graph.
sk_status learned_prepare(const sk_precond_s* M);
// Frees the coefficient planes of a learned preconditioner.
void learned_release(sk_precond_s* M);
// Coefficient planes (d, w, e, s, n, 1/d) of a 5-point FP64 CSR matrix on
// an nx x ny grid; SK_INVALID_ARG when the matrix is not such a stencil.
sk_status grid_planes(sk_matrix A, int64_t nx, int64_t ny, float* coef, cudaStream_t st);

}  // namespace sk
