// sk_vec.cuh -- one-pass element-wise kernels with fused, deterministic
// grid reductions.  A pass is a functor Op with
//   static constexpr int kNR;                 fused reductions
//   bool prepare(const Scalars*)              load scalars; false = skip
//   void operator()(i64 i, double* red)      element i
//   void finalize(const double* total)       last CTA, thread 0
// and runs as vec_kernel<Op> over [0, n) with a grid that depends on n only
// (so that the reduction tree, and hence the rounding, is reproducible).
#pragma once

#include "sk_kernels.cuh"

namespace sk {

inline int vec_grid(i64 n) {
  i64 g = (n + kThreads - 1) / kThreads;
  if (g > 148 * 8) g = 148 * 8;
  if (g < 1) g = 1;
  return static_cast<int>(g);
}

template <class Op>
__global__ void __launch_bounds__(kThreads) vec_kernel(i64 n, Op op, RedWs ws, const Scalars* sc) {
  constexpr int NR = Op::kNR;
  if (!op.prepare(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  const i64 stride = static_cast<i64>(gridDim.x) * kThreads;
  i64 i = static_cast<i64>(blockIdx.x) * kThreads + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    op(i, red);
    op(i + stride, red);
    op(i + 2 * stride, red);
    op(i + 3 * stride, red);
  }
  for (; i < n; i += stride) op(i, red);
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { op.finalize(t); });
  }
}

template <class Op>
inline void launch_vec(i64 n, Op const& op, RedWs ws, const Scalars* sc, cudaStream_t st) {
  SK_LAUNCH(vec_kernel<Op>, vec_grid(n), kThreads, 0, st, n, op, ws, sc);
}

// Single-thread kernel for the small scalar work of the solvers (Givens
// rotations, back substitution).
template <class Op>
__global__ void scalar_kernel(Op op) {
  op();
}

// ------------------------------------------------------------------
// Plain BLAS-1 passes (used by the C ABI's standalone calls)
// ------------------------------------------------------------------
template <typename T>
struct OpDot {
  static constexpr int kNR = 1;
  const T* a;
  const T* b;
  double* out;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double* red) const {
    red[0] += static_cast<double>(mul(a[i], b[i]));
  }
  __device__ void finalize(const double* t) const { *out = t[0]; }
};

template <typename T>
struct OpAxpy {  // y = alpha * x + y
  static constexpr int kNR = 0;
  T alpha;
  const T* x;
  T* y;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double*) const { y[i] = add(mul(alpha, x[i]), y[i]); }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpXpay {  // y = x + beta * y
  static constexpr int kNR = 0;
  T beta;
  const T* x;
  T* y;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double*) const { y[i] = add(x[i], mul(beta, y[i])); }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpScaleCopy {  // z = c * r
  static constexpr int kNR = 0;
  T c;
  const T* r;
  T* z;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double*) const { z[i] = mul(c, r[i]); }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpJacobi {  // z = inv_d * r   (jacobi.hpp:44-51)
  static constexpr int kNR = 0;
  const T* inv_d;
  const T* r;
  T* z;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double*) const { z[i] = mul(inv_d[i], r[i]); }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpCopy {
  static constexpr int kNR = 0;
  const T* a;
  T* b;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double*) const { b[i] = a[i]; }
  __device__ void finalize(const double*) const {}
};

// ------------------------------------------------------------------
// Chebyshev preconditioner pieces (chebyshev_preconditioner.hpp:98-169).
// Abar v = (2 A v - (lmax + lmin) v) / (lmax - lmin).
// ------------------------------------------------------------------
template <typename T>
struct ChebCoef {
  T sum, diff;
};

// b_d = c_d r ; b_{d+1} = 0
template <typename T>
struct OpChebInit {
  static constexpr int kNR = 0;
  T cd;
  const T* r;
  T* b_curr;
  T* b_prev;
  const Scalars* skip;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double*) const {
    b_curr[i] = mul(cd, r[i]);
    b_prev[i] = T(0);
  }
  __device__ void finalize(const double*) const {}
};

// SpMV epilogue: b_new = c_k r + 2 Abar b_curr - b_prev, written over b_prev.
template <typename T>
struct EpiChebStep {
  static constexpr int kNR = 0;
  T ck, sum, diff;
  const T* r;
  const T* b_curr;
  T* b_prev;  // in: b_{k+2}; out: b_k
  __device__ void operator()(int row, T av, double*) const {
    T abar = dvd(sub(mul(T(2), av), mul(sum, b_curr[row])), diff);
    b_prev[row] = sub(add(mul(ck, r[row]), mul(T(2), abar)), b_prev[row]);
  }
  __device__ void finalize(const double*) const {}
};

// Final Clenshaw step: z = c_0 r + Abar b_1 - b_2.
template <typename T>
struct EpiChebFinal {
  static constexpr int kNR = 0;
  T c0, sum, diff;
  const T* r;
  const T* b_curr;
  const T* b_prev;
  T* z;
  __device__ void operator()(int row, T av, double*) const {
    T abar = dvd(sub(mul(T(2), av), mul(sum, b_curr[row])), diff);
    z[row] = sub(add(mul(c0, r[row]), abar), b_prev[row]);
  }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpScaleCopySkip {  // z = c * r, skipped once the solve is done
  static constexpr int kNR = 0;
  T c;
  const T* r;
  T* z;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ void operator()(i64 i, double*) const { z[i] = mul(c, r[i]); }
  __device__ void finalize(const double*) const {}
};

// z = p(A) r on device.  work holds 2 n-vectors.  `sc` (may be null) makes
// every launch a no-op once a solve has finished.  vals32 selects the FP32
// value copy of an FP64 CSR handle (mixed precision, T = float).
template <typename T>
void chebyshev_apply_device(const sk_precond_s* M, const T* r, T* z, T* work, RedWs ws,
                            const Scalars* sc, cudaStream_t st, const T* vals_override = nullptr) {
  const sk_matrix_s* A = M->A;
  const i64 n = A->nrow;
  const T lmin = static_cast<T>(M->lambda_min), lmax = static_cast<T>(M->lambda_max);
  const T sum = lmax + lmin;
  const T diff = lmax - lmin;
  const i64 d = M->degree;
  auto c = [&](i64 k) { return static_cast<T>(M->coeffs[static_cast<size_t>(k)]); };
  if (d == 0 || diff == T(0)) {
    launch_vec(n, OpScaleCopySkip<T>{c(0), r, z}, ws, sc, st);
    return;
  }
  T* b_prev = work;
  T* b_curr = work + n;
  launch_vec(n, OpChebInit<T>{c(d), r, b_curr, b_prev, nullptr}, ws, sc, st);
  for (i64 k = d - 1; k >= 1; --k) {
    launch_spmv<T>(A, b_curr, EpiChebStep<T>{c(k), sum, diff, r, b_curr, b_prev}, ws, sc, st,
                   vals_override);
    T* t = b_prev;
    b_prev = b_curr;
    b_curr = t;
  }
  launch_spmv<T>(A, b_curr, EpiChebFinal<T>{c(0), sum, diff, r, b_curr, b_prev, z}, ws, sc, st,
                 vals_override);
}

}  // namespace sk
