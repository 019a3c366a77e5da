// sk_vec.cuh -- one-pass element-wise kernels with fused, deterministic
// grid reductions.  A pass is a functor Op with
//   static constexpr int kNR;                 fused reductions
//   struct In;                                the inputs of one element
//   bool prepare(const Scalars*)              load scalars; false = skip
//   In load(i64 i)                            read element i's inputs
//   void apply(i64 i, In const&, double* red) compute and store element i
//   void finalize(const double* total)       last CTA, thread 0
// vec_kernel<Op> gives each thread kUnroll elements (stride apart) and reads
// all their inputs before any store, so that the loads are in flight
// together (the stores could alias the inputs, so a fused load-compute-store
// loop would serialize them).  The grid depends on n only, so the reduction
// tree, and hence the rounding, is reproducible.
#pragma once

#include <cmath>

#include "sk_kernels.cuh"

namespace sk {

constexpr int kUnroll = 4;  // elements per thread per round (8 for small inputs)

// One wave of 8 CTAs per SM at most (148 SMs on B200); the count depends
// on n only.
inline int vec_grid(i64 n) {
  i64 g = (n + kThreads * kUnroll - 1) / (kThreads * kUnroll);
  if (g > 148 * 8) g = 148 * 8;
  if (g < 1) g = 1;
  return static_cast<int>(g);
}

template <class Op>
constexpr int vec_unroll() {
  return sizeof(typename Op::In) <= 12 ? 2 * kUnroll : kUnroll;
}

template <class Op>
__global__ void __launch_bounds__(kThreads, 4) vec_kernel(i64 n, Op op, RedWs ws, const Scalars* sc) {
  constexpr int NR = Op::kNR;
  if (!op.prepare(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  // Each warp takes contiguous segments of 32 * U elements; lane l handles
  // elements seg + 32 u + l.  The U elements of a thread are thus a
  // compile-time distance apart (one address per array plus immediate
  // offsets), and every load instruction reads 32 consecutive elements.
  constexpr int U = vec_unroll<Op>();
  constexpr i64 SEG = 32 * U;
  const int lane = threadIdx.x & 31;
  const i64 warp = (static_cast<i64>(blockIdx.x) * kThreads + threadIdx.x) >> 5;
  const i64 nwarps = static_cast<i64>(gridDim.x) * (kThreads / 32);
  for (i64 seg = warp * SEG; seg < n; seg += nwarps * SEG) {
    const i64 i0 = seg + lane;
    typename Op::In in[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const i64 i = i0 + 32 * u;
      if (i < n) in[u] = op.load(i);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const i64 i = i0 + 32 * u;
      if (i < n) reduce_terms<NR>(ws, i, red, [&](double* rr) { op.apply(i, in[u], rr); });
    }
  }
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
  struct In { T a, b; };
  const T* a;
  const T* b;
  double* out;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {a[i], b[i]}; }
  __device__ void apply(i64, In const& v, double* red) const { red[0] += static_cast<double>(mul(v.a, v.b)); }
  __device__ void finalize(const double* t) const { *out = t[0]; }
};

template <typename T>
struct OpAxpy {  // y = alpha * x + y
  static constexpr int kNR = 0;
  struct In { T x, y; };
  T alpha;
  const T* x;
  T* y;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {x[i], y[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { y[i] = add(mul(alpha, v.x), v.y); }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpXpay {  // y = x + beta * y
  static constexpr int kNR = 0;
  struct In { T x, y; };
  T beta;
  const T* x;
  T* y;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {x[i], y[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { y[i] = add(v.x, mul(beta, v.y)); }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpJacobi {  // z = inv_d * r   (jacobi.hpp:44-51)
  static constexpr int kNR = 0;
  struct In { T d, r; };
  const T* inv_d;
  const T* r;
  T* z;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {inv_d[i], r[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { z[i] = mul(v.d, v.r); }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct OpCopy {
  static constexpr int kNR = 0;
  struct In { T a; };
  const T* a;
  T* b;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {a[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { b[i] = v.a; }
  __device__ void finalize(const double*) const {}
};

// ------------------------------------------------------------------
// Chebyshev preconditioner pieces (chebyshev_preconditioner.hpp:98-169).
// Abar v = (2 A v - (lmax + lmin) v) / (lmax - lmin).
// ------------------------------------------------------------------
// b_d = c_d r ; b_{d+1} = 0
template <typename T>
struct OpChebInit {
  static constexpr int kNR = 0;
  struct In { T r; };
  T cd;
  const T* r;
  T* b_curr;
  T* b_prev;
  const Scalars* skip;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {r[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const {
    b_curr[i] = mul(cd, v.r);
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
  struct In { T r; };
  T c;
  const T* r;
  T* z;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {r[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { z[i] = mul(c, v.r); }
  __device__ void finalize(const double*) const {}
};

// Chebyshev coefficients of 1/lambda on [lmin, lmax]: the discrete cosine
// sampling of chebyshev_preconditioner.hpp:53-73, evaluated on the host in
// the value type T with the C library's cos, written into out[0..degree]
// (the caller's array: nothing is allocated).
template <typename T>
void chebyshev_coefficients(T lmin, T lmax, i64 degree, double* out) {
  const i64 d = degree;
  const i64 N = d + 1 > 64 ? d + 1 : 64;
  const T pi = static_cast<T>(3.141592653589793238462643383279502884L);
  const T center = (lmax + lmin) / T(2);
  const T half_width = (lmax - lmin) / T(2);
  for (i64 k = 0; k <= d; ++k) {
    T ck = T(0);
    for (i64 j = 0; j < N; ++j) {
      T tj = std::cos(pi * (T(j) + T(0.5)) / T(N));
      T lj = center + half_width * tj;
      T fj = T(1) / lj;
      T cos_k = std::cos(pi * T(k) * (T(j) + T(0.5)) / T(N));
      ck += fj * cos_k;
    }
    out[k] = static_cast<double>(T(2) * ck / T(N));
  }
  out[0] = static_cast<double>(static_cast<T>(out[0]) * T(0.5));
}

// z = p(A) r by the Clenshaw recurrence of chebyshev_preconditioner.hpp:98-169,
// with the coefficients co[0..d] and two n-vectors of work, w0 and w1, owned
// by the caller.  `sc` (may be null) makes every launch a no-op once a solve
// has finished.  vals_override selects the FP32 value copy of an FP64 CSR
// handle (mixed precision, T = float).
template <typename T>
void chebyshev_clenshaw(const sk_matrix_s* A, const double* co, i64 d, T lmin, T lmax, const T* r, T* z,
                        T* w0, T* w1, RedWs ws, const Scalars* sc, cudaStream_t st,
                        const T* vals_override = nullptr) {
  const i64 n = A->nrow;
  const T sum = lmax + lmin;
  const T diff = lmax - lmin;
  auto c = [&](i64 k) { return static_cast<T>(co[k]); };
  if (d == 0 || diff == T(0)) {
    launch_vec(n, OpScaleCopySkip<T>{c(0), r, z}, ws, sc, st);
    return;
  }
  T* b_prev = w0;
  T* b_curr = w1;
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

// z = M^{-1} r for a Chebyshev preconditioner handle; work holds 2 n-vectors.
template <typename T>
void chebyshev_apply_device(const sk_precond_s* M, const T* r, T* z, T* work, RedWs ws,
                            const Scalars* sc, cudaStream_t st, const T* vals_override = nullptr) {
  chebyshev_clenshaw<T>(M->A, M->coeffs.data(), M->degree, static_cast<T>(M->lambda_min),
                        static_cast<T>(M->lambda_max), r, z, work, work + M->A->nrow, ws, sc, st,
                        vals_override);
}

}  // namespace sk
