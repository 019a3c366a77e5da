// sk_lanczos.cu -- implicitly restarted Lanczos for symmetric matrices on the
// device, and the eigenvalue estimates built on it: the spectral radius and
// the [lambda_min, lambda_max] bounds that set up a Chebyshev
// preconditioner without hand-picked bounds.
//
// Follows sparkit/data/lanczos.hpp:64-503 (LanczosSolver) and
// conditioning.hpp:112-168.  The n-length work runs on the GPU, fused as in
// the Krylov solvers:
//   w = A v_j with alpha_j = <v_j, w> in the product's epilogue (:163-167);
//   w -= alpha_j v_j + beta_j v_{j-1} with the first reorthogonalisation
//     dot (:169-177, :197);
//   the two-pass reorthogonalisation (:194-205): for sk_lanczos the
//     reference's modified Gram-Schmidt as a chain of passes, each
//     subtracting h_k v_k and producing the next dot (or ||w||); for the
//     eigenvalue estimates block Gram-Schmidt, three fused passes;
//   v_{j+1} = w / beta_{j+1} (:184);
//   each sweep of Lanczos steps captured once as a CUDA graph and replayed
//     at every restart, alpha and beta read back once per sweep;
//   an implicit restart's rotations of the basis (:416-424), accumulated
//     into an m x m matrix on the host and applied as one pass that forms
//     the nev + 1 columns the restart keeps (:346-358).
// The O(m^2) work -- the tridiagonal eigensolve (dense_tridiagonal_eigen.hpp),
// the selection, the convergence test and the shifted QR steps on alpha and
// beta -- runs on the host in the value type, in the reference's operation
// order.  The start vectors are the reference's own: std::mt19937 seeded 42
// (and j + 137 after a zero beta) through uniform_real_distribution<T>{-1, 1}.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "sk_vec.cuh"

namespace sk {
namespace {

// ------------------------------------------------------------------
// Device passes
// ------------------------------------------------------------------
// w = A v_j; alpha_j = <v_j, w> (lanczos.hpp:163-167)
template <typename T>
struct EpiLzW {
  static constexpr int kNR = 1;
  T* w;
  const T* vj;
  double* alpha_out;
  __device__ void operator()(int row, T val, double* red) const {
    w[row] = val;
    red[0] += static_cast<double>(mul(vj[row], val));
  }
  __device__ void finalize(const double* t) const { *alpha_out = static_cast<double>(static_cast<T>(t[0])); }
};

// w -= alpha_j v_j; w -= beta_j v_{j-1} (:169-177); then h = <v_0, w>, the
// first dot of the reorthogonalisation (:197)
template <typename T>
struct OpLzThreeTerm {
  static constexpr int kNR = 1;
  T* w;
  const T* vj;
  const T* vjm1;  // null at j = 0
  const T* v0;
  const double* alpha;
  const double* beta;
  double* h_out;
  T a, b;
  __device__ bool prepare(const Scalars*) {
    a = static_cast<T>(*alpha);
    b = vjm1 ? static_cast<T>(*beta) : T(0);
    return true;
  }
  struct In { T w, vj, vm, v0; };
  __device__ In load(i64 i) const { return {w[i], vj[i], vjm1 ? vjm1[i] : T(0), v0[i]}; }
  __device__ void apply(i64 i, In const& q, double* red) const {
    T x = sub(q.w, mul(a, q.vj));
    if (vjm1) x = sub(x, mul(b, q.vm));
    w[i] = x;
    red[0] += static_cast<double>(mul(q.v0, x));
  }
  __device__ void finalize(const double* t) const { *h_out = static_cast<double>(static_cast<T>(t[0])); }
};

// One modified Gram-Schmidt step (:198-202, :215-220): w -= h v_k, then the
// next coefficient <v_next, w>, or with v_next null the norm ||w||.
template <typename T>
struct OpLzMgs {
  static constexpr int kNR = 1;
  T* w;
  const T* vk;
  const T* vnext;
  const double* h_in;
  double* out;
  T h;
  __device__ bool prepare(const Scalars*) {
    h = static_cast<T>(*h_in);
    return true;
  }
  struct In { T w, vk, vn; };
  __device__ In load(i64 i) const { return {w[i], vk[i], vnext ? vnext[i] : T(0)}; }
  __device__ void apply(i64 i, In const& q, double* red) const {
    const T x = sub(q.w, mul(h, q.vk));
    w[i] = x;
    red[0] += static_cast<double>(mul(vnext ? q.vn : x, x));
  }
  __device__ void finalize(const double* t) const {
    const T d = static_cast<T>(t[0]);
    *out = static_cast<double>(vnext ? d : sqrt(d));
  }
};

// <a, b> (the first dot of the random restart's orthogonalisation, :215)
template <typename T>
struct OpLzDot {
  static constexpr int kNR = 1;
  const T* a;
  const T* b;
  double* out;
  __device__ bool prepare(const Scalars*) { return true; }
  struct In { T a, b; };
  __device__ In load(i64 i) const { return {a[i], b[i]}; }
  __device__ void apply(i64, In const& q, double* red) const { red[0] += static_cast<double>(mul(q.a, q.b)); }
  __device__ void finalize(const double* t) const { *out = static_cast<double>(static_cast<T>(t[0])); }
};

// ||v|| (normalize, :483-491; the restart's new norm, :355)
template <typename T>
struct OpLzNorm {
  static constexpr int kNR = 1;
  const T* v;
  double* out;
  __device__ bool prepare(const Scalars*) { return true; }
  struct In { T v; };
  __device__ In load(i64 i) const { return {v[i]}; }
  __device__ void apply(i64, In const& q, double* red) const { red[0] += static_cast<double>(mul(q.v, q.v)); }
  __device__ void finalize(const double* t) const { *out = static_cast<double>(sqrt(static_cast<T>(t[0]))); }
};

// out = in / d when d > 0 (v_{j+1} = w / beta, :184; normalize, :487)
template <typename T>
struct OpLzDiv {
  static constexpr int kNR = 0;
  T* out;
  const T* in;
  const double* d;
  T dv;
  __device__ bool prepare(const Scalars*) {
    dv = static_cast<T>(*d);
    return dv > T(0);
  }
  struct In { T v; };
  __device__ In load(i64 i) const { return {in[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const { out[i] = dvd(q.v, dv); }
  __device__ void finalize(const double*) const {}
};

// W_c = sum_r V_r coef[r * nc + c] (r < m, in r order) for c < nc; with
// tau_v non-null the last column becomes sigma * W + tau * tau_v (:350-352)
// and its squared norm is reduced.  One thread per element reads the m
// basis entries once per column (L1-resident across columns).
template <typename T>
__global__ void __launch_bounds__(kThreads) lz_combine_kernel(i64 n, const T* __restrict__ V, i64 ldv, int m,
                                                             const double* __restrict__ coef, int nc,
                                                             T* __restrict__ W, T sigma, T tau,
                                                             const T* __restrict__ tau_v, RedWs ws,
                                                             double* norm_out) {
  double red[1] = {0.0};
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    for (int c = 0; c < nc; ++c) {
      T x = T(0);
      for (int r = 0; r < m; ++r) x = add(x, mul(static_cast<T>(coef[r * nc + c]), V[r * ldv + i]));
      if (tau_v && c == nc - 1) {
        x = add(mul(sigma, x), mul(tau, tau_v[i]));
        red[0] += static_cast<double>(mul(x, x));
      }
      W[c * ldv + i] = x;
    }
  }
  grid_reduce<1>(red, ws, [&](const double* t) {
    if (norm_out) *norm_out = static_cast<double>(sqrt(static_cast<T>(t[0])));
  });
}

// ------------------------------------------------------------------
// Block (classical) Gram-Schmidt, two passes, for nk = j + 1 <= K basis
// vectors: every coefficient of a pass from one read of the basis.
//   phase 0: w -= alpha v_j; w -= beta v_{j-1}; h1 = V^T w
//   phase 1: w -= V h1 (in k order); h2 = V^T w (the basis entries of an
//            element stay in registers between the two)
//   phase 2: w -= V h2; ||w||
// Per-CTA partial sums go to `part` (grid x K); the last CTA to arrive adds
// them in CTA order (deterministic) into h_out[0..nk) (phase 2: the norm).
// ------------------------------------------------------------------
constexpr int kBgsGrid = 148 * 2;  // CTAs at most: the grid depends on n only

inline int bgs_grid(i64 n) {
  i64 g = (n + kThreads * 4 - 1) / (kThreads * 4);
  return static_cast<int>(std::max<i64>(1, std::min<i64>(g, kBgsGrid)));
}

template <typename T, int K, int PHASE>
__global__ void __launch_bounds__(kThreads) lz_bgs_kernel(i64 n, const T* __restrict__ V, i64 ldv, int nk,
                                                         T* __restrict__ w, const T* __restrict__ vjm1,
                                                         const double* __restrict__ alpha,
                                                         const double* __restrict__ beta,
                                                         const double* __restrict__ h_in, double* part,
                                                         unsigned* counter, double* h_out) {
  constexpr int NA = PHASE == 2 ? 1 : K;
  double acc[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) acc[k] = 0.0;
  __shared__ T hs[K];  // the coefficients of phases 1 and 2 (broadcast reads)
  if (PHASE > 0) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) hs[k] = k < nk ? static_cast<T>(h_in[k]) : T(0);
    __syncthreads();
  }
  const T a = PHASE == 0 ? static_cast<T>(*alpha) : T(0);
  const T b = (PHASE == 0 && vjm1) ? static_cast<T>(*beta) : T(0);
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    T vk[K];
#pragma unroll
    for (int k = 0; k < K; ++k) vk[k] = k < nk ? V[k * ldv + i] : T(0);
    T x = w[i];
    if (PHASE == 0) {
      x = sub(x, mul(a, V[(nk - 1) * ldv + i]));  // v_j (an L1 hit: also in vk)
      if (vjm1) x = sub(x, mul(b, vjm1[i]));
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (k < nk) x = sub(x, mul(hs[k], vk[k]));
    }
    w[i] = x;
    if (PHASE == 2) {
      acc[0] += static_cast<double>(mul(x, x));
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (k < nk) acc[k] += static_cast<double>(mul(vk[k], x));
    }
  }
  // block sums: warp shuffles, then the warps in order through shared memory
  __shared__ double wsum[kThreads / 32][NA];
  __shared__ bool am_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NA; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) wsum[warp][k] = v;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < NA; k += blockDim.x) {
    double t = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) t += wsum[q][k];
    part[static_cast<size_t>(blockIdx.x) * NA + k] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  for (int k = threadIdx.x; k < (PHASE == 2 ? 1 : nk); k += blockDim.x) {
    double t = 0.0;
    for (unsigned q = 0; q < gridDim.x; ++q) t += __ldcg(part + static_cast<size_t>(q) * NA + k);
    const T tt = static_cast<T>(t);
    h_out[k] = static_cast<double>(PHASE == 2 ? sqrt(tt) : tt);
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// ------------------------------------------------------------------
// Host side: the tridiagonal eigensolver and the restart arithmetic
// ------------------------------------------------------------------
// dense_tridiagonal_eigen.hpp:58-193: implicit QR with Wilkinson shift.
// d (n) and e (n - 1) are overwritten; d receives the eigenvalues and
// Q[k * n + i] component i of eigenvector k.
template <typename T>
void tridiagonal_eigen(i64 n, std::vector<T>& d, std::vector<T>& e, T tol, i64 max_iterations,
                       std::vector<T>& Q) {
  Q.assign(static_cast<size_t>(n * n), T(0));
  for (i64 i = 0; i < n; ++i) Q[i * n + i] = T(1);
  if (n == 0) return;
  i64 hi = n - 1, total = 0;
  while (hi > 0 && total < max_iterations * n) {
    T tol_hi = tol * (std::abs(d[hi - 1]) + std::abs(d[hi]));
    if (tol_hi == T(0)) tol_hi = tol;
    if (std::abs(e[hi - 1]) <= tol_hi) {
      --hi;
      continue;
    }
    i64 lo = hi - 1;
    while (lo > 0) {
      T tol_lo = tol * (std::abs(d[lo - 1]) + std::abs(d[lo]));
      if (tol_lo == T(0)) tol_lo = tol;
      if (std::abs(e[lo - 1]) <= tol_lo) break;
      --lo;
    }
    const T delta = (d[hi - 1] - d[hi]) / T(2);
    const T e_him1 = e[hi - 1];
    T shift;
    if (delta == T(0)) {
      shift = d[hi] - std::abs(e_him1);
    } else {
      const T sign_d = delta > T(0) ? T(1) : T(-1);
      shift = d[hi] - e_him1 * e_him1 / (delta + sign_d * std::sqrt(delta * delta + e_him1 * e_him1));
    }
    T x = d[lo] - shift, z = e[lo];
    for (i64 k = lo; k < hi; ++k) {
      T cs, sn;
      const T r = std::sqrt(x * x + z * z);
      if (r == T(0)) {
        cs = T(1);
        sn = T(0);
      } else {
        cs = x / r;
        sn = z / r;
      }
      if (k > lo) e[k - 1] = r;
      const T d_k = d[k], d_k1 = d[k + 1], e_k = e[k];
      d[k] = cs * cs * d_k + T(2) * cs * sn * e_k + sn * sn * d_k1;
      d[k + 1] = sn * sn * d_k - T(2) * cs * sn * e_k + cs * cs * d_k1;
      e[k] = cs * (d_k1 - d_k) * sn + (cs * cs - sn * sn) * e_k;
      if (k + 1 < hi) {
        const T e_k1 = e[k + 1];
        z = sn * e_k1;
        e[k + 1] = cs * e_k1;
        x = e[k];
      }
      for (i64 i = 0; i < n; ++i) {
        const T q_ik = Q[k * n + i], q_ik1 = Q[(k + 1) * n + i];
        Q[k * n + i] = cs * q_ik + sn * q_ik1;
        Q[(k + 1) * n + i] = -sn * q_ik + cs * q_ik1;
      }
    }
    ++total;
  }
}

// Eigen_target order (eigen_target.hpp:13-20): does a come before b?
template <typename T>
bool target_before(int target, T a, T b) {
  switch (target) {
    case 0: return std::abs(a) > std::abs(b);
    case 1: return std::abs(a) < std::abs(b);
    case 2:
    case 4: return a > b;
    default: return a < b;
  }
}

template <typename T>
void uniform_fill(std::vector<T>& v, unsigned seed) {
  std::mt19937 rng{seed};
  std::uniform_real_distribution<T> dist{T{-1}, T{1}};
  for (auto& x : v) x = dist(rng);
}

template <typename T>
class Lanczos {
 public:
  // block_gs: reorthogonalise by block Gram-Schmidt (j + 1 <= 32), else
  // by the reference's modified Gram-Schmidt
  Lanczos(sk_matrix A, const sk_lanczos_config& cfg, cudaStream_t st, bool block_gs)
      : A_(A), cfg_(cfg), st_(st), block_gs_(block_gs) {}

  ~Lanczos() {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
    for (void* p : allocs_) cudaFreeAsync(p, st_);
  }

  sk_status run(double* eigenvalues, double* residual_norms, double* restart_residuals, T* eigenvectors,
                sk_lanczos_summary* out) {
    n_ = A_->nrow;
    m_ = cfg_.krylov_dimension;
    nev_ = cfg_.num_eigenvalues;
    if (m_ > n_) m_ = n_;  // lanczos.hpp:105-106
    if (nev_ > m_) nev_ = m_;
    tol_ = static_cast<T>(cfg_.tolerance);
    sk_status s = setup();
    if (s != SK_OK) return s;
    // init (:104-121)
    {
      std::vector<T> v0(static_cast<size_t>(n_));
      uniform_fill(v0, 42u);
      if (n_) SK_CUDA(cudaMemcpyAsync(V(0), v0.data(), n_ * sizeof(T), cudaMemcpyHostToDevice, st_));
      if ((s = normalize(V(0))) != SK_OK) return s;
    }
    alpha_.assign(static_cast<size_t>(m_), T(0));
    beta_.assign(static_cast<size_t>(m_ + 1), T(0));
    if ((s = steps(0, m_)) != SK_OK) return s;
    bool done = false;
    for (i64 r = 0; r < cfg_.max_restarts && !done; ++r) {  // run (:123-139)
      computed_restarts_ = r + 1;
      eig();
      select();
      if (converged_check(restart_residuals) || nev_ == m_) {
        if ((s = extract(eigenvalues, eigenvectors)) != SK_OK) return s;
        converged_ = true;
        done = true;
      } else if ((s = restart()) != SK_OK) {
        return s;
      }
    }
    if (!done) {
      eig();
      select();
      if ((s = extract(eigenvalues, eigenvectors)) != SK_OK) return s;
      converged_ = false;
    }
    if (residual_norms)
      for (size_t k = 0; k < res_.size(); ++k) residual_norms[k] = static_cast<double>(res_[k]);
    out->count = nev_;
    out->computed_restarts = computed_restarts_;
    out->converged_count = converged_count_;
    out->residual_count = static_cast<int64_t>(res_.size());
    out->restart_residuals_count = n_rr_;
    out->converged = converged_ ? 1 : 0;
    out->status = 0;
    SK_CUDA(cudaStreamSynchronize(st_));
    return SK_OK;
  }

 private:
  sk_matrix A_;
  sk_lanczos_config cfg_;
  cudaStream_t st_;
  bool block_gs_;
  i64 n_ = 0, m_ = 0, nev_ = 0, ldv_ = 0;
  T tol_ = T(0);
  std::vector<void*> allocs_;
  T* Vbase_ = nullptr;  // (m + 1) basis vectors
  T* W_ = nullptr;      // nev + 1 restart columns
  T* w_ = nullptr;
  double* dsc_ = nullptr;  // device scalars: alpha [m], beta [m + 1], h slots, misc
  double* coef_ = nullptr;  // m x (nev + 1) combination coefficients
  double* bgs_part_ = nullptr;  // per-CTA partial sums of the block Gram-Schmidt passes
  static constexpr int kBgsMax = 32;
  RedWs ws_{};
  std::vector<T> alpha_, beta_, tri_d_, tri_Q_, res_;
  std::vector<i64> wanted_;
  i64 computed_restarts_ = 0, converged_count_ = 0, n_rr_ = 0;
  bool converged_ = false;
  // one CUDA graph per sweep start (0, then nev for every restart)
  struct Exec {
    cudaGraphExec_t exec = nullptr;
    i64 launches = 0;
  };
  std::vector<std::pair<i64, Exec>> graphs_;

  T* V(i64 k) const { return Vbase_ + k * ldv_; }
  double* d_alpha(i64 j) const { return dsc_ + j; }
  double* d_beta(i64 j) const { return dsc_ + m_ + j; }
  // h slots: max(2 (m + 1) + 4, 2 kBgsMax) of them
  i64 nh() const { return std::max<i64>(2 * (m_ + 1) + 4, 2 * kBgsMax); }
  double* d_h(i64 s) const { return dsc_ + 2 * m_ + 1 + s; }
  double* d_misc(int k) const { return dsc_ + 2 * m_ + 1 + nh() + k; }
  i64 nsc() const { return 2 * m_ + 1 + nh() + 16; }

  template <typename P>
  sk_status alloc(P** p, size_t bytes) {
    void* q = nullptr;
    cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(bytes, 256), st_);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    allocs_.push_back(q);
    *p = static_cast<P*>(q);
    return SK_OK;
  }

  sk_status setup() {
    ldv_ = (n_ + 63) / 64 * 64 + 64;
    sk_status s;
    if ((s = alloc(&Vbase_, static_cast<size_t>((m_ + 1) * ldv_) * sizeof(T))) != SK_OK) return s;
    if ((s = alloc(&W_, static_cast<size_t>((nev_ + 1) * ldv_) * sizeof(T))) != SK_OK) return s;
    if ((s = alloc(&w_, static_cast<size_t>(ldv_) * sizeof(T))) != SK_OK) return s;
    if ((s = alloc(&dsc_, static_cast<size_t>(nsc()) * 8)) != SK_OK) return s;
    if ((s = alloc(&bgs_part_, static_cast<size_t>(kBgsGrid) * kBgsMax * 8)) != SK_OK) return s;
    if ((s = alloc(&coef_, static_cast<size_t>(m_ * (nev_ + 1) + 8) * 8)) != SK_OK) return s;
    const int cap = std::max(std::max(spmv_grid(A_), vec_grid(n_)), A_->sm_count * 8);
    if ((s = alloc(&ws_.partials, static_cast<size_t>(cap) * kMaxRed * 8)) != SK_OK) return s;
    if ((s = alloc(&ws_.counter, 64)) != SK_OK) return s;
    ws_.capacity = cap;
    SK_CUDA(cudaMemsetAsync(ws_.counter, 0, 64, st_));
    SK_CUDA(cudaMemsetAsync(Vbase_, 0, static_cast<size_t>((m_ + 1) * ldv_) * sizeof(T), st_));
    SK_CUDA(cudaMemsetAsync(dsc_, 0, static_cast<size_t>(nsc()) * 8, st_));
    return SK_OK;
  }

  sk_status read(double* host, const double* dev, size_t count) {
    SK_CUDA(cudaMemcpyAsync(host, dev, count * 8, cudaMemcpyDeviceToHost, st_));
    SK_CUDA(cudaStreamSynchronize(st_));
    return SK_OK;
  }

  // v /= ||v|| when the norm is positive (:483-491)
  sk_status normalize(T* v) {
    launch_vec(n_, OpLzNorm<T>{v, d_misc(0)}, ws_, nullptr, st_);
    launch_vec(n_, OpLzDiv<T>{v, v, d_misc(0), T(0)}, ws_, nullptr, st_);
    SK_CUDA(cudaGetLastError());
    return SK_OK;
  }

  template <int K>
  void enqueue_bgs(i64 j) {
    const int nk = static_cast<int>(j + 1);
    const int g = bgs_grid(n_);
    const T* vm = j > 0 ? V(j - 1) : nullptr;
    SK_LAUNCH((lz_bgs_kernel<T, K, 0>), g, kThreads, 0, st_, n_, Vbase_, ldv_, nk, w_, vm, d_alpha(j), d_beta(j),
              nullptr, bgs_part_, ws_.counter, d_h(0));
    SK_LAUNCH((lz_bgs_kernel<T, K, 1>), g, kThreads, 0, st_, n_, Vbase_, ldv_, nk, w_, nullptr, nullptr, nullptr,
              d_h(0), bgs_part_, ws_.counter, d_h(kBgsMax));
    SK_LAUNCH((lz_bgs_kernel<T, K, 2>), g, kThreads, 0, st_, n_, Vbase_, ldv_, nk, w_, nullptr, nullptr, nullptr,
              d_h(kBgsMax), bgs_part_, ws_.counter, d_beta(j + 1));
  }

  // The kernels of Lanczos step j (lanczos.hpp:161-187) up to the
  // division by beta_{j+1}, which skips itself when beta_{j+1} is zero.
  // With block_gs and j + 1 <= 32 basis vectors the two
  // reorthogonalisation passes run as block Gram-Schmidt (three fused
  // passes); otherwise as the reference's modified Gram-Schmidt, one pass
  // per coefficient.  The two agree to rounding, except where rounding
  // decides what the method sees: a second copy of a multiple eigenvalue,
  // which a single-vector Krylov method finds only through rounding, is
  // found (or not) as in the reference by the modified form alone.
  void enqueue_step(i64 j) {
    launch_spmv<T>(A_, V(j), EpiLzW<T>{w_, V(j), d_alpha(j)}, ws_, nullptr, st_);
    if (block_gs_ && j + 1 <= kBgsMax) {
      if (j + 1 <= 8)
        enqueue_bgs<8>(j);
      else if (j + 1 <= 16)
        enqueue_bgs<16>(j);
      else
        enqueue_bgs<32>(j);
      launch_vec(n_, OpLzDiv<T>{V(j + 1), w_, d_beta(j + 1), T(0)}, ws_, nullptr, st_);
      return;
    }
    launch_vec(n_, OpLzThreeTerm<T>{w_, V(j), j > 0 ? V(j - 1) : nullptr, V(0), d_alpha(j), d_beta(j), d_h(0)},
               ws_, nullptr, st_);
    // reorthogonalize (:194-205): slot s holds the coefficient of step s
    i64 slot = 0;
    for (int pass = 0; pass < 2; ++pass)
      for (i64 k = 0; k <= j; ++k) {
        const bool last = pass == 1 && k == j;
        const T* vnext = k < j ? V(k + 1) : (pass == 0 ? V(0) : nullptr);
        launch_vec(n_, OpLzMgs<T>{w_, V(k), vnext, d_h(slot), last ? d_beta(j + 1) : d_h(slot + 1), T(0)}, ws_,
                   nullptr, st_);
        ++slot;
      }
    launch_vec(n_, OpLzDiv<T>{V(j + 1), w_, d_beta(j + 1), T(0)}, ws_, nullptr, st_);
  }

  // lanczos_steps (:158-191).  A sweep runs as one CUDA graph (captured
  // once per start index and replayed at every restart), then alpha and
  // beta are read back together.  A zero beta_{j+1} (the reference then
  // takes a random vector, :184-186) is found afterwards: everything up to
  // step j is valid, so the sweep resumes from there with the random vector.
  sk_status steps(i64 start, i64 stop) {
    if (stop <= start) return SK_OK;
    sk_status s = run_graph(start, stop);
    if (s != SK_OK) return s;
    std::vector<double> ab(static_cast<size_t>(2 * m_ + 1));
    SK_CUDA(cudaMemcpyAsync(ab.data(), dsc_, ab.size() * 8, cudaMemcpyDeviceToHost, st_));
    SK_CUDA(cudaStreamSynchronize(st_));
    SK_CUDA(cudaGetLastError());
    for (i64 j = start; j < stop; ++j) {
      alpha_[j] = static_cast<T>(ab[j]);
      beta_[j + 1] = static_cast<T>(ab[m_ + j + 1]);
      if (!(beta_[j + 1] > T(0))) {
        if ((s = random_restart(j)) != SK_OK) return s;
        return steps_eager(j + 1, stop);
      }
    }
    return SK_OK;
  }

  // The same sweep launch by launch, reading alpha and beta after every step.
  sk_status steps_eager(i64 start, i64 stop) {
    for (i64 j = start; j < stop; ++j) {
      enqueue_step(j);
      double ab[2];
      SK_CUDA(cudaMemcpyAsync(&ab[0], d_alpha(j), 8, cudaMemcpyDeviceToHost, st_));
      SK_CUDA(cudaMemcpyAsync(&ab[1], d_beta(j + 1), 8, cudaMemcpyDeviceToHost, st_));
      SK_CUDA(cudaStreamSynchronize(st_));
      SK_CUDA(cudaGetLastError());
      alpha_[j] = static_cast<T>(ab[0]);
      beta_[j + 1] = static_cast<T>(ab[1]);
      if (!(beta_[j + 1] > T(0))) {
        sk_status s = random_restart(j);
        if (s != SK_OK) return s;
      }
    }
    return SK_OK;
  }

  sk_status run_graph(i64 start, i64 stop) {
    Exec* e = nullptr;
    for (auto& kv : graphs_)
      if (kv.first == start) e = &kv.second;
    if (!e) {
      const i64 before = g_launches.load();
      cudaGraph_t g = nullptr;
      Exec x;
      cudaError_t ce = cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal);
      if (ce == cudaSuccess) {
        for (i64 j = start; j < stop; ++j) enqueue_step(j);
        ce = cudaStreamEndCapture(st_, &g);
      }
      if (ce == cudaSuccess) ce = cudaGraphInstantiate(&x.exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (ce != cudaSuccess) return cuda_fail(ce, "Lanczos sweep capture");
      x.launches = g_launches.load() - before;
      g_launches.fetch_sub(x.launches);  // counted at each replay instead
      graphs_.emplace_back(start, x);
      e = &graphs_.back().second;
    }
    g_launches.fetch_add(e->launches);
    SK_CUDA(cudaGraphLaunch(e->exec, st_));
    return SK_OK;
  }

  // restart_with_random_vector (:207-222); beta_{j+1} stays 0
  sk_status random_restart(i64 j) {
    std::vector<T> r(static_cast<size_t>(n_));
    uniform_fill(r, static_cast<unsigned>(j + 137));
    T* v = V(j + 1);
    SK_CUDA(cudaMemcpyAsync(v, r.data(), n_ * sizeof(T), cudaMemcpyHostToDevice, st_));
    launch_vec(n_, OpLzDot<T>{V(0), v, d_h(0)}, ws_, nullptr, st_);
    for (i64 k = 0; k <= j; ++k)
      launch_vec(n_, OpLzMgs<T>{v, V(k), k < j ? V(k + 1) : nullptr, d_h(k), k < j ? d_h(k + 1) : d_misc(0), T(0)},
                 ws_, nullptr, st_);
    launch_vec(n_, OpLzDiv<T>{v, v, d_misc(0), T(0)}, ws_, nullptr, st_);
    SK_CUDA(cudaStreamSynchronize(st_));  // r leaves scope
    SK_CUDA(cudaGetLastError());
    return SK_OK;
  }

  // eigendecompose_tridiagonal (:141-151)
  void eig() {
    tri_d_.assign(alpha_.begin(), alpha_.begin() + m_);
    std::vector<T> e(beta_.begin() + 1, beta_.begin() + m_);
    tridiagonal_eigen<T>(m_, tri_d_, e, static_cast<T>(1e-15), m_ * 30, tri_Q_);
  }

  // select_wanted (:225-269).  Stable among equal Ritz values (the
  // reference's std::sort leaves their order unspecified).
  void select() {
    std::vector<i64> order(static_cast<size_t>(m_));
    for (i64 i = 0; i < m_; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](i64 a, i64 b) { return target_before<T>(cfg_.target, tri_d_[a], tri_d_[b]); });
    wanted_.assign(order.begin(), order.begin() + nev_);
  }

  // check_convergence (:153-177)
  bool converged_check(double* restart_residuals) {
    bool all = true;
    res_.clear();
    converged_count_ = 0;
    const T beta_m = beta_[m_];
    for (i64 idx : wanted_) {
      const T abs_res = std::abs(beta_m * tri_Q_[idx * m_ + (m_ - 1)]);
      const T abs_theta = std::abs(tri_d_[idx]);
      const T threshold = tol_ * std::max(abs_theta, T(1e-20));
      res_.push_back(abs_res);
      if (abs_res <= threshold)
        ++converged_count_;
      else
        all = false;
    }
    if (cfg_.collect_residuals) {
      T mx = T(0);
      for (T r : res_) mx = std::max(mx, r);
      if (restart_residuals) restart_residuals[n_rr_] = static_cast<double>(mx);
      ++n_rr_;
    }
    return all;
  }

  // implicit_restart (:314-369) with tridiagonal_qr_step (:373-434): the
  // rotations act on alpha, beta and an m x m accumulator Q; the basis is
  // then formed once as V Q for the nev + 1 columns kept.
  sk_status restart() {
    const i64 m = m_, nev = nev_;
    std::vector<char> is_wanted(static_cast<size_t>(m), 0);
    for (i64 idx : wanted_) is_wanted[idx] = 1;
    const T beta_m_saved = beta_[m];
    std::vector<T> Q(static_cast<size_t>(m * m), T(0));
    for (i64 i = 0; i < m; ++i) Q[i * m + i] = T(1);
    for (i64 u = 0; u < m; ++u) {
      if (is_wanted[u]) continue;
      const T mu = tri_d_[u];
      T x = alpha_[0] - mu, z = beta_[1];
      for (i64 k = 0; k < m - 1; ++k) {
        T cs, sn;
        const T r = std::sqrt(x * x + z * z);
        if (r == T(0)) {
          cs = T(1);
          sn = T(0);
        } else {
          cs = x / r;
          sn = z / r;
        }
        if (k > 0) beta_[k] = r;
        const T a_k = alpha_[k], a_k1 = alpha_[k + 1], b_k1 = beta_[k + 1];
        alpha_[k] = cs * cs * a_k + T(2) * cs * sn * b_k1 + sn * sn * a_k1;
        alpha_[k + 1] = sn * sn * a_k - T(2) * cs * sn * b_k1 + cs * cs * a_k1;
        beta_[k + 1] = cs * sn * (a_k1 - a_k) + (cs * cs - sn * sn) * b_k1;
        if (k + 2 < m) {
          const T b_k2 = beta_[k + 2];
          x = beta_[k + 1];
          z = sn * b_k2;
          beta_[k + 2] = cs * b_k2;
        }
        // columns k, k+1 of the accumulated rotation (rows: basis vectors);
        // row m - 1 is the reference's q_row (:412-419)
        for (i64 rr = 0; rr < m; ++rr) {
          const T q_k = Q[rr * m + k], q_k1 = Q[rr * m + k + 1];
          Q[rr * m + k] = cs * q_k + sn * q_k1;
          Q[rr * m + k + 1] = -sn * q_k + cs * q_k1;
        }
      }
    }
    const T sigma_k = beta_[nev];
    const T tau = beta_m_saved * Q[(m - 1) * m + (nev - 1)];
    const int nc = static_cast<int>(nev + 1);
    std::vector<double> coef(static_cast<size_t>(m * nc));
    for (i64 rr = 0; rr < m; ++rr)
      for (int c = 0; c < nc; ++c) coef[rr * nc + c] = static_cast<double>(Q[rr * m + c]);
    SK_CUDA(cudaMemcpyAsync(coef_, coef.data(), coef.size() * 8, cudaMemcpyHostToDevice, st_));
    const int grid = std::max(1, std::min(ceil_div(n_, kThreads), A_->sm_count * 8));
    SK_LAUNCH(lz_combine_kernel<T>, grid, kThreads, 0, st_, n_, Vbase_, ldv_, static_cast<int>(m), coef_, nc, W_,
              sigma_k, tau, V(m), ws_, d_misc(0));
    SK_CUDA(cudaMemcpy2DAsync(Vbase_, ldv_ * sizeof(T), W_, ldv_ * sizeof(T), n_ * sizeof(T), nc,
                              cudaMemcpyDeviceToDevice, st_));
    double bn = 0;
    sk_status s = read(&bn, d_misc(0), 1);
    if (s != SK_OK) return s;
    const T beta_new = static_cast<T>(bn);
    if (beta_new > T(0)) launch_vec(n_, OpLzDiv<T>{V(nev), V(nev), d_misc(0), T(0)}, ws_, nullptr, st_);
    beta_[nev] = beta_new;
    // the device recurrence reads alpha and beta from device memory
    std::vector<double> ab(static_cast<size_t>(2 * m + 1));
    for (i64 j = 0; j < m; ++j) ab[j] = static_cast<double>(alpha_[j]);
    for (i64 j = 0; j <= m; ++j) ab[m + j] = static_cast<double>(beta_[j]);
    SK_CUDA(cudaMemcpyAsync(dsc_, ab.data(), ab.size() * 8, cudaMemcpyHostToDevice, st_));
    SK_CUDA(cudaStreamSynchronize(st_));  // ab and coef leave scope
    return steps(nev, m);
  }

  // extract_ritz_pairs (:437-461)
  sk_status extract(double* eigenvalues, T* eigenvectors) {
    for (i64 w = 0; w < nev_; ++w) {
      const i64 idx = wanted_[w];
      if (eigenvalues) eigenvalues[w] = static_cast<double>(tri_d_[idx]);
      if (!eigenvectors) continue;
      std::vector<double> coef(static_cast<size_t>(m_));
      for (i64 j = 0; j < m_; ++j) coef[j] = static_cast<double>(tri_Q_[idx * m_ + j]);
      SK_CUDA(cudaMemcpyAsync(coef_, coef.data(), coef.size() * 8, cudaMemcpyHostToDevice, st_));
      T* x = eigenvectors + w * n_;
      const int grid = std::max(1, std::min(ceil_div(n_, kThreads), A_->sm_count * 8));
      // x = sum_j coeff_j v_j accumulated from zero in j order (:449-456)
      SK_LAUNCH(lz_combine_kernel<T>, grid, kThreads, 0, st_, n_, Vbase_, ldv_, static_cast<int>(m_), coef_, 1, x,
                T(1), T(0), nullptr, ws_, nullptr);
      sk_status s = normalize(x);
      if (s != SK_OK) return s;
      SK_CUDA(cudaStreamSynchronize(st_));  // coef leaves scope
    }
    SK_CUDA(cudaGetLastError());
    return SK_OK;
  }
};

static sk_status lanczos_any(sk_matrix A, const sk_lanczos_config* cfg, double* eigenvalues, double* residual_norms,
                             double* restart_residuals, void* eigenvectors, sk_lanczos_summary* out,
                             cudaStream_t st, bool block_gs) {
  SK_CHECK(A && cfg && out, SK_INVALID_ARG, "null argument");
  SK_CHECK(A->nrow == A->ncol, SK_INVALID_ARG, "Lanczos needs a square (symmetric) matrix");
  SK_CHECK(cfg->krylov_dimension >= 1 && cfg->krylov_dimension <= 4096, SK_INVALID_ARG,
           "krylov_dimension must be in [1, 4096]");
  SK_CHECK(cfg->num_eigenvalues >= 1, SK_INVALID_ARG, "num_eigenvalues must be >= 1");
  SK_CHECK(cfg->max_restarts >= 0, SK_INVALID_ARG, "negative max_restarts");
  SK_CHECK(cfg->target >= 0 && cfg->target <= 5, SK_INVALID_ARG, "target must be an sk_eigen_target");
  *out = sk_lanczos_summary{};
  if (A->nrow == 0) {
    out->converged = 1;
    return SK_OK;
  }
  SK_CUDA(cudaStreamSynchronize(A->stream));
  // the sweeps are captured as CUDA graphs, which the legacy stream cannot
  // hold: the caller's stream is drained and the handle's stream used
  if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread) {
    SK_CUDA(cudaStreamSynchronize(st));
    st = A->stream;
  }
  if (A->dtype == SK_F64) {
    Lanczos<double> L(A, *cfg, st, block_gs);
    return L.run(eigenvalues, residual_norms, restart_residuals, static_cast<double*>(eigenvectors), out);
  }
  Lanczos<float> L(A, *cfg, st, block_gs);
  return L.run(eigenvalues, residual_norms, restart_residuals, static_cast<float*>(eigenvectors), out);
}

}  // namespace
}  // namespace sk

using namespace sk;

extern "C" {

sk_status sk_lanczos(sk_matrix A, const sk_lanczos_config* cfg, double* eigenvalues, double* residual_norms,
                     double* restart_residuals, void* eigenvectors_dev, sk_lanczos_summary* out,
                     sk_stream stream) {
  cudaStream_t st = pick_stream(A, stream);
  return lanczos_any(A, cfg, eigenvalues, residual_norms, restart_residuals, eigenvectors_dev, out, st, false);
}

sk_status sk_spectral_radius(sk_matrix A, int64_t num_iter, double* rho) {
  SK_CHECK(A && rho, SK_INVALID_ARG, "null argument");
  SK_CHECK(num_iter >= 0, SK_INVALID_ARG, "negative num_iter");
  const i64 m = std::min<i64>(A->nrow, num_iter + 1);  // conditioning.hpp:114
  sk_lanczos_config cfg{1, std::max<i64>(m, 1), 1e-10, 10, SK_LARGEST_MAGNITUDE, 0};
  double ev = 0;
  sk_lanczos_summary s{};
  sk_status st = lanczos_any(A, &cfg, &ev, nullptr, nullptr, nullptr, &s, A->stream, true);
  if (st != SK_OK) return st;
  *rho = s.count ? std::abs(ev) : 0.0;
  return SK_OK;
}

sk_status sk_eigenvalue_bounds(sk_matrix A, int64_t num_iter, double* lambda_min, double* lambda_max) {
  SK_CHECK(A && lambda_min && lambda_max, SK_INVALID_ARG, "null argument");
  SK_CHECK(num_iter >= 0, SK_INVALID_ARG, "negative num_iter");
  const i64 m = std::max<i64>(std::min<i64>(A->nrow, num_iter + 1), 1);  // conditioning.hpp:135
  sk_lanczos_config cmax{1, m, 1e-10, 10, SK_LARGEST_ALGEBRAIC, 0};
  sk_lanczos_config cmin{1, m, 1e-10, 10, SK_SMALLEST_ALGEBRAIC, 0};
  double hi = 0, lo = 0;
  sk_lanczos_summary s{};
  sk_status st = lanczos_any(A, &cmax, &hi, nullptr, nullptr, nullptr, &s, A->stream, true);
  if (st != SK_OK) return st;
  if (!s.count) hi = 0;
  st = lanczos_any(A, &cmin, &lo, nullptr, nullptr, nullptr, &s, A->stream, true);
  if (st != SK_OK) return st;
  if (!s.count) lo = 0;
  *lambda_min = lo;
  *lambda_max = hi;
  return SK_OK;
}

sk_status sk_chebyshev_create_auto(sk_precond* out, sk_matrix A, int64_t degree, int64_t num_iter,
                                   double bounds[2]) {
  SK_CHECK(out && A, SK_INVALID_ARG, "null argument");
  *out = nullptr;
  double lo = 0, hi = 0;
  sk_status st = sk_eigenvalue_bounds(A, num_iter, &lo, &hi);
  if (st != SK_OK) return st;
  if (bounds) {
    bounds[0] = lo;
    bounds[1] = hi;
  }
  return sk_chebyshev_create(out, A, lo, hi, degree);
}

}  // extern "C"
