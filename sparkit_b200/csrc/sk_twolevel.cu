// sk_twolevel.cu -- a two-level preconditioner for matrices on a 2-D grid:
// a smoother (the learned network, Jacobi or Chebyshev) followed by an
// exact coarse-grid correction over agg x agg aggregates of cells.
//
// No reference counterpart: fgmres (fgmres.hpp:96-428) takes any callable
// as its variable preconditioner; this is one such callable.  The smoother
// alone cannot remove error components longer than its reach (about 40
// cells for the 4-level network, one cell per Jacobi sweep), which is why
// FGMRES(30) stalls on 512 x 512 grids; the coarse correction removes them.
//
//   z  = S(r)                       smoother
//   t  = r - A z                    SpMV with a residual epilogue
//   rc = P^T t                      restriction: sum over each aggregate
//   z += P Ac^-1 rc                 dense coarse solve, prolongation
//  [t  = r - A z;  z += S(t)]       optional post-smoothing
//
// or, coarse first, z = P Ac^-1 P^T r; z += S(r - A z): the smoother then
// only sees residuals whose aggregate sums are zero (P^T (r - A z) = 0), the
// local part that a network of limited reach can resolve.
// P is piecewise constant over the aggregates (cell (x, y) belongs to
// aggregate (x / agg, y / agg)); Ac = P^T A P is the Galerkin coarse
// operator, formed on the host from the FP64 CSR values, factored by a
// banded LU without pivoting (Ac is an M-matrix when A is: Galerkin
// aggregation keeps the signs and the diagonal dominance of the upwind
// convection-diffusion operators) and inverted column by column.  The
// inverse (nc x nc, nc <= 4096, stored in FP32) is applied as one
// deterministic GEMV with FP64 products and sums.  Solving with the banded
// factors instead would read 4 MB rather than 64 MiB, but each of its nc
// rows waits on the previous ones (a chain of nc dependent steps on one
// SM), where the GEMV spreads the rows over every SM.
// Every reduction runs in a fixed order, so applies are repeatable bit for
// bit, and the apply launches kernels only (it can be captured).
#include <algorithm>
#include <cmath>
#include <vector>

#include "sk_kernels.cuh"
#include "sk_learned.cuh"
#include "sk_twolevel.cuh"
#include "sk_vec.cuh"

namespace sk {
namespace {

constexpr i64 kMaxCoarse = 4096;

// t = r - A z
struct EpiResidStore {
  static constexpr int kNR = 0;
  const double* r;
  double* t;
  __device__ void operator()(int row, double az, double*) const { t[row] = __dsub_rn(r[row], az); }
  __device__ void finalize(const double*) const {}
};

// t = r - A z and, for a learned smoother, its input scale
// s = sqrt(mean((t / d)^2)) in the same pass (the network's scale
// reduction, summed in this product's fixed order)
struct EpiResidScale {
  static constexpr int kNR = 1;
  const double* r;
  double* t;
  const float* inv;  // 1 / d per cell
  double* s_out;
  double P;
  __device__ void operator()(int row, double az, double* red) const {
    const double ti = __dsub_rn(r[row], az);
    t[row] = ti;
    const double rt = ti * static_cast<double>(inv[row]);
    red[0] += rt * rt;
  }
  __device__ void finalize(const double* tot) const { *s_out = sqrt(tot[0] / P); }
};

// z += D^-1 t: the Jacobi smoother's apply and its addition in one pass,
// with the bits of the two (z = z + (inv_d * t))
struct OpJacobiAdd {
  static constexpr int kNR = 0;
  struct In { double d, t, z; };
  const double* inv_d;
  const double* t;
  double* z;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {inv_d[i], t[i], z[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { z[i] = __dadd_rn(v.z, __dmul_rn(v.d, v.t)); }
  __device__ void finalize(const double*) const {}
};

// rc[I] = sum of t over aggregate I, in the order of a 256-thread block
// reduction (thread T adds cells T, T + 256, ... from zero; a butterfly
// over each warp of 32 threads; a butterfly over the 8 warp sums), computed
// by one warp per aggregate: lane l plays threads l, l + 32, ..., l + 224.
__global__ void __launch_bounds__(kThreads) restrict_kernel(int nx, int agg, int mcx, int nc,
                                                            const double* __restrict__ t, double* __restrict__ rc,
                                                            const Scalars* sc) {
  constexpr int kW = kThreads / 32;
  if (solve_done(sc)) return;
  const int I = blockIdx.x * kW + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (I >= nc) return;
  const int X0 = (I % mcx) * agg, Y0 = (I / mcx) * agg;
  const int cells = agg * agg;
  double v[kW];
#pragma unroll
  for (int w = 0; w < kW; ++w) v[w] = 0.0;
  for (int c0 = 0; c0 < cells; c0 += kThreads) {
#pragma unroll
    for (int w = 0; w < kW; ++w) {
      const int c = c0 + 32 * w + lane;
      if (c < cells) v[w] += t[static_cast<i64>(Y0 + c / agg) * nx + X0 + c % agg];
    }
  }
  warp_reduce<kW>(v);
  double x[1] = {0.0};
#pragma unroll
  for (int w = 0; w < kW; ++w)
    if (lane == w) x[0] = v[w];
  warp_reduce<1>(x);
  if (lane == 0) rc[I] = x[0];
}

// zc = Ainv rc: one warp per coarse row, lane-strided partial sums and a
// shuffle tree.  The inverse is stored in FP32 (64 MiB at nc = 4096: half
// the bytes of the FP64 inverse, and within the L2) and every product is
// formed and summed in FP64; the float rounding of the inverse (relative
// 6e-8 per entry) perturbs the coarse correction of a preconditioner only.
// Each lane reads four consecutive floats (16 bytes) per step, four steps'
// loads in flight before their products are summed (in step order).
__global__ void __launch_bounds__(kThreads) coarse_gemv_kernel(int nc, const float* __restrict__ ainv,
                                                               const double* __restrict__ rc,
                                                               double* __restrict__ zc, const Scalars* sc) {
  if (solve_done(sc)) return;
  const int I = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (I >= nc) return;
  const float* row = ainv + static_cast<i64>(I) * nc;
  double s[1] = {0.0};
  int j = 4 * lane;
  if ((nc & 3) == 0) {
    for (; j < nc; j += 512) {
      float4 a[4];
      double r[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int jj = j + 128 * u;
        if (jj < nc) {
          a[u] = __ldg(reinterpret_cast<const float4*>(row + jj));
#pragma unroll
          for (int k = 0; k < 4; ++k) r[u][k] = rc[jj + k];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (j + 128 * u < nc)
          s[0] += static_cast<double>(a[u].x) * r[u][0] + static_cast<double>(a[u].y) * r[u][1] +
                  static_cast<double>(a[u].z) * r[u][2] + static_cast<double>(a[u].w) * r[u][3];
    }
  } else {
    for (j = lane; j < nc; j += 32) s[0] += static_cast<double>(row[j]) * rc[j];
  }
  warp_reduce<1>(s);
  if (lane == 0) zc[I] = s[0];
}

// z += P zc, z = P zc (set), or z += add (the smoother's share)
__global__ void __launch_bounds__(kThreads) prolong_kernel(i64 n, int nx, int agg, int mcx,
                                                           const double* __restrict__ zc, const double* add, int set,
                                                           double* z, const Scalars* sc) {
  if (solve_done(sc)) return;
  for (i64 i = blockIdx.x * static_cast<i64>(kThreads) + threadIdx.x; i < n;
       i += static_cast<i64>(gridDim.x) * kThreads) {
    const int y = static_cast<int>(i / nx), x = static_cast<int>(i % nx);
    if (zc) {
      const double c = zc[(y / agg) * mcx + x / agg];
      z[i] = set ? c : __dadd_rn(z[i], c);
    } else {
      z[i] = __dadd_rn(z[i], add[i]);
    }
  }
}

int ew_blocks(i64 n) {
  i64 g = (n + kThreads - 1) / kThreads;
  return static_cast<int>(std::max<i64>(1, std::min<i64>(g, 148 * 8)));
}

// Banded LU without pivoting of the dense nc x nc matrix a (row-major),
// lower bandwidth bl, upper bu, in place; false on a zero pivot.
bool band_lu(std::vector<double>& a, i64 nc, i64 bl, i64 bu) {
  for (i64 k = 0; k < nc; ++k) {
    const double piv = a[k * nc + k];
    if (!(std::fabs(piv) > 0.0) || !std::isfinite(piv)) return false;
    const i64 iend = std::min(nc, k + bl + 1), jend = std::min(nc, k + bu + 1);
    for (i64 i = k + 1; i < iend; ++i) {
      const double l = a[i * nc + k] / piv;
      a[i * nc + k] = l;
      if (l == 0.0) continue;
      for (i64 j = k + 1; j < jend; ++j) a[i * nc + j] -= l * a[k * nc + j];
    }
  }
  return true;
}

// Inverse from the banded LU factors, column by column (row-major out).
void band_inverse(const std::vector<double>& lu, i64 nc, i64 bl, i64 bu, std::vector<double>& inv) {
  inv.assign(static_cast<size_t>(nc * nc), 0.0);
  std::vector<double> y(static_cast<size_t>(nc));
  for (i64 c = 0; c < nc; ++c) {
    std::fill(y.begin(), y.end(), 0.0);
    y[c] = 1.0;
    for (i64 i = c + 1; i < nc; ++i) {  // L y = e_c (unit lower)
      double s = y[i];
      for (i64 j = std::max(c, i - bl); j < i; ++j) s -= lu[i * nc + j] * y[j];
      y[i] = s;
    }
    for (i64 i = nc - 1; i >= 0; --i) {  // U x = y
      double s = y[i];
      const i64 jend = std::min(nc, i + bu + 1);
      for (i64 j = i + 1; j < jend; ++j) s -= lu[i * nc + j] * y[j];
      y[i] = s / lu[i * nc + i];
    }
    for (i64 i = 0; i < nc; ++i) inv[i * nc + c] = y[i];
  }
}

}  // namespace

bool twolevel_smoother_ok(const sk_precond_s* S) {
  return !S || (S->dtype == SK_F64 && S->kind >= 1 && S->kind <= 3);
}

void twolevel_apply(const sk_precond_s* M, const double* r, double* z, RedWs ws, const Scalars* sc,
                    cudaStream_t st) {
  const sk_matrix A = M->A;
  const i64 n = M->n;
  const int nx = static_cast<int>(M->grid_nx), agg = static_cast<int>(M->agg);
  const int mcx = static_cast<int>(M->grid_nx / M->agg);
  const int nc = static_cast<int>(M->coarse_n);
  const sk_precond_s* S = M->smoother;
  auto coarse = [&](const double* t, int set) {  // z (+)= P Ac^-1 P^T t
    SK_LAUNCH(restrict_kernel, ceil_div(nc, kThreads / 32), kThreads, 0, st, nx, agg, mcx, nc, t, M->rc, sc);
    SK_LAUNCH(coarse_gemv_kernel, ceil_div(nc, kThreads / 32), kThreads, 0, st, nc,
              M->coarse_inv, M->rc, M->zc, sc);
    SK_LAUNCH(prolong_kernel, ew_blocks(n), kThreads, 0, st, n, nx, agg, mcx, M->zc, nullptr, set, z, sc);
  };
  auto smooth_add = [&]() {  // z += S(r - A z)
    if (S->kind == 3 && ws.partials && ws.capacity >= spmv_grid(A)) {
      // learned: the scale reduction in the residual product, and the last
      // convolution adds its output into z
      double* sd = learned_scale_slot(S);
      if (sd) {
        launch_spmv<double>(A, z, EpiResidScale{r, M->tbuf, S->coef + 5 * n, sd, static_cast<double>(n)}, ws, sc,
                            st);
        if (learned_apply_ex(S, M->tbuf, z, st, true, true) != SK_OK) set_error("learned smoother apply failed");
        return;
      }
    }
    launch_spmv<double>(A, z, EpiResidStore{r, M->tbuf}, RedWs{}, sc, st);
    if (S->kind == 1) {
      launch_vec(n, OpJacobiAdd{static_cast<const double*>(S->inv_diag), M->tbuf, z}, ws, sc, st);
      return;
    }
    precond_apply_dispatch(S, SK_F64, n, M->tbuf, M->tbuf2, ws, sc, st);
    SK_LAUNCH(prolong_kernel, ew_blocks(n), kThreads, 0, st, n, nx, agg, mcx, nullptr, M->tbuf2, 0, z, sc);
  };
  if (M->coarse_first) {
    coarse(r, 1);
    if (S) smooth_add();
    return;
  }
  if (S) {
    precond_apply_dispatch(S, SK_F64, n, r, z, ws, sc, st);
    launch_spmv<double>(A, z, EpiResidStore{r, M->tbuf}, RedWs{}, sc, st);
    coarse(M->tbuf, 0);
    if (M->post) smooth_add();
  } else {
    coarse(r, 1);
  }
}

void twolevel_release(sk_precond_s* M) {
  if (M->coarse_inv) cudaFree(M->coarse_inv);
  M->coarse_inv = nullptr;
  for (double** p : {&M->tbuf, &M->tbuf2, &M->rc, &M->zc, &M->cvt_in, &M->cvt_out}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
}

}  // namespace sk

using namespace sk;

extern "C" {

sk_status sk_twolevel_create(sk_precond* out, sk_matrix A, sk_precond smoother, int64_t nx, int64_t ny,
                             int64_t agg, int32_t flags) {
  SK_CHECK(out && A, SK_INVALID_ARG, "null argument");
  *out = nullptr;
  SK_CHECK(A->format == SK_CSR && A->dtype == SK_F64 && A->nrow == A->ncol, SK_NOT_SUPPORTED,
           "the two-level preconditioner needs a square FP64 CSR matrix");
  SK_CHECK(twolevel_smoother_ok(smoother), SK_INVALID_ARG,
           "the smoother must be an FP64 Jacobi, Chebyshev or learned preconditioner");
  SK_CHECK(!smoother || smoother->n == A->nrow, SK_INVALID_ARG, "smoother size differs from the matrix");
  SK_CHECK((flags & ~3) == 0, SK_INVALID_ARG, "unknown flags");
  SK_CHECK(nx > 0 && ny > 0 && nx * ny == A->nrow, SK_INVALID_ARG, "matrix size is not nx * ny");
  SK_CHECK(agg >= 1 && nx % agg == 0 && ny % agg == 0, SK_INVALID_ARG, "agg must divide both grid sides");
  const i64 mcx = nx / agg, mcy = ny / agg, nc = mcx * mcy;
  SK_CHECK(nc <= kMaxCoarse, SK_INVALID_ARG, "coarse grid above 4096 aggregates");
  const i64 n = A->nrow, nnz = A->nnz;
  // the FP64 CSR arrays, to the host once
  std::vector<int> rp(static_cast<size_t>(n + 1)), ci(static_cast<size_t>(nnz));
  std::vector<double> va(static_cast<size_t>(nnz));
  SK_CUDA(cudaStreamSynchronize(A->stream));
  SK_CUDA(cudaMemcpy(rp.data(), A->csr.row_ptr, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  if (nnz) {
    SK_CUDA(cudaMemcpy(ci.data(), A->csr.col_ind, nnz * sizeof(int), cudaMemcpyDeviceToHost));
    SK_CUDA(cudaMemcpy(va.data(), A->csr.vals, nnz * sizeof(double), cudaMemcpyDeviceToHost));
  }
  // Galerkin Ac = P^T A P and its bandwidths
  auto agg_of = [&](i64 i) { return ((i / nx) / agg) * mcx + (i % nx) / agg; };
  std::vector<double> ac(static_cast<size_t>(nc * nc), 0.0);
  i64 bl = 0, bu = 0;
  for (i64 i = 0; i < n; ++i) {
    const i64 I = agg_of(i);
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const i64 J = agg_of(ci[k]);
      ac[I * nc + J] += va[k];
      bl = std::max(bl, I - J);
      bu = std::max(bu, J - I);
    }
  }
  SK_CHECK(band_lu(ac, nc, bl, bu), SK_INVALID_ARG, "the coarse operator has a zero pivot");
  std::vector<double> inv;
  band_inverse(ac, nc, bl, bu, inv);
  for (double v : inv) SK_CHECK(std::isfinite(v), SK_INVALID_ARG, "the coarse operator is singular");
  auto* M = new sk_precond_s();
  M->kind = 4;
  M->A = A;
  M->dtype = SK_F64;
  M->n = n;
  M->smoother = smoother;
  M->grid_nx = nx;
  M->grid_ny = ny;
  M->agg = agg;
  M->coarse_n = nc;
  M->post = (flags & SK_TWOLEVEL_POST_SMOOTH) ? 1 : 0;
  M->coarse_first = (flags & SK_TWOLEVEL_COARSE_FIRST) ? 1 : 0;
  std::vector<float> inv32(inv.begin(), inv.end());
  cudaError_t e = cudaMalloc(&M->coarse_inv, static_cast<size_t>(nc * nc) * 4 + 64);
  if (e == cudaSuccess) e = cudaMalloc(&M->tbuf, static_cast<size_t>(n + 8) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&M->tbuf2, static_cast<size_t>(n + 8) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&M->rc, static_cast<size_t>(nc + 8) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&M->zc, static_cast<size_t>(nc + 8) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&M->cvt_in, static_cast<size_t>(n + 8) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&M->cvt_out, static_cast<size_t>(n + 8) * 8);
  if (e == cudaSuccess)
    e = cudaMemcpy(M->coarse_inv, inv32.data(), static_cast<size_t>(nc * nc) * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    twolevel_release(M);
    delete M;
    return cuda_fail(e, "two-level set-up");
  }
  *out = M;
  return SK_OK;
}

}  // extern "C"
