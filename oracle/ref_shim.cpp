// ref_shim.cpp -- extern "C" access to the UNMODIFIED sparkit reference.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build_ref.sh compiles this file together
// with the reference's own sources (read in place, never copied) into
// oracle/_ref/libsparkit_ref.so.  The tests use it to pin the C oracle
// bit for bit, and the benchmark's CPU-baseline leg times the reference's
// own SpMV and solvers through it.  Nothing in the product links it.
//
// Every entry point builds the reference's own matrix classes and calls its
// own templates: multiply (sparkit/data/sparse_blas.hpp:19, spmv.hpp:119,
// :148, :182), to_ellpack / to_block_sparse_row / to_jagged_diagonal
// (conversions.hpp:427, :524, :641), jacobi / jacobi_apply (jacobi.hpp:27,
// :44), chebyshev_preconditioner / _apply (chebyshev_preconditioner.hpp:46,
// :98), conjugate_gradient (conjugate_gradient.hpp:347), bicgstab
// (bicgstab.hpp:391), fgmres (fgmres.hpp:459), gmres (gmres.hpp:408), cgs
// (cgs.hpp:374), minres (minres.hpp:397), lanczos (lanczos.hpp:495),
// estimate_spectral_radius / estimate_eigenvalue_bounds (conditioning.hpp:112,
// :132), read_matrix_market / write_matrix_market (matrix_market.hpp:45,
// :119) and the matrix generators of
// matgen.hpp used by the reference's solver tests.

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <span>
#include <stdexcept>
#include <thread>
#include <vector>

#include <sparkit/data/Block_sparse_row_matrix.hpp>
#include <sparkit/data/Compressed_row_matrix.hpp>
#include <sparkit/data/Ellpack_matrix.hpp>
#include <sparkit/data/Jagged_diagonal_matrix.hpp>
#include <sparkit/data/bicgstab.hpp>
#include <sparkit/data/chebyshev_preconditioner.hpp>
#include <sparkit/data/conjugate_gradient.hpp>
#include <sparkit/data/conversions.hpp>
#include <sparkit/data/fgmres.hpp>
#include <sparkit/data/gmres.hpp>
#include <sparkit/data/cgs.hpp>
#include <sparkit/data/minres.hpp>
#include <sparkit/data/conditioning.hpp>
#include <sparkit/data/lanczos.hpp>
#include <sparkit/data/matrix_market.hpp>
#include <cstdio>
#include <sstream>
#include <sparkit/data/jacobi.hpp>
#include <sparkit/data/matgen.hpp>
#include <sparkit/data/sparse_blas.hpp>
#include <sparkit/data/spmv.hpp>

namespace sd = sparkit::data::detail;
using i64 = std::int64_t;

namespace {

  enum { F_CSR = 0, F_ELL = 1, F_JAD = 2, F_BSR = 3 };
  enum { P_IDENTITY = 0, P_JACOBI = 1, P_CHEBYSHEV = 2 };

  // A reference matrix of either value type and any of the four formats.
  template <typename T>
  struct Handle {
    int format;
    sd::Compressed_row_matrix<T>* csr = nullptr;
    sd::Ellpack_matrix<T>* ell = nullptr;
    sd::Jagged_diagonal_matrix<T>* jad = nullptr;
    sd::Block_sparse_row_matrix<T>* bsr = nullptr;
    ~Handle() {
      delete csr;
      delete ell;
      delete jad;
      delete bsr;
    }
    i64 nrow() const {
      switch (format) {
        case F_CSR: return csr->shape().row();
        case F_ELL: return ell->shape().row();
        case F_JAD: return jad->shape().row();
        default: return bsr->shape().row();
      }
    }
    std::vector<T> multiply(std::span<T const> x) const {
      switch (format) {
        case F_CSR: return sd::multiply(*csr, x);
        case F_ELL: return sd::multiply(*ell, x);
        case F_JAD: return sd::multiply(*jad, x);
        default: return sd::multiply(*bsr, x);
      }
    }
  };

  template <typename T>
  Handle<T>* make_csr(i64 nrow, i64 ncol, i64 const* rp, i64 const* ci,
                      T const* vals) {
    i64 nnz = rp[nrow];
    std::vector<sd::Index> idx;
    idx.reserve(static_cast<std::size_t>(nnz));
    for (i64 i = 0; i < nrow; ++i)
      for (i64 j = rp[i]; j < rp[i + 1]; ++j) idx.emplace_back(i, ci[j]);
    sd::Compressed_row_sparsity sp{sd::Shape{nrow, ncol}, idx.begin(),
                                   idx.end()};
    auto* h = new Handle<T>;
    h->format = F_CSR;
    h->csr = new sd::Compressed_row_matrix<T>{
      std::move(sp), std::vector<T>(vals, vals + nnz)};
    return h;
  }

  template <typename T>
  Handle<T>* wrap_csr(sd::Compressed_row_matrix<T> A) {
    auto* h = new Handle<T>;
    h->format = F_CSR;
    h->csr = new sd::Compressed_row_matrix<T>{std::move(A)};
    return h;
  }

  // Runtime-selected preconditioner with the reference's callable signature.
  template <typename T>
  struct Prec {
    int kind = P_IDENTITY;
    std::vector<T> inv_d;
    sd::Chebyshev_preconditioner<T>* cheb = nullptr;
    ~Prec() { delete cheb; }
    template <typename It, typename Out>
    void operator()(It first, It last, Out out) const {
      if (kind == P_JACOBI) {
        sd::jacobi_apply(inv_d, first, last, out);
      } else if (kind == P_CHEBYSHEV) {
        sd::chebyshev_preconditioner_apply(*cheb, first, last, out);
      } else {
        std::copy(first, last, out);
      }
    }
  };

  template <typename T>
  int setup_prec(Prec<T>& p, Handle<T> const* A, int kind, double lmin,
                 double lmax, i64 degree) {
    p.kind = kind;
    if (kind == P_JACOBI) {
      if (A->format != F_CSR) return -2;
      try {
        p.inv_d = sd::jacobi(*A->csr);
      } catch (std::invalid_argument const&) {
        return -1;
      }
    } else if (kind == P_CHEBYSHEV) {
      if (A->format != F_CSR) return -2;
      p.cheb = new sd::Chebyshev_preconditioner<T>{sd::chebyshev_preconditioner(
        *A->csr, static_cast<T>(lmin), static_cast<T>(lmax), degree)};
    }
    return 0;
  }

  struct Summary {
    double residual_norm;
    i64 computed_iterations;
    std::int32_t converged;
    std::int32_t status;
    i64 history_length;
  };

  template <typename S, typename T>
  void fill_summary(Summary* out, S const& s, double* history) {
    out->residual_norm = static_cast<double>(s.residual_norm);
    out->computed_iterations = s.computed_iterations;
    out->converged = s.converged ? 1 : 0;
    out->status = 0;
    out->history_length = static_cast<i64>(s.iteration_residuals.size());
    if (history)
      for (std::size_t i = 0; i < s.iteration_residuals.size(); ++i)
        history[i] = static_cast<double>(s.iteration_residuals[i]);
  }

  template <typename T>
  struct Op {
    Handle<T> const* A;
    template <typename It, typename Out>
    void operator()(It first, It last, Out out) const {
      std::vector<T> in(first, last);
      auto y = A->multiply(std::span<T const>{in});
      std::copy(y.begin(), y.end(), out);
    }
  };

  // The scalars of Lanczos_result<T> (lanczos.hpp:39-47).
  struct LanczosOut {
    i64 count, computed_restarts, converged_count, residual_count, restart_residuals_count;
    int converged;
  };

  template <typename T>
  void lanczos_run(Handle<T> const* A, i64 nev, i64 m, double tol, i64 max_restarts, int target,
                   int collect, T* eigenvalues, T* eigenvectors, T* residual_norms,
                   double* restart_residuals, LanczosOut* out) {
    sd::Lanczos_config<T> cfg{nev, m, static_cast<T>(tol), max_restarts,
                              static_cast<sd::Eigen_target>(target), collect != 0};
    auto r = sd::lanczos<T>(A->nrow(), cfg, Op<T>{A});
    out->count = static_cast<i64>(r.eigenvalues.size());
    out->computed_restarts = r.computed_restarts;
    out->converged_count = r.converged_count;
    out->residual_count = static_cast<i64>(r.residual_norms.size());
    out->restart_residuals_count = static_cast<i64>(r.restart_residuals.size());
    out->converged = r.converged ? 1 : 0;
    for (std::size_t k = 0; k < r.eigenvalues.size(); ++k) {
      eigenvalues[k] = r.eigenvalues[k];
      if (eigenvectors)
        std::copy(r.eigenvectors[k].begin(), r.eigenvectors[k].end(),
                  eigenvectors + k * A->nrow());
    }
    for (std::size_t k = 0; k < r.residual_norms.size(); ++k) residual_norms[k] = r.residual_norms[k];
    if (restart_residuals)
      for (std::size_t k = 0; k < r.restart_residuals.size(); ++k)
        restart_residuals[k] = static_cast<double>(r.restart_residuals[k]);
  }

  template <typename T>
  int cg(Handle<T> const* A, i64 n, T const* b, T* x, double tol,
         i64 restart, i64 max_it, int collect, int lk, int rk, double lmin,
         double lmax, i64 deg, Summary* out, double* history) {
    Prec<T> L, R;
    int e = setup_prec(L, A, lk, lmin, lmax, deg);
    if (e) return e;
    e = setup_prec(R, A, rk, lmin, lmax, deg);
    if (e) return e;
    std::vector<T> bv(b, b + n), xv(x, x + n);
    sd::CGConfig<T> cfg{static_cast<T>(tol), restart, max_it, collect != 0};
    auto s = sd::conjugate_gradient(bv.begin(), bv.end(), xv.begin(),
                                    xv.end(), cfg, Op<T>{A}, std::cref(L),
                                    std::cref(R));
    std::copy(xv.begin(), xv.end(), x);
    fill_summary<decltype(s), T>(out, s, history);
    return 0;
  }

  template <typename T>
  int bicgstab(Handle<T> const* A, i64 n, T const* b, T* x, double tol,
               i64 max_it, int collect, int lk, int rk, double lmin,
               double lmax, i64 deg, Summary* out, double* history) {
    Prec<T> L, R;
    int e = setup_prec(L, A, lk, lmin, lmax, deg);
    if (e) return e;
    e = setup_prec(R, A, rk, lmin, lmax, deg);
    if (e) return e;
    std::vector<T> bv(b, b + n), xv(x, x + n);
    sd::Bicgstab_config<T> cfg{static_cast<T>(tol), max_it, collect != 0};
    auto s = sd::bicgstab(bv.begin(), bv.end(), xv.begin(), xv.end(), cfg,
                          Op<T>{A}, std::cref(L), std::cref(R));
    std::copy(xv.begin(), xv.end(), x);
    fill_summary<decltype(s), T>(out, s, history);
    return 0;
  }

  template <typename T>
  int fgmres(Handle<T> const* A, i64 n, T const* b, T* x, double tol,
             i64 restart, i64 max_it, int collect, int pk, double lmin,
             double lmax, i64 deg, Summary* out, double* history) {
    Prec<T> P;
    int e = setup_prec(P, A, pk, lmin, lmax, deg);
    if (e) return e;
    std::vector<T> bv(b, b + n), xv(x, x + n);
    sd::Fgmres_config<T> cfg{static_cast<T>(tol), restart, max_it,
                             collect != 0};
    auto s = sd::fgmres(bv.begin(), bv.end(), xv.begin(), xv.end(), cfg,
                        Op<T>{A}, std::cref(P));
    std::copy(xv.begin(), xv.end(), x);
    fill_summary<decltype(s), T>(out, s, history);
    return 0;
  }

  template <typename T>
  int gmres(Handle<T> const* A, i64 n, T const* b, T* x, double tol,
            i64 restart, i64 max_it, int collect, int lk, int rk, double lmin,
            double lmax, i64 deg, Summary* out, double* history) {
    Prec<T> L, R;
    int e = setup_prec(L, A, lk, lmin, lmax, deg);
    if (e) return e;
    e = setup_prec(R, A, rk, lmin, lmax, deg);
    if (e) return e;
    std::vector<T> bv(b, b + n), xv(x, x + n);
    sd::Gmres_config<T> cfg{static_cast<T>(tol), restart, max_it,
                            collect != 0};
    auto s = sd::gmres(bv.begin(), bv.end(), xv.begin(), xv.end(), cfg,
                       Op<T>{A}, std::cref(L), std::cref(R));
    std::copy(xv.begin(), xv.end(), x);
    fill_summary<decltype(s), T>(out, s, history);
    return 0;
  }

  // cgs (cgs.hpp:374) and minres (minres.hpp:397): the bicgstab signature
  template <typename T, typename Cfg, typename F>
  int krylov2(Handle<T> const* A, i64 n, T const* b, T* x, double tol,
              i64 max_it, int collect, int lk, int rk, double lmin,
              double lmax, i64 deg, Summary* out, double* history, F solve) {
    Prec<T> L, R;
    int e = setup_prec(L, A, lk, lmin, lmax, deg);
    if (e) return e;
    e = setup_prec(R, A, rk, lmin, lmax, deg);
    if (e) return e;
    std::vector<T> bv(b, b + n), xv(x, x + n);
    Cfg cfg{static_cast<T>(tol), max_it, collect != 0};
    auto s = solve(bv, xv, cfg, L, R);
    std::copy(xv.begin(), xv.end(), x);
    fill_summary<decltype(s), T>(out, s, history);
    return 0;
  }

} // namespace

#define REF_API extern "C" __attribute__((visibility("default")))

#define REF_INSTANTIATE(T, S)                                                  \
  REF_API void* ref_csr_create_##S(i64 nrow, i64 ncol, i64 const* rp,          \
                                   i64 const* ci, T const* vals) {             \
    return make_csr<T>(nrow, ncol, rp, ci, vals);                              \
  }                                                                            \
  REF_API void ref_destroy_##S(void* h) { delete static_cast<Handle<T>*>(h); } \
  REF_API void ref_multiply_##S(void* h, T const* x, i64 ncol, T* y) {         \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto v = A->multiply(std::span<T const>{x, static_cast<std::size_t>(ncol)});\
    std::copy(v.begin(), v.end(), y);                                          \
  }                                                                            \
  /* Runs `reps` reference multiplies on each of `nthreads` threads at once; \
     returns the wall time in seconds. */                                      \
  REF_API double ref_multiply_threads_##S(void* h, T const* x, i64 ncol,       \
                                          int nthreads, int reps) {            \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto t0 = std::chrono::steady_clock::now();                                \
    std::vector<std::thread> pool;                                             \
    for (int t = 0; t < nthreads; ++t)                                         \
      pool.emplace_back([=] {                                                  \
        for (int r = 0; r < reps; ++r) {                                       \
          auto v = A->multiply(                                                \
            std::span<T const>{x, static_cast<std::size_t>(ncol)});            \
          asm volatile("" : : "r"(v.data()) : "memory");                       \
        }                                                                      \
      });                                                                      \
    for (auto& th : pool) th.join();                                           \
    auto t1 = std::chrono::steady_clock::now();                                \
    return std::chrono::duration<double>(t1 - t0).count();                     \
  }                                                                            \
  REF_API void* ref_to_ellpack_##S(void* h) {                                  \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto* e = new Handle<T>;                                                   \
    e->format = F_ELL;                                                         \
    e->ell = new sd::Ellpack_matrix<T>{sd::to_ellpack(*A->csr)};               \
    return e;                                                                  \
  }                                                                            \
  REF_API void* ref_to_jagged_diagonal_##S(void* h) {                          \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto* e = new Handle<T>;                                                   \
    e->format = F_JAD;                                                         \
    e->jad = new sd::Jagged_diagonal_matrix<T>{sd::to_jagged_diagonal(*A->csr)};\
    return e;                                                                  \
  }                                                                            \
  REF_API void* ref_to_block_sparse_row_##S(void* h, i64 br, i64 bc) {         \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto* e = new Handle<T>;                                                   \
    e->format = F_BSR;                                                         \
    e->bsr = new sd::Block_sparse_row_matrix<T>{                               \
      sd::to_block_sparse_row(*A->csr, br, bc)};                               \
    return e;                                                                  \
  }                                                                            \
  /* sizes: [nrow, ncol, nnz, width_or_njd_or_nblocks, nbr] */                 \
  REF_API void ref_info_##S(void* h, i64* out) {                               \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    switch (A->format) {                                                       \
      case F_CSR:                                                              \
        out[0] = A->csr->shape().row(); out[1] = A->csr->shape().column();     \
        out[2] = A->csr->size(); out[3] = 0; out[4] = 0; break;                \
      case F_ELL:                                                              \
        out[0] = A->ell->shape().row(); out[1] = A->ell->shape().column();     \
        out[2] = A->ell->size();                                               \
        out[3] = A->ell->sparsity().max_nnz_per_row(); out[4] = 0; break;      \
      case F_JAD:                                                              \
        out[0] = A->jad->shape().row(); out[1] = A->jad->shape().column();     \
        out[2] = A->jad->size();                                               \
        out[3] = static_cast<i64>(A->jad->sparsity().jdiag().size()) - 1;      \
        out[4] = 0; break;                                                     \
      default:                                                                 \
        out[0] = A->bsr->shape().row(); out[1] = A->bsr->shape().column();     \
        out[2] = A->bsr->size(); out[3] = A->bsr->sparsity().num_blocks();     \
        out[4] = A->bsr->sparsity().num_block_rows(); break;                   \
    }                                                                          \
  }                                                                            \
  /* Copies the layout out: CSR (a=row_ptr, b=col_ind), ELL (b=col_ind),     \
     JAD (a=jdiag, b=col_ind, c=perm), BSR (a=row_ptr, b=col_ind). */          \
  REF_API void ref_export_##S(void* h, i64* a, i64* b, i64* c, T* vals) {      \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto cp = [](auto span, auto* dst) {                                       \
      if (dst) std::copy(span.begin(), span.end(), dst);                       \
    };                                                                         \
    switch (A->format) {                                                       \
      case F_CSR:                                                              \
        cp(A->csr->row_ptr(), a); cp(A->csr->col_ind(), b);                    \
        cp(A->csr->values(), vals); break;                                     \
      case F_ELL:                                                              \
        cp(A->ell->sparsity().col_ind(), b); cp(A->ell->values(), vals);       \
        break;                                                                 \
      case F_JAD:                                                              \
        cp(A->jad->sparsity().jdiag(), a); cp(A->jad->sparsity().col_ind(), b);\
        cp(A->jad->sparsity().perm(), c); cp(A->jad->values(), vals); break;   \
      default:                                                                 \
        cp(A->bsr->sparsity().row_ptr(), a);                                   \
        cp(A->bsr->sparsity().col_ind(), b); cp(A->bsr->values(), vals);       \
        break;                                                                 \
    }                                                                          \
  }                                                                            \
  REF_API int ref_jacobi_##S(void* h, T* inv_d) {                              \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    try {                                                                      \
      auto d = sd::jacobi(*A->csr);                                            \
      std::copy(d.begin(), d.end(), inv_d);                                    \
    } catch (std::invalid_argument const&) {                                   \
      return -1;                                                               \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
  REF_API void ref_chebyshev_coeffs_##S(void* h, double lmin, double lmax,     \
                                        i64 degree, T* coeffs) {               \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto p = sd::chebyshev_preconditioner(*A->csr, static_cast<T>(lmin),       \
                                          static_cast<T>(lmax), degree);       \
    std::copy(p.coeffs.begin(), p.coeffs.end(), coeffs);                       \
  }                                                                            \
  REF_API void ref_chebyshev_apply_##S(void* h, double lmin, double lmax,      \
                                       i64 degree, T const* r, T* z) {         \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto p = sd::chebyshev_preconditioner(*A->csr, static_cast<T>(lmin),       \
                                          static_cast<T>(lmax), degree);       \
    i64 n = A->csr->shape().row();                                             \
    sd::chebyshev_preconditioner_apply(p, r, r + n, z);                        \
  }                                                                            \
  REF_API int ref_cg_##S(void* h, T const* b, T* x, double tol, i64 restart,   \
                         i64 max_it, int collect, int lk, int rk, double lmin, \
                         double lmax, i64 deg, Summary* out, double* hist) {   \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    return cg<T>(A, A->nrow(), b, x, tol, restart, max_it, collect, lk, rk,    \
                 lmin, lmax, deg, out, hist);                                  \
  }                                                                            \
  REF_API int ref_bicgstab_##S(void* h, T const* b, T* x, double tol,          \
                               i64 max_it, int collect, int lk, int rk,        \
                               double lmin, double lmax, i64 deg,              \
                               Summary* out, double* hist) {                   \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    return bicgstab<T>(A, A->nrow(), b, x, tol, max_it, collect, lk, rk, lmin, \
                       lmax, deg, out, hist);                                  \
  }                                                                            \
  REF_API int ref_fgmres_##S(void* h, T const* b, T* x, double tol,            \
                             i64 restart, i64 max_it, int collect, int pk,     \
                             double lmin, double lmax, i64 deg, Summary* out,  \
                             double* hist) {                                   \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    return fgmres<T>(A, A->nrow(), b, x, tol, restart, max_it, collect, pk,    \
                     lmin, lmax, deg, out, hist);                              \
  }                                                                            \
  REF_API int ref_gmres_##S(void* h, T const* b, T* x, double tol,             \
                            i64 restart, i64 max_it, int collect, int lk,      \
                            int rk, double lmin, double lmax, i64 deg,         \
                            Summary* out, double* hist) {                      \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    return gmres<T>(A, A->nrow(), b, x, tol, restart, max_it, collect, lk, rk, \
                    lmin, lmax, deg, out, hist);                               \
  }                                                                            \
  REF_API int ref_cgs_##S(void* h, T const* b, T* x, double tol, i64 max_it,   \
                          int collect, int lk, int rk, double lmin,            \
                          double lmax, i64 deg, Summary* out, double* hist) {  \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    return krylov2<T, sd::Cgs_config<T>>(                                      \
      A, A->nrow(), b, x, tol, max_it, collect, lk, rk, lmin, lmax, deg, out,  \
      hist, [&](auto& bv, auto& xv, auto cfg, auto& L, auto& R) {              \
        return sd::cgs(bv.begin(), bv.end(), xv.begin(), xv.end(), cfg,        \
                       Op<T>{A}, std::cref(L), std::cref(R));                  \
      });                                                                      \
  }                                                                            \
  REF_API int ref_minres_##S(void* h, T const* b, T* x, double tol,            \
                             i64 max_it, int collect, int lk, int rk,          \
                             double lmin, double lmax, i64 deg, Summary* out,  \
                             double* hist) {                                   \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    return krylov2<T, sd::Minres_config<T>>(                                   \
      A, A->nrow(), b, x, tol, max_it, collect, lk, rk, lmin, lmax, deg, out,  \
      hist, [&](auto& bv, auto& xv, auto cfg, auto& L, auto& R) {              \
        return sd::minres(bv.begin(), bv.end(), xv.begin(), xv.end(), cfg,     \
                          Op<T>{A}, std::cref(L), std::cref(R));               \
      });                                                                      \
  }                                                                            \
  REF_API void* ref_mm_read_##S(char const* text, i64 len, char* err,          \
                                i64 errcap) {                                  \
    try {                                                                      \
      std::istringstream is{std::string(text, static_cast<std::size_t>(len))}; \
      auto coo = sd::read_matrix_market<T>(is);                                \
      return wrap_csr<T>(sd::to_compressed_row(coo));                          \
    } catch (std::exception const& ex) {                                       \
      std::snprintf(err, static_cast<std::size_t>(errcap), "%s", ex.what());   \
      return nullptr;                                                          \
    }                                                                          \
  }                                                                            \
  REF_API i64 ref_mm_write_##S(void* h, char* buf, i64 cap) {                  \
    std::ostringstream os;                                                     \
    sd::write_matrix_market(os, *static_cast<Handle<T>*>(h)->csr);             \
    auto str = os.str();                                                       \
    if (buf && cap > 0)                                                        \
      std::memcpy(buf, str.data(),                                             \
                  std::min<std::size_t>(str.size(), static_cast<std::size_t>(cap))); \
    return static_cast<i64>(str.size());                                       \
  }                                                                            \
  REF_API void ref_lanczos_##S(void* h, i64 nev, i64 m, double tol, i64 maxr,  \
                              int target, int collect, T* ev, T* evec,         \
                              T* res, double* rr, LanczosOut* out) {           \
    lanczos_run<T>(static_cast<Handle<T>*>(h), nev, m, tol, maxr, target,      \
                   collect, ev, evec, res, rr, out);                           \
  }                                                                            \
  REF_API void ref_eigenvalue_bounds_##S(void* h, i64 num_iter, T* out2) {     \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    auto p = sd::estimate_eigenvalue_bounds<T>(A->nrow(), Op<T>{A}, num_iter); \
    out2[0] = p.first;                                                         \
    out2[1] = p.second;                                                        \
  }                                                                            \
  REF_API double ref_spectral_radius_##S(void* h, i64 num_iter) {              \
    auto* A = static_cast<Handle<T>*>(h);                                      \
    return static_cast<double>(                                                \
      sd::estimate_spectral_radius<T>(A->nrow(), Op<T>{A}, num_iter));         \
  }                                                                            \
  REF_API void* ref_poisson_2d_##S(i64 nx, i64 ny, double shift) {             \
    return wrap_csr<T>(sd::poisson_2d<T>(nx, ny, static_cast<T>(shift)));      \
  }                                                                            \
  REF_API void* ref_tridiagonal_##S(i64 n, double sub, double diag,            \
                                    double sup) {                              \
    return wrap_csr<T>(sd::tridiagonal_matrix<T>(                              \
      n, static_cast<T>(sub), static_cast<T>(diag), static_cast<T>(sup)));     \
  }                                                                            \
  REF_API void* ref_convdiff_centered_2d_##S(i64 nx, i64 ny, double d,         \
                                             double cx, double cy,             \
                                             double shift) {                   \
    return wrap_csr<T>(sd::convdiff_centered_2d<T>(                            \
      nx, ny, static_cast<T>(d), static_cast<T>(cx), static_cast<T>(cy),       \
      static_cast<T>(shift)));                                                 \
  }                                                                            \
  REF_API void* ref_convection_diffusion_2d_##S(i64 nx, i64 ny, double d,      \
                                                double cx, double cy) {        \
    return wrap_csr<T>(sd::convection_diffusion_2d<T>(                         \
      nx, ny, static_cast<T>(d), static_cast<T>(cx), static_cast<T>(cy)));     \
  }                                                                            \
  REF_API void* ref_nonsymmetric_sample_##S() {                                \
    return wrap_csr<T>(sd::nonsymmetric_sample<T>());                          \
  }

REF_INSTANTIATE(double, f64)
REF_INSTANTIATE(float, f32)
