/*
 * sparkit_b200.hpp -- the C++ drop-in of the B200 path, over the C ABI of
 * sparkit_b200.h.
 *
 * A sparkit user keeps the reference's matrix classes, config and summary
 * structs and call syntax.  What changes is the operator and
 * preconditioner arguments: device objects instead of host lambdas.
 *
 *   using namespace sparkit::data::detail;
 *   Compressed_row_matrix<double> A = ...;
 *   sk::gpu::Device_matrix<double> Ad(A);             // uploads once
 *   auto y = multiply(Ad, std::span<double const>(x)); // sparse_blas.hpp:19
 *   auto s = conjugate_gradient(b.begin(), b.end(), x.begin(), x.end(),
 *                               CGConfig<double>{1e-10, 1000, 1000},
 *                               sk::gpu::spmv(Ad), sk::gpu::jacobi(Ad),
 *                               sk::gpu::identity);   // conjugate_gradient.hpp:347
 *
 * The calls are unqualified, as the reference's tests write them.  Argument-
 * dependent lookup finds both the reference's templates and these
 * overloads, and these are the more specialised, so they are chosen.  The
 * whole solve then runs on the device, and b and x cross the host link once
 * each way.  Host callables are not run on the device.  A device operator
 * passed to a reference solver, or a host lambda passed here, fails to
 * compile with a message.  There is no CPU fallback.
 *
 * Errors: a failed call throws sk::gpu::error (a std::runtime_error that
 * holds the sk_status).  A zero diagonal in jacobi() throws
 * std::invalid_argument("jacobi: zero diagonal entry"), as jacobi.hpp:31
 * does.  Solvers report convergence in their summary, as the reference's
 * do; a Krylov breakdown the reference would loop on ends the solve
 * unconverged.
 *
 * Needs the reference's headers (sparkit/data/...) and its generated
 * sparkit/config.hpp on the include path, C++20, and libsparkit_b200.so at
 * link time.
 */
#ifndef SPARKIT_B200_HPP
#define SPARKIT_B200_HPP

#include <algorithm>
#include <cstdint>
#include <iterator>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include <sparkit/data/Block_sparse_row_matrix.hpp>
#include <sparkit/data/Compressed_row_matrix.hpp>
#include <sparkit/data/Ellpack_matrix.hpp>
#include <sparkit/data/Jagged_diagonal_matrix.hpp>
#include <sparkit/data/bicgstab.hpp>
#include <sparkit/data/conjugate_gradient.hpp>
#include <sparkit/data/fgmres.hpp>

#include "sparkit_b200.h"

namespace sk::gpu {

namespace ref = sparkit::data::detail;

// A failed C-ABI call: the status and the library's message.
class error : public std::runtime_error {
 public:
  error(sk_status s, std::string const& msg) : std::runtime_error(msg), status_(s) {}
  sk_status status() const noexcept { return status_; }

 private:
  sk_status status_;
};

inline void check(sk_status s) {
  if (s != SK_OK) {
    char const* m = sk_last_error();
    throw error(s, std::string("sparkit_b200: ") + (m ? m : "error ") + " (status " + std::to_string(s) + ")");
  }
}

template <typename T>
constexpr sk_dtype dtype_of() {
  static_assert(std::is_same_v<T, double> || std::is_same_v<T, float>,
                "the device path holds double or float values");
  return std::is_same_v<T, double> ? SK_F64 : SK_F32;
}

namespace detail {

// The reference's index spans hold size_type = std::ptrdiff_t; the C ABI
// takes int64_t.  Both are 64-bit on the supported platforms, and the
// values are passed through without change (the library narrows them to
// int32 on the device, with a range check).
template <typename I>
int64_t const* index_ptr(std::span<I const> s) {
  static_assert(sizeof(I) == sizeof(int64_t) && std::is_integral_v<I> && std::is_signed_v<I>,
                "sparkit's size_type must be a signed 64-bit integer");
  return reinterpret_cast<int64_t const*>(s.data());
}

}  // namespace detail

// A device-resident copy of one reference matrix object (the handle of
// sk_csr_create / sk_ell_create / sk_jad_create / sk_bsr_create).  Move-only.
template <typename T>
class Device_matrix {
 public:
  using value_type = T;

  // Compressed_row_matrix<T> (Compressed_row_matrix.hpp:20-132)
  explicit Device_matrix(ref::Compressed_row_matrix<T> const& A) {
    auto sh = A.shape();
    check(sk_csr_create(&h_, sh.row(), sh.column(), detail::index_ptr(A.row_ptr()), detail::index_ptr(A.col_ind()),
                        A.values().data(), dtype_of<T>()));
    nrow_ = sh.row();
    ncol_ = sh.column();
  }

  // Ellpack_matrix<T> (Ellpack_matrix.hpp:20-122)
  explicit Device_matrix(ref::Ellpack_matrix<T> const& A) {
    auto sh = A.shape();
    auto const& sp = A.sparsity();
    check(sk_ell_create(&h_, sh.row(), sh.column(), sp.max_nnz_per_row(), detail::index_ptr(sp.col_ind()),
                        A.values().data(), dtype_of<T>()));
    nrow_ = sh.row();
    ncol_ = sh.column();
  }

  // Jagged_diagonal_matrix<T> (Jagged_diagonal_matrix.hpp:20-144)
  explicit Device_matrix(ref::Jagged_diagonal_matrix<T> const& A) {
    auto sh = A.shape();
    auto const& sp = A.sparsity();
    auto jd = sp.jdiag();
    int64_t const njd = jd.empty() ? 0 : static_cast<int64_t>(jd.size()) - 1;
    auto pm = sp.perm();
    check(sk_jad_create(&h_, sh.row(), sh.column(), njd, pm.empty() ? nullptr : detail::index_ptr(pm),
                        detail::index_ptr(jd), detail::index_ptr(sp.col_ind()), A.values().data(), dtype_of<T>()));
    nrow_ = sh.row();
    ncol_ = sh.column();
  }

  // Block_sparse_row_matrix<T> (Block_sparse_row_matrix.hpp:21-150)
  explicit Device_matrix(ref::Block_sparse_row_matrix<T> const& A) {
    auto sh = A.shape();
    auto const& sp = A.sparsity();
    check(sk_bsr_create(&h_, sh.row(), sh.column(), sp.block_rows(), sp.block_cols(), detail::index_ptr(sp.row_ptr()),
                        detail::index_ptr(sp.col_ind()), A.values().data(), dtype_of<T>()));
    nrow_ = sh.row();
    ncol_ = sh.column();
  }

  Device_matrix(Device_matrix&& o) noexcept : h_(std::exchange(o.h_, nullptr)), nrow_(o.nrow_), ncol_(o.ncol_) {}
  Device_matrix& operator=(Device_matrix&& o) noexcept {
    if (this != &o) {
      reset();
      h_ = std::exchange(o.h_, nullptr);
      nrow_ = o.nrow_;
      ncol_ = o.ncol_;
    }
    return *this;
  }
  Device_matrix(Device_matrix const&) = delete;
  Device_matrix& operator=(Device_matrix const&) = delete;
  ~Device_matrix() { reset(); }

  sk_matrix handle() const noexcept { return h_; }
  int64_t rows() const noexcept { return nrow_; }
  int64_t columns() const noexcept { return ncol_; }

 private:
  void reset() noexcept {
    if (h_) sk_matrix_destroy(h_);
    h_ = nullptr;
  }
  sk_matrix h_ = nullptr;
  int64_t nrow_ = 0, ncol_ = 0;
};

// multiply(A, x) -> y (sparse_blas.hpp:19-35, spmv.hpp:119/148/182) on the
// device: x copied in, y copied out (sk_spmv_host).
template <typename T>
std::vector<T> multiply(Device_matrix<T> const& A, std::span<T const> x) {
  if (static_cast<int64_t>(x.size()) != A.columns())
    throw std::invalid_argument("multiply: x must hold one value per column");
  std::vector<T> y(static_cast<std::size_t>(A.rows()));
  check(sk_spmv_host(A.handle(), x.data(), y.data()));
  return y;
}

// The linear-operator argument of the solvers: y = A x on the device.  It
// is not a host callable: a reference solver given one fails to compile.
template <typename T>
struct spmv_op {
  Device_matrix<T> const* A;
  template <typename In, typename Out>
  void operator()(In, In, Out) const {
    static_assert(sizeof(In) == 0,
                  "sk::gpu::spmv(A) runs only inside the sk::gpu solver overloads: pass device preconditioners "
                  "(sk::gpu::jacobi, sk::gpu::chebyshev, sk::gpu::identity) so that they are chosen");
  }
};

template <typename T>
spmv_op<T> spmv(Device_matrix<T> const& A) {
  return spmv_op<T>{&A};
}

// The identity preconditioner (the reference tests' copy callable).
struct identity_t {
  sk_precond handle() const noexcept { return nullptr; }
};
inline constexpr identity_t identity{};

// A device preconditioner handle (shared by copies of the object).
class precond_base {
 public:
  sk_precond handle() const noexcept { return h_ ? h_->h : nullptr; }

 protected:
  struct holder {
    sk_precond h = nullptr;
    ~holder() {
      if (h) sk_precond_destroy(h);
    }
  };
  std::shared_ptr<holder> h_;
};

// jacobi(A) (jacobi.hpp:27-35): the inverse diagonal, on the device.
template <typename T>
class jacobi_preconditioner : public precond_base {
 public:
  explicit jacobi_preconditioner(Device_matrix<T> const& A) {
    h_ = std::make_shared<holder>();
    sk_status s = sk_jacobi_create(&h_->h, A.handle());
    if (s == SK_ZERO_DIAGONAL) throw std::invalid_argument("jacobi: zero diagonal entry");
    check(s);
  }
};

template <typename T>
jacobi_preconditioner<T> jacobi(Device_matrix<T> const& A) {
  return jacobi_preconditioner<T>(A);
}

// chebyshev_preconditioner(A, lambda_min, lambda_max, degree)
// (chebyshev_preconditioner.hpp:46-84) of a CSR handle.
template <typename T>
class chebyshev_preconditioner : public precond_base {
 public:
  chebyshev_preconditioner(Device_matrix<T> const& A, T lambda_min, T lambda_max, ref::size_type degree) {
    h_ = std::make_shared<holder>();
    check(sk_chebyshev_create(&h_->h, A.handle(), static_cast<double>(lambda_min), static_cast<double>(lambda_max),
                              static_cast<int64_t>(degree)));
  }
};

template <typename T>
chebyshev_preconditioner<T> chebyshev(Device_matrix<T> const& A, T lambda_min, T lambda_max,
                                      ref::size_type degree) {
  return chebyshev_preconditioner<T>(A, lambda_min, lambda_max, degree);
}

template <typename P>
constexpr bool is_device_preconditioner_v =
    std::is_same_v<P, identity_t> || std::is_base_of_v<precond_base, P>;

namespace detail {

template <typename P>
void require_device_preconditioner() {
  static_assert(is_device_preconditioner_v<P>,
                "the sk::gpu solver overloads take device preconditioners (sk::gpu::jacobi, sk::gpu::chebyshev, "
                "sk::gpu::identity); host callables are not run on the device");
}

template <typename T, typename XIter>
void scatter(std::vector<T> const& x, XIter xfirst, XIter xlast) {
  auto it = x.begin();
  for (; xfirst != xlast; ++xfirst, ++it) *xfirst = *it;
}

template <typename T, typename BIter, typename XIter>
void stage(BIter bfirst, BIter blast, XIter xfirst, XIter xlast, int64_t n, std::vector<T>& b, std::vector<T>& x) {
  b.assign(bfirst, blast);
  x.assign(xfirst, xlast);
  if (static_cast<int64_t>(b.size()) != n || static_cast<int64_t>(x.size()) != n)
    throw std::invalid_argument("b and x must hold one value per row of the matrix");
}

template <typename Summary, typename T>
Summary to_summary(sk_summary const& s, std::vector<double> const& hist) {
  Summary out{};
  out.residual_norm = static_cast<T>(s.residual_norm);
  out.computed_iterations = static_cast<decltype(out.computed_iterations)>(s.computed_iterations);
  out.converged = s.converged != 0;
  out.iteration_residuals.reserve(static_cast<std::size_t>(s.history_length));
  for (int64_t k = 0; k < s.history_length; ++k) out.iteration_residuals.push_back(static_cast<T>(hist[k]));
  return out;
}

}  // namespace detail

// conjugate_gradient (conjugate_gradient.hpp:339-366), the same parameter
// list and return type, with the operator and preconditioners on the device.
template <typename BIter, typename XIter, typename T, typename L, typename R>
ref::CGSummary<T> conjugate_gradient(BIter bfirst, BIter blast, XIter xfirst, XIter xlast, ref::CGConfig<T> cfg,
                                     spmv_op<T> op, L left, R right) {
  detail::require_device_preconditioner<L>();
  detail::require_device_preconditioner<R>();
  std::vector<T> b, x;
  detail::stage<T>(bfirst, blast, xfirst, xlast, op.A->rows(), b, x);
  sk_cg_config c{static_cast<double>(cfg.tolerance), static_cast<int64_t>(cfg.restart_iterations),
                 static_cast<int64_t>(cfg.max_iterations), cfg.collect_residuals ? 1 : 0};
  std::vector<double> hist(cfg.collect_residuals ? static_cast<std::size_t>(cfg.max_iterations) + 4 : 1);
  sk_summary s{};
  check(sk_cg_solve_host(op.A->handle(), left.handle(), right.handle(), b.data(), x.data(), &c, &s,
                         cfg.collect_residuals ? hist.data() : nullptr));
  detail::scatter(x, xfirst, xlast);
  return detail::to_summary<ref::CGSummary<T>, T>(s, hist);
}

// bicgstab (bicgstab.hpp:383-410).
template <typename BIter, typename XIter, typename T, typename L, typename R>
ref::Bicgstab_summary<T> bicgstab(BIter bfirst, BIter blast, XIter xfirst, XIter xlast, ref::Bicgstab_config<T> cfg,
                                  spmv_op<T> op, L left, R right) {
  detail::require_device_preconditioner<L>();
  detail::require_device_preconditioner<R>();
  std::vector<T> b, x;
  detail::stage<T>(bfirst, blast, xfirst, xlast, op.A->rows(), b, x);
  sk_bicgstab_config c{static_cast<double>(cfg.tolerance), static_cast<int64_t>(cfg.max_iterations),
                       cfg.collect_residuals ? 1 : 0};
  // one residual per half step at most
  std::vector<double> hist(cfg.collect_residuals ? 2 * static_cast<std::size_t>(cfg.max_iterations) + 4 : 1);
  sk_summary s{};
  check(sk_bicgstab_solve_host(op.A->handle(), left.handle(), right.handle(), b.data(), x.data(), &c, &s,
                               cfg.collect_residuals ? hist.data() : nullptr));
  detail::scatter(x, xfirst, xlast);
  return detail::to_summary<ref::Bicgstab_summary<T>, T>(s, hist);
}

// fgmres (fgmres.hpp:452-470).
template <typename BIter, typename XIter, typename T, typename P>
ref::Fgmres_summary<T> fgmres(BIter bfirst, BIter blast, XIter xfirst, XIter xlast, ref::Fgmres_config<T> cfg,
                              spmv_op<T> op, P preconditioner) {
  detail::require_device_preconditioner<P>();
  std::vector<T> b, x;
  detail::stage<T>(bfirst, blast, xfirst, xlast, op.A->rows(), b, x);
  sk_fgmres_config c{static_cast<double>(cfg.tolerance), static_cast<int64_t>(cfg.restart_dimension),
                     static_cast<int64_t>(cfg.max_iterations), cfg.collect_residuals ? 1 : 0};
  std::vector<double> hist(cfg.collect_residuals ? static_cast<std::size_t>(cfg.max_iterations) + 4 : 1);
  sk_summary s{};
  check(sk_fgmres_solve_host(op.A->handle(), preconditioner.handle(), b.data(), x.data(), &c, &s,
                             cfg.collect_residuals ? hist.data() : nullptr));
  detail::scatter(x, xfirst, xlast);
  return detail::to_summary<ref::Fgmres_summary<T>, T>(s, hist);
}

}  // namespace sk::gpu

#endif /* SPARKIT_B200_HPP */
