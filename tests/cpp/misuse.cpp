// Two misuses of the drop-in that must not compile (each selected by
// -DMISUSE=n), so that no host callable is silently run on the CPU and no
// device operator is handed to a host solver.
//   1: a host lambda as the preconditioner of the device overload
//   2: the device operator sk::gpu::spmv(A) given to the reference's own
//      solver (a host preconditioner selects it)
#include <vector>

#include <sparkit/data/matgen.hpp>

#include "sparkit_b200.hpp"

using namespace sparkit::data::detail;

int main() {
  auto A = tridiagonal_matrix<double>(8, -1.0, 4.0, -1.0);
  sk::gpu::Device_matrix<double> Ad(A);
  std::vector<double> b(8, 1.0), x(8, 0.0);
  auto host_prec = [](auto first, auto last, auto out) { std::copy(first, last, out); };
  CGConfig<double> cfg{.tolerance = 1e-10, .restart_iterations = 10, .max_iterations = 10};
#if MISUSE == 1
  conjugate_gradient(b.begin(), b.end(), x.begin(), x.end(), cfg, sk::gpu::spmv(Ad), host_prec, sk::gpu::identity);
#elif MISUSE == 2
  sparkit::data::detail::conjugate_gradient(b.begin(), b.end(), x.begin(), x.end(), cfg, sk::gpu::spmv(Ad),
                                            host_prec, host_prec);
#endif
  return 0;
}
