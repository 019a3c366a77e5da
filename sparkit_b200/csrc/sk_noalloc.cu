// sk_noalloc.cu -- a Chebyshev preconditioner apply that allocates nothing.
//
// Who needs it: a caller that must not allocate device memory while it is
// solving -- for example a preconditioner callback invoked from inside
// another solver library's iteration loop, where that library reserved all
// device memory up front and a cudaMalloc would fail or stall the loop.
// The regular route, sk_chebyshev_create + sk_precond_apply, allocates two
// n-vectors of work space when the preconditioner is created; this entry
// point instead keeps them in one file-scope device array.
//
// Limits and sharing:
//  - the array holds 2 x kNoAllocRows values (kNoAllocRows = 1,048,576 rows
//    per work vector, 16 MiB), for FP64 and FP32 alike; larger matrices are
//    rejected with SK_INVALID_ARG;
//  - every GPU on which this entry point runs holds the 16 MiB until the
//    process exits;
//  - all calls share the array and it keeps the last call's contents: each
//    call writes every work entry it later reads (b_{d+1} = 0 and
//    b_d = c_d r are stored before any product), so no clearing is needed,
//    but two calls that overlap on the GPU (different streams, or different
//    host threads) race on the array and must be serialized by the caller;
//  - every call looks up the array's device address on the current device
//    with cudaGetSymbolAddress; the first call on a device may load the
//    module to do so, so that first call should come before any stream
//    capture begins.
#include "sk_vec.cuh"

namespace sk {
namespace {

constexpr i64 kNoAllocRows = i64(1) << 20;
constexpr i64 kNoAllocMaxDegree = 64;

// Two work vectors of kNoAllocRows values each (read as float for FP32).
__device__ __align__(256) double sk_noalloc_cheb_scratch[2 * kNoAllocRows];

// Device address of the scratch array on the current device.  The array's
// name in host code is only a host-side stand-in, so kernels are given this
// address instead.  It is looked up on every call (no allocation, and no
// address cached across a cudaDeviceReset).
sk_status scratch_address(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, sk_noalloc_cheb_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
  *out = p;
  return SK_OK;
}

}  // namespace
}  // namespace sk

using namespace sk;

extern "C" SK_API sk_status sk_chebyshev_apply_noalloc(sk_matrix A, double lambda_min, double lambda_max,
                                                       int64_t degree, const void* r_dev, void* z_dev,
                                                       sk_stream s) {
  SK_CHECK(A, SK_INVALID_ARG, "null matrix handle");
  SK_CHECK(A->format == SK_CSR, SK_INVALID_ARG,
           "the Chebyshev preconditioner needs a CSR handle (chebyshev_preconditioner.hpp:29)");
  SK_CHECK(A->nrow == A->ncol, SK_INVALID_ARG, "the Chebyshev preconditioner needs a square matrix");
  SK_CHECK(A->nrow <= kNoAllocRows, SK_INVALID_ARG,
           "matrix has " + std::to_string(A->nrow) +
               " rows; the no-allocation Chebyshev apply holds at most 1048576 rows "
               "(use sk_chebyshev_create and sk_precond_apply for larger matrices)");
  SK_CHECK(degree >= 0 && degree <= kNoAllocMaxDegree, SK_INVALID_ARG,
           "degree must be in [0, 64] for the no-allocation Chebyshev apply");
  SK_CHECK(A->nrow == 0 || (r_dev && z_dev), SK_INVALID_ARG, "null r or z");
  if (A->nrow == 0) return SK_OK;
  int dev = -1;
  SK_CUDA(cudaGetDevice(&dev));
  SK_CHECK(dev == A->device, SK_INVALID_ARG, "the matrix handle belongs to another device than the current one");
  void* scratch = nullptr;
  sk_status st = scratch_address(&scratch);
  if (st != SK_OK) return st;
  double co[kNoAllocMaxDegree + 1];
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64) {
    chebyshev_coefficients<double>(lambda_min, lambda_max, degree, co);
    double* w = static_cast<double*>(scratch);
    chebyshev_clenshaw<double>(A, co, degree, lambda_min, lambda_max, static_cast<const double*>(r_dev),
                               static_cast<double*>(z_dev), w, w + kNoAllocRows, RedWs{}, nullptr, cs);
  } else {
    const float lmin = static_cast<float>(lambda_min), lmax = static_cast<float>(lambda_max);
    chebyshev_coefficients<float>(lmin, lmax, degree, co);
    float* w = static_cast<float*>(scratch);
    chebyshev_clenshaw<float>(A, co, degree, lmin, lmax, static_cast<const float*>(r_dev),
                              static_cast<float*>(z_dev), w, w + kNoAllocRows, RedWs{}, nullptr, cs);
  }
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}
