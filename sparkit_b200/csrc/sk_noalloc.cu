// sk_noalloc.cu -- a Chebyshev preconditioner apply that allocates nothing.
//
// Who needs it: a caller that must not allocate device memory while it is
// solving -- for example a preconditioner callback invoked from inside
// another solver library's iteration loop whose device memory is reserved
// up front, or a code path that runs while its stream is being captured
// into a CUDA graph (cudaMalloc is not permitted there).  The regular route,
// sk_chebyshev_create + sk_precond_apply, allocates two n-vectors of work
// space when the preconditioner is created; this entry point instead keeps
// them in one file-scope device array.
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
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (this may load the module), so that first call
//    must come before any stream capture begins.
#include <cmath>
#include <mutex>

#include "sk_vec.cuh"

namespace sk {
namespace {

constexpr i64 kNoAllocRows = i64(1) << 20;
constexpr i64 kNoAllocMaxDegree = 64;
constexpr int kMaxDevices = 64;

// Two work vectors of kNoAllocRows values each (read as float for FP32).
__device__ __align__(256) double sk_noalloc_cheb_scratch[2 * kNoAllocRows];

std::mutex g_scratch_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.  The array's name in host code is only a host-side stand-in,
// so kernels must be given this address instead.
sk_status scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices)
    return fail(SK_NOT_SUPPORTED, "no-alloc scratch: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, sk_noalloc_cheb_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return SK_OK;
}

// Chebyshev coefficients of 1/lambda on [lmin, lmax] in the value type T,
// by the discrete cosine sampling of chebyshev_preconditioner.hpp:53-73,
// written into a caller array (no allocation).
template <typename T>
void coefficients(T lmin, T lmax, i64 d, double* out) {
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

// The Clenshaw recurrence of chebyshev_preconditioner.hpp:98-169 with the
// two work vectors in the static scratch.
template <typename T>
void apply(const sk_matrix_s* A, const double* co, i64 d, T lmin, T lmax, const T* r, T* z,
           T* work, cudaStream_t st) {
  const i64 n = A->nrow;
  const T sum = lmax + lmin;
  const T diff = lmax - lmin;
  if (d == 0 || diff == T(0)) {
    launch_vec(n, OpScaleCopySkip<T>{static_cast<T>(co[0]), r, z}, RedWs{}, nullptr, st);
    return;
  }
  T* b_prev = work;
  T* b_curr = work + kNoAllocRows;
  launch_vec(n, OpChebInit<T>{static_cast<T>(co[d]), r, b_curr, b_prev, nullptr}, RedWs{}, nullptr, st);
  for (i64 k = d - 1; k >= 1; --k) {
    launch_spmv<T>(A, b_curr, EpiChebStep<T>{static_cast<T>(co[k]), sum, diff, r, b_curr, b_prev}, RedWs{},
                   nullptr, st);
    T* t = b_prev;
    b_prev = b_curr;
    b_curr = t;
  }
  launch_spmv<T>(A, b_curr, EpiChebFinal<T>{static_cast<T>(co[0]), sum, diff, r, b_curr, b_prev, z}, RedWs{},
                 nullptr, st);
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
  sk_status st = scratch_address(dev, &scratch);
  if (st != SK_OK) return st;
  double co[kNoAllocMaxDegree + 1];
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64) {
    coefficients<double>(lambda_min, lambda_max, degree, co);
    apply<double>(A, co, degree, lambda_min, lambda_max, static_cast<const double*>(r_dev),
                  static_cast<double*>(z_dev), static_cast<double*>(scratch), cs);
  } else {
    const float lmin = static_cast<float>(lambda_min), lmax = static_cast<float>(lambda_max);
    coefficients<float>(lmin, lmax, degree, co);
    apply<float>(A, co, degree, lmin, lmax, static_cast<const float*>(r_dev), static_cast<float*>(z_dev),
                 static_cast<float*>(scratch), cs);
  }
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}
