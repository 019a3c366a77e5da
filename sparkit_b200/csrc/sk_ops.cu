// sk_ops.cu -- C ABI of the SpMV, BLAS-1 and preconditioner operations.
#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <vector>

#include "sk_learned.cuh"
#include "sk_twolevel.cuh"
#include "sk_vec.cuh"

namespace sk {

// Reduction workspace of the standalone BLAS-1 calls: one per process,
// grown on demand, serialized by a mutex (those calls synchronize).
static std::mutex g_red_mutex;
static RedWs g_red;
static double* g_red_out = nullptr;

static sk_status global_red(int ctas, RedWs* ws, double** out) {
  if (g_red.capacity < ctas) {
    if (g_red.partials) cudaFree(g_red.partials);
    if (g_red.counter) cudaFree(g_red.counter);
    g_red = RedWs{};
    SK_CUDA(cudaMalloc(&g_red.partials, static_cast<size_t>(ctas) * kMaxRed * sizeof(double)));
    SK_CUDA(cudaMalloc(&g_red.counter, sizeof(unsigned)));
    SK_CUDA(cudaMemset(g_red.counter, 0, sizeof(unsigned)));
    g_red.capacity = ctas;
  }
  if (!g_red_out) SK_CUDA(cudaMalloc(&g_red_out, 8 * sizeof(double)));
  *ws = g_red;
  *out = g_red_out;
  return SK_OK;
}

__global__ void extract_inv_diag_kernel(i64 len, const int* __restrict__ rp,
                                        const int* __restrict__ ci, const double* __restrict__ v64,
                                        const float* __restrict__ v32, int f32, void* out,
                                        unsigned long long* zeros) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  if (i >= len) return;
  int lo = rp[i], hi = rp[i + 1];
  const int end = hi;
  while (lo < hi) {  // lower_bound of column i, unary.hpp:30-32
    int mid = lo + (hi - lo) / 2;
    if (ci[mid] < i) lo = mid + 1; else hi = mid;
  }
  const bool found = lo < end && ci[lo] == i;
  if (f32) {
    float d = found ? v32[lo] : 0.0f;
    if (d == 0.0f) atomicAdd(zeros, 1ull);
    static_cast<float*>(out)[i] = d == 0.0f ? 0.0f : __fdiv_rn(1.0f, d);
  } else {
    double d = found ? v64[lo] : 0.0;
    if (d == 0.0) atomicAdd(zeros, 1ull);
    static_cast<double*>(out)[i] = d == 0.0 ? 0.0 : __ddiv_rn(1.0, d);
  }
}

// Chebyshev coefficients (chebyshev_preconditioner.hpp:53-73) as the
// handle's host copy.
template <typename T>
static std::vector<double> cheb_coeffs(T lmin, T lmax, i64 degree) {
  std::vector<double> out(static_cast<size_t>(degree + 1));
  chebyshev_coefficients<T>(lmin, lmax, degree, out.data());
  return out;
}

// out = in converted to the other precision, skipped once a solve is done.
template <typename From, typename To>
struct OpConvert {
  static constexpr int kNR = 0;
  struct In { From v; };
  const From* in;
  To* out;
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {in[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { out[i] = static_cast<To>(v.v); }
  __device__ void finalize(const double*) const {}
};

// An FP32 apply of a preconditioner made on an FP64 handle (the inner
// solve of the mixed-precision FGMRES) uses its FP32 copies: the inverse
// diagonal rounded to float, the handle's FP32 values for the Chebyshev
// products; a two-level preconditioner runs in FP64 between a widening and
// a narrowing pass.
template <typename T>
static void precond_apply_t(const sk_precond_s* M, i64 n, const T* r, T* z, RedWs ws,
                            const Scalars* sc, cudaStream_t st) {
  constexpr bool narrow = sizeof(T) == 4;
  const bool from64 = M && M->dtype == SK_F64;
  if (!M) {
    launch_vec(n, OpCopy<T>{r, z}, ws, sc, st);
  } else if (M->kind == 1) {
    const T* inv = narrow && from64 ? reinterpret_cast<const T*>(M->inv_diag32) : static_cast<const T*>(M->inv_diag);
    launch_vec(n, OpJacobi<T>{inv, r, z}, ws, sc, st);
  } else if (M->kind == 3) {
    if constexpr (sizeof(T) == 8) {
      if (learned_apply(M, r, z, st) != SK_OK) set_error("learned preconditioner apply failed");
    }
  } else if (M->kind == 4) {
    if constexpr (sizeof(T) == 8) {
      twolevel_apply(M, r, z, ws, sc, st);
    } else {
      launch_vec(n, OpConvert<float, double>{r, M->cvt_in}, ws, sc, st);
      twolevel_apply(M, M->cvt_in, M->cvt_out, ws, sc, st);
      launch_vec(n, OpConvert<double, float>{M->cvt_out, z}, ws, sc, st);
    }
  } else {
    const T* vals = narrow && from64 ? reinterpret_cast<const T*>(f32_values(M->A)) : nullptr;
    chebyshev_apply_device<T>(M, r, z, static_cast<T*>(M->work), ws, sc, st, vals);
  }
}

sk_status precond_prepare_f32(sk_precond_s* M, cudaStream_t st) {
  if (!M || M->dtype != SK_F64) return SK_OK;
  if (M->kind == 1 && !M->inv_diag32) {
    void* p = nullptr;
    SK_CUDA(cudaMalloc(&p, static_cast<size_t>(M->n + 8) * 4));
    launch_vec(M->n, OpConvert<double, float>{static_cast<const double*>(M->inv_diag), static_cast<float*>(p)},
               RedWs{}, nullptr, st);
    SK_CUDA(cudaGetLastError());
    SK_CUDA(cudaStreamSynchronize(st));
    M->inv_diag32 = static_cast<float*>(p);
  } else if (M->kind == 2 && !f32_values(M->A)) {
    return sk_matrix_add_f32_values(M->A);
  } else if (M->kind == 3) {
    return fail(SK_NOT_SUPPORTED, "the learned preconditioner has no FP32 apply (use it as a two-level smoother)");
  }
  return SK_OK;
}

void precond_apply_dispatch(const sk_precond_s* M, sk_dtype dt, i64 n, const void* r, void* z,
                            RedWs ws, const Scalars* sc, cudaStream_t st) {
  if (dt == SK_F64)
    precond_apply_t<double>(M, n, static_cast<const double*>(r), static_cast<double*>(z), ws, sc, st);
  else
    precond_apply_t<float>(M, n, static_cast<const float*>(r), static_cast<float*>(z), ws, sc, st);
}

// Pipelined host-buffer product of a CSR handle.  The rows are cut into
// chunks of about kPipeChunkBytes of y (SELL slices or product tiles, so a
// chunk is a launch of the ordinary product kernel over its rows).  x goes
// up in pieces on one copy stream, so that piece c completes the prefix
// x[0, col_end[c]) that chunks 0..c read; chunk c's product waits for piece
// c; its y rows go down on a second copy stream while later pieces are
// still arriving.  Banded matrices (a stencil in natural order) need only
// a little more than their rows' share of x, so the two copy directions
// overlap; a matrix whose first chunk reads all of x still overlaps its
// products with the copies out.  Every row is summed by the same kernel in
// the same order as sk_spmv, so y is the same bits.
//
// Chunks of 4 MiB: with both copy directions busy the host link carries
// about 48 GB/s each way for multi-megabyte copies, and the last chunk's
// rows go down alone after the last piece of x.  Pieces of 1 MiB lose too
// much per copy to overlap (the two directions then share about 55 GB/s);
// measured on the 16.8 MB x and y of the 128^3 Laplacian: 16 chunks
// 0.63 ms, 8 chunks 0.47 ms, 4 chunks 0.435 ms, copy-product-copy 0.65 ms.
constexpr i64 kPipeChunkBytes = i64(4) << 20;
constexpr int kPipeMaxChunks = 16;

struct HostPipe {
  int chunks = 0;             // 1: the plain copy-product-copy sequence
  std::vector<i64> row_end;   // chunk c covers rows [row_end[c-1], row_end[c])
  std::vector<int> tile_end;  // tiled CSR: product tiles [tile_end[c-1], tile_end[c])
  std::vector<i64> col_end;   // x[col_end[c-1], col_end[c]) is piece c
  cudaStream_t up = nullptr, down = nullptr;
  std::vector<cudaEvent_t> ev;  // 2c: piece c landed; 2c+1: chunk c's rows computed
};

void destroy_host_pipe(HostPipe* p) {
  if (p->up) cudaStreamSynchronize(p->up);
  if (p->down) cudaStreamSynchronize(p->down);
  for (cudaEvent_t e : p->ev)
    if (e) cudaEventDestroy(e);
  if (p->up) cudaStreamDestroy(p->up);
  if (p->down) cudaStreamDestroy(p->down);
  delete p;
}

// Largest column index among the stored entries of each chunk (-1 when the
// chunk has none): CTA c reduces the entries [rp[r0], rp[r1]) of its rows.
__global__ void chunk_colmax_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                                    const long long* __restrict__ row_end, int* __restrict__ out) {
  const long long r0 = blockIdx.x ? row_end[blockIdx.x - 1] : 0, r1 = row_end[blockIdx.x];
  const long long e = rp[r1];
  int m = -1;
  for (long long k = rp[r0] + static_cast<long long>(threadIdx.x); k < e; k += blockDim.x)
    m = max(m, __ldg(ci + k));
  m = __reduce_max_sync(0xffffffffu, m);
  __shared__ int wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : -1;
    m = __reduce_max_sync(0xffffffffu, m);
    if (threadIdx.x == 0) out[blockIdx.x] = m;
  }
}

static sk_status plan_host_pipe(sk_matrix A) {
  auto* p = new HostPipe;
  // the handle keeps the plan only once it is complete
  std::unique_ptr<HostPipe, void (*)(HostPipe*)> guard(p, destroy_host_pipe);
  const size_t V = vbytes(A->dtype);
  const i64 n = A->nrow;
  int want = static_cast<int>(std::min<i64>(kPipeMaxChunks, (n * static_cast<i64>(V)) / kPipeChunkBytes));
  // (the split product of skewed rows reads x everywhere from its first
  // rows on, so it runs whole)
  if (A->format != SK_CSR || A->nnz == 0 || A->ncol == 0 || want < 2 || A->csr.hyb || A->csr.panel) {
    p->chunks = 1;
    A->pipe = guard.release();
    return SK_OK;
  }
  if (A->csr.sell) {
    for (int c = 1; c <= want; ++c) {
      i64 r = c == want ? n : std::min(n, (n * c / want + 31) / 32 * 32);
      if (r > (p->row_end.empty() ? 0 : p->row_end.back())) p->row_end.push_back(r);
    }
  } else {
    const int np = A->csr.nparts;
    std::vector<int2> tiles(static_cast<size_t>(np) + 1);
    SK_CUDA(cudaMemcpyAsync(tiles.data(), A->csr.tiles, tiles.size() * sizeof(int2), cudaMemcpyDeviceToHost,
                            A->stream));
    SK_CUDA(cudaStreamSynchronize(A->stream));
    int t = 0;
    for (int c = 1; c <= want; ++c) {
      const i64 target = n * c / want;
      while (t < np && tiles[static_cast<size_t>(t)].x < target) ++t;
      const i64 r = c == want ? n : tiles[static_cast<size_t>(t)].x;
      if (r > (p->row_end.empty() ? 0 : p->row_end.back())) {
        p->row_end.push_back(r);
        p->tile_end.push_back(c == want ? np : t);
      }
    }
  }
  const int P = static_cast<int>(p->row_end.size());
  if (P < 2) {
    p->row_end.clear();
    p->tile_end.clear();
    p->chunks = 1;
    A->pipe = guard.release();
    return SK_OK;
  }
  long long* d_rows = nullptr;
  int* d_max = nullptr;
  SK_CUDA(cudaMalloc(&d_rows, P * sizeof(long long) + P * sizeof(int)));
  d_max = reinterpret_cast<int*>(d_rows + P);
  std::vector<long long> rows(p->row_end.begin(), p->row_end.end());
  std::vector<int> colmax(static_cast<size_t>(P));
  cudaError_t e = cudaMemcpyAsync(d_rows, rows.data(), P * sizeof(long long), cudaMemcpyHostToDevice, A->stream);
  if (e == cudaSuccess) {
    SK_LAUNCH(chunk_colmax_kernel, P, 1024, 0, A->stream, A->csr.row_ptr, A->csr.col_ind, d_rows, d_max);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(colmax.data(), d_max, P * sizeof(int), cudaMemcpyDeviceToHost, A->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
  cudaFree(d_rows);
  if (e != cudaSuccess) return cuda_fail(e, "host pipeline plan");
  i64 have = 0;
  for (int c = 0; c < P; ++c) {
    have = std::max<i64>(have, static_cast<i64>(colmax[static_cast<size_t>(c)]) + 1);
    p->col_end.push_back(c + 1 == P ? A->ncol : std::min<i64>(have, A->ncol));
  }
  SK_CUDA(cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking));
  SK_CUDA(cudaStreamCreateWithFlags(&p->down, cudaStreamNonBlocking));
  p->ev.resize(2 * static_cast<size_t>(P), nullptr);
  for (auto& ev : p->ev) SK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  p->chunks = P;
  A->pipe = guard.release();
  return SK_OK;
}

// The product over rows [r0, r1) of chunk c (y indexed by absolute row).
template <typename T>
static void launch_chunk(const sk_matrix_s* A, const HostPipe& p, int c, const T* x, T* y, cudaStream_t st) {
  using Tune = SpmvTune<T, EpiStore<T>>;
  const i64 r0 = c ? p.row_end[static_cast<size_t>(c) - 1] : 0, r1 = p.row_end[static_cast<size_t>(c)];
  if (A->csr.dia_n) {
    SK_LAUNCH((dia_spmv_kernel<T, EpiStore<T>, Tune::kDiaMinB>), static_cast<int>(ceil_div(r1 - r0, kThreads)),
              kThreads, 0, st, dia_args(A, r0, r1), static_cast<const T*>(A->csr.dia_vals), x, EpiStore<T>{y},
              RedWs{}, nullptr);
  } else if (A->csr.sell) {
    SK_LAUNCH((sell_spmv_kernel<T, EpiStore<T>, Tune::kSellU, Tune::kSellPred, Tune::kSellMinB>),
              static_cast<int>(ceil_div(r1 - r0, kThreads)), kThreads, 0, st, static_cast<int>(r1 - r0),
              A->csr.sell_off + r0 / 32, A->csr.sell_len + r0, A->csr.sell_col,
              static_cast<const T*>(A->csr.sell_vals), x, EpiStore<T>{y + r0}, RedWs{}, nullptr);
  } else {
    const int t0 = c ? p.tile_end[static_cast<size_t>(c) - 1] : 0, t1 = p.tile_end[static_cast<size_t>(c)];
    SK_LAUNCH((csr_spmv_kernel<T, EpiStore<T>>), t1 - t0, kThreads, 0, st, A->csr.row_ptr, A->csr.col_ind,
              static_cast<const T*>(A->csr.vals), x, A->csr.tiles + t0, A->csr.lanes + t0, EpiStore<T>{y},
              RedWs{}, nullptr);
  }
}

}  // namespace sk

using namespace sk;

extern "C" {

sk_status sk_spmv(sk_matrix A, const void* x_dev, void* y_dev, sk_stream s) {
  SK_CHECK(A, SK_INVALID_ARG, "null handle");
  SK_CHECK((x_dev || A->ncol == 0) && (y_dev || A->nrow == 0), SK_INVALID_ARG, "null vector");
  cudaStream_t st = pick_stream(A, s);
  if (A->dtype == SK_F64)
    launch_spmv<double>(A, static_cast<const double*>(x_dev),
                        EpiStore<double>{static_cast<double*>(y_dev)}, RedWs{}, nullptr, st);
  else
    launch_spmv<float>(A, static_cast<const float*>(x_dev),
                       EpiStore<float>{static_cast<float*>(y_dev)}, RedWs{}, nullptr, st);
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

sk_status sk_spmv_f32(sk_matrix A, const float* x_dev, float* y_dev, sk_stream s) {
  SK_CHECK(A, SK_INVALID_ARG, "null handle");
  cudaStream_t st = pick_stream(A, s);
  if (A->dtype == SK_F32) return sk_spmv(A, x_dev, y_dev, s);
  SK_CHECK(A->format == SK_CSR && f32_values(A), SK_INVALID_ARG,
           "no FP32 value copy: call sk_matrix_add_f32_values first");
  launch_spmv<float>(A, x_dev, EpiStore<float>{y_dev}, RedWs{}, nullptr, st, f32_values(A));
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}


sk_status sk_spmv_host(sk_matrix A, const void* x_host, void* y_host) {
  SK_CHECK(A, SK_INVALID_ARG, "null handle");
  SK_CHECK((x_host || A->ncol == 0) && (y_host || A->nrow == 0), SK_INVALID_ARG, "null vector");
  const size_t V = A->dtype == SK_F64 ? 8 : 4;
  if (!A->io) SK_CUDA(cudaMalloc(&A->io, (A->ncol + A->nrow + 16) * V));
  if (!A->pipe) {
    sk_status st = plan_host_pipe(A);
    if (st != SK_OK) return st;
  }
  char* xd = static_cast<char*>(A->io);
  char* yd = xd + ((A->ncol + 8) * V);
  const HostPipe& p = *A->pipe;
  if (p.chunks == 1) {
    if (A->ncol) SK_CUDA(cudaMemcpyAsync(xd, x_host, A->ncol * V, cudaMemcpyHostToDevice, A->stream));
    sk_status st = sk_spmv(A, xd, yd, A->stream);
    if (st != SK_OK) return st;
    if (A->nrow) SK_CUDA(cudaMemcpyAsync(y_host, yd, A->nrow * V, cudaMemcpyDeviceToHost, A->stream));
    SK_CUDA(cudaStreamSynchronize(A->stream));
    return SK_OK;
  }
  // all pieces of x first, then the products, then the copies out: each
  // loop only enqueues, so pageable host buffers cannot stall a later stage
  const char* xh = static_cast<const char*>(x_host);
  char* yh = static_cast<char*>(y_host);
  for (int c = 0; c < p.chunks; ++c) {
    const i64 lo = c ? p.col_end[static_cast<size_t>(c) - 1] : 0, hi = p.col_end[static_cast<size_t>(c)];
    if (hi > lo) SK_CUDA(cudaMemcpyAsync(xd + lo * V, xh + lo * V, (hi - lo) * V, cudaMemcpyHostToDevice, p.up));
    SK_CUDA(cudaEventRecord(p.ev[2 * static_cast<size_t>(c)], p.up));
  }
  for (int c = 0; c < p.chunks; ++c) {
    SK_CUDA(cudaStreamWaitEvent(A->stream, p.ev[2 * static_cast<size_t>(c)], 0));
    if (A->dtype == SK_F64)
      launch_chunk<double>(A, p, c, reinterpret_cast<const double*>(xd), reinterpret_cast<double*>(yd),
                           A->stream);
    else
      launch_chunk<float>(A, p, c, reinterpret_cast<const float*>(xd), reinterpret_cast<float*>(yd), A->stream);
    SK_CUDA(cudaGetLastError());
    SK_CUDA(cudaEventRecord(p.ev[2 * static_cast<size_t>(c) + 1], A->stream));
  }
  for (int c = 0; c < p.chunks; ++c) {
    const i64 r0 = c ? p.row_end[static_cast<size_t>(c) - 1] : 0, r1 = p.row_end[static_cast<size_t>(c)];
    SK_CUDA(cudaStreamWaitEvent(p.down, p.ev[2 * static_cast<size_t>(c) + 1], 0));
    SK_CUDA(cudaMemcpyAsync(yh + r0 * V, yd + r0 * V, (r1 - r0) * V, cudaMemcpyDeviceToHost, p.down));
  }
  SK_CUDA(cudaStreamSynchronize(p.down));
  return SK_OK;
}

sk_status sk_dot(sk_dtype dtype, int64_t n, const void* a_dev, const void* b_dev, double* result,
                 sk_stream s) {
  SK_CHECK(result && n >= 0, SK_INVALID_ARG, "bad arguments");
  SK_CHECK(n == 0 || (a_dev && b_dev), SK_INVALID_ARG, "null vector");
  if (n == 0) {
    *result = 0.0;
    return SK_OK;
  }
  std::lock_guard<std::mutex> lock(g_red_mutex);
  RedWs ws;
  double* out = nullptr;
  sk_status st = global_red(vec_grid(n), &ws, &out);
  if (st != SK_OK) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(s);
  if (dtype == SK_F64)
    launch_vec(n, OpDot<double>{static_cast<const double*>(a_dev), static_cast<const double*>(b_dev), out},
               ws, nullptr, cs);
  else
    launch_vec(n, OpDot<float>{static_cast<const float*>(a_dev), static_cast<const float*>(b_dev), out},
               ws, nullptr, cs);
  SK_CUDA(cudaGetLastError());
  SK_CUDA(cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, cs));
  SK_CUDA(cudaStreamSynchronize(cs));
  return SK_OK;
}

sk_status sk_nrm2(sk_dtype dtype, int64_t n, const void* a_dev, double* result, sk_stream s) {
  sk_status st = sk_dot(dtype, n, a_dev, a_dev, result, s);
  if (st == SK_OK) *result = std::sqrt(*result);
  return st;
}

sk_status sk_axpy(sk_dtype dtype, int64_t n, double alpha, const void* x_dev, void* y_dev,
                  sk_stream s) {
  SK_CHECK(n >= 0 && (n == 0 || (x_dev && y_dev)), SK_INVALID_ARG, "bad arguments");
  if (n == 0) return SK_OK;
  cudaStream_t cs = static_cast<cudaStream_t>(s);
  if (dtype == SK_F64)
    launch_vec(n, OpAxpy<double>{alpha, static_cast<const double*>(x_dev), static_cast<double*>(y_dev)},
               RedWs{}, nullptr, cs);
  else
    launch_vec(n, OpAxpy<float>{static_cast<float>(alpha), static_cast<const float*>(x_dev),
                                static_cast<float*>(y_dev)},
               RedWs{}, nullptr, cs);
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

sk_status sk_xpay(sk_dtype dtype, int64_t n, const void* x_dev, double beta, void* y_dev,
                  sk_stream s) {
  SK_CHECK(n >= 0 && (n == 0 || (x_dev && y_dev)), SK_INVALID_ARG, "bad arguments");
  if (n == 0) return SK_OK;
  cudaStream_t cs = static_cast<cudaStream_t>(s);
  if (dtype == SK_F64)
    launch_vec(n, OpXpay<double>{beta, static_cast<const double*>(x_dev), static_cast<double*>(y_dev)},
               RedWs{}, nullptr, cs);
  else
    launch_vec(n, OpXpay<float>{static_cast<float>(beta), static_cast<const float*>(x_dev),
                                static_cast<float*>(y_dev)},
               RedWs{}, nullptr, cs);
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

sk_status sk_jacobi_create(sk_precond* out, sk_matrix A) {
  SK_CHECK(out && A, SK_INVALID_ARG, "null argument");
  *out = nullptr;
  SK_CHECK(A->format == SK_CSR, SK_INVALID_ARG, "jacobi needs a CSR handle (jacobi.hpp:27)");
  const i64 len = std::min(A->nrow, A->ncol);
  const size_t V = A->dtype == SK_F64 ? 8 : 4;
  auto* M = new sk_precond_s;
  M->kind = 1;
  M->A = A;
  M->dtype = A->dtype;
  M->n = len;
  unsigned long long* zeros = nullptr;
  cudaError_t e = cudaMalloc(&M->inv_diag, (len + 8) * V);
  if (e == cudaSuccess) e = cudaMalloc(&zeros, 8);
  if (e != cudaSuccess) {
    cudaFree(M->inv_diag);
    delete M;
    return cuda_fail(e, "cudaMalloc");
  }
  cudaMemsetAsync(zeros, 0, 8, A->stream);
  if (len > 0)
    SK_LAUNCH(extract_inv_diag_kernel, ceil_div(len, kThreads), kThreads, 0, A->stream, len,
              A->csr.row_ptr, A->csr.col_ind, static_cast<const double*>(A->csr.vals),
              static_cast<const float*>(A->csr.vals), A->dtype == SK_F32 ? 1 : 0, M->inv_diag, zeros);
  unsigned long long nz = 0;
  cudaMemcpyAsync(&nz, zeros, 8, cudaMemcpyDeviceToHost, A->stream);
  e = cudaStreamSynchronize(A->stream);
  cudaFree(zeros);
  if (e != cudaSuccess) {
    cudaFree(M->inv_diag);
    delete M;
    return cuda_fail(e, "jacobi set-up");
  }
  if (nz) {
    cudaFree(M->inv_diag);
    delete M;
    return fail(SK_ZERO_DIAGONAL, "jacobi: zero diagonal entry");
  }
  *out = M;
  return SK_OK;
}

sk_status sk_chebyshev_create(sk_precond* out, sk_matrix A, double lambda_min, double lambda_max,
                              int64_t degree) {
  SK_CHECK(out && A, SK_INVALID_ARG, "null argument");
  *out = nullptr;
  SK_CHECK(A->format == SK_CSR, SK_INVALID_ARG,
           "chebyshev preconditioner needs a CSR handle (chebyshev_preconditioner.hpp:29)");
  SK_CHECK(degree >= 0, SK_INVALID_ARG, "negative degree");
  SK_CHECK(A->nrow == A->ncol, SK_INVALID_ARG, "chebyshev preconditioner needs a square matrix");
  auto* M = new sk_precond_s;
  M->kind = 2;
  M->A = A;
  M->dtype = A->dtype;
  M->n = A->nrow;
  M->lambda_min = lambda_min;
  M->lambda_max = lambda_max;
  M->degree = degree;
  if (A->dtype == SK_F64)
    M->coeffs = cheb_coeffs<double>(lambda_min, lambda_max, degree);
  else
    M->coeffs = cheb_coeffs<float>(static_cast<float>(lambda_min), static_cast<float>(lambda_max), degree);
  const size_t V = A->dtype == SK_F64 ? 8 : 4;
  cudaError_t e = cudaMalloc(&M->work, (2 * A->nrow + 16) * V);
  if (e != cudaSuccess) {
    delete M;
    return cuda_fail(e, "cudaMalloc");
  }
  *out = M;
  return SK_OK;
}

sk_status sk_precond_apply(sk_precond M, int64_t n, const void* r_dev, void* z_dev, sk_stream s) {
  SK_CHECK(n >= 0 && (n == 0 || (r_dev && z_dev)), SK_INVALID_ARG, "bad arguments");
  if (n == 0) return SK_OK;
  if (M) SK_CHECK(n == M->n, SK_INVALID_ARG, "vector length differs from the preconditioner's");
  cudaStream_t cs = M ? pick_stream(M->A, s) : static_cast<cudaStream_t>(s);
  // NULL preconditioner: identity on the FP64 path unless told otherwise.
  sk_dtype dt = M ? M->dtype : SK_F64;
  if (M && M->kind == 3) {
    sk_status ls = learned_apply(M, static_cast<const double*>(r_dev), static_cast<double*>(z_dev), cs);
    if (ls != SK_OK) return ls;
    SK_CUDA(cudaGetLastError());
    return SK_OK;
  }
  precond_apply_dispatch(M, dt, n, r_dev, z_dev, RedWs{}, nullptr, cs);
  SK_CUDA(cudaGetLastError());
  if (M && M->kind == 4 && M->smoother && M->smoother->kind == 3) return sk_net_status(M->smoother->net);
  return SK_OK;
}

sk_status sk_precond_values(sk_precond M, void* host_out, int64_t capacity, int64_t* count) {
  SK_CHECK(M && count, SK_INVALID_ARG, "null argument");
  const size_t V = M->dtype == SK_F64 ? 8 : 4;
  if (M->kind == 1) {
    *count = M->n;
    if (host_out && capacity >= M->n && M->n > 0) {
      SK_CUDA(cudaStreamSynchronize(M->A->stream));
      SK_CUDA(cudaMemcpy(host_out, M->inv_diag, M->n * V, cudaMemcpyDeviceToHost));
    }
  } else {
    *count = static_cast<int64_t>(M->coeffs.size());
    if (host_out && capacity >= *count) {
      for (size_t k = 0; k < M->coeffs.size(); ++k) {
        if (M->dtype == SK_F64)
          static_cast<double*>(host_out)[k] = M->coeffs[k];
        else
          static_cast<float*>(host_out)[k] = static_cast<float>(M->coeffs[k]);
      }
    }
  }
  return SK_OK;
}

sk_status sk_precond_destroy(sk_precond M) {
  if (!M) return SK_OK;
  // cudaFree waits for the device; the matrix M->A may already be gone.
  if (M->kind == 3) learned_release(M);
  if (M->kind == 4) twolevel_release(M);
  if (M->inv_diag) cudaFree(M->inv_diag);
  if (M->inv_diag32) cudaFree(M->inv_diag32);
  if (M->work) cudaFree(M->work);
  delete M;
  return SK_OK;
}

}  // extern "C"
