// sk_dia.cu -- the diagonal copy of a CSR handle (sk_matrix_add_diagonals).
//
// No reference counterpart: the copy is a second device layout of the
// reference's Compressed_row_matrix (Compressed_row_matrix.hpp:20-132), as
// the SELL-32 copy is, for matrices whose entries lie on a few diagonals (a
// stencil in natural order).  The product over it (dia_spmv_kernel) reads
// no column indices and no gathered x, and sums each row's stored entries
// in ascending column order, which is the row's CSR order when the row
// holds its columns in ascending order; the copy is built only then, so
// every product gives the bits of the CSR product.
//
// Two passes over the CSR arrays: one collects the distinct offsets c - r
// (a set of kDiaMax slots per CTA in shared memory, merged into one in
// global memory) and checks that every row's columns ascend; the second
// writes each entry into its diagonal's segment of its row's 32-row slice
// and each row's mask of stored diagonals.
#include <algorithm>
#include <climits>
#include <vector>

#include "sk_internal.cuh"

namespace sk {
namespace {

constexpr int kEmpty = INT_MIN;  // c - r > INT_MIN for every entry

// Inserts v into the kDiaMax-slot set s (slots fill from 0, never change
// once set).  False: the set is full and does not hold v.
__device__ __forceinline__ bool set_insert(int* s, int v) {
  volatile int* vs = s;
  for (int k = 0; k < kDiaMax; ++k) {
    const int cur = vs[k];
    if (cur == v) return true;
    if (cur == kEmpty) {
      const int old = atomicCAS(s + k, kEmpty, v);
      if (old == kEmpty || old == v) return true;
    }
  }
  return false;
}

// flags bit 0: a row whose columns do not strictly ascend; bit 1: more
// than kDiaMax distinct offsets.
__global__ void dia_scan_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci, int* gset,
                                int* flags) {
  __shared__ int set[kDiaMax];
  if (threadIdx.x < kDiaMax) set[threadIdx.x] = kEmpty;
  __syncthreads();
  int bad = 0;
  for (i64 r = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; r < n && !(bad & 2);
       r += static_cast<i64>(gridDim.x) * blockDim.x) {
    const int b = rp[r], e = rp[r + 1];
    int prev = -1;
    for (int k = b; k < e; ++k) {
      const int c = ci[k];
      if (c <= prev) bad |= 1;
      prev = c;
      if (!set_insert(set, c - static_cast<int>(r))) {
        bad |= 2;
        break;
      }
    }
  }
  if (bad) atomicOr(flags, bad);
  __syncthreads();
  if (threadIdx.x < kDiaMax) {
    const int v = set[threadIdx.x];
    if (v != kEmpty && !set_insert(gset, v)) atomicOr(flags, 2);
  }
}

struct Offsets {
  int n;
  int off[kDiaMax];
};

template <typename T>
__global__ void dia_fill_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci,
                                const T* __restrict__ va, Offsets o, T* __restrict__ planes,
                                unsigned short* __restrict__ mask) {
  for (i64 r = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<i64>(gridDim.x) * blockDim.x) {
    unsigned m = 0;
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
      const int off = ci[k] - static_cast<int>(r);
      int d = 0;
      while (d + 1 < o.n && o.off[d] != off) ++d;  // every offset is in the set
      planes[((r >> 5) * o.n + d) * 32 + (r & 31)] = va[k];
      m |= 1u << d;
    }
    mask[r] = static_cast<unsigned short>(m);
  }
}

__global__ void dia_to_float_kernel(const double* __restrict__ in, float* __restrict__ out, i64 n) {
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<i64>(gridDim.x) * blockDim.x)
    out[i] = static_cast<float>(in[i]);
}

}  // namespace

sk_status dia_pattern(sk_matrix A, std::vector<int>* offsets) {
  offsets->clear();
  const i64 n = A->nrow;
  if (A->format != SK_CSR || n == 0 || A->nnz == 0 || n > INT_MAX / 2) return SK_OK;
  if (A->csr.dia_n) {
    offsets->assign(A->csr.dia_off, A->csr.dia_off + A->csr.dia_n);
    return SK_OK;
  }
  int* scratch = nullptr;
  SK_CUDA(cudaMalloc(&scratch, (kDiaMax + 1) * sizeof(int)));
  std::vector<int> h(kDiaMax + 1, kEmpty);
  h[kDiaMax] = 0;
  cudaError_t e = cudaMemcpyAsync(scratch, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, A->stream);
  if (e == cudaSuccess) {
    SK_LAUNCH(dia_scan_kernel, grid_for(n), kThreads, 0, A->stream, n, A->csr.row_ptr, A->csr.col_ind, scratch,
              scratch + kDiaMax);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h.data(), scratch, h.size() * sizeof(int), cudaMemcpyDeviceToHost, A->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
  cudaFree(scratch);
  if (e != cudaSuccess) return cuda_fail(e, "diagonal scan");
  if (h[kDiaMax] != 0) return SK_OK;  // unsorted rows or too many diagonals
  std::vector<int> offs;
  for (int k = 0; k < kDiaMax; ++k)
    if (h[k] != kEmpty) offs.push_back(h[k]);
  std::sort(offs.begin(), offs.end());
  const i64 nd = static_cast<i64>(offs.size());
  if (nd == 0 || nd * n > 2 * A->nnz) return SK_OK;  // planes more than half empty
  *offsets = offs;
  return SK_OK;
}

sk_status build_dia_f32(sk_matrix A) {
  if (!A->csr.dia_n || A->csr.dia_vals32 || A->dtype != SK_F64) return SK_OK;
  const i64 len = A->csr.dia_len;
  void* p = nullptr;
  sk_status st = dev_alloc(A, &p, len * 4 + 64);
  if (st != SK_OK) return st;
  SK_LAUNCH(dia_to_float_kernel, grid_for(len), kThreads, 0, A->stream, static_cast<const double*>(A->csr.dia_vals),
            static_cast<float*>(p), len);
  SK_CUDA(cudaGetLastError());
  SK_CUDA(cudaStreamSynchronize(A->stream));
  A->csr.dia_vals32 = static_cast<float*>(p);
  return SK_OK;
}

}  // namespace sk

using namespace sk;

extern "C" {

sk_status sk_matrix_add_diagonals(sk_matrix A, int* built) {
  SK_CHECK(A && built, SK_INVALID_ARG, "null argument");
  *built = 0;
  SK_CHECK(A->format == SK_CSR, SK_NOT_SUPPORTED, "the diagonal copy is for CSR handles");
  if (A->csr.dia_n) {
    *built = 1;
    return SK_OK;
  }
  const i64 n = A->nrow;
  std::vector<int> offs;
  sk_status st0 = dia_pattern(A, &offs);
  if (st0 != SK_OK) return st0;
  if (offs.empty()) return SK_OK;  // not a pattern of few diagonals
  const i64 nd = static_cast<i64>(offs.size());
  // slice-major: the nd segments of a 32-row slice are adjacent, so that a
  // warp's loads of one row group stay within one page (separate planes
  // put each of a row's nd loads on its own page)
  const i64 len = (n + 31) / 32 * 32 * nd;
  const size_t V = vbytes(A->dtype);
  void *planes = nullptr, *mask = nullptr;
  sk_status st;
  if ((st = dev_alloc(A, &planes, len * V + 64)) != SK_OK) return st;
  if ((st = dev_alloc(A, &mask, (n + 64) * 2)) != SK_OK) return st;
  SK_CUDA(cudaMemsetAsync(planes, 0, len * V + 64, A->stream));
  Offsets o{};
  o.n = static_cast<int>(nd);
  for (i64 d = 0; d < nd; ++d) o.off[d] = offs[static_cast<size_t>(d)];
  if (A->dtype == SK_F64)
    SK_LAUNCH(dia_fill_kernel<double>, grid_for(n), kThreads, 0, A->stream, n, A->csr.row_ptr, A->csr.col_ind,
              static_cast<const double*>(A->csr.vals), o, static_cast<double*>(planes),
              static_cast<unsigned short*>(mask));
  else
    SK_LAUNCH(dia_fill_kernel<float>, grid_for(n), kThreads, 0, A->stream, n, A->csr.row_ptr, A->csr.col_ind,
              static_cast<const float*>(A->csr.vals), o, static_cast<float*>(planes),
              static_cast<unsigned short*>(mask));
  SK_CUDA(cudaGetLastError());
  SK_CUDA(cudaStreamSynchronize(A->stream));
  A->csr.dia_vals = planes;
  A->csr.dia_mask = static_cast<unsigned short*>(mask);
  A->csr.dia_len = len;
  for (i64 d = 0; d < nd; ++d) A->csr.dia_off[d] = offs[static_cast<size_t>(d)];
  A->csr.dia_n = static_cast<int>(nd);
  // a handle that already carries its FP32 value copy gets the FP32 planes
  if (A->csr.vals32 && (st = build_dia_f32(A)) != SK_OK) return st;
  *built = 1;
  return SK_OK;
}

}  // extern "C"
