// sk_convert.cu -- the ELLPACK, jagged-diagonal and BSR handles built on the
// device from a device-resident CSR handle (the reference builds them on the
// host with sorts over int64 index lists, conversions.hpp:427-691), and the
// export of every handle back to the reference's host arrays.
//
// Every conversion is a handful of streaming passes over the CSR arrays:
//   ELL  width = longest row (a max reduction), then one thread per row
//        writes its slots; a warp stores one slot of 32 rows as one segment.
//   JAD  rows ordered by decreasing length, ties by row index (a stable LSD
//        radix sort on the key maxlen - len, 8 bits per pass: one pass when
//        every row is shorter than 256), the diagonal widths from the sorted
//        lengths, then one thread per permuted row writes its diagonals.
//   BSR  a group of lanes per block row merges the sorted block columns of
//        its rows, once to count the blocks and once to fill them.
#include <algorithm>
#include <climits>
#include <type_traits>
#include <vector>

#include "sk_sort.cuh"

namespace sk {
namespace {

// ------------------------------------------------------------------
// Device time of a conversion: events around each run of kernels, so that
// the host's allocations between them are not counted
// ------------------------------------------------------------------
struct SegTimer {
  cudaStream_t st;
  std::vector<cudaEvent_t> ev;  // begin, end, begin, end, ...
  explicit SegTimer(cudaStream_t s) : st(s) {}
  ~SegTimer() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
  void mark() {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) == cudaSuccess) {
      cudaEventRecord(e, st);
      ev.push_back(e);
    }
  }
  // after the stream has been synchronised
  double total_ms() const {
    double t = 0;
    for (size_t i = 0; i + 1 < ev.size(); i += 2) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) == cudaSuccess) t += ms;
    }
    return t;
  }
};

// ------------------------------------------------------------------
// Row lengths and their maximum
// ------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) row_len_kernel(const int* __restrict__ rp, i64 n, int* __restrict__ len,
                               int* __restrict__ maxlen) {
  int m = 0;
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) {
    const int l = rp[i + 1] - rp[i];
    if (len) len[i] = l;
    m = max(m, l);
  }
  // one atomic per CTA (one per warp serialises tens of thousands of
  // atomics on a single address)
  __shared__ int wm[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; ++w) m = max(m, wm[w]);
    if (m > 0) atomicMax(maxlen, m);
  }
}

static sk_status max_row_length(const int* rp, i64 n, int* len, int* dmax, cudaStream_t st, int* out,
                                SegTimer& tm) {
  tm.mark();
  SK_CUDA(cudaMemsetAsync(dmax, 0, sizeof(int), st));
  if (n > 0) SK_LAUNCH(row_len_kernel, grid_for(n), kThreads, 0, st, rp, n, len, dmax);
  tm.mark();
  SK_CUDA(cudaMemcpyAsync(out, dmax, sizeof(int), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  return SK_OK;
}

// ------------------------------------------------------------------
// CSR -> ELL
// ------------------------------------------------------------------
// One thread per slot row i < ld: entry k of row i to k * ld + i, the
// slots past the row's length (and the rows past nrow) zero.
// One thread per slot row i < ld: entry k of row i to k * ld + i, the
// slots past the row's length (and the rows past nrow) zero.  A warp
// stores one slot of 32 rows as one segment, padding included: clearing
// the arrays first and writing the entries alone measured slower when
// padding dominates (partial-sector writes).
template <typename T>
__global__ void csr_to_ell_kernel(i64 n, i64 ld, i64 width, const int* __restrict__ rp,
                                  const int* __restrict__ ci, const T* __restrict__ va,
                                  int* __restrict__ col, T* __restrict__ val, int* __restrict__ rowlen) {
  const i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  if (i >= ld) return;
  int a = 0, len = 0;
  if (i < n) {
    a = rp[i];
    len = rp[i + 1] - a;
    rowlen[i] = len;
  }
  for (i64 k = 0; k < width; ++k) {
    const bool in = k < len;
    col[k * ld + i] = in ? ci[a + k] : 0;
    val[k * ld + i] = in ? va[a + k] : T(0);
  }
}

// ------------------------------------------------------------------
// CSR -> JAD
// ------------------------------------------------------------------
__global__ void jad_keys_kernel(const int* __restrict__ len, i64 n, unsigned maxlen,
                                unsigned* __restrict__ keys) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) keys[i] = maxlen - static_cast<unsigned>(len[i]);
}

// perm, plen from the sorted keys; width[k] = rows longer than k, written
// by the last sorted row of at least k + 1 entries.
__global__ void jad_perm_kernel(const unsigned* __restrict__ skeys, const int* __restrict__ sidx, i64 n,
                                unsigned maxlen, int* __restrict__ perm, int* __restrict__ plen,
                                int* __restrict__ width) {
  i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; p < n; p += stride) {
    const int l = static_cast<int>(maxlen - skeys[p]);
    const int next = p + 1 < n ? static_cast<int>(maxlen - skeys[p + 1]) : 0;
    perm[p] = sidx[p];
    plen[p] = l;
    for (int k = next; k < l; ++k) width[k] = static_cast<int>(p + 1);
  }
}

// Entry k of row perm[p] goes to jdiag[k] + p.  The permuted rows are
// sorted by decreasing length, so each warp's 32 rows p0 .. p0 + 31 have
// the longest first.  Warps whose rows have at most 32 entries: one lane
// per row (jad_short_kernel).  Longer rows: 32 x 32 tiles through shared
// memory, read along each row (one coalesced segment per row) and written
// along each diagonal (one segment per diagonal) (jad_long_kernel); kept
// apart so that the short rows run at full occupancy.
constexpr int kJadWarps = 4;

template <typename T>
__global__ void jad_short_kernel(i64 n, const int* __restrict__ perm, const int* __restrict__ plen,
                                 const int* __restrict__ jdiag, const int* __restrict__ rp,
                                 const int* __restrict__ ci, const T* __restrict__ va, int* __restrict__ col,
                                 T* __restrict__ val) {
  const i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  const int L0 = plen[p & ~static_cast<i64>(31)];
  if (L0 > 32) return;
  const int a = rp[perm[p]], l = plen[p];
  for (int k = 0; k < l; ++k) {
    const i64 dst = static_cast<i64>(__ldg(jdiag + k)) + p;
    col[dst] = ci[a + k];
    val[dst] = va[a + k];
  }
}

template <typename V>
__device__ __forceinline__ void jad_tile(V (*buf)[33], const V* __restrict__ src, V* __restrict__ dst, int lane,
                                         int a_me, int l_me, int k0, int kn, i64 p0, const int* __restrict__ jdiag) {
  for (int r = 0; r < 32; ++r) {
    const int a = __shfl_sync(0xffffffffu, a_me, r);
    const int l = __shfl_sync(0xffffffffu, l_me, r);
    if (k0 + lane < l) buf[r][lane] = src[a + k0 + lane];
  }
  __syncwarp();
  for (int k = 0; k < kn; ++k)
    if (k0 + k < l_me) dst[static_cast<i64>(__ldg(jdiag + k0 + k)) + p0 + lane] = buf[lane][k];
  __syncwarp();
}

// Covers the warps of rows longer than 32 entries: permuted rows
// 0 .. nlong - 1 (nlong = rows of more than 32 entries); blockIdx.y picks
// a range of kJadChunk diagonals, so that the longest rows are spread over
// many warps instead of one warp walking them alone.
constexpr int kJadChunk = 256;

template <typename T>
__global__ void __launch_bounds__(kJadWarps * 32) jad_long_kernel(
    i64 n, const int* __restrict__ perm, const int* __restrict__ plen, const int* __restrict__ jdiag,
    const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ va, int* __restrict__ col,
    T* __restrict__ val) {
  __shared__ T tile[kJadWarps][32][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const i64 p0 = (static_cast<i64>(blockIdx.x) * kJadWarps + w) * 32;
  if (p0 >= n) return;
  const i64 p = p0 + lane;
  const bool in = p < n;
  const int a = in ? rp[perm[p]] : 0;
  const int l = in ? plen[p] : 0;
  const int L0 = __shfl_sync(0xffffffffu, l, 0);
  if (L0 <= 32) return;
  auto* tb = tile[w];
  auto* ib = reinterpret_cast<int(*)[33]>(&tile[w][0][0]);
  const int kbeg = blockIdx.y * kJadChunk;
  const int kend = min(L0, kbeg + kJadChunk);
  for (int k0 = kbeg; k0 < kend; k0 += 32) {
    const int kn = min(32, kend - k0);
    jad_tile<int>(ib, ci, col, lane, a, l, k0, kn, p0, jdiag);
    jad_tile<T>(tb, va, val, lane, a, l, k0, kn, p0, jdiag);
  }
}

__global__ void iota_kernel(int* __restrict__ p, i64 n) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) p[i] = static_cast<int>(i);
}

// ------------------------------------------------------------------
// CSR -> BSR
// ------------------------------------------------------------------
// A group of G lanes (a power of two, G >= min(br, 32)) per block row; lane
// gl of the group holds rows gl, gl + G, ... (at most 8) of the block row.
// Each step takes the smallest block column at the heads of the rows (a
// min over the group), then every lane moves past its entries in that
// block column, which FILL scatters into the block.
constexpr int kBsrRowsPerLane = 8;

// R: rows per lane (1 when block_rows <= 32); BC: the block width when it
// is a small constant (divisions become multiplications), 0 otherwise.
template <typename T, bool FILL, int R, int BC>
__global__ void __launch_bounds__(kThreads) csr_to_bsr_kernel(
    i64 nrow, i64 nbr, int br, int bc_rt, int G, const int* __restrict__ rp, const int* __restrict__ ci,
    const T* __restrict__ va, int* __restrict__ cnt, const i64* __restrict__ brp, int* __restrict__ bcol,
    T* __restrict__ bval) {
  const int bc = BC > 0 ? BC : bc_rt;
  const int lane = threadIdx.x & 31;
  const i64 warp_id = (blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x) >> 5;
  const int gpw = 32 / G;
  const int g = lane / G, gl = lane - g * G;
  const i64 I = warp_id * gpw + g;
  const bool active = I < nbr;
  int pos[R], end[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int lr = gl + G * j;
    const i64 r = I * br + lr;
    if (active && lr < br && r < nrow) {
      pos[j] = rp[r];
      end[j] = rp[r + 1];
    } else {
      pos[j] = end[j] = 0;
    }
  }
  const i64 bsz = static_cast<i64>(br) * bc;
  const i64 first = (FILL && active) ? brp[I] : 0;
  int count = 0;
  for (;;) {
    int h = INT_MAX;
#pragma unroll
    for (int j = 0; j < R; ++j)
      if (pos[j] < end[j]) h = min(h, ci[pos[j]] / bc);
    for (int o = G >> 1; o > 0; o >>= 1) h = min(h, __shfl_xor_sync(0xffffffffu, h, o));
    if (!__any_sync(0xffffffffu, h != INT_MAX)) break;
    if (h == INT_MAX) continue;
    const i64 blk = first + count;
    if (FILL && gl == 0) bcol[blk] = h;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      if (FILL) {
        // the lane's row of the block, zeros included, so that every
        // block is written whole (no clearing pass, no partial sectors)
        const int lr = gl + G * j;
        if (active && lr < br) {
          T* out = bval + blk * bsz + static_cast<i64>(lr) * bc;
          const int c0 = h * bc;
          for (int c = 0; c < bc; ++c) {
            T v = T(0);
            if (pos[j] < end[j] && ci[pos[j]] == c0 + c) v = va[pos[j]++];
            out[c] = v;
          }
        }
      } else {
        while (pos[j] < end[j] && ci[pos[j]] / bc == h) ++pos[j];
      }
    }
    ++count;
  }
  if (!FILL && active && gl == 0) cnt[I] = count;
}

// ------------------------------------------------------------------
// Exports (device layout -> the reference's host arrays)
// ------------------------------------------------------------------
__global__ void widen_kernel(const int* __restrict__ in, i64 n, long long* __restrict__ out) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) out[i] = in[i];
}

// Row-major slots g0 .. g0 + count of the reference's ELL layout: -1 and 0
// past each row's length (Ellpack_sparsity_Impl.cpp:35-37).
template <typename T>
__global__ void ell_export_kernel(i64 g0, i64 count, i64 width, i64 ld, const int* __restrict__ col,
                                  const T* __restrict__ val, const int* __restrict__ rowlen,
                                  long long* __restrict__ ocol, T* __restrict__ oval) {
  i64 t = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; t < count; t += stride) {
    const i64 g = g0 + t, i = g / width, k = g - i * width;
    const bool in = k < rowlen[i];
    ocol[t] = in ? col[k * ld + i] : -1;
    oval[t] = in ? val[k * ld + i] : T(0);
  }
}

static sk_status download_indices(const int* dev, i64 count, int64_t* host, cudaStream_t st) {
  if (count == 0) return SK_OK;
  SK_CHECK(host, SK_INVALID_ARG, "null output array");
  Temps tmp(st);
  long long* stage = nullptr;
  const i64 chunk = std::min(count, kChunk);
  sk_status s = tmp.get(&stage, chunk);
  if (s != SK_OK) return s;
  for (i64 off = 0; off < count; off += chunk) {
    const i64 c = std::min(chunk, count - off);
    SK_LAUNCH(widen_kernel, grid_for(c), kThreads, 0, st, dev + off, c, stage);
    SK_CUDA(cudaMemcpyAsync(host + off, stage, c * sizeof(long long), cudaMemcpyDeviceToHost, st));
    SK_CUDA(cudaStreamSynchronize(st));
  }
  return SK_OK;
}

static sk_status download_values(const void* dev, i64 count, sk_dtype dt, void* host, cudaStream_t st) {
  if (count == 0) return SK_OK;
  SK_CHECK(host, SK_INVALID_ARG, "null output array");
  SK_CUDA(cudaMemcpyAsync(host, dev, count * vbytes(dt), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  return SK_OK;
}

static sk_status check_source(sk_matrix* out, sk_matrix csr) {
  SK_CHECK(out, SK_INVALID_ARG, "null output handle");
  *out = nullptr;
  SK_CHECK(csr, SK_INVALID_ARG, "null CSR handle");
  SK_CHECK(csr->format == SK_CSR, SK_INVALID_ARG, "the source handle must be CSR");
  SK_CUDA(cudaSetDevice(csr->device));
  SK_CUDA(cudaStreamSynchronize(csr->stream));
  return SK_OK;
}

template <typename T>
static sk_status ell_from_csr(sk_matrix A, sk_matrix C) {
  cudaStream_t st = A->stream;
  const i64 n = C->nrow;
  Temps tmp(st);
  int* dmax = nullptr;
  sk_status s;
  if ((s = tmp.get(&dmax, 1)) != SK_OK) return s;
  SegTimer tm(st);
  int width = 0;
  if ((s = max_row_length(C->csr.row_ptr, n, nullptr, dmax, st, &width, tm)) != SK_OK) return s;
  const i64 ld = (n + 31) / 32 * 32 + 96;  // the slot stride of sk_ell_create
  A->ell.width = width;
  A->ell.ld = ld;
  A->nnz = C->nnz;
  const i64 stored = ld * width;
  void *col = nullptr, *va = nullptr, *rl = nullptr;
  if ((s = dev_alloc(A, &col, (stored + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &va, (stored + 8) * sizeof(T))) != SK_OK) return s;
  if ((s = dev_alloc(A, &rl, (n + 8) * 4)) != SK_OK) return s;
  A->ell.col = static_cast<int*>(col);
  A->ell.vals = va;
  A->ell.rowlen = static_cast<int*>(rl);
  tm.mark();
  if (n > 0)
    SK_LAUNCH(csr_to_ell_kernel<T>, ceil_div(ld, kThreads), kThreads, 0, st, n, ld, static_cast<i64>(width),
              C->csr.row_ptr, C->csr.col_ind, static_cast<const T*>(C->csr.vals), A->ell.col,
              static_cast<T*>(va), A->ell.rowlen);
  tm.mark();
  SK_CUDA(cudaGetLastError());
  SK_CUDA(cudaStreamSynchronize(st));
  A->build_ms = tm.total_ms();
  return SK_OK;
}

template <typename T>
static sk_status jad_from_csr(sk_matrix A, sk_matrix C) {
  cudaStream_t st = A->stream;
  const i64 n = C->nrow, nnz = C->nnz;
  Temps tmp(st);
  sk_status s;
  int *len = nullptr, *dmax = nullptr;
  if ((s = tmp.get(&len, n)) != SK_OK) return s;
  if ((s = tmp.get(&dmax, 1)) != SK_OK) return s;
  SegTimer tm(st);
  int maxlen = 0;
  if ((s = max_row_length(C->csr.row_ptr, n, len, dmax, st, &maxlen, tm)) != SK_OK) return s;
  const i64 njd = nnz > 0 ? maxlen : 0;
  A->nnz = nnz;
  A->jad.njd = njd;
  void *pm = nullptr, *jd = nullptr, *ci = nullptr, *va = nullptr, *pl = nullptr;
  if ((s = dev_alloc(A, &pm, (n + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &jd, (njd + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &ci, (nnz + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &va, (nnz + 8) * sizeof(T))) != SK_OK) return s;
  if ((s = dev_alloc(A, &pl, (n + 8) * 4 + 64)) != SK_OK) return s;
  A->jad.perm = static_cast<int*>(pm);
  A->jad.jdiag = static_cast<int*>(jd);
  A->jad.col = static_cast<int*>(ci);
  A->jad.vals = va;
  A->jad.plen = static_cast<int*>(pl);
  if (njd == 0) {
    // An empty matrix: no diagonals (Jagged_diagonal_sparsity_Impl.cpp:28-31);
    // the identity order serves the product, every row sums to zero.
    tm.mark();
    SK_CUDA(cudaMemsetAsync(jd, 0, 4, st));
    SK_CUDA(cudaMemsetAsync(pl, 0, (n + 8) * 4, st));
    if (n > 0) SK_LAUNCH(iota_kernel, grid_for(n), kThreads, 0, st, A->jad.perm, n);
    tm.mark();
    SK_CUDA(cudaGetLastError());
    SK_CUDA(cudaStreamSynchronize(st));
    A->build_ms = tm.total_ms();
    return SK_OK;
  }
  unsigned *k1 = nullptr, *k2 = nullptr, *sk = nullptr;
  int *i1 = nullptr, *i2 = nullptr, *si = nullptr, *width = nullptr;
  i64* jd64 = nullptr;
  if ((s = tmp.get(&k1, n)) != SK_OK) return s;
  if ((s = tmp.get(&k2, n)) != SK_OK) return s;
  if ((s = tmp.get(&i1, n)) != SK_OK) return s;
  if ((s = tmp.get(&i2, n)) != SK_OK) return s;
  if ((s = tmp.get(&width, njd)) != SK_OK) return s;
  if ((s = tmp.get(&jd64, njd + 1)) != SK_OK) return s;
  tm.mark();
  SK_LAUNCH(jad_keys_kernel, grid_for(n), kThreads, 0, st, len, n, static_cast<unsigned>(maxlen), k1);
  if ((s = stable_radix_sort<unsigned>(k1, k2, i1, i2, n, static_cast<unsigned>(maxlen), tmp, st, &sk, &si)) !=
      SK_OK)
    return s;
  SK_LAUNCH(jad_perm_kernel, grid_for(n), kThreads, 0, st, sk, si, n, static_cast<unsigned>(maxlen),
            A->jad.perm, A->jad.plen, width);
  if ((s = exclusive_scan(width, njd, jd64, tmp, st)) != SK_OK) return s;
  SK_LAUNCH(narrow_i64_kernel, grid_for(njd + 1), kThreads, 0, st, jd64, njd + 1, A->jad.jdiag);
  const int* rp_ = C->csr.row_ptr;
  const int* ci_ = C->csr.col_ind;
  const T* va_ = static_cast<const T*>(C->csr.vals);
  SK_LAUNCH(jad_short_kernel<T>, ceil_div(n, kThreads), kThreads, 0, st, n, A->jad.perm, A->jad.plen, A->jad.jdiag,
            rp_, ci_, va_, A->jad.col, static_cast<T*>(va));
  tm.mark();
  if (maxlen > 32) {
    // rows of more than 32 entries = the width of diagonal 32
    int w32[2] = {0, 0};
    SK_CUDA(cudaMemcpyAsync(w32, A->jad.jdiag + 32, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    SK_CUDA(cudaStreamSynchronize(st));
    const i64 nlong = w32[1] - w32[0];
    const dim3 grid(ceil_div(nlong, 32 * kJadWarps), ceil_div(maxlen, kJadChunk));
    tm.mark();
    SK_LAUNCH(jad_long_kernel<T>, grid, 32 * kJadWarps, 0, st, n, A->jad.perm,
              A->jad.plen, A->jad.jdiag, rp_, ci_, va_, A->jad.col, static_cast<T*>(va));
    tm.mark();
  }
  SK_CUDA(cudaGetLastError());
  SK_CUDA(cudaStreamSynchronize(st));
  A->build_ms = tm.total_ms();
  return SK_OK;
}

template <typename T>
static sk_status bsr_from_csr(sk_matrix A, sk_matrix C, int br, int bc) {
  cudaStream_t st = A->stream;
  const i64 n = C->nrow;
  const i64 nbr = (n + br - 1) / br;
  const i64 bsz = static_cast<i64>(br) * bc;
  auto& b = A->bsr;
  b.br = br;
  b.bc = bc;
  b.nbr = nbr;
  b.nbr_mult = n / br;
  Temps tmp(st);
  sk_status s;
  int* cnt = nullptr;
  i64* rp64 = nullptr;
  if ((s = tmp.get(&cnt, nbr)) != SK_OK) return s;
  if ((s = tmp.get(&rp64, nbr + 1)) != SK_OK) return s;
  int G = 1;
  while (G < br && G < 32) G <<= 1;
  const i64 warps = (nbr + (32 / G) - 1) / (32 / G);
  const int grid = ceil_div(warps * 32, kThreads);
  const auto merge = [&](auto fill, int* c, const i64* r, int* bcol, T* bval) {
    constexpr bool F = decltype(fill)::value;
    const int* rp_ = C->csr.row_ptr;
    const int* ci_ = C->csr.col_ind;
    const T* va_ = static_cast<const T*>(C->csr.vals);
    if (br > 32)
      SK_LAUNCH((csr_to_bsr_kernel<T, F, kBsrRowsPerLane, 0>), grid, kThreads, 0, st, n, nbr, br, bc, G, rp_, ci_,
                va_, c, r, bcol, bval);
    else if (bc == 1)
      SK_LAUNCH((csr_to_bsr_kernel<T, F, 1, 1>), grid, kThreads, 0, st, n, nbr, br, bc, G, rp_, ci_, va_, c, r,
                bcol, bval);
    else if (bc == 2)
      SK_LAUNCH((csr_to_bsr_kernel<T, F, 1, 2>), grid, kThreads, 0, st, n, nbr, br, bc, G, rp_, ci_, va_, c, r,
                bcol, bval);
    else if (bc == 3)
      SK_LAUNCH((csr_to_bsr_kernel<T, F, 1, 3>), grid, kThreads, 0, st, n, nbr, br, bc, G, rp_, ci_, va_, c, r,
                bcol, bval);
    else if (bc == 4)
      SK_LAUNCH((csr_to_bsr_kernel<T, F, 1, 4>), grid, kThreads, 0, st, n, nbr, br, bc, G, rp_, ci_, va_, c, r,
                bcol, bval);
    else
      SK_LAUNCH((csr_to_bsr_kernel<T, F, 1, 0>), grid, kThreads, 0, st, n, nbr, br, bc, G, rp_, ci_, va_, c, r,
                bcol, bval);
  };
  SegTimer tm(st);
  tm.mark();
  if (nbr > 0) merge(std::false_type{}, cnt, nullptr, nullptr, nullptr);
  if ((s = exclusive_scan(cnt, nbr, rp64, tmp, st)) != SK_OK) return s;
  tm.mark();
  std::vector<int64_t> rp(static_cast<size_t>(nbr) + 1);
  SK_CUDA(cudaMemcpyAsync(rp.data(), rp64, (nbr + 1) * sizeof(i64), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  const i64 nblocks = rp[static_cast<size_t>(nbr)];
  SK_CHECK(nblocks * bsz < (i64(1) << 31) - 16, SK_INDEX_OVERFLOW, "block values do not fit int32");
  b.nblocks = nblocks;
  A->nnz = nblocks * bsz;
  void *drp = nullptr, *dci = nullptr, *dva = nullptr;
  if ((s = dev_alloc(A, &drp, (nbr + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &dci, (nblocks + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &dva, (nblocks * bsz + 8) * sizeof(T))) != SK_OK) return s;
  b.row_ptr = static_cast<int*>(drp);
  b.col = static_cast<int*>(dci);
  b.vals = dva;
  tm.mark();
  SK_LAUNCH(narrow_i64_kernel, grid_for(nbr + 1), kThreads, 0, st, rp64, nbr + 1, b.row_ptr);
  if (nbr > 0) merge(std::true_type{}, nullptr, rp64, b.col, static_cast<T*>(dva));
  tm.mark();
  SK_CUDA(cudaGetLastError());
  // the product's partition of block rows into CTA tiles is a greedy walk
  // over the block row pointers, taken on the host copy above
  std::vector<int> part;
  bsr_partition(rp.data(), nbr, br, bsz, part);
  b.nparts = static_cast<int>(part.size()) - 1;
  if ((s = upload_vector(A, part, &b.part, st)) != SK_OK) return s;
  // the sliced product copy is built as for an uploaded handle (host
  // offsets, one scatter kernel) and is not counted in build_ms
  if ((s = build_bsr_sell(A, rp.data(), st)) != SK_OK) return s;
  SK_CUDA(cudaStreamSynchronize(st));
  A->build_ms = tm.total_ms();
  return SK_OK;
}

}  // namespace
}  // namespace sk

using namespace sk;

extern "C" {

sk_status sk_ell_from_csr(sk_matrix* out, sk_matrix csr) {
  sk_status s = check_source(out, csr);
  if (s != SK_OK) return s;
  if ((s = new_handle(out, SK_ELL, csr->dtype, csr->nrow, csr->ncol)) != SK_OK) return s;
  HandleGuard guard{out};
  s = csr->dtype == SK_F64 ? ell_from_csr<double>(*out, csr) : ell_from_csr<float>(*out, csr);
  if (s != SK_OK) return s;
  guard.ok = true;
  return SK_OK;
}

sk_status sk_jad_from_csr(sk_matrix* out, sk_matrix csr) {
  sk_status s = check_source(out, csr);
  if (s != SK_OK) return s;
  if ((s = new_handle(out, SK_JAD, csr->dtype, csr->nrow, csr->ncol)) != SK_OK) return s;
  HandleGuard guard{out};
  s = csr->dtype == SK_F64 ? jad_from_csr<double>(*out, csr) : jad_from_csr<float>(*out, csr);
  if (s != SK_OK) return s;
  guard.ok = true;
  return SK_OK;
}

sk_status sk_bsr_from_csr(sk_matrix* out, sk_matrix csr, int64_t block_rows, int64_t block_cols) {
  sk_status s = check_source(out, csr);
  if (s != SK_OK) return s;
  SK_CHECK(block_rows >= 1 && block_cols >= 1 && block_rows <= kThreads &&
               block_rows * block_cols <= kBsrTileVals,
           SK_INVALID_ARG, "block shape must be >= 1, block_rows <= 256, block size <= 4096");
  if ((s = new_handle(out, SK_BSR, csr->dtype, csr->nrow, csr->ncol)) != SK_OK) return s;
  HandleGuard guard{out};
  const int br = static_cast<int>(block_rows), bc = static_cast<int>(block_cols);
  s = csr->dtype == SK_F64 ? bsr_from_csr<double>(*out, csr, br, bc) : bsr_from_csr<float>(*out, csr, br, bc);
  if (s != SK_OK) return s;
  guard.ok = true;
  return SK_OK;
}

sk_status sk_matrix_build_ms(sk_matrix A, double* ms) {
  SK_CHECK(A && ms, SK_INVALID_ARG, "null handle or output");
  *ms = A->build_ms;
  return SK_OK;
}

sk_status sk_csr_export(sk_matrix A, int64_t* row_ptr, int64_t* col_ind, void* values) {
  SK_CHECK(A && A->format == SK_CSR, SK_INVALID_ARG, "not a CSR handle");
  cudaStream_t st = A->stream;
  SK_CUDA(cudaStreamSynchronize(st));
  sk_status s;
  if ((s = download_indices(A->csr.row_ptr, A->nrow + 1, row_ptr, st)) != SK_OK) return s;
  if ((s = download_indices(A->csr.col_ind, A->nnz, col_ind, st)) != SK_OK) return s;
  return download_values(A->csr.vals, A->nnz, A->dtype, values, st);
}

sk_status sk_ell_export(sk_matrix A, int64_t* col_ind, void* values) {
  SK_CHECK(A && A->format == SK_ELL, SK_INVALID_ARG, "not an ELL handle");
  cudaStream_t st = A->stream;
  SK_CUDA(cudaStreamSynchronize(st));
  const i64 slots = A->nrow * A->ell.width;
  if (slots == 0) return SK_OK;
  SK_CHECK(col_ind && values, SK_INVALID_ARG, "null output array");
  const size_t V = vbytes(A->dtype);
  Temps tmp(st);
  long long* stage = nullptr;
  char* vstage = nullptr;
  const i64 chunk = std::min(slots, kChunk);
  sk_status s;
  if ((s = tmp.get(&stage, chunk)) != SK_OK) return s;
  if ((s = tmp.get(&vstage, chunk * static_cast<i64>(V))) != SK_OK) return s;
  for (i64 off = 0; off < slots; off += chunk) {
    const i64 c = std::min(chunk, slots - off);
    if (A->dtype == SK_F64)
      SK_LAUNCH(ell_export_kernel<double>, grid_for(c), kThreads, 0, st, off, c, A->ell.width, A->ell.ld,
                A->ell.col, static_cast<const double*>(A->ell.vals), A->ell.rowlen, stage,
                reinterpret_cast<double*>(vstage));
    else
      SK_LAUNCH(ell_export_kernel<float>, grid_for(c), kThreads, 0, st, off, c, A->ell.width, A->ell.ld,
                A->ell.col, static_cast<const float*>(A->ell.vals), A->ell.rowlen, stage,
                reinterpret_cast<float*>(vstage));
    SK_CUDA(cudaMemcpyAsync(col_ind + off, stage, c * sizeof(long long), cudaMemcpyDeviceToHost, st));
    SK_CUDA(cudaMemcpyAsync(static_cast<char*>(values) + off * V, vstage, c * V, cudaMemcpyDeviceToHost, st));
    SK_CUDA(cudaStreamSynchronize(st));
  }
  return SK_OK;
}

sk_status sk_jad_export(sk_matrix A, int64_t* perm, int64_t* jdiag, int64_t* col_ind, void* values) {
  SK_CHECK(A && A->format == SK_JAD, SK_INVALID_ARG, "not a JAD handle");
  SK_CHECK(jdiag, SK_INVALID_ARG, "null jdiag");
  cudaStream_t st = A->stream;
  SK_CUDA(cudaStreamSynchronize(st));
  sk_status s;
  if (A->jad.njd > 0 && (s = download_indices(A->jad.perm, A->nrow, perm, st)) != SK_OK) return s;
  if ((s = download_indices(A->jad.jdiag, A->jad.njd + 1, jdiag, st)) != SK_OK) return s;
  if ((s = download_indices(A->jad.col, A->nnz, col_ind, st)) != SK_OK) return s;
  return download_values(A->jad.vals, A->nnz, A->dtype, values, st);
}

sk_status sk_bsr_export(sk_matrix A, int64_t* row_ptr, int64_t* col_ind, void* values) {
  SK_CHECK(A && A->format == SK_BSR, SK_INVALID_ARG, "not a BSR handle");
  cudaStream_t st = A->stream;
  SK_CUDA(cudaStreamSynchronize(st));
  const auto& b = A->bsr;
  sk_status s;
  if ((s = download_indices(b.row_ptr, b.nbr + 1, row_ptr, st)) != SK_OK) return s;
  if ((s = download_indices(b.col, b.nblocks, col_ind, st)) != SK_OK) return s;
  return download_values(b.vals, b.nblocks * b.br * b.bc, A->dtype, values, st);
}

}  // extern "C"
