// sk_core.cu -- library plumbing (status, device memory) and the upload of
// the reference's four storage layouts into device-resident handles.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "sk_internal.cuh"

namespace sk {

std::atomic<i64> g_launches{0};

constexpr unsigned long long kDefaultWaitNs = 2000000000ull;  // 2 s per barrier wait
static std::atomic<unsigned long long> g_wait_ns{kDefaultWaitNs};
static std::atomic<unsigned> g_wait_bias{0};
static std::atomic<int> g_sum_order{0};
bool summation_sequential() { return g_sum_order.load(std::memory_order_relaxed) != 0; }
unsigned long long wait_limit_ns() { return g_wait_ns.load(std::memory_order_relaxed); }
unsigned wait_target_bias() { return g_wait_bias.load(std::memory_order_relaxed); }
static thread_local std::string t_last_error;

void set_error(std::string const& msg) { t_last_error = msg; }
sk_status fail(sk_status st, std::string const& msg) {
  t_last_error = msg;
  return st;
}
sk_status cuda_fail(cudaError_t e, char const* what) {
  t_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return SK_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SK_NO_DEVICE;
  return SK_CUDA_ERROR;
}

cudaStream_t pick_stream(sk_matrix A, sk_stream s) {
  if (s) return static_cast<cudaStream_t>(s);
  return A ? A->stream : nullptr;
}

sk_status dev_alloc(sk_matrix A, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  if (A) {
    A->allocations.push_back(*p);
    A->device_bytes += static_cast<i64>(bytes);
  }
  return SK_OK;
}

// ------------------------------------------------------------------
// Narrowing of int64 index arrays to int32 on the device, with a range
// check [lo, hi) (allow_neg1: -1 also accepted, the ELL sentinel).
// ------------------------------------------------------------------
__global__ void narrow_kernel(const long long* __restrict__ in, int* __restrict__ out,
                              i64 count, long long lo, long long hi, int allow_neg1,
                              unsigned long long* bad) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < count; i += stride) {
    long long v = in[i];
    bool ok = (v >= lo && v < hi) || (allow_neg1 && v == -1);
    if (!ok) atomicAdd(bad, 1ull);
    out[i] = ok ? static_cast<int>(v) : 0;
  }
}

// ELL row-major chunk -> slot-major arrays; rowlen[i] = first -1 slot.
template <typename T>
__global__ void ell_transpose_kernel(const long long* __restrict__ col_rm,
                                     const T* __restrict__ val_rm, i64 g0, i64 count,
                                     i64 ld, i64 width, long long ncol,
                                     int* __restrict__ col_sm, T* __restrict__ val_sm,
                                     int* __restrict__ rowlen, unsigned long long* bad) {
  i64 t = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; t < count; t += stride) {
    i64 g = g0 + t;
    i64 i = g / width, k = g - i * width;
    long long c = col_rm[t];
    size_t dst = static_cast<size_t>(k) * static_cast<size_t>(ld) + static_cast<size_t>(i);
    if (c == -1) {
      atomicMin(rowlen + i, static_cast<int>(k));
      col_sm[dst] = 0;
      val_sm[dst] = T(0);
    } else {
      if (c < 0 || c >= ncol) atomicAdd(bad, 1ull);
      col_sm[dst] = (c >= 0 && c < ncol) ? static_cast<int>(c) : 0;
      val_sm[dst] = val_rm[t];
    }
  }
}

// Scatters CSR rows into the SELL-32 copy: entry k of row i goes to
// off[i / 32] + 32 k + i % 32; padding stays zero (column 0, value 0, never
// read because len[i] bounds every row).
template <typename T>
__global__ void csr_to_sell_kernel(i64 nrow, const int* __restrict__ rp, const int* __restrict__ ci,
                                   const T* __restrict__ va, const int* __restrict__ off,
                                   int* __restrict__ scol, T* __restrict__ sval,
                                   unsigned char* __restrict__ len) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  if (i >= nrow) return;
  const int a = rp[i], b = rp[i + 1];
  len[i] = static_cast<unsigned char>(b - a);
  const i64 base = off[i >> 5] + (i & 31);
  for (int k = 0; k < b - a; ++k) {
    scol[base + 32 * k] = ci[a + k];
    sval[base + 32 * k] = va[a + k];
  }
}

// Scatters BSR block rows into the sliced copy (layout in sk_internal.cuh).
template <typename T>
__global__ void bsr_to_sell_kernel(i64 nbr, int bsz, const int* __restrict__ rp, const int* __restrict__ bc,
                                   const T* __restrict__ va, const int* __restrict__ off,
                                   int* __restrict__ scol, T* __restrict__ sval,
                                   unsigned char* __restrict__ len) {
  i64 I = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  if (I >= nbr) return;
  const int a = rp[I], b = rp[I + 1];
  len[I] = static_cast<unsigned char>(b - a);
  const i64 o = off[I >> 5];
  const i64 l = I & 31;
  for (int k = 0; k < b - a; ++k) {
    scol[o + 32 * k + l] = bc[a + k];
    for (int e = 0; e < bsz; ++e)
      sval[(o + 32 * k) * bsz + 32 * e + l] = va[static_cast<i64>(a + k) * bsz + e];
  }
}

__global__ void fill_int_kernel(int* p, i64 n, int v) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) p[i] = v;
}

template <typename T>
__global__ void to_float_kernel(const T* __restrict__ in, float* __restrict__ out, i64 n) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) out[i] = static_cast<float>(in[i]);
}

int grid_for(i64 n) {
  i64 g = (n + kThreads - 1) / kThreads;
  return static_cast<int>(std::max<i64>(1, std::min<i64>(g, 148 * 32)));
}


// Copies count int64 host indices to int32 device memory, checking range.
static sk_status upload_indices(const int64_t* host, i64 count, int* dev, long long lo,
                                long long hi, bool allow_neg1, cudaStream_t st,
                                const char* what) {
  if (count == 0) return SK_OK;
  long long* stage = nullptr;
  unsigned long long* bad = nullptr;
  i64 chunk = std::min(count, kChunk);
  SK_CUDA(cudaMalloc(&stage, chunk * sizeof(long long)));
  cudaError_t e = cudaMalloc(&bad, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    cudaFree(stage);
    return cuda_fail(e, "cudaMalloc");
  }
  cudaMemsetAsync(bad, 0, sizeof(unsigned long long), st);
  for (i64 off = 0; off < count; off += chunk) {
    i64 c = std::min(chunk, count - off);
    cudaMemcpyAsync(stage, host + off, c * sizeof(long long), cudaMemcpyHostToDevice, st);
    SK_LAUNCH(narrow_kernel, grid_for(c), kThreads, 0, st, stage, dev + off, c, lo, hi,
              allow_neg1 ? 1 : 0, bad);
  }
  unsigned long long nbad = 0;
  cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  cudaFree(stage);
  cudaFree(bad);
  if (e != cudaSuccess) return cuda_fail(e, "upload_indices");
  if (nbad)
    return fail(SK_INDEX_OVERFLOW, std::string(what) + ": " + std::to_string(nbad) +
                                       " index value(s) outside the valid int32 range");
  return SK_OK;
}

// Row-block partition of a CSR row_ptr for csr_spmv_kernel: blocks of at
// most kRowsMax rows and kTileNnz entries, or one row longer than a tile.
// lanes[b] = 1 when every row of the block has at most 32 entries (one
// thread sums each row in order), else the lane count for the longest row.
static void csr_partition(const int64_t* rp, i64 n, std::vector<int>& part,
                          std::vector<unsigned char>& lanes) {
  part.clear();
  lanes.clear();
  part.push_back(0);
  i64 r = 0;
  while (r < n) {
    i64 r0 = r, nnz = 0, maxlen = 0;
    i64 len0 = rp[r + 1] - rp[r];
    if (len0 > kTileNnz) {
      ++r;
      part.push_back(static_cast<int>(r));
      lanes.push_back(32);
      continue;
    }
    // Rows of up to 32 entries and longer rows go to separate tiles, so a
    // short row is always summed by one lane in storage order.
    const bool long0 = len0 > 32;
    while (r < n && r - r0 < kRowsMax) {
      i64 len = rp[r + 1] - rp[r];
      if (nnz + len > kTileNnz || (len > 32) != long0) break;
      nnz += len;
      maxlen = std::max(maxlen, len);
      ++r;
    }
    part.push_back(static_cast<int>(r));
    unsigned char L = 1;
    if (maxlen > 32) L = maxlen <= 64 ? 4 : (maxlen <= 128 ? 8 : (maxlen <= 512 ? 16 : 32));
    lanes.push_back(L);
  }
}

// BSR block-row partition: at most kThreads / br block rows and a tile's
// worth of block values per CTA; a longer block row gets a CTA alone (the
// kernel then walks it tile by tile).
void bsr_partition(const int64_t* rp, i64 nbr, i64 br, i64 bsz, std::vector<int>& part) {
  part.clear();
  part.push_back(0);
  i64 max_rows = std::max<i64>(1, kThreads / br);
  i64 tile_blocks = std::min<i64>(1024, std::max<i64>(1, kBsrTileVals / bsz));
  i64 I = 0;
  while (I < nbr) {
    i64 I0 = I, nb = 0;
    while (I < nbr && I - I0 < max_rows) {
      i64 len = rp[I + 1] - rp[I];
      if (I > I0 && nb + len > tile_blocks) break;
      nb += len;
      ++I;
    }
    part.push_back(static_cast<int>(I));
  }
}

sk_status new_handle(sk_matrix* out, sk_format f, sk_dtype dt, i64 nrow, i64 ncol) {
  SK_CHECK(out != nullptr, SK_INVALID_ARG, "null output handle");
  *out = nullptr;
  SK_CHECK(dt == SK_F64 || dt == SK_F32, SK_INVALID_ARG, "dtype must be SK_F64 or SK_F32");
  SK_CHECK(nrow >= 0 && ncol >= 0, SK_INVALID_ARG, "negative shape");
  SK_CHECK(nrow < (i64(1) << 31) - 8 && ncol < (i64(1) << 31) - 8, SK_INDEX_OVERFLOW,
           "shape does not fit int32 indices");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(SK_NO_DEVICE, "no CUDA device available");
  auto* A = new sk_matrix_s;
  A->format = f;
  A->dtype = dt;
  A->nrow = nrow;
  A->ncol = ncol;
  cudaGetDevice(&A->device);
  cudaDeviceGetAttribute(&A->sm_count, cudaDevAttrMultiProcessorCount, A->device);
  if (A->sm_count <= 0) A->sm_count = 148;
  e = cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete A;
    return cuda_fail(e, "cudaStreamCreate");
  }
  *out = A;
  return SK_OK;
}

void destroy_handle(sk_matrix A) {
  if (!A) return;
  if (A->stream) cudaStreamSynchronize(A->stream);
  for (void* p : A->allocations) cudaFree(p);
  if (A->io) cudaFree(A->io);
  if (A->pipe) destroy_host_pipe(A->pipe);
  if (A->ws) cudaFree(A->ws);
  if (A->ws2) cudaFree(A->ws2);
  if (A->stream) cudaStreamDestroy(A->stream);
  delete A;
}

// Adds the SELL-32 copy of a CSR handle when every row has at most
// kSellMaxRow entries and the padding stays within a quarter of nnz.
static sk_status build_sell(sk_matrix A, const int64_t* rp, cudaStream_t st_) {
  const i64 n = A->nrow;
  if (n == 0 || A->nnz == 0) return SK_OK;
  const i64 nslices = (n + 31) / 32;
  std::vector<int> off(static_cast<size_t>(nslices) + 1, 0);
  i64 total = 0;
  for (i64 s = 0; s < nslices; ++s) {
    i64 w = 0;
    for (i64 i = 32 * s; i < std::min(n, 32 * s + 32); ++i) w = std::max<i64>(w, rp[i + 1] - rp[i]);
    if (w > kSellMaxRow) return SK_OK;
    off[static_cast<size_t>(s)] = static_cast<int>(total);
    total += 32 * w;
    if (total > (i64(1) << 31) - 64) return SK_OK;
  }
  off[static_cast<size_t>(nslices)] = static_cast<int>(total);
  if (total > A->nnz + A->nnz / 4 + 64) return SK_OK;
  const size_t V = vbytes(A->dtype);
  void *col = nullptr, *val = nullptr, *len = nullptr;
  sk_status st;
  if ((st = dev_alloc(A, &col, (total + 64) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &val, (total + 64) * V)) != SK_OK) return st;
  if ((st = dev_alloc(A, &len, n + 64)) != SK_OK) return st;
  SK_CUDA(cudaMemsetAsync(col, 0, (total + 64) * 4, st_));
  SK_CUDA(cudaMemsetAsync(val, 0, (total + 64) * V, st_));
  if ((st = upload_vector(A, off, &A->csr.sell_off, st_)) != SK_OK) return st;
  A->csr.sell_col = static_cast<int*>(col);
  A->csr.sell_vals = val;
  A->csr.sell_len = static_cast<unsigned char*>(len);
  A->csr.sell_entries = total;
  if (A->dtype == SK_F64)
    SK_LAUNCH(csr_to_sell_kernel<double>, ceil_div(n, kThreads), kThreads, 0, st_, n, A->csr.row_ptr,
              A->csr.col_ind, static_cast<const double*>(A->csr.vals), A->csr.sell_off, A->csr.sell_col,
              static_cast<double*>(val), A->csr.sell_len);
  else
    SK_LAUNCH(csr_to_sell_kernel<float>, ceil_div(n, kThreads), kThreads, 0, st_, n, A->csr.row_ptr,
              A->csr.col_ind, static_cast<const float*>(A->csr.vals), A->csr.sell_off, A->csr.sell_col,
              static_cast<float*>(val), A->csr.sell_len);
  SK_CUDA(cudaGetLastError());
  A->csr.sell = true;
  return SK_OK;
}

// The split product's row lists (long rows by decreasing length, ties in
// row order; short rows in row order) for a CSR handle without SELL-32
// whose rows longer than kHybLong hold at least half of the entries.  The
// long rows' share of the wave follows their share of the work, a short
// row's entry counting twice (its loads are not coalesced).
static sk_status build_hybrid(sk_matrix A, const int64_t* rp, cudaStream_t st_) {
  const i64 n = A->nrow;
  if (n == 0 || A->nnz == 0) return SK_OK;
  std::vector<int> shorts, longs;
  i64 long_nnz = 0;
  for (i64 i = 0; i < n; ++i) {
    const i64 len = rp[i + 1] - rp[i];
    if (len > kHybLong) {
      longs.push_back(static_cast<int>(i));
      long_nnz += len;
    } else {
      shorts.push_back(static_cast<int>(i));
    }
  }
  if (2 * long_nnz < A->nnz) return SK_OK;
  std::stable_sort(longs.begin(), longs.end(), [&](int a, int b) { return rp[a + 1] - rp[a] > rp[b + 1] - rp[b]; });
  sk_status st;
  if (!shorts.empty() && (st = upload_vector(A, shorts, &A->csr.hyb_short, st_)) != SK_OK) return st;
  if ((st = upload_vector(A, longs, &A->csr.hyb_long, st_)) != SK_OK) return st;
  A->csr.hyb_nshort = static_cast<int>(shorts.size());
  A->csr.hyb_nlong = static_cast<int>(longs.size());
  const double short_work = 2.0 * static_cast<double>(A->nnz - long_nnz);
  A->csr.hyb_long_frac = static_cast<double>(long_nnz) / (static_cast<double>(long_nnz) + short_work);
  A->csr.hyb = true;
  return SK_OK;
}

// Adds the sliced copy of a 2x2 or 3x3 BSR handle when every block row has
// at most kSellMaxRow blocks and the padding stays within a quarter.
sk_status build_bsr_sell(sk_matrix A, const int64_t* rp, cudaStream_t st_) {
  auto& B = A->bsr;
  if (!((B.br == 3 && B.bc == 3) || (B.br == 2 && B.bc == 2))) return SK_OK;
  const i64 nbr = B.nbr;
  if (nbr == 0 || B.nblocks == 0) return SK_OK;
  const i64 nslices = (nbr + 31) / 32;
  std::vector<int> off(static_cast<size_t>(nslices) + 1, 0);
  i64 total = 0;
  const i64 bsz = B.br * B.bc;
  for (i64 s = 0; s < nslices; ++s) {
    i64 w = 0;
    for (i64 I = 32 * s; I < std::min(nbr, 32 * s + 32); ++I) w = std::max<i64>(w, rp[I + 1] - rp[I]);
    if (w > kSellMaxRow) return SK_OK;
    off[static_cast<size_t>(s)] = static_cast<int>(total);
    total += 32 * w;
    if (total * bsz > (i64(1) << 31) - 64) return SK_OK;
  }
  off[static_cast<size_t>(nslices)] = static_cast<int>(total);
  if (total > B.nblocks + B.nblocks / 4 + 64) return SK_OK;
  const size_t V = vbytes(A->dtype);
  void *col = nullptr, *val = nullptr, *len = nullptr;
  sk_status st;
  if ((st = dev_alloc(A, &col, (total + 64) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &val, (total * bsz + 64) * V)) != SK_OK) return st;
  if ((st = dev_alloc(A, &len, nbr + 64)) != SK_OK) return st;
  SK_CUDA(cudaMemsetAsync(col, 0, (total + 64) * 4, st_));
  SK_CUDA(cudaMemsetAsync(val, 0, (total * bsz + 64) * V, st_));
  if ((st = upload_vector(A, off, &B.sell_off, st_)) != SK_OK) return st;
  B.sell_col = static_cast<int*>(col);
  B.sell_vals = val;
  B.sell_len = static_cast<unsigned char*>(len);
  B.sell_blocks = total;
  if (A->dtype == SK_F64)
    SK_LAUNCH(bsr_to_sell_kernel<double>, ceil_div(nbr, kThreads), kThreads, 0, st_, nbr, static_cast<int>(bsz),
              B.row_ptr, B.col, static_cast<const double*>(B.vals), B.sell_off, B.sell_col,
              static_cast<double*>(val), B.sell_len);
  else
    SK_LAUNCH(bsr_to_sell_kernel<float>, ceil_div(nbr, kThreads), kThreads, 0, st_, nbr, static_cast<int>(bsz),
              B.row_ptr, B.col, static_cast<const float*>(B.vals), B.sell_off, B.sell_col,
              static_cast<float*>(val), B.sell_len);
  SK_CUDA(cudaGetLastError());
  B.sell = true;
  return SK_OK;
}

// The product's tables of a CSR handle whose arrays are on the device:
// the row-block partition and its tiles, and the SELL-32 copy, all from the
// host copy of the row pointers.
sk_status csr_finish(sk_matrix A, const int64_t* row_ptr, cudaStream_t st_) {
  sk_status st;
  std::vector<int> part;
  std::vector<unsigned char> lanes;
  csr_partition(row_ptr, A->nrow, part, lanes);
  A->csr.nparts = static_cast<int>(part.size()) - 1;
  std::vector<int2> tiles(part.size());
  for (size_t b = 0; b < part.size(); ++b)
    tiles[b] = make_int2(part[b], static_cast<int>(row_ptr[part[b]]));
  if ((st = upload_vector(A, tiles, &A->csr.tiles, st_)) != SK_OK) return st;
  if ((st = upload_vector(A, lanes, &A->csr.lanes, st_)) != SK_OK) return st;
  if ((st = build_sell(A, row_ptr, st_)) != SK_OK) return st;
  return A->csr.sell ? SK_OK : build_hybrid(A, row_ptr, st_);
}

}  // namespace sk

using namespace sk;

i64 sk_matrix_s::spmv_bytes() const {
  const i64 V = dtype == SK_F64 ? 8 : 4;
  switch (format) {
    case SK_CSR:
      if (csr.dia_n) return (V * csr.dia_n + 2) * nrow + V * ncol + V * nrow;  // planes, mask, x, y
      return V * nnz + 4 * nnz + 4 * (nrow + 1) + V * ncol + V * nrow;
    case SK_ELL: return (V + 4) * nnz + V * ncol + V * nrow;
    case SK_JAD: return (V + 4) * nnz + 4 * (jad.njd + 1) + 4 * nrow + V * ncol + V * nrow;
    case SK_BSR:
      return bsr.nblocks * (bsr.br * bsr.bc * V + 4) + 4 * (bsr.nbr + 1) + V * ncol + V * nrow;
  }
  return 0;
}

extern "C" {

const char* sk_version(void) { return "sparkit_b200 0.1.0 (sm_100a)"; }

const char* sk_last_error(void) { return t_last_error.c_str(); }

sk_status sk_device_count(int* count) {
  SK_CHECK(count, SK_INVALID_ARG, "null count");
  *count = 0;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    cudaGetLastError();
  }
  return SK_OK;
}

sk_status sk_launch_count(int64_t* count) {
  SK_CHECK(count, SK_INVALID_ARG, "null count");
  *count = g_launches.load();
  return SK_OK;
}

sk_status sk_set_summation_order(int32_t order) {
  SK_CHECK(order == SK_SUM_TREE || order == SK_SUM_SEQUENTIAL, SK_INVALID_ARG, "unknown summation order");
  g_sum_order.store(order);
  return SK_OK;
}

sk_status sk_get_summation_order(int32_t* order) {
  SK_CHECK(order, SK_INVALID_ARG, "null pointer");
  *order = g_sum_order.load();
  return SK_OK;
}

sk_status sk_debug_set_wait(uint64_t limit_ns, int32_t unmeetable) {
  SK_CHECK(limit_ns <= 10000000000ull, SK_INVALID_ARG, "wait limit above 10 s");
  g_wait_ns.store(limit_ns ? limit_ns : kDefaultWaitNs);
  g_wait_bias.store(unmeetable ? 1u : 0u);
  return SK_OK;
}

sk_status sk_device_alloc(void** dev, size_t bytes) {
  SK_CHECK(dev, SK_INVALID_ARG, "null pointer");
  return dev_alloc(nullptr, dev, bytes);
}
sk_status sk_device_free(void* dev) {
  SK_CUDA(cudaFree(dev));
  return SK_OK;
}
sk_status sk_memcpy_h2d(void* dev, const void* host, size_t bytes, sk_stream s) {
  SK_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(s)));
  SK_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(s)));
  return SK_OK;
}
sk_status sk_memcpy_d2h(void* host, const void* dev, size_t bytes, sk_stream s) {
  SK_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(s)));
  SK_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(s)));
  return SK_OK;
}
sk_status sk_stream_synchronize(sk_stream s) {
  SK_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(s)));
  return SK_OK;
}

sk_status sk_csr_create(sk_matrix* out, int64_t nrow, int64_t ncol, const int64_t* row_ptr,
                        const int64_t* col_ind, const void* values, sk_dtype dtype) {
  sk_status st = new_handle(out, SK_CSR, dtype, nrow, ncol);
  if (st != SK_OK) return st;
  HandleGuard guard{out};
  sk_matrix A = *out;
  SK_CHECK(row_ptr, SK_INVALID_ARG, "null row_ptr");
  SK_CHECK(row_ptr[0] == 0, SK_INVALID_ARG, "row_ptr[0] must be 0");
  for (i64 i = 0; i < nrow; ++i)
    SK_CHECK(row_ptr[i + 1] >= row_ptr[i], SK_INVALID_ARG, "row_ptr must be non-decreasing");
  const i64 nnz = row_ptr[nrow];
  SK_CHECK(nnz < (i64(1) << 31) - 16, SK_INDEX_OVERFLOW, "nnz does not fit int32 row pointers");
  SK_CHECK(nnz == 0 || (col_ind && values), SK_INVALID_ARG, "null col_ind or values");
  A->nnz = nnz;
  cudaStream_t st_ = A->stream;
  const size_t V = vbytes(dtype);
  void *rp = nullptr, *ci = nullptr, *va = nullptr;
  if ((st = dev_alloc(A, &rp, (nrow + 1 + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &ci, (nnz + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &va, (nnz + 8) * V)) != SK_OK) return st;
  SK_CUDA(cudaMemsetAsync(ci, 0, (nnz + 8) * 4, st_));
  SK_CUDA(cudaMemsetAsync(va, 0, (nnz + 8) * V, st_));
  A->csr.row_ptr = static_cast<int*>(rp);
  A->csr.col_ind = static_cast<int*>(ci);
  A->csr.vals = va;
  if ((st = upload_indices(row_ptr, nrow + 1, A->csr.row_ptr, 0, nnz + 1, false, st_, "row_ptr")) != SK_OK)
    return st;
  if ((st = upload_indices(col_ind, nnz, A->csr.col_ind, 0, ncol, false, st_, "col_ind")) != SK_OK)
    return st;
  if (nnz) SK_CUDA(cudaMemcpyAsync(va, values, nnz * V, cudaMemcpyHostToDevice, st_));
  if ((st = csr_finish(A, row_ptr, st_)) != SK_OK) return st;
  SK_CUDA(cudaStreamSynchronize(st_));
  guard.ok = true;
  return SK_OK;
}

sk_status sk_ell_create(sk_matrix* out, int64_t nrow, int64_t ncol, int64_t width,
                        const int64_t* col_ind, const void* values, sk_dtype dtype) {
  sk_status st = new_handle(out, SK_ELL, dtype, nrow, ncol);
  if (st != SK_OK) return st;
  HandleGuard guard{out};
  sk_matrix A = *out;
  SK_CHECK(width >= 0 && width < (i64(1) << 31), SK_INVALID_ARG, "bad ELL width");
  const i64 slots = nrow * width;
  SK_CHECK(slots == 0 || (col_ind && values), SK_INVALID_ARG, "null col_ind or values");
  cudaStream_t st_ = A->stream;
  const size_t V = vbytes(dtype);
  A->ell.width = width;
  // slot stride: nrow rounded up to 32 plus 96, so that the slot streams a
  // warp reads together never sit a large power of two apart
  const i64 ld = (nrow + 31) / 32 * 32 + 96;
  A->ell.ld = ld;
  const i64 stored = ld * width;
  void *col = nullptr, *va = nullptr, *rl = nullptr;
  if ((st = dev_alloc(A, &col, (stored + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &va, (stored + 8) * V)) != SK_OK) return st;
  if ((st = dev_alloc(A, &rl, (nrow + 8) * 4)) != SK_OK) return st;
  A->ell.col = static_cast<int*>(col);
  A->ell.vals = va;
  A->ell.rowlen = static_cast<int*>(rl);
  SK_LAUNCH(fill_int_kernel, grid_for(nrow + 1), kThreads, 0, st_, A->ell.rowlen, nrow,
            static_cast<int>(width));
  if (slots > 0) {
    i64 chunk = std::min(slots, kChunk);
    long long* stage = nullptr;
    void* vstage = nullptr;
    unsigned long long* bad = nullptr;
    SK_CUDA(cudaMalloc(&stage, chunk * 8));
    SK_CUDA(cudaMalloc(&vstage, chunk * V));
    SK_CUDA(cudaMalloc(&bad, 8));
    SK_CUDA(cudaMemsetAsync(bad, 0, 8, st_));
    for (i64 off = 0; off < slots; off += chunk) {
      i64 c = std::min(chunk, slots - off);
      SK_CUDA(cudaMemcpyAsync(stage, col_ind + off, c * 8, cudaMemcpyHostToDevice, st_));
      SK_CUDA(cudaMemcpyAsync(vstage, static_cast<const char*>(values) + off * V, c * V,
                              cudaMemcpyHostToDevice, st_));
        if (dtype == SK_F64)
        SK_LAUNCH(ell_transpose_kernel<double>, grid_for(c), kThreads, 0, st_, stage,
                  static_cast<const double*>(vstage), off, c, ld, width, ncol, A->ell.col,
                  static_cast<double*>(va), A->ell.rowlen, bad);
      else
        SK_LAUNCH(ell_transpose_kernel<float>, grid_for(c), kThreads, 0, st_, stage,
                  static_cast<const float*>(vstage), off, c, ld, width, ncol, A->ell.col,
                  static_cast<float*>(va), A->ell.rowlen, bad);
    }
    unsigned long long nbad = 0;
    cudaMemcpyAsync(&nbad, bad, 8, cudaMemcpyDeviceToHost, st_);
    cudaError_t e = cudaStreamSynchronize(st_);
    cudaFree(stage);
    cudaFree(vstage);
    cudaFree(bad);
    if (e != cudaSuccess) return cuda_fail(e, "ell upload");
    if (nbad) return fail(SK_INDEX_OVERFLOW, "ELL col_ind holds values outside [0, ncol) other than -1");
  }
  // stored entries = sum of row lengths
  std::vector<int> rl_h(static_cast<size_t>(nrow));
  if (nrow) SK_CUDA(cudaMemcpy(rl_h.data(), A->ell.rowlen, nrow * 4, cudaMemcpyDeviceToHost));
  i64 nnz = 0;
  for (int v : rl_h) nnz += v;
  A->nnz = nnz;
  guard.ok = true;
  return SK_OK;
}

sk_status sk_jad_create(sk_matrix* out, int64_t nrow, int64_t ncol, int64_t njd,
                        const int64_t* perm, const int64_t* jdiag, const int64_t* col_ind,
                        const void* values, sk_dtype dtype) {
  sk_status st = new_handle(out, SK_JAD, dtype, nrow, ncol);
  if (st != SK_OK) return st;
  HandleGuard guard{out};
  sk_matrix A = *out;
  SK_CHECK(njd >= 0 && jdiag, SK_INVALID_ARG, "bad jagged-diagonal count or null jdiag");
  SK_CHECK(jdiag[0] == 0, SK_INVALID_ARG, "jdiag[0] must be 0");
  i64 prev_w = nrow;
  std::vector<int> plen(static_cast<size_t>(nrow) + 1, 0);
  for (i64 k = 0; k < njd; ++k) {
    i64 w = jdiag[k + 1] - jdiag[k];
    SK_CHECK(w >= 0 && w <= prev_w, SK_INVALID_ARG,
             "jagged-diagonal widths must be non-increasing and at most nrow");
    prev_w = w;
    plen[0] += 1;
    plen[static_cast<size_t>(w)] -= 1;
  }
  for (i64 i = 1; i < nrow; ++i) plen[i] += plen[i - 1];
  plen.resize(static_cast<size_t>(nrow));
  const i64 nnz = jdiag[njd];
  SK_CHECK(nnz < (i64(1) << 31) - 16, SK_INDEX_OVERFLOW, "nnz does not fit int32");
  // An empty reference JAD has no perm (Jagged_diagonal_sparsity_Impl.cpp:28-31):
  // every row is then zero and the identity order serves.
  std::vector<int64_t> ident;
  if (njd == 0 && perm == nullptr) {
    ident.resize(static_cast<size_t>(nrow));
    for (i64 i = 0; i < nrow; ++i) ident[static_cast<size_t>(i)] = i;
    perm = ident.data();
  }
  SK_CHECK(nrow == 0 || perm, SK_INVALID_ARG, "null perm");
  SK_CHECK(nnz == 0 || (col_ind && values), SK_INVALID_ARG, "null col_ind or values");
  A->nnz = nnz;
  A->jad.njd = njd;
  cudaStream_t st_ = A->stream;
  const size_t V = vbytes(dtype);
  void *pm = nullptr, *jd = nullptr, *ci = nullptr, *va = nullptr;
  if ((st = dev_alloc(A, &pm, (nrow + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &jd, (njd + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &ci, (nnz + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &va, (nnz + 8) * V)) != SK_OK) return st;
  A->jad.perm = static_cast<int*>(pm);
  A->jad.jdiag = static_cast<int*>(jd);
  A->jad.col = static_cast<int*>(ci);
  A->jad.vals = va;
  if ((st = upload_indices(perm, nrow, A->jad.perm, 0, nrow, false, st_, "perm")) != SK_OK) return st;
  if ((st = upload_indices(jdiag, njd + 1, A->jad.jdiag, 0, nnz + 1, false, st_, "jdiag")) != SK_OK)
    return st;
  if ((st = upload_indices(col_ind, nnz, A->jad.col, 0, ncol, false, st_, "col_ind")) != SK_OK) return st;
  if (nnz) SK_CUDA(cudaMemcpyAsync(va, values, nnz * V, cudaMemcpyHostToDevice, st_));
  if ((st = upload_vector(A, plen, &A->jad.plen, st_)) != SK_OK) return st;
  SK_CUDA(cudaStreamSynchronize(st_));
  guard.ok = true;
  return SK_OK;
}

sk_status sk_bsr_create(sk_matrix* out, int64_t nrow, int64_t ncol, int64_t block_rows,
                        int64_t block_cols, const int64_t* row_ptr, const int64_t* col_ind,
                        const void* values, sk_dtype dtype) {
  sk_status st = new_handle(out, SK_BSR, dtype, nrow, ncol);
  if (st != SK_OK) return st;
  HandleGuard guard{out};
  sk_matrix A = *out;
  SK_CHECK(block_rows >= 1 && block_cols >= 1 && block_rows <= kThreads &&
               block_rows * block_cols <= kBsrTileVals,
           SK_INVALID_ARG, "block shape must be >= 1, block_rows <= 256, block size <= 4096");
  SK_CHECK(row_ptr, SK_INVALID_ARG, "null row_ptr");
  const i64 nbr = (nrow + block_rows - 1) / block_rows;
  const i64 nbc = (ncol + block_cols - 1) / block_cols;
  SK_CHECK(row_ptr[0] == 0, SK_INVALID_ARG, "row_ptr[0] must be 0");
  for (i64 i = 0; i < nbr; ++i)
    SK_CHECK(row_ptr[i + 1] >= row_ptr[i], SK_INVALID_ARG, "row_ptr must be non-decreasing");
  const i64 nblocks = row_ptr[nbr];
  const i64 bsz = block_rows * block_cols;
  SK_CHECK(nblocks * bsz < (i64(1) << 31) - 16, SK_INDEX_OVERFLOW, "block values do not fit int32");
  SK_CHECK(nblocks == 0 || (col_ind && values), SK_INVALID_ARG, "null col_ind or values");
  auto& b = A->bsr;
  b.br = block_rows;
  b.bc = block_cols;
  b.nbr = nbr;
  b.nbr_mult = nrow / block_rows;
  b.nblocks = nblocks;
  A->nnz = nblocks * bsz;
  cudaStream_t st_ = A->stream;
  const size_t V = vbytes(dtype);
  void *rp = nullptr, *ci = nullptr, *va = nullptr;
  if ((st = dev_alloc(A, &rp, (nbr + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &ci, (nblocks + 8) * 4)) != SK_OK) return st;
  if ((st = dev_alloc(A, &va, (nblocks * bsz + 8) * V)) != SK_OK) return st;
  SK_CUDA(cudaMemsetAsync(va, 0, (nblocks * bsz + 8) * V, st_));
  b.row_ptr = static_cast<int*>(rp);
  b.col = static_cast<int*>(ci);
  b.vals = va;
  if ((st = upload_indices(row_ptr, nbr + 1, b.row_ptr, 0, nblocks + 1, false, st_, "row_ptr")) != SK_OK)
    return st;
  if ((st = upload_indices(col_ind, nblocks, b.col, 0, nbc, false, st_, "col_ind")) != SK_OK) return st;
  if (nblocks) SK_CUDA(cudaMemcpyAsync(va, values, nblocks * bsz * V, cudaMemcpyHostToDevice, st_));
  std::vector<int> part;
  bsr_partition(row_ptr, nbr, block_rows, bsz, part);
  b.nparts = static_cast<int>(part.size()) - 1;
  if ((st = upload_vector(A, part, &b.part, st_)) != SK_OK) return st;
  if ((st = build_bsr_sell(A, row_ptr, st_)) != SK_OK) return st;
  SK_CUDA(cudaStreamSynchronize(st_));
  guard.ok = true;
  return SK_OK;
}

sk_status sk_matrix_destroy(sk_matrix A) {
  destroy_handle(A);
  return SK_OK;
}

sk_status sk_matrix_info(sk_matrix A, int64_t info[8]) {
  SK_CHECK(A && info, SK_INVALID_ARG, "null handle or info");
  info[0] = A->format;
  info[1] = A->dtype;
  info[2] = A->nrow;
  info[3] = A->ncol;
  info[4] = A->nnz;
  info[5] = A->format == SK_ELL ? A->ell.width
            : A->format == SK_JAD ? A->jad.njd
            : A->format == SK_BSR ? A->bsr.nblocks
                                  : 0;
  info[6] = A->device_bytes;
  info[7] = A->spmv_bytes();
  return SK_OK;
}

sk_status sk_matrix_layout(sk_matrix A, int32_t* layout) {
  SK_CHECK(A && layout, SK_INVALID_ARG, "null handle or layout");
  *layout = SK_LAYOUT_NATIVE;
  if (A->format == SK_CSR) {
    const auto& C = A->csr;
    *layout = C.dia_n ? SK_LAYOUT_DIAGONALS
              : C.sell ? SK_LAYOUT_SELL
              : C.panel ? SK_LAYOUT_PANELS
              : C.hyb ? SK_LAYOUT_SPLIT
                      : SK_LAYOUT_NATIVE;
  } else if (A->format == SK_BSR && A->bsr.sell) {
    *layout = SK_LAYOUT_SELL;
  }
  return SK_OK;
}

sk_status sk_matrix_add_f32_values(sk_matrix A) {
  SK_CHECK(A, SK_INVALID_ARG, "null handle");
  SK_CHECK(A->format == SK_CSR, SK_NOT_SUPPORTED, "FP32 value copy is for CSR handles");
  if (A->dtype == SK_F32) return SK_OK;
  if (A->csr.vals32) return build_dia_f32(A);  // planes added after the copy
  void* p = nullptr;
  sk_status st = dev_alloc(A, &p, (A->nnz + 8) * 4);
  if (st != SK_OK) return st;
  SK_CUDA(cudaMemsetAsync(p, 0, (A->nnz + 8) * 4, A->stream));
  if (A->nnz)
    SK_LAUNCH(to_float_kernel<double>, grid_for(A->nnz), kThreads, 0, A->stream,
              static_cast<const double*>(A->csr.vals), static_cast<float*>(p), A->nnz);
  A->csr.vals32 = static_cast<float*>(p);
  if (A->csr.sell) {
    void* q = nullptr;
    st = dev_alloc(A, &q, (A->csr.sell_entries + 64) * 4);
    if (st != SK_OK) return st;
    SK_CUDA(cudaMemsetAsync(q, 0, (A->csr.sell_entries + 64) * 4, A->stream));
    SK_LAUNCH(to_float_kernel<double>, grid_for(A->csr.sell_entries), kThreads, 0, A->stream,
              static_cast<const double*>(A->csr.sell_vals), static_cast<float*>(q), A->csr.sell_entries);
    A->csr.sell_vals32 = static_cast<float*>(q);
  }
  SK_CUDA(cudaStreamSynchronize(A->stream));
  return build_dia_f32(A);
}

}  // extern "C"
