// sk_mm.cu -- Matrix Market text into a device CSR handle, and back.
//
// Reading follows read_matrix_market<T> (sparkit/data/matrix_market.hpp:45-115,
// banner: matrix_market.cpp:28-87) followed by to_compressed_row of the
// resulting Coordinate_matrix (Coordinate_matrix.hpp:36-41: a map keyed by
// (row, column), so the last of duplicate entries wins, then sorted):
//   host threads   split the (memory-mapped) text at line boundaries and
//                  parse their pieces with std::from_chars (correctly
//                  rounded, as the reference's istream >> T);
//   device         mirrors the entries of a symmetric file, sorts the
//                  (row, column) keys with a stable LSD radix sort, keeps
//                  the last entry of every key and builds the row pointers:
//                  the O(nnz log nnz) work the reference does in a std::map.
// Writing follows write_matrix_market (matrix_market.hpp:119-150): the same
// banner, size line and "row col value" lines, values as ostream << T
// prints them (6 significant digits) unless a precision is given.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "sk_sort.cuh"

namespace sk {
namespace {

enum { MM_COORDINATE, MM_ARRAY };
enum { MM_REAL, MM_INTEGER, MM_COMPLEX, MM_PATTERN };
enum { MM_GENERAL, MM_SYMMETRIC, MM_SKEW_SYMMETRIC, MM_HERMITIAN };

inline bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

std::string lower(std::string s) {
  for (auto& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}

// The whitespace-separated words of [b, e), as istream >> std::string reads them.
std::vector<std::string> words(const char* b, const char* e, size_t maxn) {
  std::vector<std::string> out;
  while (b < e && out.size() < maxn) {
    while (b < e && is_space(*b)) ++b;
    const char* s = b;
    while (b < e && !is_space(*b)) ++b;
    if (b > s) out.emplace_back(s, b);
  }
  return out;
}

// parse_banner (matrix_market.cpp:28-87)
sk_status parse_banner(const char* b, const char* e, int* format, int* field, int* symmetry) {
  auto w = words(b, e, 5);
  w.resize(5);
  if (lower(w[0]) != "%%matrixmarket") return fail(SK_INVALID_ARG, "matrix market: invalid banner header: " + w[0]);
  const std::string f = lower(w[2]), d = lower(w[3]), s = lower(w[4]);
  if (f == "coordinate")
    *format = MM_COORDINATE;
  else if (f == "array")
    *format = MM_ARRAY;
  else
    return fail(SK_INVALID_ARG, "matrix market: unknown format: " + f);
  if (d == "real")
    *field = MM_REAL;
  else if (d == "integer")
    *field = MM_INTEGER;
  else if (d == "complex")
    *field = MM_COMPLEX;
  else if (d == "pattern")
    *field = MM_PATTERN;
  else
    return fail(SK_INVALID_ARG, "matrix market: unknown field: " + d);
  if (s == "general")
    *symmetry = MM_GENERAL;
  else if (s == "symmetric")
    *symmetry = MM_SYMMETRIC;
  else if (s == "skew-symmetric")
    *symmetry = MM_SKEW_SYMMETRIC;
  else if (s == "hermitian")
    *symmetry = MM_HERMITIAN;
  else
    return fail(SK_INVALID_ARG, "matrix market: unknown symmetry: " + s);
  return SK_OK;
}

// istream >> integer: leading whitespace, an optional sign, digits.
bool parse_int(const char*& p, const char* e, long long* v) {
  while (p < e && is_space(*p)) ++p;
  if (p < e && *p == '+') ++p;
  auto r = std::from_chars(p, e, *v);
  if (r.ec != std::errc()) return false;
  p = r.ptr;
  return true;
}

// istream >> T for a real: leading whitespace, then the decimal form
// (std::from_chars rounds correctly, like the strtod behind istream).  A
// value beyond the type's range reads as libstdc++'s num_get reads it: an
// overflow as the largest finite value of its sign, an underflow as
// strtod's (strtof's) zero or subnormal.
template <typename T>
bool parse_real(const char*& p, const char* e, T* v) {
  while (p < e && is_space(*p)) ++p;
  if (p < e && *p == '+') ++p;
  auto r = std::from_chars(p, e, *v, std::chars_format::general);
  if (r.ec == std::errc::result_out_of_range) {
    char buf[128];
    const size_t n = std::min<size_t>(static_cast<size_t>(r.ptr - p), sizeof(buf) - 1);
    std::memcpy(buf, p, n);
    buf[n] = 0;
    const double d = sizeof(T) == 4 ? static_cast<double>(std::strtof(buf, nullptr)) : std::strtod(buf, nullptr);
    *v = std::isinf(d) ? std::copysign(std::numeric_limits<T>::max(), static_cast<T>(d)) : static_cast<T>(d);
  } else if (r.ec != std::errc()) {
    return false;
  }
  p = r.ptr;
  return true;
}

const char* line_end(const char* p, const char* e) {
  const void* q = std::memchr(p, '\n', static_cast<size_t>(e - p));
  return q ? static_cast<const char*>(q) : e;
}

// ------------------------------------------------------------------
// Device assembly
// ------------------------------------------------------------------
// 0-based keys row * ncol + col in file order, each mirrored entry of a
// symmetric file right after its original (matrix_market.hpp:104-106).
template <typename T>
__global__ void mm_keys_kernel(i64 nnz, const int* __restrict__ rows, const int* __restrict__ cols,
                               const T* __restrict__ vals, const i64* __restrict__ mirror_before, i64 ncol,
                               unsigned long long* __restrict__ keys, T* __restrict__ vexp) {
  i64 k = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; k < nnz; k += stride) {
    const i64 r = rows[k] - 1, c = cols[k] - 1;
    const T v = vals[k];
    const i64 pos = mirror_before ? k + mirror_before[k] : k;
    keys[pos] = static_cast<unsigned long long>(r) * ncol + c;
    vexp[pos] = v;
    if (mirror_before && r != c) {
      keys[pos + 1] = static_cast<unsigned long long>(c) * ncol + r;
      vexp[pos + 1] = v;
    }
  }
}

__global__ void mm_mirror_flags_kernel(i64 nnz, const int* __restrict__ rows, const int* __restrict__ cols,
                                       int* __restrict__ flag) {
  i64 k = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; k < nnz; k += stride) flag[k] = rows[k] != cols[k] ? 1 : 0;
}

// 1 for the last entry of each run of equal keys (std::map's
// insert_or_assign keeps the last value given for a key)
__global__ void mm_last_flags_kernel(i64 n, const unsigned long long* __restrict__ keys, int* __restrict__ flag) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) flag[i] = (i + 1 == n || keys[i] != keys[i + 1]) ? 1 : 0;
}

template <typename T>
__global__ void mm_compact_kernel(i64 n, const unsigned long long* __restrict__ keys,
                                  const int* __restrict__ order, const T* __restrict__ vexp,
                                  const int* __restrict__ flag, const i64* __restrict__ pos, i64 ncol,
                                  unsigned long long* __restrict__ ukeys, int* __restrict__ col, T* __restrict__ val) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) {
    if (!flag[i]) continue;
    const i64 d = pos[i];
    const unsigned long long k = keys[i];
    ukeys[d] = k;
    col[d] = static_cast<int>(k % static_cast<unsigned long long>(ncol));
    val[d] = vexp[order[i]];
  }
}

// row_ptr[r] = first entry whose key is at least r * ncol (r = 0 .. nrow)
__global__ void mm_row_ptr_kernel(i64 nrow, i64 nu, const unsigned long long* __restrict__ ukeys, i64 ncol,
                                  int* __restrict__ row_ptr) {
  i64 r = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; r <= nrow; r += stride) {
    const unsigned long long target = static_cast<unsigned long long>(r) * ncol;
    i64 lo = 0, hi = nu;
    while (lo < hi) {
      const i64 mid = (lo + hi) / 2;
      if (ukeys[mid] < target)
        lo = mid + 1;
      else
        hi = mid;
    }
    row_ptr[r] = static_cast<int>(lo);
  }
}

template <typename T>
sk_status mm_read(sk_matrix* out, const char* text, i64 len, sk_dtype dt, int threads) {
  SK_CHECK(out, SK_INVALID_ARG, "null output handle");
  *out = nullptr;
  SK_CHECK(text || len == 0, SK_INVALID_ARG, "null text");
  const char* p = text;
  const char* end = text + len;
  if (len == 0) return fail(SK_INVALID_ARG, "matrix market: unexpected end of input");
  // banner (matrix_market.hpp:49-64)
  const char* eol = line_end(p, end);
  int format = 0, field = 0, symmetry = 0;
  sk_status s = parse_banner(p, eol, &format, &field, &symmetry);
  if (s != SK_OK) return s;
  if (format != MM_COORDINATE) return fail(SK_INVALID_ARG, "matrix market: only coordinate format is supported");
  if (field == MM_COMPLEX) return fail(SK_INVALID_ARG, "matrix market: complex field is not yet supported");
  // comments and empty lines before the size line (:66-68)
  p = eol < end ? eol + 1 : end;
  while (p < end) {
    eol = line_end(p, end);
    if (eol > p && *p != '%') break;
    p = eol < end ? eol + 1 : end;
  }
  SK_CHECK(p < end, SK_INVALID_ARG, "matrix market: missing size line");
  long long rows = 0, cols = 0, nnz = 0;
  {
    const char* q = p;
    if (parse_int(q, eol, &rows) && parse_int(q, eol, &cols)) parse_int(q, eol, &nnz);
  }
  // Shape (Shape.cpp:8-10) rejects a side of 1 or less
  SK_CHECK(rows > 1 && cols > 1, SK_INVALID_ARG, "invalid matrix shape");
  SK_CHECK(nnz >= 0, SK_INVALID_ARG, "matrix market: negative entry count");
  const char* data = eol < end ? eol + 1 : end;
  const bool pattern = field == MM_PATTERN;
  // skew-symmetric and hermitian files are read as stored (:99-100)
  const bool symmetric = symmetry == MM_SYMMETRIC;

  // -- host: the entry lines, split among threads at line boundaries; each
  // thread parses its piece into its own arrays (first touch in parallel),
  // a prefix over the pieces' line counts places them, and the lines past
  // the first nnz are ignored, as the reference never reads them
  int nt = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
  nt = std::max(1, std::min({nt, 64, static_cast<int>((end - data) / (1 << 20)) + 1}));
  std::vector<const char*> cut(static_cast<size_t>(nt) + 1);
  cut[0] = data;
  cut[nt] = end;
  for (int t = 1; t < nt; ++t) {
    const char* c = std::max(data + (end - data) * t / nt, cut[t - 1]);
    const char* q = line_end(c, end);
    cut[t] = q < end ? q + 1 : end;
  }
  struct Piece {
    std::vector<int> r, c;
    std::vector<T> v;
    i64 bad = -1;  // first malformed line of the piece
  };
  std::vector<Piece> piece(static_cast<size_t>(nt));
  {
    std::vector<std::thread> pool;
    auto parse = [&](int t) {
      Piece& P = piece[t];
      const size_t guess = static_cast<size_t>(cut[t + 1] - cut[t]) / 16 + 16;
      P.r.reserve(guess);
      P.c.reserve(guess);
      P.v.reserve(guess);
      for (const char* q = cut[t]; q < cut[t + 1];) {
        const char* e2 = line_end(q, cut[t + 1]);
        const char* r = q;
        long long a = 0, b = 0;
        T v = T(1);  // pattern entries are 1 (:90-92)
        bool ok = parse_int(r, e2, &a) && parse_int(r, e2, &b) && (pattern || parse_real<T>(r, e2, &v));
        ok = ok && a >= 1 && a <= rows && b >= 1 && b <= cols;
        if (!ok && P.bad < 0) P.bad = static_cast<i64>(P.r.size());
        P.r.push_back(ok ? static_cast<int>(a) : 1);
        P.c.push_back(ok ? static_cast<int>(b) : 1);
        P.v.push_back(v);
        q = e2 < cut[t + 1] ? e2 + 1 : cut[t + 1];
      }
    };
    for (int t = 1; t < nt; ++t) pool.emplace_back(parse, t);
    parse(0);
    for (auto& th : pool) th.join();
  }
  std::vector<i64> first(static_cast<size_t>(nt) + 1, 0);
  for (int t = 0; t < nt; ++t) first[t + 1] = first[t] + static_cast<i64>(piece[t].r.size());
  if (first[nt] < nnz)
    return fail(SK_INVALID_ARG, "matrix market: unexpected end of input (" + std::to_string(first[nt]) + " of " +
                                    std::to_string(nnz) + " entry lines)");
  for (int t = 0; t < nt; ++t)
    if (piece[t].bad >= 0 && first[t] + piece[t].bad < nnz)
      return fail(SK_INVALID_ARG, "matrix market: entry line " + std::to_string(first[t] + piece[t].bad + 1) +
                                      " is not 'row col" + (pattern ? "" : " value") +
                                      "' with 1-based indices in range");

  // -- device: mirror, sort, keep the last of each key, row pointers
  if ((s = new_handle(out, SK_CSR, dt, rows, cols)) != SK_OK) return s;
  HandleGuard guard{out};
  sk_matrix A = *out;
  cudaStream_t st = A->stream;
  Temps tmp(st);
  int *dr = nullptr, *dc = nullptr;
  T* dv = nullptr;
  if ((s = tmp.get(&dr, nnz)) != SK_OK) return s;
  if ((s = tmp.get(&dc, nnz)) != SK_OK) return s;
  if ((s = tmp.get(&dv, nnz)) != SK_OK) return s;
  for (int t = 0; t < nt; ++t) {
    const i64 cnt = std::min<i64>(static_cast<i64>(piece[t].r.size()), nnz - first[t]);
    if (cnt <= 0) break;
    SK_CUDA(cudaMemcpyAsync(dr + first[t], piece[t].r.data(), cnt * sizeof(int), cudaMemcpyHostToDevice, st));
    SK_CUDA(cudaMemcpyAsync(dc + first[t], piece[t].c.data(), cnt * sizeof(int), cudaMemcpyHostToDevice, st));
    SK_CUDA(cudaMemcpyAsync(dv + first[t], piece[t].v.data(), cnt * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  i64 nexp = nnz;
  i64* mirror_before = nullptr;
  if (symmetric && nnz) {
    int* flag = nullptr;
    if ((s = tmp.get(&flag, nnz)) != SK_OK) return s;
    if ((s = tmp.get(&mirror_before, nnz + 1)) != SK_OK) return s;
    SK_LAUNCH(mm_mirror_flags_kernel, grid_for(nnz), kThreads, 0, st, nnz, dr, dc, flag);
    if ((s = exclusive_scan(flag, nnz, mirror_before, tmp, st)) != SK_OK) return s;
    i64 m = 0;
    SK_CUDA(cudaMemcpyAsync(&m, mirror_before + nnz, sizeof(i64), cudaMemcpyDeviceToHost, st));
    SK_CUDA(cudaStreamSynchronize(st));
    nexp = nnz + m;
  }
  SK_CHECK(nexp < (i64(1) << 31) - 16, SK_INDEX_OVERFLOW, "entries do not fit int32 positions");
  unsigned long long *k1 = nullptr, *k2 = nullptr, *sk = nullptr;
  int *i1 = nullptr, *i2 = nullptr, *si = nullptr, *lastf = nullptr;
  T* vexp = nullptr;
  i64* lpos = nullptr;
  if ((s = tmp.get(&k1, nexp)) != SK_OK) return s;
  if ((s = tmp.get(&k2, nexp)) != SK_OK) return s;
  if ((s = tmp.get(&i1, nexp)) != SK_OK) return s;
  if ((s = tmp.get(&i2, nexp)) != SK_OK) return s;
  if ((s = tmp.get(&vexp, nexp)) != SK_OK) return s;
  if ((s = tmp.get(&lastf, nexp)) != SK_OK) return s;
  if ((s = tmp.get(&lpos, nexp + 1)) != SK_OK) return s;
  i64 nu = 0;
  if (nexp) {
    SK_LAUNCH(mm_keys_kernel<T>, grid_for(nnz), kThreads, 0, st, nnz, dr, dc, dv, mirror_before,
              static_cast<i64>(cols), k1, vexp);
    const unsigned long long maxkey = static_cast<unsigned long long>(rows) * cols - 1;
    if ((s = stable_radix_sort<unsigned long long>(k1, k2, i1, i2, nexp, maxkey, tmp, st, &sk, &si)) != SK_OK)
      return s;
    SK_LAUNCH(mm_last_flags_kernel, grid_for(nexp), kThreads, 0, st, nexp, sk, lastf);
    if ((s = exclusive_scan(lastf, nexp, lpos, tmp, st)) != SK_OK) return s;
    SK_CUDA(cudaMemcpyAsync(&nu, lpos + nexp, sizeof(i64), cudaMemcpyDeviceToHost, st));
    SK_CUDA(cudaStreamSynchronize(st));
  }
  A->nnz = nu;
  const size_t V = sizeof(T);
  void *rp = nullptr, *ci = nullptr, *va = nullptr;
  unsigned long long* ukeys = nullptr;
  if ((s = tmp.get(&ukeys, nu)) != SK_OK) return s;
  if ((s = dev_alloc(A, &rp, (rows + 1 + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &ci, (nu + 8) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &va, (nu + 8) * V)) != SK_OK) return s;
  SK_CUDA(cudaMemsetAsync(ci, 0, (nu + 8) * 4, st));
  SK_CUDA(cudaMemsetAsync(va, 0, (nu + 8) * V, st));
  A->csr.row_ptr = static_cast<int*>(rp);
  A->csr.col_ind = static_cast<int*>(ci);
  A->csr.vals = va;
  if (nexp)
    SK_LAUNCH(mm_compact_kernel<T>, grid_for(nexp), kThreads, 0, st, nexp, sk, si, vexp, lastf, lpos,
              static_cast<i64>(cols), ukeys, A->csr.col_ind, static_cast<T*>(va));
  SK_LAUNCH(mm_row_ptr_kernel, grid_for(rows + 1), kThreads, 0, st, static_cast<i64>(rows), nu, ukeys,
            static_cast<i64>(cols), A->csr.row_ptr);
  SK_CUDA(cudaGetLastError());
  std::vector<int> rp32(static_cast<size_t>(rows) + 1);
  SK_CUDA(cudaMemcpyAsync(rp32.data(), A->csr.row_ptr, (rows + 1) * 4, cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  std::vector<int64_t> rp64(rp32.begin(), rp32.end());
  if ((s = csr_finish(A, rp64.data(), st)) != SK_OK) return s;
  SK_CUDA(cudaStreamSynchronize(st));
  guard.ok = true;
  return SK_OK;
}

sk_status read_any(sk_matrix* out, const char* text, i64 len, sk_dtype dt, int threads) {
  SK_CHECK(dt == SK_F64 || dt == SK_F32, SK_INVALID_ARG, "dtype must be SK_F64 or SK_F32");
  return dt == SK_F64 ? mm_read<double>(out, text, len, dt, threads) : mm_read<float>(out, text, len, dt, threads);
}

// write_matrix_market (matrix_market.hpp:119-150); precision 0 prints
// values as ostream << T does by default (%g, 6 significant digits).
template <typename T>
sk_status mm_write(sk_matrix A, FILE* f, int precision, int threads) {
  const i64 n = A->nrow, nnz = A->nnz;
  std::vector<int> rp(static_cast<size_t>(n) + 1), ci(static_cast<size_t>(nnz));
  std::vector<T> v(static_cast<size_t>(nnz));
  cudaStream_t st = A->stream;
  SK_CUDA(cudaMemcpyAsync(rp.data(), A->csr.row_ptr, (n + 1) * 4, cudaMemcpyDeviceToHost, st));
  if (nnz) {
    SK_CUDA(cudaMemcpyAsync(ci.data(), A->csr.col_ind, nnz * 4, cudaMemcpyDeviceToHost, st));
    SK_CUDA(cudaMemcpyAsync(v.data(), A->csr.vals, nnz * sizeof(T), cudaMemcpyDeviceToHost, st));
  }
  SK_CUDA(cudaStreamSynchronize(st));
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%lld %lld %lld\n", static_cast<long long>(n),
               static_cast<long long>(A->ncol), static_cast<long long>(nnz));
  int nt = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
  nt = std::max(1, std::min({nt, 64, static_cast<int>(nnz / 100000) + 1}));
  std::vector<std::string> buf(static_cast<size_t>(nt));
  const int prec = precision > 0 ? precision : 6;
  auto fmt = [&](int t) {
    const i64 r0 = n * t / nt, r1 = n * (t + 1) / nt;
    std::string& o = buf[t];
    o.reserve(static_cast<size_t>(rp[r1] - rp[r0]) * 32);
    char line[96];
    for (i64 r = r0; r < r1; ++r)
      for (int j = rp[r]; j < rp[r + 1]; ++j) {
        const int k = std::snprintf(line, sizeof(line), "%lld %d %.*g\n", static_cast<long long>(r + 1), ci[j] + 1,
                                    prec, static_cast<double>(v[j]));
        o.append(line, static_cast<size_t>(k));
      }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(fmt, t);
  fmt(0);
  for (auto& th : pool) th.join();
  for (auto& o : buf)
    if (std::fwrite(o.data(), 1, o.size(), f) != o.size()) return fail(SK_INVALID_ARG, "matrix market: write failed");
  return SK_OK;
}

}  // namespace
}  // namespace sk

using namespace sk;

extern "C" {

sk_status sk_matrix_market_read_buffer(sk_matrix* out, const char* text, int64_t length, sk_dtype dtype,
                                       int32_t threads) {
  SK_CHECK(length >= 0, SK_INVALID_ARG, "negative length");
  return read_any(out, text, length, dtype, threads);
}

sk_status sk_matrix_market_read(sk_matrix* out, const char* path, sk_dtype dtype, int32_t threads) {
  SK_CHECK(out && path, SK_INVALID_ARG, "null argument");
  *out = nullptr;
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) return fail(SK_INVALID_ARG, std::string("matrix market: cannot open file: ") + path);
  struct stat sb;
  if (::fstat(fd, &sb) != 0) {
    ::close(fd);
    return fail(SK_INVALID_ARG, std::string("matrix market: cannot read file: ") + path);
  }
  const size_t len = static_cast<size_t>(sb.st_size);
  if (len == 0) {
    ::close(fd);
    return read_any(out, "", 0, dtype, threads);
  }
  // the page cache mapped read-only: no copy of the text
  void* m = ::mmap(nullptr, len, PROT_READ, MAP_PRIVATE, fd, 0);
  ::close(fd);
  if (m == MAP_FAILED) return fail(SK_INVALID_ARG, std::string("matrix market: cannot map file: ") + path);
  sk_status s = read_any(out, static_cast<const char*>(m), static_cast<i64>(len), dtype, threads);
  ::munmap(m, len);
  return s;
}

sk_status sk_matrix_market_write(sk_matrix A, const char* path, int32_t precision, int32_t threads) {
  SK_CHECK(A && path, SK_INVALID_ARG, "null argument");
  SK_CHECK(A->format == SK_CSR, SK_INVALID_ARG, "write_matrix_market takes a CSR matrix");
  SK_CHECK(precision >= 0 && precision <= 40, SK_INVALID_ARG, "precision must be in [0, 40]");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(SK_INVALID_ARG, std::string("matrix market: cannot open file: ") + path);
  sk_status s =
      A->dtype == SK_F64 ? mm_write<double>(A, f, precision, threads) : mm_write<float>(A, f, precision, threads);
  if (std::fclose(f) != 0 && s == SK_OK) s = fail(SK_INVALID_ARG, "matrix market: write failed");
  return s;
}

}  // extern "C"
