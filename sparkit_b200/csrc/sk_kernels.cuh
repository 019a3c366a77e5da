// sk_kernels.cuh -- device code shared by the SpMV, BLAS-1, preconditioner
// and solver translation units.
//
// Arithmetic policy: products and sums are written with the _rn
// intrinsics, so nvcc never contracts a multiply and an add into an FMA.
// With the sequential per-row order used below this reproduces the
// reference's rounding bit for bit wherever a row is summed by one thread
// (CSR rows in blocks of short rows, every ELL, JAD and BSR row), and every
// element-wise update of the solvers.  Only the dot products (grid
// reductions in a fixed tree) round differently from the reference's
// sequential std::inner_product.
#pragma once

#include <cuda_runtime.h>

#include "sk_internal.cuh"

namespace sk {

// ------------------------------------------------------------------
// Rounding-explicit arithmetic
// ------------------------------------------------------------------
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }

// Streaming (evict-first) loads for matrix data that is read once per
// product, so that the vectors stay in L2.
__device__ __forceinline__ void load4_stream(const double* p, double (&o)[4]) {
  double2 a = __ldcs(reinterpret_cast<const double2*>(p));
  double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void load4_stream(const float* p, float (&o)[4]) {
  float4 a = __ldcs(reinterpret_cast<const float4*>(p));
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}
__device__ __forceinline__ void load4_stream(const int* p, int (&o)[4]) {
  int4 a = __ldcs(reinterpret_cast<const int4*>(p));
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}

// ------------------------------------------------------------------
// Deterministic block and grid reductions of NR doubles
// ------------------------------------------------------------------
template <int NR>
__device__ __forceinline__ void warp_reduce(double (&v)[NR]) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] += __shfl_xor_sync(0xffffffffu, v[j], off);
}

// Result valid in thread 0.  Any whole number of warps up to 1024 threads.
template <int NR>
__device__ __forceinline__ void block_reduce(double (&v)[NR]) {
  __shared__ double red_smem[32][NR > 0 ? NR : 1];
  warp_reduce<NR>(v);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < NR; ++j) red_smem[warp][j] = v[j];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] = lane < static_cast<int>(blockDim.x >> 5) ? red_smem[lane][j] : 0.0;
    warp_reduce<NR>(v);
  }
}

// Sums v over the whole grid; the last CTA to arrive calls fin(total) on
// thread 0.  Deterministic: CTA partials are summed in CTA order.
// The sequential order: warp j sums term j of elements 0 .. n-1 in element
// order (s = s + t_i from s = 0, in the value type), each lane holding the
// same running sum; the 32 terms of the next group are loaded while the
// current group is added.  Result in t[j] of every lane of warp j.
template <int NR>
__device__ __forceinline__ void sequential_sums(RedWs const& ws, double (&t)[NR]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= NR) return;
  const double* src = ws.seq + static_cast<size_t>(warp) * ws.seq_ld;
  const i64 n = ws.seq_n;
  double s64 = 0.0;
  float s32 = 0.0f;
  double nxt = lane < n ? __ldcg(src + lane) : 0.0;
  for (i64 i0 = 0; i0 < n; i0 += 32) {
    const double cur = nxt;
    nxt = i0 + 32 + lane < n ? __ldcg(src + i0 + 32 + lane) : 0.0;
    const int cnt = n - i0 < 32 ? static_cast<int>(n - i0) : 32;
    if (ws.seq_f32) {
      for (int k = 0; k < cnt; ++k) s32 = __fadd_rn(s32, static_cast<float>(__shfl_sync(0xffffffffu, cur, k)));
    } else {
      for (int k = 0; k < cnt; ++k) s64 = __dadd_rn(s64, __shfl_sync(0xffffffffu, cur, k));
    }
  }
#pragma unroll
  for (int j = 0; j < NR; ++j)
    if (j == warp) t[j] = ws.seq_f32 ? static_cast<double>(s32) : s64;
}

template <int NR, class Fin>
__device__ __forceinline__ void grid_reduce(double (&v)[NR], RedWs ws, Fin const& fin) {
  __shared__ bool am_last;
  __shared__ double seq_tot[NR];
  block_reduce<NR>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NR; ++j) ws.partials[static_cast<size_t>(blockIdx.x) * kMaxRed + j] = v[j];
    __threadfence();
    unsigned prev = atomicAdd(ws.counter, 1u);
    am_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double t[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) t[j] = 0.0;
  if (ws.seq) {
    sequential_sums<NR>(ws, t);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < NR && lane == 0) seq_tot[warp] = t[warp];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int j = 0; j < NR; ++j) t[j] = seq_tot[j];
      fin(t);
      *ws.counter = 0u;
    }
    return;
  }
  // 4 partials per thread in flight at a time: the loads are independent,
  // only their (fixed-order) sum is sequential
  unsigned b = threadIdx.x;
  for (; b + 3 * blockDim.x < gridDim.x; b += 4 * blockDim.x) {
    double q[4][NR];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int j = 0; j < NR; ++j)
        q[u][j] = __ldcg(ws.partials + static_cast<size_t>(b + u * blockDim.x) * kMaxRed + j);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int j = 0; j < NR; ++j) t[j] += q[u][j];
  }
  for (; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int j = 0; j < NR; ++j) t[j] += __ldcg(ws.partials + static_cast<size_t>(b) * kMaxRed + j);
  block_reduce<NR>(t);
  if (threadIdx.x == 0) {
    fin(t);
    *ws.counter = 0u;
  }
}

__device__ __forceinline__ bool solve_done(const Scalars* sc) {
  return sc != nullptr && *reinterpret_cast<const volatile int*>(&sc->done) != 0;
}

// Hands element i's contribution to a fused reduction: accumulated into
// red (the tree order), or, in the sequential order, stored as element i's
// terms for the last CTA to sum in element order.
template <int NR, class F>
__device__ __forceinline__ void reduce_terms(RedWs const& ws, i64 i, double* red, F const& f) {
  if constexpr (NR > 0) {
    if (ws.seq) {
      double e[NR];
#pragma unroll
      for (int j = 0; j < NR; ++j) e[j] = 0.0;
      f(e);
#pragma unroll
      for (int j = 0; j < NR; ++j) ws.seq[static_cast<size_t>(j) * ws.seq_ld + i] = e[j];
      return;
    }
  }
  f(red);
}

// ------------------------------------------------------------------
// SpMV epilogues.  operator()(row, value, red) receives each finished row
// exactly once; red[] accumulates the fused reductions (kNR of them);
// finalize(total) runs once, on the last CTA, with the grid totals.
// ------------------------------------------------------------------
template <typename T>
struct EpiStore {
  static constexpr int kNR = 0;
  T* y;
  __device__ void operator()(int row, T v, double*) const { y[row] = v; }
  __device__ void finalize(const double*) const {}
};

// ------------------------------------------------------------------
// Asynchronous 16-byte global -> shared copies (cp.async, L2 only).
// ------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
// One element (4 or 8 bytes) global -> shared, asynchronously.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(sizeof(T)) : "memory");
}

// ------------------------------------------------------------------
// CSR: one CTA per tile of rows (tiles[b] = {first row, first entry};
// at most 256 rows and 2048 entries, or one longer row).  Every thread
// starts all of its work's loads at once: the tile's row pointers (one per
// thread), the 8 values it owns straight into shared memory (cp.async, no
// register held while in flight) and their 8 column indices; then the 8
// gathers of x, so that the random gathers of skewed matrices overlap
// instead of being walked row by row.  The rounded products replace the
// values in shared memory.  Then each row is summed from there by one
// thread in storage order (bit-exact with the reference), or, in tiles
// holding a row longer than 32 entries, by L lanes with strided partial
// sums and a shuffle tree.  Six CTAs share an SM (at most 40 registers).
// ------------------------------------------------------------------
template <typename T, class Epi>
__global__ void __launch_bounds__(kThreads, 6)
csr_spmv_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                const T* __restrict__ va, const T* __restrict__ x,
                const int2* __restrict__ tiles,
                const unsigned char* __restrict__ lanes, Epi epi, RedWs ws,
                const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  __shared__ __align__(16) T sval[kTileNnz + 8];
  __shared__ int srp[kRowsMax + 1];
  if (solve_done(sc)) return;
  const int tid = threadIdx.x;
  const int2 t0 = tiles[blockIdx.x];
  const int2 t1 = tiles[blockIdx.x + 1];
  const int r0 = t0.x, nr = t1.x - t0.x;
  const int s = t0.y, e = t1.y;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;

  if (e - s > kTileNnz) {
    // A single row longer than a tile: strided partial sums + tree.
    double acc[1] = {0.0};
    T part_sum = T(0);
    for (int k = s + tid; k < e; k += kThreads)
      part_sum = add(part_sum, mul(__ldcs(va + k), __ldg(x + __ldcs(ci + k))));
    acc[0] = static_cast<double>(part_sum);
    block_reduce<1>(acc);
    if (tid == 0) reduce_terms<NR>(ws, r0, red, [&](double* rr) { epi(r0, static_cast<T>(acc[0]), rr); });
  } else {
    // Thread tid owns entries s + tid + 256 j (j < 8).  Row 0 of the tile
    // starts at s and row nr ends at e, so only rows 1..nr-1 need rp.
    constexpr int J = kTileNnz / kThreads;
    T* sprod = sval;
    int rpv = 0;
    if (tid > 0 && tid < nr) rpv = __ldg(rp + r0 + tid);
    int cj[J];
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k = s + tid + j * kThreads;
      if (k < e) {
        cp_async_elem(sprod + tid + j * kThreads, va + k);
        cj[j] = __ldcs(ci + k);
      }
    }
    T xj[J];
#pragma unroll
    for (int j = 0; j < J; ++j)
      if (s + tid + j * kThreads < e) xj[j] = __ldg(x + cj[j]);
    cp_async_commit_wait_all();  // this thread's own values have landed
#pragma unroll
    for (int j = 0; j < J; ++j)
      if (s + tid + j * kThreads < e) sprod[tid + j * kThreads] = mul(sprod[tid + j * kThreads], xj[j]);
    if (tid == 0) {
      srp[0] = 0;
      srp[nr] = e - s;
    } else if (tid < nr) {
      srp[tid] = rpv - s;
    }
    __syncthreads();
    const int L = lanes[blockIdx.x];
    if (L == 1) {
      if (tid < nr) {
        const int a = srp[tid], b = srp[tid + 1];
        T sum = T(0);
        for (int k = a; k < b; ++k) sum = add(sum, sprod[k]);
        reduce_terms<NR>(ws, r0 + tid, red, [&](double* rr) { epi(r0 + tid, sum, rr); });
      }
    } else {
      // L lanes per row (a power of two chosen at upload from the tile's
      // longest row), strided partial sums then a shuffle tree.
      const int rows_per_pass = kThreads / L;
      const int npass = (nr + rows_per_pass - 1) / rows_per_pass;
      const int lane = tid & (L - 1);
      for (int pass = 0; pass < npass; ++pass) {
        const int row = pass * rows_per_pass + tid / L;
        T sum = T(0);
        if (row < nr) {
          const int a = srp[row], b = srp[row + 1];
          for (int k = a + lane; k < b; k += L) sum = add(sum, sprod[k]);
        }
        for (int off = L >> 1; off > 0; off >>= 1)
          sum = add(sum, __shfl_xor_sync(0xffffffffu, sum, off));
        if (row < nr && lane == 0) reduce_terms<NR>(ws, r0 + row, red, [&](double* rr) { epi(r0 + row, sum, rr); });
      }
    }
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// Sum over one row of v_k * x[c_k], k = 0..n-1, accumulated from 0 in
// storage order (the reference's order, so the result is bit-exact);
// fetch(k, c, v) loads entry k.  PRED: rounds of U entries whose loads are
// all issued together (predicated); otherwise rounds of U plus a serial
// tail, which needs fewer registers.  The measured best per value type is
// chosen in launch_spmv.
// ------------------------------------------------------------------
template <typename T, int U, bool PRED, class Fetch>
__device__ __forceinline__ T row_dot(int n, const T* __restrict__ x, Fetch const& fetch) {
  T sum = T(0);
  if constexpr (PRED) {
    for (int k = 0; k < n; k += U) {
      int c[U];
      T v[U];
#pragma unroll
      for (int j = 0; j < U; ++j)
        if (k + j < n) fetch(k + j, c[j], v[j]);
      T xv[U];
#pragma unroll
      for (int j = 0; j < U; ++j)
        if (k + j < n) xv[j] = __ldg(x + c[j]);
#pragma unroll
      for (int j = 0; j < U; ++j)
        if (k + j < n) sum = add(sum, mul(v[j], xv[j]));
    }
  } else {
    int k = 0;
    for (; k + U <= n; k += U) {
      int c[U];
      T v[U];
#pragma unroll
      for (int j = 0; j < U; ++j) fetch(k + j, c[j], v[j]);
      T p[U];
#pragma unroll
      for (int j = 0; j < U; ++j) p[j] = mul(v[j], __ldg(x + c[j]));
#pragma unroll
      for (int j = 0; j < U; ++j) sum = add(sum, p[j]);
    }
    for (; k < n; ++k) {
      int c;
      T v;
      fetch(k, c, v);
      sum = add(sum, mul(v, __ldg(x + c)));
    }
  }
  return sum;
}

// ------------------------------------------------------------------
// CSR through its SELL-32 copy: one warp per slice of 32 rows, one thread
// per row.  Slot k of the 32 rows is one contiguous segment, so every load
// of column indices and values is a full coalesced line, and a thread's
// slots are independent loads issued together (8 at a time).  Each row is
// summed in storage order from 0, exactly as sparse_blas.hpp:25-28.
// ------------------------------------------------------------------
template <typename T, class Epi, int U, bool PRED, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
sell_spmv_kernel(int nrow, const int* __restrict__ off, const unsigned char* __restrict__ len,
                 const int* __restrict__ col, const T* __restrict__ va, const T* __restrict__ x,
                 Epi epi, RedWs ws, const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  if (solve_done(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  // grid-stride over rows: a kernel that carries a reduction runs at most
  // one wave of CTAs, so that few CTAs take part in the grid reduction
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < nrow; i += gridDim.x * kThreads) {
    const int n = len[i];
    const int* cp = col + __ldg(off + (i >> 5)) + (i & 31);
    const T* vp = va + (cp - col);
    const T sum = row_dot<T, U, PRED>(n, x, [&](int k, int& c, T& v) {
      c = __ldcs(cp + 32 * k);
      v = __ldcs(vp + 32 * k);
    });
    reduce_terms<NR>(ws, i, red, [&](double* rr) { epi(i, sum, rr); });
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// CSR split by row length, for skewed matrices (a few rows hold most of
// the entries).  One wave of CTAs: the last long_ctas CTAs take the long
// rows (more than kHybLong entries, by decreasing length, round robin over
// their warps), one warp per row: each lane sums the entries k = lane,
// lane + 32, ... into four independent partial sums (four loads of the
// contiguous row segment and four gathers of x in flight per lane), which
// a fixed shuffle tree then adds.  The other CTAs take the short rows in
// row order, one thread per row, each summed in storage order from 0 (the
// bits of sparse_blas.hpp:25-28).  No shared memory, so the L1 serves the
// random gathers of x only.
// ------------------------------------------------------------------
template <typename T, class Epi, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
hyb_spmv_kernel(const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ va,
                const T* __restrict__ x, const int* __restrict__ short_rows, int nshort,
                const int* __restrict__ long_rows, int nlong, int long_ctas, Epi epi, RedWs ws,
                const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  if (solve_done(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  const int short_ctas = static_cast<int>(gridDim.x) - long_ctas;
  if (static_cast<int>(blockIdx.x) >= short_ctas) {
    constexpr int W = kThreads / 32;
    const int lane = threadIdx.x & 31;
    const int nw = long_ctas * W;
    for (int w = (static_cast<int>(blockIdx.x) - short_ctas) * W + (threadIdx.x >> 5); w < nlong; w += nw) {
      const int row = __ldg(long_rows + w);
      const int b = __ldg(rp + row), e = __ldg(rp + row + 1);
      T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
      int k = b + lane;
      for (; k + 96 < e; k += 128) {
        const int c0 = __ldcs(ci + k), c1 = __ldcs(ci + k + 32), c2 = __ldcs(ci + k + 64), c3 = __ldcs(ci + k + 96);
        const T v0 = __ldcs(va + k), v1 = __ldcs(va + k + 32), v2 = __ldcs(va + k + 64), v3 = __ldcs(va + k + 96);
        const T x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
        a0 = add(a0, mul(v0, x0));
        a1 = add(a1, mul(v1, x1));
        a2 = add(a2, mul(v2, x2));
        a3 = add(a3, mul(v3, x3));
      }
      for (; k < e; k += 32) a0 = add(a0, mul(__ldcs(va + k), __ldg(x + __ldcs(ci + k))));
      T sum = add(add(a0, a1), add(a2, a3));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum = add(sum, __shfl_xor_sync(0xffffffffu, sum, o));
      if (lane == 0) reduce_terms<NR>(ws, row, red, [&](double* rr) { epi(row, sum, rr); });
    }
  } else {
    for (int t = blockIdx.x * kThreads + threadIdx.x; t < nshort; t += short_ctas * kThreads) {
      const int row = __ldg(short_rows + t);
      const int b = __ldg(rp + row), n = __ldg(rp + row + 1) - b;
      const T sum = row_dot<T, 4, true>(n, x, [&](int k, int& c, T& v) {
        c = __ldcs(ci + b + k);
        v = __ldcs(va + b + k);
      });
      reduce_terms<NR>(ws, row, red, [&](double* rr) { epi(row, sum, rr); });
    }
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// CSR through its column-panel copy (sk_panel.cu): CTA b owns rows
// row0[b] .. row0[b+1]-1 with a running sum each in shared memory, and
// walks the column panels in order, panel k of x in one half of a double
// buffer (cp.async) while panel k + 1 fills the other.  The matrix stream
// arrives in chunks (a panel's entries for this block, cut to fit a
// stage): thread 0 keeps kPanelStages chunks in flight, each moved by
// three bulk copies (values, column offsets, slice table) that complete
// on the stage's mbarrier, so the warps read nothing but shared memory.  A
// warp takes a slice (or a piece of one) of up to 32 row segments
// (lengths non-increasing over the lanes); each lane adds its entries to
// its row's sum one after another.  Slot j
// of a piece holds the entries j of lanes 0 .. c_j - 1 (c_j from a
// ballot), stored after slot j - 1.  A row has at most one segment per
// panel (the later pieces of a slice in later chunks), and the CTA
// synchronizes between chunks, so no two lanes touch the same sum at once
// and every row is summed in ascending column order.  Stage waits are bounded in time; a wait that
// runs out sets *err and the CTA skips the remaining work.
// ------------------------------------------------------------------
constexpr int kPanelThreads = 1024;

struct PanelArgs {
  const int* row0;
  const int* chunk_ptr;
  const int4* chunk;
  const int* chunk_kn;
  const unsigned* meta;
  const unsigned short* col;
  int panels, width, ncol, run_bytes, stage_bytes;
  int x16;  // x is 16-byte aligned
  int* err;
  unsigned long long wait_ns;
};

inline PanelArgs panel_args(const sk_matrix_s* A, const void* x) {
  const auto& C = A->csr;
  PanelArgs g{};
  g.row0 = C.pn_row0;
  g.chunk_ptr = C.pn_chunk_ptr;
  g.chunk = C.pn_chunk;
  g.chunk_kn = C.pn_chunk_kn;
  g.meta = C.pn_meta;
  g.col = C.pn_col;
  g.panels = C.pn_panels;
  g.width = C.pn_width;
  g.ncol = static_cast<int>(A->ncol);
  g.stage_bytes = C.pn_stage_bytes;
  g.run_bytes = C.pn_smem - 2 * C.pn_width * static_cast<int>(A->dtype == SK_F64 ? 8 : 4) -
                kPanelStages * C.pn_stage_bytes;
  g.x16 = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
  g.err = C.pn_err;
  g.wait_ns = wait_limit_ns();
  return g;
}

template <typename T>
__device__ __forceinline__ void panel_stage(T* dst, const T* __restrict__ x, int c0, int cnt, bool x16) {
  constexpr int E = 16 / static_cast<int>(sizeof(T));
  int done = 0;
  if (x16) {
    const int n16 = cnt / E;
    for (int i = threadIdx.x; i < n16; i += blockDim.x) cp_async16(dst + i * E, x + c0 + i * E);
    done = n16 * E;
  }
  for (int i = done + threadIdx.x; i < cnt; i += blockDim.x) cp_async_elem(dst + i, x + c0 + i);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ unsigned pn_smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void pn_bulk(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   pn_smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(pn_smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void pn_l2_prefetch(const void* p, unsigned bytes) {
  if (bytes) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool pn_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(pn_smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for a stage: false once wait_ns have passed.
__device__ __forceinline__ bool pn_wait(unsigned long long* bar, unsigned parity, unsigned long long wait_ns) {
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (pn_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (t0 == 0) {
        t0 = t;
      } else if (t - t0 > wait_ns) {
        return false;
      }
    }
  }
}

template <typename T, class Epi>
__global__ void __launch_bounds__(kPanelThreads, 1)
panel_spmv_kernel(PanelArgs g, const T* __restrict__ va, const T* __restrict__ x, Epi epi, RedWs ws,
                  const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  constexpr int SC = kPanelChunkEntries;
  constexpr unsigned V = sizeof(T);
  if (solve_done(sc)) return;
  extern __shared__ __align__(16) unsigned char panel_smem[];
  __shared__ __align__(8) unsigned long long bars[kPanelStages];
  __shared__ int s_fail;
  T* run = reinterpret_cast<T*>(panel_smem);
  T* xs = reinterpret_cast<T*>(panel_smem + g.run_bytes);
  unsigned char* stages = panel_smem + g.run_bytes + 2 * g.width * V;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  const int b = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const int r0 = __ldg(g.row0 + b), nr = __ldg(g.row0 + b + 1) - r0;
  const int c0 = __ldg(g.chunk_ptr + b), nch = __ldg(g.chunk_ptr + b + 1) - c0;
  for (int i = threadIdx.x; i < nr; i += blockDim.x) run[i] = T(0);
  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int j = 0; j < kPanelStages; ++j)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pn_smem_addr(&bars[j])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // chunk i into stage i % kPanelStages (thread 0)
  auto issue = [&](int i) {
    const int4 ch = __ldg(g.chunk + c0 + i);
    unsigned long long* bar = &bars[i % kPanelStages];
    unsigned char* st = stages + (i % kPanelStages) * g.stage_bytes;
    const unsigned bytes = static_cast<unsigned>(ch.y) * (V + 2u) + static_cast<unsigned>(ch.w) * 4u;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(pn_smem_addr(bar)), "r"(bytes)
                 : "memory");
    if (ch.y) {
      pn_bulk(st, va + ch.x, static_cast<unsigned>(ch.y) * V, bar);
      pn_bulk(st + SC * V, g.col + ch.x, static_cast<unsigned>(ch.y) * 2u, bar);
    }
    if (ch.w) pn_bulk(st + SC * (V + 2u), g.meta + ch.z, static_cast<unsigned>(ch.w) * 4u, bar);
    if (i + kPanelStages < nch) {  // the chunk after the stages in flight: into L2
      const int4 cn = __ldg(g.chunk + c0 + i + kPanelStages);
      pn_l2_prefetch(va + cn.x, static_cast<unsigned>(cn.y) * V);
      pn_l2_prefetch(g.col + cn.x, static_cast<unsigned>(cn.y) * 2u);
    }
  };
  if (threadIdx.x == 0)
    for (int i = 0; i < nch && i < kPanelStages; ++i) issue(i);
  panel_stage(xs, x, 0, min(g.width, g.ncol), g.x16 != 0);
  if (g.panels > 1) panel_stage(xs + g.width, x, g.width, min(g.width, g.ncol - g.width), g.x16 != 0);
  bool ok = true;
  int kprev = -1;
  for (int i = 0; i < nch; ++i) {
    const int kn = __ldg(g.chunk_kn + c0 + i);
    const int k = kn & 0xffff, ns = kn >> 16;
    if (k != kprev) {
      if (k + 1 < g.panels) {
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
      } else {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      }
      __syncthreads();  // panel k of x visible; the sums of panel k - 1 written
      kprev = k;
    }
    if (ok && !pn_wait(&bars[i % kPanelStages], (i / kPanelStages) & 1, g.wait_ns)) {
      ok = false;
      atomicExch(g.err, 1);
    }
    if (ok) {
      const unsigned char* st = stages + (i % kPanelStages) * g.stage_bytes;
      const T* sv = reinterpret_cast<const T*>(st);
      const unsigned short* scl = reinterpret_cast<const unsigned short*>(st + SC * V);
      const unsigned* rel = reinterpret_cast<const unsigned*>(st + SC * (V + 2u));
      const unsigned* segw = rel + ((ns + 3) & ~3);
      const T* xp = xs + (k & 1) * g.width;
      for (int t = warp; t < ns; t += nwarps) {
        const unsigned w = segw[t * 32 + lane];
        const int len = static_cast<int>(w >> 16), row = static_cast<int>(w & 0xffffu);
        const int base = static_cast<int>(rel[t]);
        const int maxlen = __shfl_sync(0xffffffffu, len, 0);  // lane 0 holds the longest segment
        T acc = len > 0 ? run[row] : T(0);
        int off = 0;
        for (int j = 0; j < maxlen; j += 4) {
          unsigned short c[4];
          T v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const unsigned m = __ballot_sync(0xffffffffu, len > j + u);
            if (len > j + u) {
              const int e = base + off + lane;
              c[u] = scl[e];
              v[u] = sv[e];
            }
            off += __popc(m);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (len > j + u) acc = add(acc, mul(v[u], xp[c[u]]));
        }
        if (len > 0) run[row] = acc;
      }
    }
    __syncthreads();  // stage i is free; after a panel's last chunk, its x buffer too
    if (threadIdx.x == 0 && i + kPanelStages < nch) issue(i + kPanelStages);
    const bool last = i + 1 == nch || (__ldg(g.chunk_kn + c0 + i + 1) & 0xffff) != k;
    if (last && k + 2 < g.panels) {
      const int c2 = (k + 2) * g.width;
      panel_stage(xs + (k & 1) * g.width, x, c2, min(g.width, g.ncol - c2), g.x16 != 0);
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (!ok) s_fail = 1;
  __syncthreads();
  if (s_fail) {
    // copies still in flight land before the CTA leaves (bounded)
    if (threadIdx.x == 0)
      for (int i = nch - kPanelStages < 0 ? 0 : nch - kPanelStages; i < nch; ++i)
        pn_wait(&bars[i % kPanelStages], (i / kPanelStages) & 1, g.wait_ns);
    __syncthreads();
    return;
  }
  for (int i = threadIdx.x; i < nr; i += blockDim.x)
    reduce_terms<NR>(ws, r0 + i, red, [&](double* rr) { epi(r0 + i, run[i], rr); });
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// CSR through its diagonal copy: one thread per row.  Diagonal d of a
// warp's 32 rows is one contiguous 32-value segment of the slice-major copy
// (a slice's segments are adjacent), and x[i + off[d]] is contiguous too,
// so neither the matrix stream nor the reads of x are gathers, and no
// column index is read.  The loads do not wait for the row's mask: a diagonal the row does
// not store reads a zero plane entry and a clamped x, and the mask leaves
// both out of the sum.  A row sums its stored entries in ascending column
// order from 0: the order of its CSR row, so the bits of sparse_blas.hpp:
// 25-28.  Rows r0 .. r1 - 1; y indexed by the absolute row.
// ------------------------------------------------------------------
struct DiaArgs {
  int n;  // diagonals
  int r0, r1;
  int ncol;
  const unsigned short* mask;
  int off[kDiaMax];
};

inline DiaArgs dia_args(const sk_matrix_s* A, i64 r0, i64 r1) {
  DiaArgs g{};
  g.n = A->csr.dia_n;
  g.r0 = static_cast<int>(r0);
  g.r1 = static_cast<int>(r1);
  g.ncol = static_cast<int>(A->ncol);
  g.mask = A->csr.dia_mask;
  for (int d = 0; d < kDiaMax; ++d) g.off[d] = A->csr.dia_off[d];
  return g;
}

template <typename T, class Epi, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
dia_spmv_kernel(DiaArgs g, const T* __restrict__ va, const T* __restrict__ x, Epi epi, RedWs ws,
                const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  if (solve_done(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  for (int i = g.r0 + blockIdx.x * kThreads + threadIdx.x; i < g.r1; i += gridDim.x * kThreads) {
    const unsigned m = __ldcs(g.mask + i);
    const T* vs = va + static_cast<long long>(i >> 5) * (32 * g.n) + (i & 31);
    // groups of G diagonals: the loads of a group are issued together
    constexpr int G = sizeof(T) == 8 ? 2 : 4;
    T sum = T(0);
#pragma unroll
    for (int d0 = 0; d0 < kDiaMax; d0 += G) {
      if (d0 >= g.n) break;
      T v[G], xv[G];
#pragma unroll
      for (int j = 0; j < G; ++j)
        if (d0 + j < g.n) {
          v[j] = __ldcs(vs + 32 * (d0 + j));
          xv[j] = __ldg(x + min(max(i + g.off[d0 + j], 0), g.ncol - 1));
        }
#pragma unroll
      for (int j = 0; j < G; ++j)
        if (d0 + j < g.n && ((m >> (d0 + j)) & 1u)) sum = add(sum, mul(v[j], xv[j]));
    }
    reduce_terms<NR>(ws, i, red, [&](double* rr) { epi(i, sum, rr); });
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// ELLPACK (slot-major): one thread per row, sequential over its slots,
// stopping at the row's length (the reference stops at the first -1).
// ------------------------------------------------------------------
template <typename T, class Epi, int U, bool PRED, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
ell_spmv_kernel(int nrow, long long ld, const int* __restrict__ col, const T* __restrict__ va,
                const int* __restrict__ rowlen, const T* __restrict__ x,
                Epi epi, RedWs ws, const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  if (solve_done(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < nrow; i += gridDim.x * kThreads) {
    const int* cp = col + i;
    const T* vp = va + i;
    const T sum = row_dot<T, U, PRED>(rowlen[i], x, [&](int k, int& c, T& v) {
      c = __ldcs(cp + k * ld);
      v = __ldcs(vp + k * ld);
    });
    reduce_terms<NR>(ws, i, red, [&](double* rr) { epi(i, sum, rr); });
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// Jagged diagonal: one thread per permuted position i, sweeping the
// diagonals that reach it (coalesced across i), then y[perm[i]] = sum.
// ------------------------------------------------------------------
template <typename T, class Epi, int U, bool PRED, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
jad_spmv_kernel(int nrow, const int* __restrict__ perm, const int* __restrict__ jd,
                const int* __restrict__ col, const T* __restrict__ va,
                const int* __restrict__ plen, const T* __restrict__ x,
                Epi epi, RedWs ws, const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  if (solve_done(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < nrow; i += gridDim.x * kThreads) {
    const T sum = row_dot<T, U, PRED>(plen[i], x, [&](int k, int& c, T& v) {
      const int idx = __ldg(jd + k) + i;
      c = __ldcs(col + idx);
      v = __ldcs(va + idx);
    });
    reduce_terms<NR>(ws, perm[i], red, [&](double* rr) { epi(perm[i], sum, rr); });
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// BSR: one CTA per block-row range; block values staged through shared
// memory (16-byte streaming loads) as products with x, then one thread per
// scalar row sums its block row in the reference's order:
// y = ((0 + s_0) + s_1) + ..., s_b = sequential sum over the block's row.
// Block rows at or past nrow / br (a partial last block row) give 0, as the
// reference's truncating loop bound does.  BR/BC > 0 fixes the block shape
// at compile time; 0 reads it at run time.
// ------------------------------------------------------------------
template <typename T, int BR, int BC, class Epi>
__global__ void __launch_bounds__(kThreads)
bsr_spmv_kernel(int nrow, int ncol, int br_rt, int bc_rt, int nbr_trunc,
                const int* __restrict__ rp, const int* __restrict__ bcol,
                const T* __restrict__ va, const T* __restrict__ x,
                const int* __restrict__ part, Epi epi, RedWs ws,
                const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  constexpr int kMaxTileBlocks = 1024;
  __shared__ T prod[kBsrTileVals];
  __shared__ int srp[kThreads + 1];
  __shared__ int scol[kMaxTileBlocks];
  if (solve_done(sc)) return;
  const int br = BR > 0 ? BR : br_rt;
  const int bc = BC > 0 ? BC : bc_rt;
  const int bsz = br * bc;
  const int tid = threadIdx.x;
  const int I0 = part[blockIdx.x];
  const int nb = part[blockIdx.x + 1] - I0;  // block rows of this CTA
  for (int t = tid; t <= nb; t += kThreads) srp[t] = rp[I0 + t];
  __syncthreads();
  const int bs = srp[0], be = srp[nb];
  int tile_blocks = kBsrTileVals / bsz;
  if (tile_blocks > kMaxTileBlocks) tile_blocks = kMaxTileBlocks;

  // thread -> (block row, row within block)
  const int my_I = tid / br;
  const int my_r = tid - my_I * br;
  const bool active = my_I < nb;
  T acc = T(0);
  int my_b = active ? srp[my_I] : 0;
  const int my_e = active ? srp[my_I + 1] : 0;

  for (int cb = bs; cb < be; cb += tile_blocks) {
    const int ce = cb + tile_blocks < be ? cb + tile_blocks : be;
    __syncthreads();
    for (int t = tid; t < ce - cb; t += kThreads) scol[t] = bcol[cb + t];
    __syncthreads();
    const size_t vs = static_cast<size_t>(cb) * bsz, ve = static_cast<size_t>(ce) * bsz;
    const size_t as = vs & ~static_cast<size_t>(3);
    const int ngroups = static_cast<int>((((ve + 3) & ~static_cast<size_t>(3)) - as) >> 2);
    for (int g = tid; g < ngroups; g += kThreads) {
      const size_t e0 = as + 4 * static_cast<size_t>(g);
      T v[4];
      load4_stream(va + e0, v);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const size_t e = e0 + j;
        if (e >= vs && e < ve) {
          const int local = static_cast<int>(e - vs);
          const int lb = local / bsz;
          const int rem = local - lb * bsz;
          const int c = rem % bc;
          const int xc = scol[lb] * bc + c;
          prod[local] = xc < ncol ? mul(v[j], __ldg(x + xc)) : T(0);
        }
      }
    }
    __syncthreads();
    if (active) {
      for (; my_b < my_e && my_b < ce; ++my_b) {
        const int base = (my_b - cb) * bsz + my_r * bc;
        T s = T(0);
        for (int c = 0; c < bc; ++c) s = add(s, prod[base + c]);
        acc = add(acc, s);
      }
    }
  }
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  if (active) {
    const int I = I0 + my_I;
    const int row = I * br + my_r;
    if (row < nrow) reduce_terms<NR>(ws, row, red, [&](double* rr) { epi(row, I < nbr_trunc ? acc : T(0), rr); });
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// ------------------------------------------------------------------
// BSR through its sliced copy (2x2 / 3x3 blocks): one thread per block
// row, reading each block's column and its BR*BC elements as coalesced
// 32-lane segments; row r of the block row accumulates
// y = ((0 + s_0) + s_1) + ..., s_b the sequential sum over the block's row r
// (spmv.hpp:158-170).  Block rows at or past nrow / br give 0.
// ------------------------------------------------------------------
template <typename T, int BR, int BC, class Epi>
__global__ void __launch_bounds__(kThreads, 4)
bsr_sell_kernel(int nrow, int ncol, int nbr, int nbr_trunc, const int* __restrict__ off,
                const unsigned char* __restrict__ len, const int* __restrict__ col,
                const T* __restrict__ va, const T* __restrict__ x, Epi epi, RedWs ws,
                const Scalars* sc) {
  constexpr int NR = Epi::kNR;
  constexpr int BSZ = BR * BC;
  if (solve_done(sc)) return;
  double red[NR > 0 ? NR : 1];
#pragma unroll
  for (int j = 0; j < (NR > 0 ? NR : 1); ++j) red[j] = 0.0;
  for (int I = blockIdx.x * kThreads + threadIdx.x; I < nbr; I += gridDim.x * kThreads) {
    const int n = I < nbr_trunc ? len[I] : 0;
    const int o = __ldg(off + (I >> 5));
    const int l = I & 31;
    T acc[BR];
#pragma unroll
    for (int r = 0; r < BR; ++r) acc[r] = T(0);
    for (int k = 0; k < n; ++k) {
      const int J = __ldcs(col + o + 32 * k + l);
      const T* vp = va + static_cast<size_t>(o + 32 * k) * BSZ + l;
      T v[BSZ];
#pragma unroll
      for (int e = 0; e < BSZ; ++e) v[e] = __ldcs(vp + 32 * e);
      T xv[BC];
#pragma unroll
      for (int c = 0; c < BC; ++c) {
        const int xc = J * BC + c;
        xv[c] = xc < ncol ? __ldg(x + xc) : T(0);
      }
#pragma unroll
      for (int r = 0; r < BR; ++r) {
        T sum = T(0);
#pragma unroll
        for (int c = 0; c < BC; ++c) sum = add(sum, mul(v[r * BC + c], xv[c]));
        acc[r] = add(acc[r], sum);
      }
    }
#pragma unroll
    for (int r = 0; r < BR; ++r) {
      const int row = I * BR + r;
      if (row < nrow) reduce_terms<NR>(ws, row, red, [&](double* rr) { epi(row, acc[r], rr); });
    }
  }
  if constexpr (NR > 0) {
    grid_reduce<NR>(red, ws, [&](const double* t) { epi.finalize(t); });
  }
}

// Grid size of the SpMV launch for a handle (for sizing RedWs).
inline int spmv_grid(const sk_matrix_s* A) {
  switch (A->format) {
    case SK_CSR:
      return A->csr.sell || A->csr.dia_n ? ceil_div(A->nrow, kThreads)
                                         : (A->csr.nparts > A->csr.pn_blocks ? A->csr.nparts : A->csr.pn_blocks);
    case SK_BSR: return A->bsr.sell ? ceil_div(A->bsr.nbr, kThreads) : A->bsr.nparts;
    default: return ceil_div(A->nrow, kThreads);
  }
}

// Row-loop variants per value type, as measured on B200 (3-D 7-point
// Laplacian, 128^3): FP64 rows run fastest as rounds of 4 plus a serial tail
// at 8 CTAs per SM (32 registers, with or without a fused reduction, no
// spills: so a 262,144-row product with a reduction is one wave of 1024
// CTAs, not 888 and a tail); FP32 SELL rows as predicated rounds of 8 at 5
// CTAs per SM.  The general CSR kernel with a fused reduction needs more
// registers and is bounded at 6 CTAs per SM.  Every variant sums each row in
// the same order, so the choice never changes a row's result.
template <typename T, class Epi>
struct SpmvTune {
  static constexpr int kMinB = Epi::kNR > 0 ? 6 : 8;
  static constexpr int kSellU = sizeof(T) == 8 ? 4 : 8;
  static constexpr bool kSellPred = sizeof(T) != 8;
  static constexpr int kSellMinB = sizeof(T) == 8 ? 8 : 5;
  // the diagonal kernel runs the SELL grid at the SELL residency, so that
  // a fused reduction sums the same rows in the same CTAs (the same bits)
  static constexpr int kDiaMinB = kSellMinB;
};

// Grid of a thread-per-row product over `rows` rows: one CTA per 256
// rows, or, when the epilogue carries a reduction, at most one wave
// (SMs x resident CTAs per SM) looping over the rows.
template <class Epi>
inline int row_grid(const sk_matrix_s* A, i64 rows, int minb) {
  const int full = ceil_div(rows, kThreads);
  if (Epi::kNR == 0) return full > 0 ? full : 1;
  const int wave = A->sm_count * minb;
  return full < wave ? (full > 0 ? full : 1) : wave;
}

// Launches y-epilogue SpMV on any format.  vals_override lets the
// mixed-precision path run the FP32 copy of an FP64 CSR handle.
template <typename T, class Epi>
void launch_spmv(const sk_matrix_s* A, const T* x, Epi const& epi, RedWs ws,
                 const Scalars* sc, cudaStream_t st,
                 const T* vals_override = nullptr) {
  if (A->nrow == 0) return;
  switch (A->format) {
    case SK_CSR: {
      if (A->csr.dia_n) {
        const T* v = vals_override ? vals_override : static_cast<const T*>(A->csr.dia_vals);
        SK_LAUNCH((dia_spmv_kernel<T, Epi, SpmvTune<T, Epi>::kDiaMinB>),
                  row_grid<Epi>(A, A->nrow, SpmvTune<T, Epi>::kSellMinB), kThreads, 0, st,
                  dia_args(A, 0, A->nrow), v, x, epi, ws, sc);
        break;
      }
      if (A->csr.sell) {
        const T* v = vals_override ? vals_override : static_cast<const T*>(A->csr.sell_vals);
        SK_LAUNCH((sell_spmv_kernel<T, Epi, SpmvTune<T, Epi>::kSellU, SpmvTune<T, Epi>::kSellPred,
                                    SpmvTune<T, Epi>::kSellMinB>),
                  row_grid<Epi>(A, A->nrow, SpmvTune<T, Epi>::kSellMinB), kThreads, 0, st,
                  static_cast<int>(A->nrow), A->csr.sell_off, A->csr.sell_len, A->csr.sell_col, v, x,
                  epi, ws, sc);
        break;
      }
      if (A->csr.panel && !vals_override) {
        static const bool attr_set = [] {
          return cudaFuncSetAttribute(panel_spmv_kernel<T, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kPanelSmem) == cudaSuccess;
        }();
        if (!attr_set) {
          set_error("panel product: shared-memory attribute refused");
          break;
        }
        SK_LAUNCH((panel_spmv_kernel<T, Epi>), A->csr.pn_blocks, kPanelThreads, A->csr.pn_smem, st,
                  panel_args(A, x), static_cast<const T*>(A->csr.pn_vals), x, epi, ws, sc);
        break;
      }
      const T* v = vals_override ? vals_override : static_cast<const T*>(A->csr.vals);
      if (A->csr.hyb) {
        constexpr int MB = 6;  // 40 registers: four loads and gathers in flight per lane without spills
        const int grid = A->sm_count * MB;
        const int nl = A->csr.hyb_nlong, ns = A->csr.hyb_nshort;
        int lc = static_cast<int>(grid * A->csr.hyb_long_frac + 0.5);
        lc = nl == 0 ? 0 : ns == 0 ? grid : (lc < 1 ? 1 : lc > grid - 1 ? grid - 1 : lc);
        SK_LAUNCH((hyb_spmv_kernel<T, Epi, MB>), grid, kThreads, 0, st, A->csr.row_ptr, A->csr.col_ind, v, x,
                  A->csr.hyb_short, ns, A->csr.hyb_long, nl, lc, epi, ws, sc);
        break;
      }
      SK_LAUNCH((csr_spmv_kernel<T, Epi>), A->csr.nparts, kThreads, 0, st,
                A->csr.row_ptr, A->csr.col_ind, v, x, A->csr.tiles, A->csr.lanes, epi,
                ws, sc);
      break;
    }
    case SK_ELL:
      SK_LAUNCH((ell_spmv_kernel<T, Epi, 4, false, SpmvTune<T, Epi>::kMinB>),
                row_grid<Epi>(A, A->nrow, SpmvTune<T, Epi>::kMinB), kThreads, 0, st,
                static_cast<int>(A->nrow), static_cast<long long>(A->ell.ld), A->ell.col,
                static_cast<const T*>(A->ell.vals),
                A->ell.rowlen, x, epi, ws, sc);
      break;
    case SK_JAD:
      SK_LAUNCH((jad_spmv_kernel<T, Epi, 4, false, SpmvTune<T, Epi>::kMinB>),
                row_grid<Epi>(A, A->nrow, SpmvTune<T, Epi>::kMinB), kThreads, 0, st,
                static_cast<int>(A->nrow), A->jad.perm, A->jad.jdiag, A->jad.col,
                static_cast<const T*>(A->jad.vals), A->jad.plen, x, epi, ws, sc);
      break;
    case SK_BSR: {
      const auto& b = A->bsr;
      if (b.sell) {
        const T* sv = static_cast<const T*>(b.sell_vals);
        if (b.br == 3)
          SK_LAUNCH((bsr_sell_kernel<T, 3, 3, Epi>), row_grid<Epi>(A, b.nbr, 4), kThreads, 0, st,
                    static_cast<int>(A->nrow), static_cast<int>(A->ncol), static_cast<int>(b.nbr),
                    static_cast<int>(b.nbr_mult), b.sell_off, b.sell_len, b.sell_col, sv, x, epi, ws, sc);
        else
          SK_LAUNCH((bsr_sell_kernel<T, 2, 2, Epi>), row_grid<Epi>(A, b.nbr, 4), kThreads, 0, st,
                    static_cast<int>(A->nrow), static_cast<int>(A->ncol), static_cast<int>(b.nbr),
                    static_cast<int>(b.nbr_mult), b.sell_off, b.sell_len, b.sell_col, sv, x, epi, ws, sc);
        break;
      }
      const T* v = static_cast<const T*>(b.vals);
      if (b.br == 3 && b.bc == 3)
        SK_LAUNCH((bsr_spmv_kernel<T, 3, 3, Epi>), b.nparts, kThreads, 0, st,
                  static_cast<int>(A->nrow), static_cast<int>(A->ncol), 3, 3,
                  static_cast<int>(b.nbr_mult), b.row_ptr, b.col, v, x, b.part, epi, ws, sc);
      else if (b.br == 2 && b.bc == 2)
        SK_LAUNCH((bsr_spmv_kernel<T, 2, 2, Epi>), b.nparts, kThreads, 0, st,
                  static_cast<int>(A->nrow), static_cast<int>(A->ncol), 2, 2,
                  static_cast<int>(b.nbr_mult), b.row_ptr, b.col, v, x, b.part, epi, ws, sc);
      else
        SK_LAUNCH((bsr_spmv_kernel<T, 0, 0, Epi>), b.nparts, kThreads, 0, st,
                  static_cast<int>(A->nrow), static_cast<int>(A->ncol),
                  static_cast<int>(b.br), static_cast<int>(b.bc),
                  static_cast<int>(b.nbr_mult), b.row_ptr, b.col, v, x, b.part, epi, ws, sc);
      break;
    }
  }
}

}  // namespace sk
