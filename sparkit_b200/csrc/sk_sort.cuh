// sk_sort.cuh -- device scans and a stable radix sort shared by the format
// conversions (sk_convert.cu) and the Matrix Market assembly (sk_mm.cu):
// reduce-then-scan exclusive scans to int64, and a stable LSD radix sort of
// (key, position) pairs, 8 bits per pass, with each tile's ranks taken by
// warp match and per-warp digit counts so that equal keys keep their order.
#pragma once

#include <algorithm>
#include <vector>

#include "sk_internal.cuh"

namespace sk {
namespace {

constexpr int kScanTile = 4096;   // scan: items per CTA (256 threads x 16)
constexpr int kRadixTile = 4096;  // radix sort: keys per CTA (16 rounds of 256)

// ------------------------------------------------------------------
// Temporary device buffers of one conversion: stream-ordered, so that
// releasing them does not synchronise the device
// ------------------------------------------------------------------
struct Temps {
  cudaStream_t st;
  std::vector<void*> p;
  explicit Temps(cudaStream_t s) : st(s) {}
  ~Temps() {
    for (void* q : p) cudaFreeAsync(q, st);
  }
  template <typename V>
  sk_status get(V** out, i64 count) {
    void* q = nullptr;
    cudaError_t e = cudaMallocAsync(&q, static_cast<size_t>(std::max<i64>(count, 1) + 8) * sizeof(V), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    p.push_back(q);
    *out = static_cast<V*>(q);
    return SK_OK;
  }
};

// ------------------------------------------------------------------
// Exclusive scan to int64 (reduce, scan the tile sums, scan the tiles)
// ------------------------------------------------------------------
// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ i64 block_excl_scan(i64 v, i64* excl, i64* warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  i64 inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const i64 t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    i64 w = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const i64 t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < nw) warp_tot[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const i64 before = warp > 0 ? warp_tot[warp - 1] : 0;
  *excl = before + inc - v;
  const i64 total = warp_tot[(blockDim.x >> 5) - 1];
  __syncthreads();
  return total;
}

template <typename In>
__global__ void __launch_bounds__(kThreads) scan_sums_kernel(const In* __restrict__ in, i64 n,
                                                             i64* __restrict__ sums) {
  __shared__ i64 wt[kThreads / 32];
  const i64 base = static_cast<i64>(blockIdx.x) * kScanTile;
  i64 s = 0;
  for (int r = 0; r < kScanTile / kThreads; ++r) {
    const i64 i = base + r * kThreads + threadIdx.x;
    if (i < n) s += static_cast<i64>(in[i]);
  }
  i64 excl;
  const i64 tot = block_excl_scan(s, &excl, wt);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// In-place exclusive scan of the tile sums by one CTA.
__global__ void __launch_bounds__(1024) scan_single_kernel(i64* __restrict__ v, i64 n) {
  __shared__ i64 wt[32];
  i64 carry = 0;
  for (i64 base = 0; base < n; base += blockDim.x) {
    const i64 i = base + threadIdx.x;
    const i64 x = i < n ? v[i] : 0;
    i64 excl;
    const i64 tot = block_excl_scan(x, &excl, wt);
    if (i < n) v[i] = carry + excl;
    carry += tot;
  }
}

// out[i] = offset of the tile + exclusive scan inside it; out[n] = total.
template <typename In>
__global__ void __launch_bounds__(kThreads) scan_tiles_kernel(const In* __restrict__ in, i64 n,
                                                              const i64* __restrict__ tile_off,
                                                              i64* __restrict__ out) {
  __shared__ i64 buf[kScanTile];
  __shared__ i64 wt[kThreads / 32];
  const i64 base = static_cast<i64>(blockIdx.x) * kScanTile;
  for (int r = 0; r < kScanTile / kThreads; ++r) {
    const int j = r * kThreads + threadIdx.x;
    buf[j] = base + j < n ? static_cast<i64>(in[base + j]) : 0;
  }
  __syncthreads();
  constexpr int kPer = kScanTile / kThreads;
  i64 s = 0;
  for (int k = 0; k < kPer; ++k) s += buf[threadIdx.x * kPer + k];
  i64 excl;
  const i64 tot = block_excl_scan(s, &excl, wt);
  i64 run = tile_off[blockIdx.x] + excl;
  for (int k = 0; k < kPer; ++k) {
    const i64 x = buf[threadIdx.x * kPer + k];
    buf[threadIdx.x * kPer + k] = run;
    run += x;
  }
  __syncthreads();
  for (int r = 0; r < kScanTile / kThreads; ++r) {
    const int j = r * kThreads + threadIdx.x;
    if (base + j < n) out[base + j] = buf[j];
  }
  if (base + kScanTile >= n && threadIdx.x == 0) out[n] = tile_off[blockIdx.x] + tot;
}

// out[0..n] = exclusive scan of in[0..n) with the total at out[n].
template <typename In>
sk_status exclusive_scan(const In* in, i64 n, i64* out, Temps& tmp, cudaStream_t st) {
  if (n == 0) {
    SK_CUDA(cudaMemsetAsync(out, 0, sizeof(i64), st));
    return SK_OK;
  }
  const i64 nt = (n + kScanTile - 1) / kScanTile;
  i64* sums = nullptr;
  sk_status s = tmp.get(&sums, nt);
  if (s != SK_OK) return s;
  SK_LAUNCH(scan_sums_kernel<In>, static_cast<unsigned>(nt), kThreads, 0, st, in, n, sums);
  SK_LAUNCH(scan_single_kernel, 1, 1024, 0, st, sums, nt);
  SK_LAUNCH(scan_tiles_kernel<In>, static_cast<unsigned>(nt), kThreads, 0, st, in, n, sums, out);
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

__global__ void narrow_i64_kernel(const i64* __restrict__ in, i64 n, int* __restrict__ out) {
  i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  for (; i < n; i += stride) out[i] = static_cast<int>(in[i]);
}

// ------------------------------------------------------------------
// Stable LSD radix sort of (key, index) pairs, 8 bits per pass
// ------------------------------------------------------------------
template <typename Key>
__global__ void __launch_bounds__(kThreads) radix_hist_kernel(const Key* __restrict__ keys, i64 n,
                                                              int shift, int* __restrict__ hist,
                                                              i64 ntiles) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const i64 base = static_cast<i64>(blockIdx.x) * kRadixTile;
  for (int r = 0; r < kRadixTile / kThreads; ++r) {
    const i64 i = base + r * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&cnt[static_cast<int>((keys[i] >> shift) & Key(255))], 1);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// Keys of one tile go out in position order within each digit: round by
// round, warp by warp within a round, lane by lane within a warp.
template <typename Key>
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(
    const Key* __restrict__ kin, const int* __restrict__ vin, Key* __restrict__ kout,
    int* __restrict__ vout, i64 n, int shift, const i64* __restrict__ off, i64 ntiles) {
  __shared__ int run[256];
  __shared__ int wcnt[kThreads / 32][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  run[tid] = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) wcnt[w][tid] = 0;
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  const i64 base = static_cast<i64>(blockIdx.x) * kRadixTile;
  for (int r = 0; r < kRadixTile / kThreads; ++r) {
    const i64 i = base + r * kThreads + tid;
    const bool valid = i < n;
    const Key key = valid ? kin[i] : Key(0);
    const int d = valid ? static_cast<int>((key >> shift) & Key(255)) : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int lrank = __popc(peers & lt);
    if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pos = run[d] + lrank;
      for (int w = 0; w < warp; ++w) pos += wcnt[w][d];
      const i64 dst = off[static_cast<i64>(d) * ntiles + blockIdx.x] + pos;
      kout[dst] = key;
      vout[dst] = vin ? vin[i] : static_cast<int>(i);
    }
    __syncthreads();
    int s = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
      s += wcnt[w][tid];
      wcnt[w][tid] = 0;
    }
    run[tid] += s;
    __syncthreads();
  }
}

// Sorts keys[0..n) (values <= maxkey) stably; on return *keys_out and
// *idx_out hold the sorted keys and the original positions (either the
// input buffers or the scratch ones).
template <typename Key>
sk_status stable_radix_sort(Key* keys, Key* keys2, int* idx, int* idx2, i64 n, Key maxkey, Temps& tmp,
                            cudaStream_t st, Key** keys_out, int** idx_out) {
  const i64 ntiles = (n + kRadixTile - 1) / kRadixTile;
  int* hist = nullptr;
  i64* off = nullptr;
  sk_status s;
  if ((s = tmp.get(&hist, 256 * ntiles)) != SK_OK) return s;
  if ((s = tmp.get(&off, 256 * ntiles + 1)) != SK_OK) return s;
  Key *ka = keys, *kb = keys2;
  int *va = nullptr, *vb = idx;
  int shift = 0;
  do {
    SK_LAUNCH(radix_hist_kernel<Key>, static_cast<unsigned>(ntiles), kThreads, 0, st, ka, n, shift, hist, ntiles);
    if ((s = exclusive_scan(hist, 256 * ntiles, off, tmp, st)) != SK_OK) return s;
    SK_LAUNCH(radix_scatter_kernel<Key>, static_cast<unsigned>(ntiles), kThreads, 0, st, ka, va, kb, vb, n, shift,
              off, ntiles);
    SK_CUDA(cudaGetLastError());
    std::swap(ka, kb);
    va = vb;
    vb = (vb == idx) ? idx2 : idx;
    shift += 8;
  } while (shift < static_cast<int>(8 * sizeof(Key)) && (maxkey >> shift) != 0);
  *keys_out = ka;
  *idx_out = va;
  return SK_OK;
}


}  // namespace
}  // namespace sk
