// sk_learned.cu -- the learned variable preconditioner of FGMRES: a small
// convolutional encoder-decoder over the 2-D grid of a 5-point matrix,
// trained on the device on (residual, error) pairs harvested from the plain
// solver's own runs, and applied inside FGMRES (fgmres.hpp:96-428 takes any
// callable as its variable preconditioner; the reference has no learned
// one).
//
// Network (3x3 convolutions, zero padding; NHWC BF16 tensors, FP32
// accumulation and FP32 master weights):
//   level 0 (H x W): e0 = relu(conv0(x; 8->16))
//   level 1 (H/2):   e1 = relu(conv1(pool(e0); 16->32))
//   level 2 (H/4):   e2 = relu(conv2(pool(e1); 32->64))
//   level 3 (H/8):   e3 = relu(conv3(pool(e2); 64->64)); b3 = relu(conv4(e3))
//   level 2:         d2 = relu(conv5(up(b3) + e2; 64->32))
//   level 1:         d1 = relu(conv6(up(d2) + e1; 32->16))
//   level 0:         d0 = relu(conv7(up(d1) + e0; 16->16)); y = conv8(d0; 16->1)
// pool = 2x2 average, up = nearest-neighbour.  Input features of a vector v
// with the coefficient planes (d, w, e, s, n) of the matrix: rt = v / d,
// s = rms(rt), x = [rt / s, w/d, e/d, s/d, n/d, 0, 0, 0]; the
// preconditioner returns z = s * y.
//
// Every convolution (forward, and the input gradient as a convolution with
// the flipped, transposed weights) is one implicit GEMM per CTA tile of
// 16 x 8 output pixels (M = 128) by all output channels (N = 16..64) with
// K = 9 taps x input channels:
//   * TMA (cp.async.bulk.tensor, 4-D map over [batch][H][W][C]) stages the
//     18 x 10 halo tile of each 8-channel chunk as one [18][10][8] BF16
//     plane; the zero padding of the convolution is the TMA's out-of-bounds
//     fill.  The packed weights arrive by one bulk copy.
//   * Each plane is directly a K-major no-swizzle UMMA operand: a core
//     matrix is 8 consecutive pixels of one tile row (8 x 16 B), the 16 tile
//     rows are core matrices 160 B apart (SBO), and the second 8-channel
//     half of a K = 16 step is the next plane (LBO) -- or, for 8 input
//     channels, the next tap.  A tap is only a start-address offset, so no
//     im2col copy exists anywhere.
//   * One thread issues 9 * Cin / 16 tcgen05.mma (kind::f16, BF16 inputs,
//     FP32 accumulator of 128 lanes x N columns in tensor memory); the four
//     warps read the accumulator back with tcgen05.ld (thread = pixel) and
//     apply bias, ReLU or the ReLU mask of the backward pass, and store
//     16-byte vectors.
//   * Variants: two tiles per CTA for the full-resolution 16-channel layers
//     (one wave of resident CTAs at 512^2), two threads per pixel for the
//     upsample-and-add epilogues, and a first layer that computes the
//     vector's feature channel into its staged planes (the matrix's fixed
//     channels are built once per preconditioner).
// The weight gradient (training only) is a GEMM over pixels with
// mma.sync.m16n8k16 on the same staged planes.
#include <cuda.h>
#include <cuda_bf16.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <random>
#include <set>
#include <utility>
#include <vector>

#include "sk_kernels.cuh"
#include "sk_learned.cuh"

namespace sk {

using bf16 = __nv_bfloat16;

// ------------------------------------------------------------------
// Network description
// ------------------------------------------------------------------
constexpr int kNL = 9;
constexpr int kCin[kNL] = {8, 16, 32, 64, 64, 64, 32, 16, 16};
constexpr int kCout[kNL] = {16, 32, 64, 64, 64, 32, 16, 16, 1};

constexpr int kTileH = 16, kTileW = 8;              // output tile: M = 128 pixels
constexpr int kHaloH = kTileH + 2, kHaloW = kTileW + 2;
constexpr int kPlaneBytes = kHaloH * kHaloW * 16;    // 2880: one [18][10][8] BF16 chunk
constexpr int kPlaneStride = 2944;                   // 128-byte aligned plane stride
constexpr int kGPlaneBytes = kTileH * kTileW * 16;   // 2048: one [16][8][8] chunk without halo
constexpr long long kSpinLimit = 1ll << 24;          // bounded mbarrier waits
constexpr int kConvThreads = 128;

inline int pad_n(int c) { return c < 16 ? 16 : c; }
inline int kchunks(int cin) {  // 8-channel K chunks of 9 taps, rounded to an even count
  const int kc = 9 * cin / 8;
  return (kc + 1) & ~1;
}

// ------------------------------------------------------------------
// PTX wrappers: mbarrier, TMA, tcgen05, ldmatrix / mma.sync
// ------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(phase)
      : "memory");
  return ok != 0;
}
// Waits with an iteration limit; on timeout records `code` and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned phase, int* err, int code) {
  for (long long i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(b, phase)) return true;
  if (err) atomicExch(err, code);
  return false;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// D[tmem] (+)= A[smem] * B[smem]^T, M = 128, N from idesc, K = 16 (BF16).
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle (version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major.
constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t (&r)[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2(uint32_t addr, uint32_t (&r)[2]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t (&r)[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t addr, uint32_t (&r)[2]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(addr));
}
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ------------------------------------------------------------------
// Convolution (forward, or input gradient with flipped weights)
// ------------------------------------------------------------------
__device__ __forceinline__ void unpack8(uint4 u, float (&f)[8]) {
  const bf16* h = reinterpret_cast<const bf16*>(&u);
#pragma unroll
  for (int j = 0; j < 8; ++j) f[j] = __bfloat162float(h[j]);
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 u;
  bf16* h = reinterpret_cast<bf16*>(&u);
#pragma unroll
  for (int j = 0; j < 8; ++j) h[j] = __float2bfloat16_rn(f[j]);
  return u;
}

enum ConvOut : int { OUT_BF16 = 0, OUT_F32 = 1, OUT_Z64 = 2 };

struct ConvArgs {
  int B, H, W;
  const bf16* wpk;      // packed weights, kchunks(CIN) x (N/8) core matrices of 8 x 16 B
  const float* bias;    // null: none
  int relu;
  const bf16* mask;     // null: none; else out = 0 where mask <= 0 (same layout as out)
  int out_kind;
  bf16* out;            // OUT_BF16: [B][H][W][N]
  bf16* pool_out;       // OUT_BF16, optional: 2x2 average of out, [B][H/2][W/2][N]
  const bf16* up_skip;  // OUT_BF16, optional: up_out = up(out) + up_skip at [B][2H][2W][N]
  bf16* up_out;
  float* outf;          // OUT_F32: channel 0 only, [B][H][W]
  double* outz;         // OUT_Z64: z = s[b] * (float)(acc0 + bias0)
  const double* scale;  // OUT_Z64: s per sample
  int z_add;            // OUT_Z64: z += s[b] * (float)(acc0 + bias0) instead
  // first layer of an apply (one sample): channel 0 of the staged input
  // planes replaced by the feature v * (1/d) / s, computed from these
  const double* feat_v;
  const float* feat_inv;
  const double* feat_s;
  int* err;
};

// Thread = output pixel (x, y) of sample b with the NC accumulators v of
// channels c0 .. c0 + NC - 1 of its N (the bias already added).  All
// threads of the CTA call it (the 2x2 pooling exchanges values between the
// lanes of a warp: x + 1 is lane + 1, y + 1 is lane + 8).
template <int N, bool UP, int NC = N>
__device__ __forceinline__ void conv_epilogue(ConvArgs const& a, int b, int y, int x, const float* v, int c0 = 0) {
  const bool valid = y < a.H && x < a.W;
  const i64 p = (static_cast<i64>(b) * a.H + y) * a.W + x;
  if (a.out_kind == OUT_F32) {
    if (valid && c0 == 0) a.outf[p] = v[0];
    return;
  }
  if (a.out_kind == OUT_Z64) {
    if (valid && c0 == 0) {
      const double zv = a.scale[b] * static_cast<double>(v[0]);
      a.outz[p] = a.z_add ? __dadd_rn(a.outz[p], zv) : zv;
    }
    return;
  }
  const int q0 = c0 / 8;  // first 16-byte channel group of this thread
  uint4* __restrict__ dst = reinterpret_cast<uint4*>(a.out + p * N) + q0;
  const uint4* __restrict__ msk =
      (a.mask && valid) ? reinterpret_cast<const uint4*>(a.mask + p * N) + q0 : nullptr;
  const bool pool_writer = valid && ((x & 1) == 0) && ((y & 1) == 0);
  const int h2 = a.H / 2, w2 = a.W / 2;
  // the reads of the epilogue (mask, the skip vectors of the four upsampled
  // pixels) are issued before the stores of their group of channels, up to
  // 32 channels at a time, so that their latencies overlap instead of
  // following the stores one by one
  const bool up = UP && valid;
  const uint4* __restrict__ skip = reinterpret_cast<const uint4*>(a.up_skip);
  constexpr int G = NC / 8 < 4 ? NC / 8 : 4;
#pragma unroll
  for (int cb = 0; cb < NC / 8; cb += G) {
    uint4 skv[UP ? G : 1][4];
    uint4 mvv[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      mvv[g] = msk ? __ldg(msk + cb + g) : make_uint4(0, 0, 0, 0);
      if constexpr (UP) {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          const i64 fp = (static_cast<i64>(b) * 2 * a.H + 2 * y + (d >> 1)) * (2 * a.W) + 2 * x + (d & 1);
          skv[g][d] = up ? __ldg(skip + fp * (N / 8) + q0 + cb + g) : make_uint4(0, 0, 0, 0);
        }
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int c = cb + g;
      const bf16* mb = reinterpret_cast<const bf16*>(&mvv[g]);
      uint4 o;
      bf16* ob = reinterpret_cast<bf16*>(&o);
      float r[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        float t = v[c * 8 + j];
        if (a.relu) t = fmaxf(t, 0.0f);
        if (msk && !(__bfloat162float(mb[j]) > 0.0f)) t = 0.0f;
        ob[j] = __float2bfloat16_rn(t);
        r[j] = __bfloat162float(ob[j]);
      }
      if (valid) dst[c] = o;
      if (a.pool_out) {
        float q[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float r01 = __shfl_down_sync(0xffffffffu, r[j], 1);
          const float r10 = __shfl_down_sync(0xffffffffu, r[j], 8);
          const float r11 = __shfl_down_sync(0xffffffffu, r[j], 9);
          q[j] = 0.25f * ((r[j] + r01) + (r10 + r11));
        }
        if (pool_writer)
          reinterpret_cast<uint4*>(a.pool_out)[((static_cast<i64>(b) * h2 + y / 2) * w2 + x / 2) * (N / 8) + q0 + c] =
              pack8(q);
      }
      if constexpr (UP) {
        if (up) {
#pragma unroll
        for (int d = 0; d < 4; ++d) {
          const i64 fp = (static_cast<i64>(b) * 2 * a.H + 2 * y + (d >> 1)) * (2 * a.W) + 2 * x + (d & 1);
          float sk[8], u[8];
          unpack8(skv[g][d], sk);
#pragma unroll
          for (int j = 0; j < 8; ++j) u[j] = r[j] + sk[j];
          reinterpret_cast<uint4*>(a.up_out)[fp * (N / 8) + q0 + c] = pack8(u);
        }
        }
      }
    }
  }
}

// The implicit GEMM of one 16 x 8 tile: 9 * CIN / 16 tcgen05.mma into the
// accumulator at tmem, from the staged planes at pbase (K-major, one
// [18][10][8] BF16 plane per 8 input channels) and the packed weights at
// wbase.  Issued by one thread.
template <int CIN, int N>
__device__ __forceinline__ void conv_issue_mma(uint32_t pbase, uint32_t wbase, uint32_t tmem) {
  constexpr uint32_t idesc = umma_idesc(128, N);
  constexpr int KC = (9 * CIN / 8 + 1) & ~1;
#pragma unroll
  for (int s = 0; s < KC / 2; ++s) {  // every tap offset a constant
    const int kc0 = 2 * s, kc1 = 2 * s + 1;
    uint32_t a0, lbo;
    if constexpr (CIN == 8) {
      // the two K halves are taps kc0 and kc1 of the single plane
      const int t0 = kc0, t1 = kc1 < 9 ? kc1 : kc0;
      const uint32_t o0 = ((t0 / 3) * kHaloW + t0 % 3) * 16, o1 = ((t1 / 3) * kHaloW + t1 % 3) * 16;
      a0 = pbase + o0;
      lbo = o1 - o0;
    } else {
      constexpr int P = CIN / 8;
      const int t = kc0 / P, c = kc0 % P;  // kc1 is plane c + 1 of the same tap
      a0 = pbase + c * kPlaneStride + ((t / 3) * kHaloW + t % 3) * 16;
      lbo = kPlaneStride;
    }
    const uint64_t ad = umma_desc(a0, lbo, kHaloW * 16);
    const uint64_t bd = umma_desc(wbase + kc0 * (N / 8) * 128, (N / 8) * 128, 128);
    umma_bf16(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
  }
}

// Shared memory of one conv CTA (TM tiles side by side along x).
template <int CIN, int N, bool TC, int TM = 1>
struct ConvSmem {
  static constexpr int kPlanes = CIN / 8;
  static constexpr int kKC = (9 * CIN / 8 + 1) & ~1;
  static constexpr int kWBytes = kKC * (N / 8) * 128;
  static constexpr int kIn = 0;
  static constexpr int kW = TM * kPlanes * kPlaneStride;
  static constexpr int kStage = kW + kWBytes;  // mma.sync path only: [128][N + 4] floats
  static constexpr int kBar = kStage + (TC ? 0 : 128 * (N + 4) * 4);
  static constexpr int kBytes = kBar + 64;
};

// TC = true: tcgen05 (product path); false: the same tile with mma.sync
// (cross-check of the tcgen05 path in the tests).  UP: the epilogue also
// writes the upsampled sum with the skip tensor (a.up_out); the other
// layers leave out its registers.  TM: 16 x 8 tiles per CTA side by side
// along x (tcgen05 only), each with its own TMEM accumulator columns, so
// that the full-resolution layers fit in one wave of resident CTAs.  CS:
// threads per pixel (tcgen05 only); with CS = 2 the second 128 threads read
// the upper half of the accumulator columns of the same TMEM lanes and run
// the epilogue of those channels, which halves each thread's chain of
// upsample-and-add loads and stores.  FEAT: the first layer of an apply
// (8 input channels, one sample) computes channel 0 of its input, the
// scaled vector v / d / s, into the staged planes itself; the other
// channels come from a tensor that holds the matrix's fixed features.
template <int CIN, int N, bool TC, bool UP, int TM = 1, int CS = 1, bool FEAT = false>
__global__ void __launch_bounds__(kConvThreads * CS) conv3x3_kernel(const __grid_constant__ CUtensorMap in_map,
                                                                    ConvArgs a) {
  static_assert(TC || TM == 1, "several tiles per CTA only on the tcgen05 path");
  static_assert(!FEAT || (CIN == 8 && TC), "fused features only for the first layer on the tcgen05 path");
  static_assert(CS == 1 || (TC && N / CS >= 16), "channel split only on the tcgen05 path, 16 columns or more");
  constexpr int NC = N / CS;
  using S = ConvSmem<CIN, N, TC, TM>;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* planes = smem + S::kIn;
  unsigned char* wsm = smem + S::kW;
  uint64_t* bar_load = reinterpret_cast<uint64_t*>(smem + S::kBar);
  uint64_t* bar_mma = bar_load + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_load + 2);
  __shared__ int ok_load;
  __shared__ float s_bias[N];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int px = tid & (kConvThreads - 1), cbase = (tid / kConvThreads) * NC;  // pixel, first channel
  const int x0 = blockIdx.x * kTileW * TM, y0 = blockIdx.y * kTileH, b = blockIdx.z;
  constexpr uint32_t kCols = TM * N < 32 ? 32 : TM * N;

  // Launched as a programmatic dependent of the previous layer: this CTA
  // sets up (barriers, tensor memory), then lets the next layer launch, and
  // touches no global memory until the previous grid has completed
  // (griddepcontrol.wait).  The next layer can launch only once every CTA
  // of this one holds its tensor memory, so no CTA of this layer ever waits
  // for columns held by a CTA that waits for this layer.
  if (tid == 0) {
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if constexpr (TC) {
    if (warp == 0) tmem_alloc(tmem_slot, kCols);
    tc_fence_before();
  }
  __syncthreads();
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // The weights and biases are written only between passes (packing after
  // an optimizer step), before the first layer of a pass starts, and that
  // layer starts only after every earlier kernel has completed; so they
  // are fetched while the previous layer finishes.  The input planes are
  // the previous layer's output: they wait for it.
  // (a single-channel output has one bias value)
  if (tid < N) s_bias[tid] = a.bias && (a.out_kind == OUT_BF16 || tid == 0) ? __ldg(a.bias + tid) : 0.0f;
  if (tid == 0) {
    mbar_expect_tx(bar_load, TM * S::kPlanes * kPlaneBytes + S::kWBytes);
    bulk_load(wsm, a.wpk, S::kWBytes, bar_load);
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (tid == 0) {
    for (int t = 0; t < TM; ++t)
      for (int c = 0; c < S::kPlanes; ++c)
        tma_load_4d(planes + (t * S::kPlanes + c) * kPlaneStride, &in_map, c * 8, x0 + t * kTileW - 1, y0 - 1, b,
                    bar_load);
  }
  // While the tiles arrive: FEAT loads the vector channel of its halo
  // pixels, (float)(v * (double)(1/d) / s), zero outside the grid (the
  // convolution's padding) or for s = 0; UP brings the skip vectors that
  // its epilogue adds into L1.
  constexpr int kHalo = TM * kHaloH * kHaloW;
  constexpr int kFeatPer = FEAT ? (kHalo + kConvThreads * CS - 1) / (kConvThreads * CS) : 1;
  float feat[kFeatPer];
  if constexpr (FEAT) {
    const double sb = *a.feat_s;
#pragma unroll
    for (int k = 0; k < kFeatPer; ++k) {
      const int idx = tid + k * kConvThreads * CS;
      const int t = idx / (kHaloH * kHaloW), h = idx % (kHaloH * kHaloW);
      const int gy = y0 - 1 + h / kHaloW, gx = x0 + t * kTileW - 1 + h % kHaloW;
      float f = 0.0f;
      if (idx < kHalo && gy >= 0 && gy < a.H && gx >= 0 && gx < a.W && sb > 0.0) {
        const i64 p = static_cast<i64>(gy) * a.W + gx;
        f = static_cast<float>(a.feat_v[p] * static_cast<double>(a.feat_inv[p]) / sb);
      }
      feat[k] = f;
    }
  }
  if constexpr (UP) {
    const int y = y0 + (px >> 3), x = x0 + (px & 7);
    if (a.up_skip && y < a.H && x < a.W) {
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        const i64 fp = (static_cast<i64>(b) * 2 * a.H + 2 * y + (d >> 1)) * (2 * a.W) + 2 * x + (d & 1);
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.up_skip + fp * N + cbase));
      }
    }
  }
  if (tid == 0) ok_load = mbar_wait(bar_load, 0, a.err, 1) ? 1 : 0;
  __syncthreads();
  const bool ok = ok_load != 0;
  if constexpr (FEAT) {
    // channel 0 of every halo pixel, over the tile copy's (zero) channel 0
    if (ok) {
#pragma unroll
      for (int k = 0; k < kFeatPer; ++k) {
        const int idx = tid + k * kConvThreads * CS;
        if (idx < kHalo) {
          const int t = idx / (kHaloH * kHaloW), h = idx % (kHaloH * kHaloW);
          *reinterpret_cast<bf16*>(planes + t * S::kPlanes * kPlaneStride + h * 16) = __float2bfloat16_rn(feat[k]);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
    }
    __syncthreads();
  }

  float v[NC];
  if constexpr (TC) {
    uint32_t tmem = 0;
    tc_fence_after();
    tmem = *tmem_slot;
    bool mma_ok = ok;
    if (tid == 0 && ok) {
#pragma unroll
      for (int t = 0; t < TM; ++t)
        conv_issue_mma<CIN, N>(smem_u32(planes) + t * S::kPlanes * kPlaneStride, smem_u32(wsm), tmem + t * N);
      umma_commit(bar_mma);
    }
    __syncthreads();
    if (ok) mma_ok = mbar_wait(bar_mma, 0, a.err, 2);
    mma_ok = __syncthreads_and(mma_ok ? 1 : 0) != 0;
    tc_fence_after();
    // warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31
    const uint32_t row = tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16);
#pragma unroll 1
    for (int t = 0; t < TM && mma_ok; ++t) {
#pragma unroll
      for (int c = 0; c < NC / 16; ++c) {
        float u[16];
        tmem_ld16(row + t * N + cbase + c * 16, u);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j) v[c * 16 + j] = u[j];
      }
      if (t + 1 < TM) {  // the earlier tiles' epilogues; the last one runs below
        if (a.bias) {
#pragma unroll
          for (int j = 0; j < NC; ++j) v[j] += s_bias[cbase + j];
        }
        conv_epilogue<N, UP, NC>(a, b, y0 + (px >> 3), x0 + t * kTileW + (px & 7), v, cbase);
      }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kCols);
    if (!mma_ok) return;
  } else {
    if (!ok) return;
    // warp w: tile rows 4w..4w+3 as two m16 tiles; all N / 8 n tiles
    float acc[2][N / 8][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < N / 8; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.0f;
    const uint32_t pbase = smem_u32(planes), wbase = smem_u32(wsm);
    const int r = lane & 15, half = lane >> 4;
#pragma unroll 1
    for (int s = 0; s < S::kKC / 2; ++s) {
      const int kc = 2 * s + half;  // this lane's K half
      uint32_t abase;
      if constexpr (CIN == 8) {
        const int t = kc < 9 ? kc : 8;
        abase = pbase + ((t / 3) * kHaloW + t % 3) * 16;
      } else {
        constexpr int P = CIN / 8;
        const int t = kc / P, c = kc % P;
        abase = pbase + c * kPlaneStride + ((t / 3) * kHaloW + t % 3) * 16;
      }
      uint32_t af[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int ty = 4 * warp + 2 * mt + (r >> 3), tx = r & 7;
        ldsm_x4(abase + (ty * kHaloW + tx) * 16, af[mt]);
      }
#pragma unroll
      for (int nt = 0; nt < N / 8; ++nt) {
        uint32_t bf[2];
        // lanes 0-7: rows of chunk 2s, lanes 8-15: rows of chunk 2s+1
        const int l = lane & 15;
        ldsm_x2(wbase + ((2 * s + (l >> 3)) * (N / 8) + nt) * 128 + (l & 7) * 16, bf);
        mma16816(acc[0][nt], af[0], bf);
        mma16816(acc[1][nt], af[1], bf);
      }
    }
    float* stage = reinterpret_cast<float*>(smem + S::kStage);
    constexpr int LD = N + 4;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < N / 8; ++nt) {
        const int m = 32 * warp + 16 * mt + (lane >> 2), n = nt * 8 + 2 * (lane & 3);
        stage[m * LD + n] = acc[mt][nt][0];
        stage[m * LD + n + 1] = acc[mt][nt][1];
        stage[(m + 8) * LD + n] = acc[mt][nt][2];
        stage[(m + 8) * LD + n + 1] = acc[mt][nt][3];
      }
    __syncthreads();
#pragma unroll
    for (int n = 0; n < N; ++n) v[n] = stage[tid * LD + n];
  }
  if (a.bias) {
#pragma unroll
    for (int j = 0; j < NC; ++j) v[j] += s_bias[cbase + j];
  }
  conv_epilogue<N, UP, NC>(a, b, y0 + (px >> 3), x0 + (TM - 1) * kTileW + (px & 7), v, cbase);
}

// ------------------------------------------------------------------
// Weight gradient: dW[co][t][ci] = sum_p G[p][co] X[p + off_t][ci],
// db[co] = sum_p G[p][co].  Grid: (ctas per tap, 9 taps); each CTA walks
// tiles blockIdx.x, + gridDim.x, ... accumulating in registers with
// mma.sync (M = co, N = ci, K = 16 pixels), then writes its partial.
// ------------------------------------------------------------------
struct WgradArgs {
  int B, H, W, ntiles_x, ntiles_y;
  float* part;   // [9][gridDim.x][CO][CI]
  float* bpart;  // [gridDim.x][CO] (written by the tap-0 CTAs)
  int* err;
};

template <int CI, int CO>
__global__ void __launch_bounds__(kConvThreads) wgrad_kernel(const __grid_constant__ CUtensorMap x_map,
                                                             const __grid_constant__ CUtensorMap g_map,
                                                             WgradArgs a) {
  constexpr int XP = CI / 8, GP = CO / 8;
  constexpr int NT = CI / 8, MT = CO / 16;
  constexpr int NTW = (NT + 3) / 4;  // n tiles per warp
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* xs = smem;
  unsigned char* gs = smem + XP * kPlaneStride;
  uint64_t* bar = reinterpret_cast<uint64_t*>(gs + GP * kGPlaneBytes);
  __shared__ int ok_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tap = blockIdx.y, dy = tap / 3, dx = tap % 3;
  float acc[MT][NTW][4];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NTW; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.0f;
  float bacc = 0.0f;
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  const int ntiles = a.ntiles_x * a.ntiles_y * a.B;
  unsigned phase = 0;
  bool alive = true;
  for (int tile = blockIdx.x; tile < ntiles && alive; tile += gridDim.x) {
    const int tx = tile % a.ntiles_x, ty = (tile / a.ntiles_x) % a.ntiles_y, b = tile / (a.ntiles_x * a.ntiles_y);
    const int x0 = tx * kTileW, y0 = ty * kTileH;
    __syncthreads();  // previous tile's planes are consumed
    if (tid == 0) {
      mbar_expect_tx(bar, XP * kPlaneBytes + GP * kGPlaneBytes);
      for (int c = 0; c < XP; ++c) tma_load_4d(xs + c * kPlaneStride, &x_map, c * 8, x0 - 1, y0 - 1, b, bar);
      for (int c = 0; c < GP; ++c) tma_load_4d(gs + c * kGPlaneBytes, &g_map, c * 8, x0, y0, b, bar);
      ok_s = mbar_wait(bar, phase, a.err, 3) ? 1 : 0;
    }
    __syncthreads();
    phase ^= 1u;
    if (!ok_s) {
      alive = false;
      break;
    }
    const uint32_t xb = smem_u32(xs), gb = smem_u32(gs);
#pragma unroll 1
    for (int s = 0; s < kTileH / 2; ++s) {
      // K step: tile rows 2s, 2s+1 (16 pixels)
      const int j = lane & 15;  // pixel of the step this lane addresses
      const int py = 2 * s + (j >> 3), px = j & 7;
      uint32_t af[MT][4];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        // matrices: (co 0-7, k 0-7), (co 8-15, k 0-7), (co 0-7, k 8-15), (co 8-15, k 8-15)
        const int q = lane >> 3;  // which 8x8 matrix this lane addresses
        const int kpix = (q >> 1) * 8 + (lane & 7);
        const int cyy = 2 * s + (kpix >> 3), cxx = kpix & 7;
        const int cchunk = 2 * mt + (q & 1);
        ldsm_x4_t(gb + cchunk * kGPlaneBytes + (cyy * kTileW + cxx) * 16, af[mt]);
      }
#pragma unroll
      for (int jn = 0; jn < NTW; ++jn) {
        const int nt = warp + 4 * jn;
        if (nt < NT) {
          uint32_t bfr[2];
          ldsm_x2_t(xb + nt * kPlaneStride + ((py + dy) * kHaloW + px + dx) * 16, bfr);
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) mma16816(acc[mt][jn], af[mt], bfr);
        }
      }
    }
    if (tap == 0 && tid < CO) {
      const bf16* gsh = reinterpret_cast<const bf16*>(gs + (tid / 8) * kGPlaneBytes);
      for (int pix = 0; pix < kTileH * kTileW; ++pix) bacc += __bfloat162float(gsh[pix * 8 + (tid & 7)]);
    }
  }
  float* part = a.part + (static_cast<size_t>(tap) * gridDim.x + blockIdx.x) * CO * CI;
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int jn = 0; jn < NTW; ++jn) {
      const int nt = warp + 4 * jn;
      if (nt < NT) {
        const int co = mt * 16 + (lane >> 2), ci = nt * 8 + 2 * (lane & 3);
        part[co * CI + ci] = acc[mt][jn][0];
        part[co * CI + ci + 1] = acc[mt][jn][1];
        part[(co + 8) * CI + ci] = acc[mt][jn][2];
        part[(co + 8) * CI + ci + 1] = acc[mt][jn][3];
      }
    }
  if (tap == 0 && tid < CO) a.bpart[static_cast<size_t>(blockIdx.x) * CO + tid] = bacc;
}

// grad[w_off + (co * 9 + t) * CI + ci] = sum_k part[t][k][co][ci] (k in
// order); grad[b_off + co] = sum_k bpart[k][co]; co < cout_true only.
__global__ void wgrad_reduce_kernel(const float* part, const float* bpart, int nctas, int CO, int CI, int cout_true,
                                    float* grad_w, float* grad_b) {
  const int total = 9 * cout_true * CI;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total + cout_true; i += gridDim.x * blockDim.x) {
    if (i < total) {
      const int ci = i % CI, t = (i / CI) % 9, co = i / (CI * 9);
      float s = 0.0f;
      for (int k = 0; k < nctas; ++k) s += part[((static_cast<size_t>(t) * nctas + k) * CO + co) * CI + ci];
      grad_w[i] = s;
    } else {
      const int co = i - total;
      float s = 0.0f;
      for (int k = 0; k < nctas; ++k) s += bpart[static_cast<size_t>(k) * CO + co];
      grad_b[co] = s;
    }
  }
}

// ------------------------------------------------------------------
// Element-wise kernels over NHWC BF16 tensors (8 channels per thread)
// ------------------------------------------------------------------
// g[B][H/2][W/2][C] = (act > 0) ? sum of the 4 fine gradients : 0
__global__ void upadd_bwd_kernel(int B, int H, int W, int C, const bf16* dfine, const bf16* act, bf16* g) {
  const int h = H / 2, w = W / 2, cc = C / 8;
  const i64 total = static_cast<i64>(B) * h * w * cc;
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<i64>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(i % cc);
    const i64 pix = i / cc;
    const int x = static_cast<int>(pix % w), y = static_cast<int>((pix / w) % h), b = static_cast<int>(pix / (static_cast<i64>(w) * h));
    const uint4* src = reinterpret_cast<const uint4*>(dfine);
    const i64 base = ((static_cast<i64>(b) * H + 2 * y) * W + 2 * x) * cc + c;
    float p00[8], p01[8], p10[8], p11[8], m[8], o[8];
    unpack8(src[base], p00);
    unpack8(src[base + cc], p01);
    unpack8(src[base + static_cast<i64>(W) * cc], p10);
    unpack8(src[base + static_cast<i64>(W) * cc + cc], p11);
    unpack8(reinterpret_cast<const uint4*>(act)[i], m);
#pragma unroll
    for (int j = 0; j < 8; ++j) o[j] = m[j] > 0.0f ? (p00[j] + p01[j]) + (p10[j] + p11[j]) : 0.0f;
    reinterpret_cast<uint4*>(g)[i] = pack8(o);
  }
}

// g[B][H][W][C] = (act > 0) ? dskip + 0.25 up(dpool) : 0
__global__ void pool_bwd_kernel(int B, int H, int W, int C, const bf16* dskip, const bf16* dpool, const bf16* act,
                                bf16* g) {
  const int cc = C / 8, h = H / 2, w = W / 2;
  const i64 total = static_cast<i64>(B) * H * W * cc;
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<i64>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(i % cc);
    const i64 pix = i / cc;
    const int x = static_cast<int>(pix % W), y = static_cast<int>((pix / W) % H), b = static_cast<int>(pix / (static_cast<i64>(W) * H));
    float s[8], d[8], m[8], o[8];
    unpack8(reinterpret_cast<const uint4*>(dskip)[i], s);
    unpack8(reinterpret_cast<const uint4*>(dpool)[((static_cast<i64>(b) * h + y / 2) * w + x / 2) * cc + c], d);
    unpack8(reinterpret_cast<const uint4*>(act)[i], m);
#pragma unroll
    for (int j = 0; j < 8; ++j) o[j] = m[j] > 0.0f ? s[j] + 0.25f * d[j] : 0.0f;
    reinterpret_cast<uint4*>(g)[i] = pack8(o);
  }
}

// ------------------------------------------------------------------
// Features, scales, loss
// ------------------------------------------------------------------
// Source of sample b's residual: vector r (apply: double) or pair idx[b]
// of the training set (float).
struct SampleSrc {
  const double* v64;     // apply: the FGMRES vector (one sample)
  const float* R;        // training: residuals [npairs][P]
  const float* E;        // training: errors [npairs][P]
  const int* idx;        // training: pair of each sample
  const int* pair_inst;  // training: instance of each pair
  const float* coef;     // [ninst][6][P] (apply: one instance)
  i64 P;
  __device__ double r(int b, i64 p) const {
    if (v64) return v64[p];
    return static_cast<double>(R[static_cast<i64>(idx[b]) * P + p]);
  }
  __device__ double e(int b, i64 p) const { return static_cast<double>(E[static_cast<i64>(idx[b]) * P + p]); }
  __device__ const float* planes(int b) const {
    if (v64) return coef;
    return coef + static_cast<i64>(pair_inst[idx[b]]) * 6 * P;
  }
};

constexpr int kRedBlocks = 256;  // CTAs per sample of the per-sample reductions

// s[b] = sqrt(mean((r * invd)^2)); grid (kRedBlocks, B), block kThreads.
__global__ void __launch_bounds__(kThreads) scale_kernel(SampleSrc src, double* partial, unsigned* counter,
                                                         double* s) {
  const int b = blockIdx.y;
  const float* cf = src.planes(b);
  double acc[1] = {0.0};
  const i64 stride = static_cast<i64>(gridDim.x) * blockDim.x;
  i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  for (; p + 3 * stride < src.P; p += 4 * stride) {  // 4 independent loads in flight
    double rt[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) rt[u] = src.r(b, p + u * stride) * static_cast<double>(cf[5 * src.P + p + u * stride]);
#pragma unroll
    for (int u = 0; u < 4; ++u) acc[0] += rt[u] * rt[u];
  }
  for (; p < src.P; p += stride) {
    const double rt = src.r(b, p) * static_cast<double>(cf[5 * src.P + p]);
    acc[0] += rt * rt;
  }
  block_reduce<1>(acc);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partial[b * kRedBlocks + blockIdx.x] = acc[0];
    __threadfence();
    last = atomicAdd(counter + b, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {  // the last CTA sums the partials with all its threads (a fixed tree)
    __threadfence();
    double t[1] = {0.0};
    for (int k = threadIdx.x; k < static_cast<int>(gridDim.x); k += blockDim.x)
      t[0] += __ldcg(partial + b * kRedBlocks + k);
    block_reduce<1>(t);
    if (threadIdx.x == 0) {
      s[b] = sqrt(t[0] / static_cast<double>(src.P));
      counter[b] = 0u;
    }
  }
}

// x[b][p][0..7] (BF16): rt / s, w/d, e/d, s/d, n/d, 0, 0, 0
__global__ void features_kernel(SampleSrc src, int B, const double* s, bf16* x) {
  const i64 total = static_cast<i64>(B) * src.P;
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<i64>(gridDim.x) * blockDim.x) {
    const int b = static_cast<int>(i / src.P);
    const i64 p = i % src.P;
    const float* cf = src.planes(b);
    const float inv = cf[5 * src.P + p];
    const double sb = s[b];
    float f[8];
    f[0] = sb > 0.0 ? static_cast<float>(src.r(b, p) * static_cast<double>(inv) / sb) : 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) f[1 + k] = __fmul_rn(cf[(1 + k) * src.P + p], inv);
    f[5] = f[6] = f[7] = 0.0f;
    reinterpret_cast<uint4*>(x)[i] = pack8(f);
  }
}

// x[p][0..7] (BF16) of one instance: 0, w/d, e/d, s/d, n/d, 0, 0, 0 -- the
// features that do not depend on the vector (features_kernel's channels
// 1-4, bit for bit); the first convolution of an apply fills channel 0.
__global__ void fixed_features_kernel(const float* cf, i64 P, bf16* x) {
  for (i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; p < P;
       p += static_cast<i64>(gridDim.x) * blockDim.x) {
    const float inv = cf[5 * P + p];
    float f[8];
    f[0] = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) f[1 + k] = __fmul_rn(cf[(1 + k) * P + p], inv);
    f[5] = f[6] = f[7] = 0.0f;
    reinterpret_cast<uint4*>(x)[p] = pack8(f);
  }
}

struct LossArgs {
  SampleSrc src;
  int B, H, W;
  const double* s;
  const float* y;    // network output [B][P]
  float* rho;        // [B][P]
  double* partial;   // [B][kRedBlocks][4]
  unsigned* counter; // [B]
  double* wts;       // [B][3]: wr, wt, loss_b
  double mu;
  bf16* g8;          // [B][P][16]
  double* loss_out;  // mean loss (written by loss2's first thread)
};

__device__ __forceinline__ float loss_dif(LossArgs const& a, int b, i64 p) {
  const double sb = a.s[b];
  const float tg = sb > 0.0 ? static_cast<float>(a.src.e(b, p) / sb) : 0.0f;
  return a.y[static_cast<i64>(b) * a.src.P + p] - tg;
}

// rho = A (y - tgt), and per sample |rho|^2, |r/s|^2, |tgt|^2, |dif|^2
__global__ void __launch_bounds__(kThreads) loss1_kernel(LossArgs a) {
  const int b = blockIdx.y;
  const i64 P = a.src.P;
  const float* cf = a.src.planes(b);
  const double sb = a.s[b];
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; p < P;
       p += static_cast<i64>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(p % a.W), y = static_cast<int>(p / a.W);
    const float dp = loss_dif(a, b, p);
    float v = __fmul_rn(cf[p], dp);
    if (x > 0) v = __fadd_rn(v, __fmul_rn(cf[P + p], loss_dif(a, b, p - 1)));
    if (x + 1 < a.W) v = __fadd_rn(v, __fmul_rn(cf[2 * P + p], loss_dif(a, b, p + 1)));
    if (y > 0) v = __fadd_rn(v, __fmul_rn(cf[3 * P + p], loss_dif(a, b, p - a.W)));
    if (y + 1 < a.H) v = __fadd_rn(v, __fmul_rn(cf[4 * P + p], loss_dif(a, b, p + a.W)));
    a.rho[static_cast<i64>(b) * P + p] = v;
    const double rs = sb > 0.0 ? a.src.r(b, p) / sb : 0.0;
    const float tg = sb > 0.0 ? static_cast<float>(a.src.e(b, p) / sb) : 0.0f;
    acc[0] += static_cast<double>(v) * v;
    acc[1] += rs * rs;
    acc[2] += static_cast<double>(tg) * tg;
    acc[3] += static_cast<double>(dp) * dp;
  }
  block_reduce<4>(acc);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    for (int j = 0; j < 4; ++j) a.partial[(b * kRedBlocks + blockIdx.x) * 4 + j] = acc[j];
    __threadfence();
    last = atomicAdd(a.counter + b, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < static_cast<int>(gridDim.x); ++k)
      for (int j = 0; j < 4; ++j) t[j] += __ldcg(a.partial + (b * kRedBlocks + k) * 4 + j);
    const double wr = t[1] > 0.0 ? 1.0 / t[1] : 0.0;
    const double wt = t[2] > 0.0 ? a.mu / t[2] : 0.0;
    a.wts[b * 3 + 0] = wr;
    a.wts[b * 3 + 1] = wt;
    a.wts[b * 3 + 2] = t[0] * wr + t[3] * wt;
    a.counter[b] = 0u;
  }
}

// g8[b][p][0] = (2/B) (A^T rho * wr + dif * wt), channels 1..15 zero;
// the first thread also writes the mean loss.
__global__ void loss2_kernel(LossArgs a) {
  const i64 P = a.src.P;
  const i64 total = static_cast<i64>(a.B) * P;
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.loss_out) {
    double l = 0.0;
    for (int b = 0; b < a.B; ++b) l += a.wts[b * 3 + 2];
    *a.loss_out = l / a.B;
  }
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<i64>(gridDim.x) * blockDim.x) {
    const int b = static_cast<int>(i / P);
    const i64 p = i % P;
    const int x = static_cast<int>(p % a.W), y = static_cast<int>(p / a.W);
    const float* cf = a.src.planes(b);
    const float* rh = a.rho + static_cast<i64>(b) * P;
    float v = __fmul_rn(cf[p], rh[p]);
    if (x > 0) v = __fadd_rn(v, __fmul_rn(cf[2 * P + p - 1], rh[p - 1]));
    if (x + 1 < a.W) v = __fadd_rn(v, __fmul_rn(cf[P + p + 1], rh[p + 1]));
    if (y > 0) v = __fadd_rn(v, __fmul_rn(cf[4 * P + p - a.W], rh[p - a.W]));
    if (y + 1 < a.H) v = __fadd_rn(v, __fmul_rn(cf[3 * P + p + a.W], rh[p + a.W]));
    const double g = (2.0 / a.B) * (static_cast<double>(v) * a.wts[b * 3] + static_cast<double>(loss_dif(a, b, p)) * a.wts[b * 3 + 1]);
    float f[8] = {static_cast<float>(g), 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float z[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    uint4* dst = reinterpret_cast<uint4*>(a.g8 + i * 16);
    dst[0] = pack8(f);
    dst[1] = pack8(z);
  }
}

// ------------------------------------------------------------------
// Adam on the flat FP32 parameters, then the BF16 packed weights
// ------------------------------------------------------------------
__global__ void adam_kernel(i64 n, float* p, float* m, float* v, const float* g, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<i64>(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

struct PackLayer {
  int cin, cout, np;  // np: padded output channels of the forward conv
  long long w_off;    // FP32 weights W[cout][9][cin]
  bf16* fwd;          // kchunks(cin) x (np / 8) core matrices
  bf16* dgrad;        // flipped: conv of cout (padded np) channels to cin; null for layer 0
  int kcf, kcd;
};
struct PackTable {
  PackLayer l[kNL];
};

// Packed element (n, kc, j) at ((kc * (N / 8) + n / 8) * 8 + n % 8) * 8 + j
// of a conv with CIN input channels: chunk kc = t * (CIN / 8) + c holds
// input channels 8c..8c+7 of tap t (CIN = 8: chunk kc = tap kc).
__global__ void pack_kernel(const float* params, PackTable tab) {
  const PackLayer L = tab.l[blockIdx.y];
  // forward: N = np, CIN = cin
  const int nf = L.kcf * L.np * 8;
  const int nd = L.dgrad ? L.kcd * L.cin * 8 : 0;  // dgrad: N = cin (>= 16), CIN' = np
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf + nd; i += gridDim.x * blockDim.x) {
    if (i < nf) {
      const int j = i % 8, rown = (i / 8) % 8, grp = (i / 64) % (L.np / 8), kc = i / (64 * (L.np / 8));
      const int n = grp * 8 + rown;
      float w = 0.0f;
      const int P = L.cin / 8;
      const int t = L.cin == 8 ? kc : kc / P, c = L.cin == 8 ? 0 : kc % P;
      if (t < 9 && n < L.cout) w = params[L.w_off + (static_cast<long long>(n) * 9 + t) * L.cin + c * 8 + j];
      L.fwd[i] = __float2bfloat16_rn(w);
    } else {
      const int k = i - nf;
      const int j = k % 8, rown = (k / 8) % 8, grp = (k / 64) % (L.cin / 8), kc = k / (64 * (L.cin / 8));
      const int n = grp * 8 + rown;  // dgrad output channel = forward input channel
      // dgrad input channels = forward output channels (np of them, 8 per chunk)
      const int P = L.np / 8;
      const int t = kc / P, c = kc % P;
      const int co = c * 8 + j;
      float w = 0.0f;
      if (t < 9 && co < L.cout) w = params[L.w_off + (static_cast<long long>(co) * 9 + (8 - t)) * L.cin + n];
      L.dgrad[k] = __float2bfloat16_rn(w);
    }
  }
}

// ------------------------------------------------------------------
// Coefficient planes of a 5-point matrix on an nx x ny grid
// ------------------------------------------------------------------
// coef[0..5][p] = d, w, e, s, n (float of the entries, 0 when absent) and
// float(1 / d).  Rows with any other column, or a zero diagonal, set bad.
__global__ void planes_kernel(i64 n, int nx, const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ v, float* coef, unsigned* bad) {
  for (i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<i64>(gridDim.x) * blockDim.x) {
    float c[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    double d = 0.0;
    const int x = static_cast<int>(p % nx);
    bool ok = true;
    for (int k = rp[p]; k < rp[p + 1]; ++k) {
      const i64 off = ci[k] - p;
      const float fv = static_cast<float>(v[k]);
      if (off == 0) {
        c[0] = fv;
        d = v[k];
      } else if (off == -1 && x > 0) c[1] = fv;
      else if (off == 1 && x + 1 < nx) c[2] = fv;
      else if (off == -nx) c[3] = fv;
      else if (off == nx) c[4] = fv;
      else if (v[k] != 0.0) ok = false;
    }
    if (d == 0.0) ok = false;
    for (int k = 0; k < 5; ++k) coef[k * n + p] = c[k];
    coef[5 * n + p] = d != 0.0 ? static_cast<float>(1.0 / d) : 0.0f;
    if (!ok) atomicAdd(bad, 1u);
  }
}

// pairs: R[k][p] = float(r), E[k][p] = float(e)
__global__ void store_pair_kernel(i64 n, const double* r, const double* e, float* R, float* E) {
  for (i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<i64>(gridDim.x) * blockDim.x) {
    R[p] = static_cast<float>(r[p]);
    E[p] = static_cast<float>(e[p]);
  }
}

// r = b - A x (any handle through the SpMV epilogue is overkill here: a
// plain CSR row loop), e = xs - x
__global__ void resid_err_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci,
                                 const double* __restrict__ v, const double* b, const double* x, const double* xs,
                                 double* r, double* e) {
  for (i64 p = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<i64>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int k = rp[p]; k < rp[p + 1]; ++k) s += v[k] * x[ci[k]];
    r[p] = b[p] - s;
    e[p] = xs[p] - x[p];
  }
}

// ------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

// Raises a kernel's dynamic shared-memory limit once per (kernel, device).
template <class K>
static bool attr_once(K kernel, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
  std::lock_guard<std::mutex> g(mu);
  if (done.count(key)) return true;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) return false;
  done.insert(key);
  return true;
}

// 4-D map over a BF16 NHWC tensor [B][H][W][C], box {8, bw, bh, 1}.
static sk_status make_map(CUtensorMap* m, const void* base, int B, int H, int W, int C, int bw, int bh) {
  EncodeTiled enc = encode_fn();
  SK_CHECK(enc, SK_CUDA_ERROR, "cuTensorMapEncodeTiled is not available from the driver");
  SK_CHECK(C % 8 == 0 && (reinterpret_cast<uintptr_t>(base) & 15) == 0, SK_INVALID_ARG, "tensor map alignment");
  cuuint64_t dims[4] = {static_cast<cuuint64_t>(C), static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
                        static_cast<cuuint64_t>(B)};
  cuuint64_t strides[3] = {static_cast<cuuint64_t>(C) * 2, static_cast<cuuint64_t>(W) * C * 2,
                           static_cast<cuuint64_t>(H) * W * C * 2};
  cuuint32_t box[4] = {8, static_cast<cuuint32_t>(bw), static_cast<cuuint32_t>(bh), 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  SK_CHECK(r == CUDA_SUCCESS, SK_CUDA_ERROR, "cuTensorMapEncodeTiled failed");
  return SK_OK;
}

// Encoded maps by (address, shape, box), so that repeated applies encode
// nothing; the entries stay valid for as long as the buffer keeps its shape.
struct MapCache {
  std::map<std::array<long long, 7>, CUtensorMap> maps;
  sk_status get(const void* base, int B, int H, int W, int C, int bw, int bh, CUtensorMap* out) {
    const std::array<long long, 7> key{reinterpret_cast<long long>(base), B, H, W, C, bw, bh};
    auto it = maps.find(key);
    if (it != maps.end()) {
      *out = it->second;
      return SK_OK;
    }
    if (maps.size() > 512) maps.clear();
    sk_status s = make_map(out, base, B, H, W, C, bw, bh);
    if (s == SK_OK) maps.emplace(key, *out);
    return s;
  }
};

// More tiles than this many CTAs per SM could hold at once: the layers
// with 16 output channels take two tiles per CTA (one wave instead of two).
constexpr int kConvWaveCtas = 8 * 148;

template <int CIN, int N, bool TC>
static sk_status launch_conv(MapCache& mc, const void* in, ConvArgs const& a, cudaStream_t st) {
  CUtensorMap m;
  sk_status s = mc.get(in, a.B, a.H, a.W, CIN, kHaloW, kHaloH, &m);
  if (s != SK_OK) return s;
  const int ntiles = ceil_div(a.W, kTileW) * ceil_div(a.H, kTileH) * a.B;
  int tm = 1, cs = 1;
  auto kernel = a.up_out ? conv3x3_kernel<CIN, N, TC, true> : conv3x3_kernel<CIN, N, TC, false>;
  int bytes = ConvSmem<CIN, N, TC>::kBytes;
  if constexpr (TC && N == 16) {
    if (!a.up_out && ntiles > kConvWaveCtas) {
      tm = 2;
      kernel = conv3x3_kernel<CIN, N, TC, false, 2>;
      bytes = ConvSmem<CIN, N, TC, 2>::kBytes;
    }
  }
  if constexpr (TC && N >= 32) {  // the upsample-and-add epilogue split over two threads per pixel
    if (a.up_out) {
      cs = 2;
      kernel = conv3x3_kernel<CIN, N, TC, true, 1, 2>;
    }
  }
  if (a.feat_v) {
    if constexpr (TC && CIN == 8 && N == 16) {
      SK_CHECK(a.B == 1 && !a.up_out, SK_INVALID_ARG, "fused features take one sample");
      kernel = tm == 2 ? conv3x3_kernel<CIN, N, TC, false, 2, 1, true> : conv3x3_kernel<CIN, N, TC, false, 1, 1, true>;
    } else {
      return fail(SK_NOT_SUPPORTED, "fused features only in the first layer on the tcgen05 path");
    }
  }
  if (!attr_once(kernel, bytes)) return fail(SK_CUDA_ERROR, "cudaFuncSetAttribute");
  // programmatic dependent launch: the set-up of this layer's CTAs (barrier
  // init, tensor-memory allocation) overlaps the tail of the previous one
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  const int ntx = ceil_div(a.W, kTileW * tm), nty = ceil_div(a.H, kTileH);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(ntx, nty, a.B);
  cfg.blockDim = dim3(kConvThreads * cs);
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  SK_CUDA(cudaLaunchKernelEx(&cfg, kernel, m, a));
  return SK_OK;
}

template <bool TC>
static sk_status conv_dispatch(MapCache& mc, int cin, int n, const void* in, ConvArgs const& a, cudaStream_t st) {
#define SK_CONV_CASE(CI, NN) \
  if (cin == CI && n == NN) return launch_conv<CI, NN, TC>(mc, in, a, st);
  SK_CONV_CASE(8, 16)
  SK_CONV_CASE(16, 16)
  SK_CONV_CASE(16, 32)
  SK_CONV_CASE(32, 16)
  SK_CONV_CASE(32, 64)
  SK_CONV_CASE(64, 32)
  SK_CONV_CASE(64, 64)
#undef SK_CONV_CASE
  return fail(SK_NOT_SUPPORTED, "no convolution instance for these channel counts");
}

template <int CI, int CO>
static sk_status launch_wgrad(MapCache& mc, const void* x, const void* g, WgradArgs a, int nctas, cudaStream_t st) {
  CUtensorMap xm, gm;
  sk_status s = mc.get(x, a.B, a.H, a.W, CI, kHaloW, kHaloH, &xm);
  if (s != SK_OK) return s;
  if ((s = mc.get(g, a.B, a.H, a.W, CO, kTileW, kTileH, &gm)) != SK_OK) return s;
  const int bytes = (CI / 8) * kPlaneStride + (CO / 8) * kGPlaneBytes + 64;
  if (!attr_once(wgrad_kernel<CI, CO>, bytes)) return fail(SK_CUDA_ERROR, "cudaFuncSetAttribute");
  SK_LAUNCH((wgrad_kernel<CI, CO>), dim3(nctas, 9), kConvThreads, bytes, st, xm, gm, a);
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

static sk_status wgrad_dispatch(MapCache& mc, int ci, int co, const void* x, const void* g, WgradArgs a,
                                int nctas, cudaStream_t st) {
#define SK_WG_CASE(CI, CO) \
  if (ci == CI && co == CO) return launch_wgrad<CI, CO>(mc, x, g, a, nctas, st);
  SK_WG_CASE(8, 16)
  SK_WG_CASE(16, 32)
  SK_WG_CASE(32, 64)
  SK_WG_CASE(64, 64)
  SK_WG_CASE(64, 32)
  SK_WG_CASE(32, 16)
  SK_WG_CASE(16, 16)
#undef SK_WG_CASE
  return fail(SK_NOT_SUPPORTED, "no weight-gradient instance for these channel counts");
}

inline int ew_grid(i64 n) {
  i64 g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return static_cast<int>(g < 1 ? 1 : g);
}

}  // namespace sk

// ------------------------------------------------------------------
// Handles
// ------------------------------------------------------------------
using namespace sk;

struct sk_net_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  i64 np = 0;
  long long w_off[kNL], b_off[kNL];
  float* params = nullptr;  // FP32 master
  float* grad = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  bf16* wf[kNL] = {};
  bf16* wd[kNL] = {};
  long long step = 0;
  int legacy_mma = 0;  // cross-check hook: convolutions on mma.sync
  sk_status host_err = SK_OK;  // first failed apply inside a solver (sticky until read)
  MapCache maps;
  int* err = nullptr;
  // activation / gradient workspace for one (B, H, W)
  int B = 0, H = 0, W = 0;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  bf16 *x0, *e0, *p0, *e1, *p1, *e2, *p2, *e3, *b3, *u2, *d2, *u1, *d1, *u0, *d0;
  float* y;
  bf16 *g8, *g7, *du0, *g6, *du1, *g5, *du2, *g4, *g3, *dp2, *g2, *dp1, *g1, *dp0, *g0;
  float* rho;
  double *s, *red, *wts, *loss;
  unsigned* counter;
  float *part, *bpart;
  int wg_ctas = 0;
  std::vector<void*> allocs;
};

struct sk_pairs_s {
  int nx = 0, ny = 0;
  i64 P = 0, cap = 0, count = 0;
  int cap_inst = 0, ninst = 0;
  float* R = nullptr;
  float* E = nullptr;
  int* inst = nullptr;      // per pair
  float* coef = nullptr;    // [cap_inst][6][P]
  std::vector<int> inst_host;
  void* scratch = nullptr;  // harvest: r, e, x (doubles)
};

namespace sk {

static sk_status net_alloc(sk_net N, void** p, size_t bytes) {
  SK_CUDA(cudaMalloc(p, bytes));
  N->allocs.push_back(*p);
  return SK_OK;
}

// Carves the workspace of a (B, H, W) configuration (grow-only).
static sk_status net_workspace(sk_net N, int B, int H, int W) {
  if (N->B == B && N->H == H && N->W == W && N->ws) return SK_OK;
  SK_CHECK(H % 8 == 0 && W % 8 == 0 && H >= 8 && W >= 8, SK_INVALID_ARG, "grid sides must be multiples of 8");
  const size_t P0 = static_cast<size_t>(B) * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  struct Item { void** dst; size_t bytes; };
  const int ctas = 2 * 148;
  std::vector<Item> items = {
      {(void**)&N->x0, P0 * 8 * 2},   {(void**)&N->e0, P0 * 16 * 2}, {(void**)&N->p0, P1 * 16 * 2},
      {(void**)&N->e1, P1 * 32 * 2},  {(void**)&N->p1, P2 * 32 * 2}, {(void**)&N->e2, P2 * 64 * 2},
      {(void**)&N->p2, P3 * 64 * 2},  {(void**)&N->e3, P3 * 64 * 2}, {(void**)&N->b3, P3 * 64 * 2},
      {(void**)&N->u2, P2 * 64 * 2},  {(void**)&N->d2, P2 * 32 * 2}, {(void**)&N->u1, P1 * 32 * 2},
      {(void**)&N->d1, P1 * 16 * 2},  {(void**)&N->u0, P0 * 16 * 2}, {(void**)&N->d0, P0 * 16 * 2},
      {(void**)&N->y, P0 * 4},        {(void**)&N->g8, P0 * 16 * 2}, {(void**)&N->g7, P0 * 16 * 2},
      {(void**)&N->du0, P0 * 16 * 2}, {(void**)&N->g6, P1 * 16 * 2}, {(void**)&N->du1, P1 * 32 * 2},
      {(void**)&N->g5, P2 * 32 * 2},  {(void**)&N->du2, P2 * 64 * 2}, {(void**)&N->g4, P3 * 64 * 2},
      {(void**)&N->g3, P3 * 64 * 2},  {(void**)&N->dp2, P3 * 64 * 2}, {(void**)&N->g2, P2 * 64 * 2},
      {(void**)&N->dp1, P2 * 32 * 2}, {(void**)&N->g1, P1 * 32 * 2}, {(void**)&N->dp0, P1 * 16 * 2},
      {(void**)&N->g0, P0 * 16 * 2},  {(void**)&N->rho, P0 * 4},     {(void**)&N->s, static_cast<size_t>(B) * 8},
      {(void**)&N->red, static_cast<size_t>(B) * kRedBlocks * 4 * 8},
      {(void**)&N->wts, static_cast<size_t>(B) * 3 * 8},              {(void**)&N->loss, 8},
      {(void**)&N->counter, static_cast<size_t>(B) * 4},
      {(void**)&N->part, static_cast<size_t>(9) * ctas * 64 * 64 * 4},
      {(void**)&N->bpart, static_cast<size_t>(ctas) * 64 * 4}};
  size_t total = 0;
  for (auto& it : items) total += (it.bytes + 255) & ~size_t(255);
  if (total > N->ws_bytes) {
    if (N->ws) {
      cudaStreamSynchronize(N->stream);
      cudaFree(N->ws);
      N->ws = nullptr;
    }
    SK_CUDA(cudaMalloc(&N->ws, total));
    N->ws_bytes = total;
  }
  char* p = static_cast<char*>(N->ws);
  for (auto& it : items) {
    *it.dst = p;
    p += (it.bytes + 255) & ~size_t(255);
  }
  SK_CUDA(cudaMemsetAsync(N->counter, 0, static_cast<size_t>(B) * 4, N->stream));
  SK_CUDA(cudaMemsetAsync(N->ws, 0, total, N->stream));
  N->B = B;
  N->H = H;
  N->W = W;
  N->wg_ctas = ctas;
  return SK_OK;
}

static sk_status net_pack(sk_net N) {
  PackTable tab{};
  for (int l = 0; l < kNL; ++l) {
    PackLayer& L = tab.l[l];
    L.cin = kCin[l];
    L.cout = kCout[l];
    L.np = pad_n(kCout[l]);
    L.w_off = N->w_off[l];
    L.fwd = N->wf[l];
    L.dgrad = l > 0 ? N->wd[l] : nullptr;
    L.kcf = kchunks(L.cin);
    L.kcd = kchunks(L.np);
  }
  SK_LAUNCH(pack_kernel, dim3(32, kNL), 256, 0, N->stream, N->params, tab);
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

static const float* bias_of(sk_net N, int l) { return N->params + N->b_off[l]; }

template <bool TC>
static sk_status conv_fwd(sk_net N, int l, const bf16* in, int H, int W, ConvArgs a) {
  a.B = N->B;
  a.H = H;
  a.W = W;
  a.wpk = N->wf[l];
  a.bias = bias_of(N, l);
  a.err = N->err;
  return conv_dispatch<TC>(N->maps, kCin[l], pad_n(kCout[l]), in, a, N->stream);
}

static sk_status run_conv(sk_net N, int l, const bf16* in, int H, int W, ConvArgs a) {
  return N->legacy_mma ? conv_fwd<false>(N, l, in, H, W, a) : conv_fwd<true>(N, l, in, H, W, a);
}

// input gradient of layer l (a conv from pad_n(cout) to cin channels),
// masked by `mask` (the activation feeding layer l) when non-null
static sk_status run_dgrad(sk_net N, int l, const bf16* g, int H, int W, bf16* out, const bf16* mask) {
  ConvArgs a{};
  a.B = N->B;
  a.H = H;
  a.W = W;
  a.wpk = N->wd[l];
  a.bias = nullptr;
  a.relu = 0;
  a.mask = mask;
  a.out_kind = OUT_BF16;
  a.out = out;
  a.err = N->err;
  const int cin = pad_n(kCout[l]);
  return N->legacy_mma ? conv_dispatch<false>(N->maps, cin, kCin[l], g, a, N->stream)
                       : conv_dispatch<true>(N->maps, cin, kCin[l], g, a, N->stream);
}

static sk_status run_wgrad(sk_net N, int l, const bf16* x, const bf16* g, int H, int W) {
  WgradArgs a{};
  a.B = N->B;
  a.H = H;
  a.W = W;
  a.ntiles_x = ceil_div(W, kTileW);
  a.ntiles_y = ceil_div(H, kTileH);
  a.part = N->part;
  a.bpart = N->bpart;
  a.err = N->err;
  const int ntiles = a.ntiles_x * a.ntiles_y * a.B;
  const int nctas = std::min(N->wg_ctas / 9 + 1, ntiles);
  const int co = pad_n(kCout[l]);
  sk_status s = wgrad_dispatch(N->maps, kCin[l], co, x, g, a, nctas, N->stream);
  if (s != SK_OK) return s;
  const int total = 9 * kCout[l] * kCin[l] + kCout[l];
  SK_LAUNCH(wgrad_reduce_kernel, ceil_div(total, 256), 256, 0, N->stream, N->part, N->bpart, nctas, co, kCin[l],
            kCout[l], N->grad + N->w_off[l], N->grad + N->b_off[l]);
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

// Forward pass from N->x0; the last layer writes per `last`.  Pooling and
// the upsample-and-add of the skip connections run in the epilogues of the
// convolutions that produce their inputs.
static sk_status net_forward(sk_net N, ConvArgs last, const bf16* xin = nullptr, const ConvArgs* feat = nullptr) {
  const int H = N->H, W = N->W, H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  sk_status s;
  auto fwd = [&](int l, const bf16* in, int h, int w, bf16* out, bf16* pool, const bf16* skip, bf16* up) {
    ConvArgs a{};
    a.relu = 1;
    a.out_kind = OUT_BF16;
    a.out = out;
    a.pool_out = pool;
    a.up_skip = skip;
    a.up_out = up;
    if (l == 0 && feat) {
      a.feat_v = feat->feat_v;
      a.feat_inv = feat->feat_inv;
      a.feat_s = feat->feat_s;
    }
    return run_conv(N, l, in, h, w, a);
  };
  if ((s = fwd(0, xin ? xin : N->x0, H, W, N->e0, N->p0, nullptr, nullptr)) != SK_OK) return s;
  if ((s = fwd(1, N->p0, H1, W1, N->e1, N->p1, nullptr, nullptr)) != SK_OK) return s;
  if ((s = fwd(2, N->p1, H2, W2, N->e2, N->p2, nullptr, nullptr)) != SK_OK) return s;
  if ((s = fwd(3, N->p2, H3, W3, N->e3, nullptr, nullptr, nullptr)) != SK_OK) return s;
  if ((s = fwd(4, N->e3, H3, W3, N->b3, nullptr, N->e2, N->u2)) != SK_OK) return s;
  if ((s = fwd(5, N->u2, H2, W2, N->d2, nullptr, N->e1, N->u1)) != SK_OK) return s;
  if ((s = fwd(6, N->u1, H1, W1, N->d1, nullptr, N->e0, N->u0)) != SK_OK) return s;
  if ((s = fwd(7, N->u0, H, W, N->d0, nullptr, nullptr, nullptr)) != SK_OK) return s;
  last.relu = 0;
  return run_conv(N, 8, N->d0, H, W, last);
}

static sk_status net_backward(sk_net N) {
  const int H = N->H, W = N->W, H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  const int B = N->B;
  cudaStream_t st = N->stream;
  sk_status s;
  if ((s = run_wgrad(N, 8, N->d0, N->g8, H, W)) != SK_OK) return s;
  if ((s = run_dgrad(N, 8, N->g8, H, W, N->g7, N->d0)) != SK_OK) return s;
  if ((s = run_wgrad(N, 7, N->u0, N->g7, H, W)) != SK_OK) return s;
  if ((s = run_dgrad(N, 7, N->g7, H, W, N->du0, nullptr)) != SK_OK) return s;
  SK_LAUNCH(upadd_bwd_kernel, ew_grid(static_cast<i64>(B) * H1 * W1 * 2), 256, 0, st, B, H, W, 16, N->du0, N->d1,
            N->g6);
  if ((s = run_wgrad(N, 6, N->u1, N->g6, H1, W1)) != SK_OK) return s;
  if ((s = run_dgrad(N, 6, N->g6, H1, W1, N->du1, nullptr)) != SK_OK) return s;
  SK_LAUNCH(upadd_bwd_kernel, ew_grid(static_cast<i64>(B) * H2 * W2 * 4), 256, 0, st, B, H1, W1, 32, N->du1, N->d2,
            N->g5);
  if ((s = run_wgrad(N, 5, N->u2, N->g5, H2, W2)) != SK_OK) return s;
  if ((s = run_dgrad(N, 5, N->g5, H2, W2, N->du2, nullptr)) != SK_OK) return s;
  SK_LAUNCH(upadd_bwd_kernel, ew_grid(static_cast<i64>(B) * H3 * W3 * 8), 256, 0, st, B, H2, W2, 64, N->du2, N->b3,
            N->g4);
  if ((s = run_wgrad(N, 4, N->e3, N->g4, H3, W3)) != SK_OK) return s;
  if ((s = run_dgrad(N, 4, N->g4, H3, W3, N->g3, N->e3)) != SK_OK) return s;
  if ((s = run_wgrad(N, 3, N->p2, N->g3, H3, W3)) != SK_OK) return s;
  if ((s = run_dgrad(N, 3, N->g3, H3, W3, N->dp2, nullptr)) != SK_OK) return s;
  SK_LAUNCH(pool_bwd_kernel, ew_grid(static_cast<i64>(B) * H2 * W2 * 8), 256, 0, st, B, H2, W2, 64, N->du2, N->dp2,
            N->e2, N->g2);
  if ((s = run_wgrad(N, 2, N->p1, N->g2, H2, W2)) != SK_OK) return s;
  if ((s = run_dgrad(N, 2, N->g2, H2, W2, N->dp1, nullptr)) != SK_OK) return s;
  SK_LAUNCH(pool_bwd_kernel, ew_grid(static_cast<i64>(B) * H1 * W1 * 4), 256, 0, st, B, H1, W1, 32, N->du1, N->dp1,
            N->e1, N->g1);
  if ((s = run_wgrad(N, 1, N->p0, N->g1, H1, W1)) != SK_OK) return s;
  if ((s = run_dgrad(N, 1, N->g1, H1, W1, N->dp0, nullptr)) != SK_OK) return s;
  SK_LAUNCH(pool_bwd_kernel, ew_grid(static_cast<i64>(B) * H * W * 2), 256, 0, st, B, H, W, 16, N->du0, N->dp0,
            N->e0, N->g0);
  if ((s = run_wgrad(N, 0, N->x0, N->g0, H, W)) != SK_OK) return s;
  SK_CUDA(cudaGetLastError());
  return SK_OK;
}

static sk_status check_err(sk_net N) {
  int e = 0;
  SK_CUDA(cudaMemcpyAsync(&e, N->err, 4, cudaMemcpyDeviceToHost, N->stream));
  SK_CUDA(cudaStreamSynchronize(N->stream));
  if (e) {
    cudaMemsetAsync(N->err, 0, 4, N->stream);
    return fail(SK_TIMEOUT, "a network kernel gave up waiting on its tile copies or tensor-core work");
  }
  return SK_OK;
}

// features of a batch into N->x0 (and scales into N->s)
static void net_features(sk_net N, SampleSrc const& src, int B) {
  SK_LAUNCH(scale_kernel, dim3(kRedBlocks, B), kThreads, 0, N->stream, src, N->red, N->counter, N->s);
  SK_LAUNCH(features_kernel, ew_grid(static_cast<i64>(B) * src.P), 256, 0, N->stream, src, B, N->s, N->x0);
}

// loss and dL/dy of the batch whose forward pass is in N (y)
static void net_loss(sk_net N, SampleSrc const& src, double mu, double* loss_out) {
  LossArgs a{};
  a.src = src;
  a.B = N->B;
  a.H = N->H;
  a.W = N->W;
  a.s = N->s;
  a.y = N->y;
  a.rho = N->rho;
  a.partial = N->red;
  a.counter = N->counter;
  a.wts = N->wts;
  a.mu = mu;
  a.g8 = N->g8;
  a.loss_out = loss_out;
  SK_LAUNCH(loss1_kernel, dim3(kRedBlocks, N->B), kThreads, 0, N->stream, a);
  SK_LAUNCH(loss2_kernel, ew_grid(static_cast<i64>(N->B) * src.P), 256, 0, N->stream, a);
}

static SampleSrc pair_src(sk_pairs D, const int* idx_dev) {
  SampleSrc src{};
  src.R = D->R;
  src.E = D->E;
  src.idx = idx_dev;
  src.pair_inst = D->inst;
  src.coef = D->coef;
  src.P = D->P;
  return src;
}

// forward + loss + backward of pairs idx_dev[0..B) (gradient into N->grad)
static sk_status net_step_grad(sk_net N, sk_pairs D, const int* idx_dev, int B, double mu, double* loss_dev) {
  sk_status s = net_workspace(N, B, D->ny, D->nx);
  if (s != SK_OK) return s;
  SampleSrc src = pair_src(D, idx_dev);
  net_features(N, src, B);
  ConvArgs last{};
  last.out_kind = OUT_F32;
  last.outf = N->y;
  if ((s = net_forward(N, last)) != SK_OK) return s;
  net_loss(N, src, mu, loss_dev);
  return net_backward(N);
}

}  // namespace sk

// ------------------------------------------------------------------
// Learned preconditioner apply (precond kind 3), used by precond dispatch
// ------------------------------------------------------------------
namespace sk {

sk_status learned_apply(const sk_precond_s* M, const double* v, double* z, cudaStream_t st) {
  return learned_apply_ex(M, v, z, st, false, false);
}

double* learned_scale_slot(const sk_precond_s* M) {
  sk_net N = M->net;
  if (net_workspace(N, 1, static_cast<int>(M->grid_ny), static_cast<int>(M->grid_nx)) != SK_OK) return nullptr;
  return N->s;
}

// On the tcgen05 path the first convolution computes the scaled vector
// channel itself (the other input channels are the matrix's, fixed at
// creation), so an apply is the scale reduction and the nine convolutions.
sk_status learned_apply_ex(const sk_precond_s* M, const double* v, double* z, cudaStream_t st, bool add,
                           bool scale_ready) {
  sk_net N = M->net;
  N->stream = st;
  sk_status s = net_workspace(N, 1, static_cast<int>(M->grid_ny), static_cast<int>(M->grid_nx));
  if (s != SK_OK) return s;
  SampleSrc src{};
  src.v64 = v;
  src.coef = M->coef;
  src.P = M->n;
  if (!scale_ready)
    SK_LAUNCH(scale_kernel, dim3(kRedBlocks, 1), kThreads, 0, N->stream, src, N->red, N->counter, N->s);
  ConvArgs last{};
  last.out_kind = OUT_Z64;
  last.outz = z;
  last.scale = N->s;
  last.z_add = add ? 1 : 0;
  if (!N->legacy_mma && M->xfeat) {
    ConvArgs f{};
    f.feat_v = v;
    f.feat_inv = M->coef + 5 * M->n;
    f.feat_s = N->s;
    s = net_forward(N, last, static_cast<const bf16*>(M->xfeat), &f);
  } else {
    SK_LAUNCH(features_kernel, ew_grid(src.P), 256, 0, N->stream, src, 1, N->s, N->x0);
    s = net_forward(N, last);
  }
  if (s != SK_OK && N->host_err == SK_OK) N->host_err = s;
  return s;
}

template <bool TC>
static sk_status conv_attrs() {
  bool ok = true;
  auto both = [&](auto k_plain, auto k_up, int bytes) { ok = ok && attr_once(k_plain, bytes) && attr_once(k_up, bytes); };
#define SK_CONV_ATTR(CI, NN) \
  both(conv3x3_kernel<CI, NN, TC, false>, conv3x3_kernel<CI, NN, TC, true>, ConvSmem<CI, NN, TC>::kBytes);
  if constexpr (TC) {
    ok = ok && attr_once(conv3x3_kernel<8, 16, TC, false, 2>, ConvSmem<8, 16, TC, 2>::kBytes) &&
         attr_once(conv3x3_kernel<16, 16, TC, false, 2>, ConvSmem<16, 16, TC, 2>::kBytes) &&
         attr_once(conv3x3_kernel<32, 16, TC, false, 2>, ConvSmem<32, 16, TC, 2>::kBytes) &&
         attr_once(conv3x3_kernel<8, 16, TC, false, 1, 1, true>, ConvSmem<8, 16, TC>::kBytes) &&
         attr_once(conv3x3_kernel<8, 16, TC, false, 2, 1, true>, ConvSmem<8, 16, TC, 2>::kBytes);
#define SK_CONV_ATTR_CS(CI, NN) \
  ok = ok && attr_once(conv3x3_kernel<CI, NN, TC, true, 1, 2>, ConvSmem<CI, NN, TC>::kBytes);
    SK_CONV_ATTR_CS(16, 32)
    SK_CONV_ATTR_CS(32, 64)
    SK_CONV_ATTR_CS(64, 32)
    SK_CONV_ATTR_CS(64, 64)
#undef SK_CONV_ATTR_CS
  }
  SK_CONV_ATTR(8, 16)
  SK_CONV_ATTR(16, 16)
  SK_CONV_ATTR(16, 32)
  SK_CONV_ATTR(32, 16)
  SK_CONV_ATTR(32, 64)
  SK_CONV_ATTR(64, 32)
  SK_CONV_ATTR(64, 64)
#undef SK_CONV_ATTR
  return ok ? SK_OK : fail(SK_CUDA_ERROR, "cudaFuncSetAttribute");
}

sk_status learned_prepare(const sk_precond_s* M) {
  sk_net N = M->net;
  N->stream = nullptr;
  sk_status s = net_workspace(N, 1, static_cast<int>(M->grid_ny), static_cast<int>(M->grid_nx));
  if (s != SK_OK) return s;
  SK_CUDA(cudaStreamSynchronize(nullptr));
  return N->legacy_mma ? conv_attrs<false>() : conv_attrs<true>();
}

void learned_release(sk_precond_s* M) {
  if (M->coef) cudaFree(M->coef);
  M->coef = nullptr;
  if (M->xfeat) cudaFree(M->xfeat);
  M->xfeat = nullptr;
}

}  // namespace sk

// ------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------
extern "C" {

sk_status sk_net_create(sk_net* out, uint64_t seed) {
  SK_CHECK(out, SK_INVALID_ARG, "null output");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SK_NO_DEVICE, "no CUDA device");
  auto* N = new sk_net_s();
  cudaGetDevice(&N->device);
  long long off = 0;
  for (int l = 0; l < kNL; ++l) {
    N->w_off[l] = off;
    off += static_cast<long long>(kCout[l]) * 9 * kCin[l];
    N->b_off[l] = off;
    off += kCout[l];
  }
  N->np = off;
  sk_status s = SK_OK;
  auto bail = [&](sk_status st) {
    sk_net_destroy(N);
    return st;
  };
  for (float** p : {&N->params, &N->grad, &N->m, &N->v})
    if ((s = net_alloc(N, reinterpret_cast<void**>(p), N->np * 4 + 64)) != SK_OK) return bail(s);
  for (int l = 0; l < kNL; ++l) {
    const size_t fb = static_cast<size_t>(kchunks(kCin[l])) * pad_n(kCout[l]) * 8 * 2;
    if ((s = net_alloc(N, reinterpret_cast<void**>(&N->wf[l]), fb)) != SK_OK) return bail(s);
    if (l > 0) {
      const size_t db = static_cast<size_t>(kchunks(pad_n(kCout[l]))) * kCin[l] * 8 * 2;
      if ((s = net_alloc(N, reinterpret_cast<void**>(&N->wd[l]), db)) != SK_OK) return bail(s);
    }
  }
  if ((s = net_alloc(N, reinterpret_cast<void**>(&N->err), 16)) != SK_OK) return bail(s);
  // He initialisation (normal, std sqrt(2 / fan_in)), zero biases
  std::vector<float> h(N->np, 0.0f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  for (int l = 0; l < kNL; ++l) {
    const float sd = std::sqrt(2.0f / (9.0f * kCin[l]));
    for (long long i = 0; i < static_cast<long long>(kCout[l]) * 9 * kCin[l]; ++i) h[N->w_off[l] + i] = sd * nd(rng);
  }
  if (cudaMemcpy(N->params, h.data(), N->np * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(N->m, 0, N->np * 4) != cudaSuccess || cudaMemset(N->v, 0, N->np * 4) != cudaSuccess ||
      cudaMemset(N->grad, 0, N->np * 4) != cudaSuccess || cudaMemset(N->err, 0, 16) != cudaSuccess)
    return bail(fail(SK_CUDA_ERROR, "network initialisation copy failed"));
  if ((s = net_pack(N)) != SK_OK) return bail(s);
  if (cudaStreamSynchronize(N->stream) != cudaSuccess) return bail(fail(SK_CUDA_ERROR, "pack failed"));
  *out = N;
  return SK_OK;
}

sk_status sk_net_destroy(sk_net N) {
  if (!N) return SK_OK;
  cudaDeviceSynchronize();
  for (void* p : N->allocs) cudaFree(p);
  if (N->ws) cudaFree(N->ws);
  delete N;
  return SK_OK;
}

int64_t sk_net_param_count(void) {
  long long n = 0;
  for (int l = 0; l < kNL; ++l) n += static_cast<long long>(kCout[l]) * 9 * kCin[l] + kCout[l];
  return n;
}

sk_status sk_net_get_params(sk_net N, float* host, int64_t capacity) {
  SK_CHECK(N && host && capacity >= N->np, SK_INVALID_ARG, "null network or short buffer");
  SK_CUDA(cudaStreamSynchronize(N->stream));
  SK_CUDA(cudaMemcpy(host, N->params, N->np * 4, cudaMemcpyDeviceToHost));
  return SK_OK;
}

sk_status sk_net_set_params(sk_net N, const float* host, int64_t count) {
  SK_CHECK(N && host && count == N->np, SK_INVALID_ARG, "null network or wrong parameter count");
  SK_CUDA(cudaStreamSynchronize(N->stream));
  SK_CUDA(cudaMemcpy(N->params, host, N->np * 4, cudaMemcpyHostToDevice));
  SK_CUDA(cudaMemset(N->m, 0, N->np * 4));
  SK_CUDA(cudaMemset(N->v, 0, N->np * 4));
  N->step = 0;
  sk_status s = net_pack(N);
  if (s != SK_OK) return s;
  SK_CUDA(cudaStreamSynchronize(N->stream));
  return SK_OK;
}

sk_status sk_net_set_legacy_mma(sk_net N, int32_t on) {
  SK_CHECK(N, SK_INVALID_ARG, "null network");
  N->legacy_mma = on ? 1 : 0;
  return SK_OK;
}

sk_status sk_pairs_create(sk_pairs* out, int64_t nx, int64_t ny, int64_t capacity, int32_t max_instances) {
  SK_CHECK(out, SK_INVALID_ARG, "null output");
  *out = nullptr;
  SK_CHECK(nx >= 8 && ny >= 8 && nx % 8 == 0 && ny % 8 == 0, SK_INVALID_ARG, "grid sides must be multiples of 8");
  SK_CHECK(capacity >= 1 && max_instances >= 1, SK_INVALID_ARG, "empty capacity");
  auto* D = new sk_pairs_s();
  D->nx = static_cast<int>(nx);
  D->ny = static_cast<int>(ny);
  D->P = nx * ny;
  D->cap = capacity;
  D->cap_inst = max_instances;
  cudaError_t e = cudaMalloc(&D->R, static_cast<size_t>(capacity) * D->P * 4);
  if (e == cudaSuccess) e = cudaMalloc(&D->E, static_cast<size_t>(capacity) * D->P * 4);
  if (e == cudaSuccess) e = cudaMalloc(&D->inst, static_cast<size_t>(capacity) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&D->coef, static_cast<size_t>(max_instances) * 6 * D->P * 4);
  if (e == cudaSuccess) e = cudaMalloc(&D->scratch, static_cast<size_t>(D->P) * 3 * 8 + 64);
  if (e != cudaSuccess) {
    sk_pairs_destroy(D);
    return cuda_fail(e, "cudaMalloc (pairs)");
  }
  *out = D;
  return SK_OK;
}

sk_status sk_pairs_destroy(sk_pairs D) {
  if (!D) return SK_OK;
  cudaDeviceSynchronize();
  for (void* p : {static_cast<void*>(D->R), static_cast<void*>(D->E), static_cast<void*>(D->inst),
                  static_cast<void*>(D->coef), D->scratch})
    if (p) cudaFree(p);
  delete D;
  return SK_OK;
}

sk_status sk_pairs_count(sk_pairs D, int64_t* count) {
  SK_CHECK(D && count, SK_INVALID_ARG, "null argument");
  *count = D->count;
  return SK_OK;
}

}  // extern "C"

namespace sk {

// Extracts the six coefficient planes of a 5-point FP64 CSR matrix on an
// nx x ny grid into `coef` (6 n floats).
sk_status grid_planes(sk_matrix A, int64_t nx, int64_t ny, float* coef, cudaStream_t st) {
  SK_CHECK(A && A->format == SK_CSR && A->dtype == SK_F64, SK_NOT_SUPPORTED,
           "the learned preconditioner needs an FP64 CSR matrix");
  SK_CHECK(A->nrow == A->ncol && A->nrow == nx * ny, SK_INVALID_ARG, "matrix size is not nx * ny");
  unsigned* bad = nullptr;
  SK_CUDA(cudaMalloc(&bad, 4));
  cudaMemsetAsync(bad, 0, 4, st);
  SK_LAUNCH(planes_kernel, ew_grid(A->nrow), 256, 0, st, A->nrow, static_cast<int>(nx), A->csr.row_ptr,
            A->csr.col_ind, static_cast<const double*>(A->csr.vals), coef, bad);
  unsigned h = 0;
  cudaMemcpyAsync(&h, bad, 4, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(bad);
  SK_CUDA(e);
  SK_CHECK(h == 0, SK_INVALID_ARG, "matrix is not a 5-point stencil with a nonzero diagonal on the given grid");
  return SK_OK;
}

}  // namespace sk

extern "C" {

sk_status sk_pairs_add_instance(sk_pairs D, sk_matrix A, int32_t* instance) {
  SK_CHECK(D && A && instance, SK_INVALID_ARG, "null argument");
  SK_CHECK(D->ninst < D->cap_inst, SK_INVALID_ARG, "instance capacity exhausted");
  cudaStream_t st = A->stream;
  sk_status s = grid_planes(A, D->nx, D->ny, D->coef + static_cast<i64>(D->ninst) * 6 * D->P, st);
  if (s != SK_OK) return s;
  *instance = D->ninst++;
  return SK_OK;
}

sk_status sk_pairs_add(sk_pairs D, int32_t instance, const double* r_dev, const double* e_dev, sk_stream s) {
  SK_CHECK(D && r_dev && e_dev, SK_INVALID_ARG, "null argument");
  SK_CHECK(instance >= 0 && instance < D->ninst, SK_INVALID_ARG, "unknown instance");
  SK_CHECK(D->count < D->cap, SK_INVALID_ARG, "pair capacity exhausted");
  cudaStream_t st = static_cast<cudaStream_t>(s);
  SK_LAUNCH(store_pair_kernel, ew_grid(D->P), 256, 0, st, D->P, r_dev, e_dev, D->R + D->count * D->P,
            D->E + D->count * D->P);
  SK_CUDA(cudaMemcpyAsync(D->inst + D->count, &instance, 4, cudaMemcpyHostToDevice, st));
  SK_CUDA(cudaStreamSynchronize(st));
  D->inst_host.push_back(instance);
  ++D->count;
  return SK_OK;
}

sk_status sk_learned_harvest(sk_pairs D, int32_t instance, sk_matrix A, const double* b_dev,
                             const double* xstar_dev, int64_t restart, int64_t cycles, int64_t* added) {
  SK_CHECK(D && A && b_dev && xstar_dev && added, SK_INVALID_ARG, "null argument");
  SK_CHECK(instance >= 0 && instance < D->ninst, SK_INVALID_ARG, "unknown instance");
  SK_CHECK(A->nrow == D->P && A->format == SK_CSR && A->dtype == SK_F64, SK_INVALID_ARG,
           "harvest needs the instance's FP64 CSR matrix");
  *added = 0;
  cudaStream_t st = A->stream;
  double* r = static_cast<double*>(D->scratch);
  double* e = r + D->P;
  double* x = e + D->P;
  SK_CUDA(cudaMemsetAsync(x, 0, D->P * 8, st));
  sk_precond J = nullptr;
  sk_status s = sk_jacobi_create(&J, A);
  if (s != SK_OK) return s;
  sk_fgmres_config cfg{0.0, restart, restart, 0};
  for (int64_t c = 0; c < cycles && D->count < D->cap; ++c) {
    sk_summary sum{};
    s = sk_fgmres_solve(A, J, b_dev, x, &cfg, &sum, nullptr, st);
    if (s != SK_OK) break;
    SK_LAUNCH(resid_err_kernel, ew_grid(D->P), 256, 0, st, D->P, A->csr.row_ptr, A->csr.col_ind,
              static_cast<const double*>(A->csr.vals), b_dev, x, xstar_dev, r, e);
    if ((s = sk_pairs_add(D, instance, r, e, st)) != SK_OK) break;
    ++*added;
  }
  sk_precond_destroy(J);
  return s;
}

sk_status sk_net_loss_grad(sk_net N, sk_pairs D, const int32_t* pairs_host, int32_t batch, double mu,
                           double* loss, float* grad_host, int64_t capacity) {
  SK_CHECK(N && D && pairs_host && loss && batch >= 1, SK_INVALID_ARG, "null argument");
  for (int b = 0; b < batch; ++b)
    SK_CHECK(pairs_host[b] >= 0 && pairs_host[b] < D->count, SK_INVALID_ARG, "pair index out of range");
  int* idx = nullptr;
  SK_CUDA(cudaMalloc(&idx, batch * 4));
  SK_CUDA(cudaMemcpy(idx, pairs_host, batch * 4, cudaMemcpyHostToDevice));
  N->stream = nullptr;
  sk_status s = net_workspace(N, batch, D->ny, D->nx);  // N->loss lives in it
  if (s == SK_OK) s = net_step_grad(N, D, idx, batch, mu, N->loss);
  if (s == SK_OK) s = check_err(N);
  if (s == SK_OK) {
    cudaMemcpy(loss, N->loss, 8, cudaMemcpyDeviceToHost);
    if (grad_host && capacity >= N->np) cudaMemcpy(grad_host, N->grad, N->np * 4, cudaMemcpyDeviceToHost);
  }
  cudaFree(idx);
  return s;
}

sk_status sk_net_train(sk_net N, sk_pairs D, const sk_train_config* cfg, sk_train_summary* out,
                       double* loss_history) {
  SK_CHECK(N && D && cfg && out, SK_INVALID_ARG, "null argument");
  SK_CHECK(D->count >= 1, SK_INVALID_ARG, "no training pairs");
  SK_CHECK(cfg->batch >= 1 && cfg->steps >= 0, SK_INVALID_ARG, "bad batch or step count");
  *out = sk_train_summary{};
  const int B = cfg->batch;
  const auto t0 = std::chrono::steady_clock::now();
  // all sample indices up front: one copy
  std::vector<int> idx(static_cast<size_t>(cfg->steps) * B);
  std::mt19937_64 rng(cfg->seed);
  std::uniform_int_distribution<int64_t> pick(0, D->count - 1);
  for (auto& v : idx) v = static_cast<int>(pick(rng));
  int* idx_dev = nullptr;
  double* loss_dev = nullptr;
  SK_CUDA(cudaMalloc(&idx_dev, idx.size() * 4 + 16));
  SK_CUDA(cudaMalloc(&loss_dev, (cfg->steps + 1) * 8));
  N->stream = nullptr;
  sk_status s = SK_OK;
  if (!idx.empty()) s = (cudaMemcpy(idx_dev, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess)
                            ? SK_OK
                            : fail(SK_CUDA_ERROR, "index upload");
  for (int64_t k = 0; k < cfg->steps && s == SK_OK; ++k) {
    s = net_step_grad(N, D, idx_dev + k * B, B, cfg->mu, loss_dev + k);
    if (s != SK_OK) break;
    ++N->step;
    // cosine decay from lr to lr * lr_final_ratio
    const double frac = cfg->steps > 1 ? static_cast<double>(k) / (cfg->steps - 1) : 1.0;
    const float lr = static_cast<float>(cfg->lr * (cfg->lr_final_ratio + (1.0 - cfg->lr_final_ratio) * 0.5 *
                                                                            (1.0 + std::cos(3.141592653589793 * frac))));
    const float c1 = 1.0f - std::pow(cfg->beta1, static_cast<float>(N->step));
    const float c2 = 1.0f - std::pow(cfg->beta2, static_cast<float>(N->step));
    SK_LAUNCH(adam_kernel, ew_grid(N->np), 256, 0, N->stream, N->np, N->params, N->m, N->v, N->grad, lr,
              cfg->beta1, cfg->beta2, cfg->eps, c1, c2);
    s = net_pack(N);
  }
  if (s == SK_OK) s = check_err(N);
  if (s == SK_OK && cfg->steps > 0) {
    std::vector<double> h(cfg->steps);
    cudaMemcpy(h.data(), loss_dev, cfg->steps * 8, cudaMemcpyDeviceToHost);
    out->first_loss = h.front();
    out->last_loss = h.back();
    if (loss_history) std::memcpy(loss_history, h.data(), h.size() * 8);
  }
  out->steps = cfg->steps;
  out->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  cudaFree(idx_dev);
  cudaFree(loss_dev);
  return s;
}

sk_status sk_learned_create(sk_precond* out, sk_matrix A, sk_net net, int64_t nx, int64_t ny) {
  SK_CHECK(out && A && net, SK_INVALID_ARG, "null argument");
  *out = nullptr;
  SK_CHECK(nx >= 8 && ny >= 8 && nx % 8 == 0 && ny % 8 == 0, SK_INVALID_ARG, "grid sides must be multiples of 8");
  auto* M = new sk_precond_s();
  M->kind = 3;
  M->A = A;
  M->dtype = SK_F64;
  M->n = A->nrow;
  M->net = net;
  M->grid_nx = nx;
  M->grid_ny = ny;
  cudaError_t e = cudaMalloc(&M->coef, static_cast<size_t>(6) * nx * ny * 4);
  if (e != cudaSuccess) {
    delete M;
    return cuda_fail(e, "cudaMalloc (planes)");
  }
  sk_status s = grid_planes(A, nx, ny, M->coef, A->stream);
  if (s == SK_OK && cudaMalloc(&M->xfeat, static_cast<size_t>(nx) * ny * 16) != cudaSuccess)
    s = fail(SK_OUT_OF_MEMORY, "cudaMalloc (fixed features)");
  if (s == SK_OK) {
    SK_LAUNCH(fixed_features_kernel, ew_grid(M->n), 256, 0, A->stream, M->coef, M->n,
              static_cast<bf16*>(M->xfeat));
    if (cudaGetLastError() != cudaSuccess) s = fail(SK_CUDA_ERROR, "fixed features");
  }
  if (s != SK_OK) {
    learned_release(M);
    delete M;
    return s;
  }
  *out = M;
  return SK_OK;
}

sk_status sk_learned_planes(sk_precond M, float* host, int64_t capacity) {
  SK_CHECK(M && M->kind == 3 && host && capacity >= 6 * M->n, SK_INVALID_ARG, "not a learned preconditioner");
  SK_CUDA(cudaDeviceSynchronize());
  SK_CUDA(cudaMemcpy(host, M->coef, static_cast<size_t>(6) * M->n * 4, cudaMemcpyDeviceToHost));
  return SK_OK;
}

sk_status sk_net_status(sk_net N) {
  SK_CHECK(N, SK_INVALID_ARG, "null network");
  if (N->host_err != SK_OK) {
    const sk_status e = N->host_err;
    N->host_err = SK_OK;
    return fail(e, "a learned preconditioner apply inside the solve failed");
  }
  return check_err(N);
}

}  // extern "C"
