// sk_mixed.cu -- the FP32 inner solve of the mixed-precision solver as one
// persistent cooperative launch.
//
// No reference counterpart as a whole: the iteration is the reference's
// conjugate gradient (conjugate_gradient.hpp:122-312, Jacobi or identity
// left preconditioner, true residual only at k = 0) in FP32, without a
// kernel boundary per step.  One CTA per SM (two over the diagonal copy)
// stays resident for the whole solve.
//
// The Jacobi inner solve runs on the symmetrically scaled matrix
// S = D^-1/2 A D^-1/2 (D = diag(A)), whose diagonal is 1 and is not stored:
// CG on S y = D^-1/2 r0 with d = D^-1/2 y takes, in exact arithmetic, the
// same steps as Jacobi-preconditioned CG on A d = r0 (<r_S, r_S> is
// <r, D^-1 r>), but reads no inverse diagonal and streams one entry per row
// less.  The unpreconditioned inner solve runs on A itself.  Either way the
// preconditioned residual is the residual, so each iteration is two phases
// separated by grid-wide reductions:
//
//   S  w = M r for this CTA's rows (M = S or A); p = r + beta p and
//      q = w + beta q, which equals M p by linearity, so no second product
//      is needed; <p, q>                                          -> alpha
//   U  d += alpha p, r -= alpha q, <r, r> and the unscaled ||r||^2
//      (the sum of a_ii r_i^2 on S)                               -> test, beta
//
// The convergence test is the reference's ||r|| / ||r0|| < tol on the
// residual of A d = r0 (conjugate_gradient.hpp:264-276).  The dot products
// are reduced deterministically: each CTA publishes its partial in a slot
// before the barrier, and after it every CTA sums all the slots in the same
// fixed order, so every CTA holds the same scalars and takes the same
// decision.  Barrier waits are bounded in time; a wait that runs out sets
// an error word that makes every other CTA leave at its next wait, and the
// host reports SK_TIMEOUT.
//
// The vectors (r, d, p, q and the diagonal, 5 x 4 B per row) stay in L2 (a
// persisting window set by the caller) while the matrix streams through it
// with evict-first loads.
#include <climits>
#include <vector>

#include "sk_kernels.cuh"
#include "sk_mixed.cuh"

namespace sk {
namespace {

constexpr int kPT = 512;   // threads per CTA (SELL: one CTA per SM, up to 128 registers;
                           // diagonal copy: two CTAs per SM, up to 64)
constexpr int kPW = kPT / 32;
constexpr int kPU = 8;     // SELL slots loaded together
constexpr int kSlot = 4;   // doubles per CTA and reduction

struct SyncWords {
  unsigned long long arrived;  // total arrivals, never reset during a solve
  int err;
  int converged;
  long long iterations;
  double rnorm;
  double pad[4];
};

struct PArgs {
  int n;
  const int* off;  // SELL-32 form
  const unsigned char* len;
  const int* col;
  const float* val;  // SELL-32 values, or the diagonal planes
  int dia_n;         // diagonal form: planes, row masks and offsets
  const unsigned short* dia_mask;
  int dia_off[kDiaMax];
  const float* wdiag;  // a_ii of A when the matrix is the scaled S, else null
  float* r;
  float* d;
  float* p;
  float* q;
  double* slots;  // [2][grid][kSlot]
  SyncWords* sync;
  float tol;
  long long max_iters;
  unsigned long long wait_ns;  // bound of each barrier wait
  unsigned bias;               // extra arrivals a barrier waits for (timeout tests)
};

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Publishes this CTA's writes (ordered before by bar.sync) and arrives.
__device__ __forceinline__ void arrive_release(unsigned long long* p) {
  asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u64 [%0], 1;" ::"l"(p) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid barrier on one monotonic arrival counter: barrier number e (from 1)
// is passed when the counter reaches e * gridDim.x (+ bias, which only the
// timeout tests set).  False: a wait ran out (here or in another CTA) and
// the kernel must return.  The clock and the error word are read once per
// 256 polls.
__device__ bool grid_barrier(SyncWords* s, unsigned& epoch, unsigned long long wait_ns, unsigned bias) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    epoch += 1;
    const unsigned long long target = static_cast<unsigned long long>(epoch) * gridDim.x + bias;
    arrive_release(&s->arrived);
    unsigned long long t0 = 0;
    for (unsigned spins = 0; ld_acquire(&s->arrived) < target; ++spins) {
      if ((spins & 255u) == 255u) {
        if (*reinterpret_cast<volatile int*>(&s->err) != 0) {
          ok = 0;
          break;
        }
        const unsigned long long t = global_ns();
        if (t0 == 0) {
          t0 = t;
        } else if (t - t0 > wait_ns) {
          atomicExch(&s->err, 1);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sums v over the grid into every thread of every CTA (the same bits
// everywhere): block tree, then CTA slots summed in CTA order by warp 0.
// Consecutive reductions alternate between the two slot sets.
template <int NR>
__device__ __forceinline__ bool grid_allreduce(double (&v)[NR], PArgs const& a, int set, unsigned& epoch) {
  __shared__ double s_part[kPW][kSlot];
  __shared__ double s_tot[kSlot];
  warp_reduce<NR>(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < NR; ++j) s_part[warp][j] = v[j];
  __syncthreads();
  double* slot = a.slots + static_cast<size_t>(set) * gridDim.x * kSlot;
  if (warp == 0) {
    double t[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) t[j] = lane < kPW ? s_part[lane][j] : 0.0;
    warp_reduce<NR>(t);
    if (lane == 0)
#pragma unroll
      for (int j = 0; j < NR; ++j) slot[static_cast<size_t>(blockIdx.x) * kSlot + j] = t[j];
  }
  if (!grid_barrier(a.sync, epoch, a.wait_ns, a.bias)) return false;
  // every thread below gridDim.x reads one CTA's slot (one round trip),
  // then a fixed tree over the CTA
  double t[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j)
    t[j] = threadIdx.x < gridDim.x ? __ldcg(slot + static_cast<size_t>(threadIdx.x) * kSlot + j) : 0.0;
  warp_reduce<NR>(t);
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < NR; ++j) s_part[warp][j] = t[j];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < NR; ++j) t[j] = lane < kPW ? s_part[lane][j] : 0.0;
    warp_reduce<NR>(t);
    if (lane == 0)
#pragma unroll
      for (int j = 0; j < NR; ++j) s_tot[j] = t[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NR; ++j) v[j] = s_tot[j];
  return true;
}

// Row i's SELL position: its length and the offset of its slot 0.
__device__ __forceinline__ void row_meta(PArgs const& a, int i, int& len, int& base) {
  len = 0;
  base = 0;
  if (i < a.n) {
    len = __ldg(a.len + i);
    base = __ldg(a.off + (i >> 5)) + (i & 31);
  }
}

// Streams slots k..k+kPU-1 of a row (evict-first: read once per product).
__device__ __forceinline__ void row_fetch(PArgs const& a, int len, int base, int k, int (&c)[kPU], float (&v)[kPU]) {
#pragma unroll
  for (int j = 0; j < kPU; ++j)
    if (k + j < len) {
      const int e = base + 32 * (k + j);
      c[j] = __ldcs(a.col + e);
      v[j] = __ldcs(a.val + e);
    }
}

// The direction update of one row from its product w = (M r)_i: p = r +
// beta p, q = w + beta q (p = r, q = w at the first step); returns p q.
template <bool FIRST>
__device__ __forceinline__ double row_direction(PArgs const& a, int i, float ri, float w, float pi, float qi,
                                                float beta) {
  const float pn = FIRST ? ri : add(ri, mul(beta, pi));
  const float qn = FIRST ? w : add(w, mul(beta, qi));
  a.p[i] = pn;
  a.q[i] = qn;
  return static_cast<double>(mul(pn, qn));
}

// Phase S over SELL rows: each row's product summed from r_i (UNIT: the
// unit diagonal of S) or from 0, then its stored entries in storage order.
// Three rows are in flight per thread: the slots of row k+2 stream from
// HBM while the gathers of row k+1 return and row k is summed, so neither
// the matrix stream nor the gathers wait on each other.  Returns this
// thread's share of <p, q>.
template <bool UNIT, bool FIRST>
__device__ __forceinline__ double phase_s_sell(PArgs const& a, int t0, int T, float beta) {
  double pq = 0.0;
  // row a: summed this step; row b: slots arrived, gathers issued this
  // step; row c: slots issued this step
  int ia = t0, la, basea, lb, bb, lc, bc;
  float va[kPU], ga[kPU], ra = 0.0f, pa = 0.0f, qa = 0.0f;
  int cb[kPU];
  float vb[kPU];
  row_meta(a, ia, la, basea);
  row_fetch(a, la, basea, 0, cb, vb);
#pragma unroll
  for (int j = 0; j < kPU; ++j) {
    va[j] = vb[j];
    ga[j] = (j < la) ? a.r[cb[j]] : 0.0f;
  }
  if (ia < a.n) {
    ra = a.r[ia];
    if (!FIRST) {
      pa = a.p[ia];
      qa = a.q[ia];
    }
  }
  row_meta(a, ia + T, lb, bb);
  row_fetch(a, lb, bb, 0, cb, vb);
  row_meta(a, ia + 2 * T, lc, bc);
  while (ia < a.n) {
    // slots of row c (issued first, so that a wait on row b's indices
    // below does not hold the HBM stream back), position of row d
    int cc[kPU];
    float vc[kPU];
    row_fetch(a, lc, bc, 0, cc, vc);
    int ld, bd;
    row_meta(a, ia + 3 * T, ld, bd);
    // gathers and own values of row b
    float gb[kPU];
#pragma unroll
    for (int j = 0; j < kPU; ++j)
      if (j < lb) gb[j] = a.r[cb[j]];
    const int ib = ia + T;
    float rb = 0.0f, pb = 0.0f, qb = 0.0f;
    if (ib < a.n) {
      rb = a.r[ib];
      if (!FIRST) {
        pb = a.p[ib];
        qb = a.q[ib];
      }
    }
    // sum of row a
    float sum = UNIT ? ra : 0.0f;
#pragma unroll
    for (int j = 0; j < kPU; ++j)
      if (j < la) sum = add(sum, mul(va[j], ga[j]));
    for (int k = kPU; k < la; k += kPU) {  // rows longer than kPU slots
      int c[kPU];
      float v[kPU], g[kPU];
      row_fetch(a, la, basea, k, c, v);
#pragma unroll
      for (int j = 0; j < kPU; ++j)
        if (k + j < la) g[j] = a.r[c[j]];
#pragma unroll
      for (int j = 0; j < kPU; ++j)
        if (k + j < la) sum = add(sum, mul(v[j], g[j]));
    }
    pq += row_direction<FIRST>(a, ia, ra, sum, pa, qa, beta);
    // rotate a <- b <- c <- d
    ia = ib;
    la = lb;
    basea = bb;
    ra = rb;
    pa = pb;
    qa = qb;
    lb = lc;
    bb = bc;
    lc = ld;
    bc = bd;
#pragma unroll
    for (int j = 0; j < kPU; ++j) {
      va[j] = vb[j];
      ga[j] = gb[j];
      cb[j] = cc[j];
      vb[j] = vc[j];
    }
  }
  return pq;
}

// Phase S over diagonal planes.  The values of a warp's rows for one
// diagonal are one 32-value segment and the reads of r at row + off[d] are
// contiguous, so no load depends on another: each thread issues the value
// and r loads of kDiaRows rows for kDiaGroup diagonals at a time without
// waiting for the rows' masks (a diagonal a row does not store reads a zero
// value and a clamped r, and the mask leaves both out of the sum).  The
// kernel runs 2 CTAs per SM here (this phase needs few registers), which
// hides the load latency better than a deeper register pipeline at one CTA
// per SM.  Each row is summed from r_i (UNIT) or 0 over its stored
// diagonals in ascending column order.  Returns this thread's share of
// <p, q>.
constexpr int kDiaRows = 2;
constexpr int kDiaGroup = 4;

template <bool UNIT, bool FIRST>
__device__ __forceinline__ double phase_s_dia(PArgs const& a, int t0, int T, float beta) {
  constexpr int R = kDiaRows, C = kDiaGroup;
  double pq = 0.0;
  const int last = a.n - 1;
  const long long sl = 32 * a.dia_n;
  for (int i = t0; i < a.n; i += R * T) {
    unsigned m[R];
    float s[R], ro[R], po[R], qo[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int row = i + r * T;
      const bool in = row < a.n;
      m[r] = in ? __ldcs(a.dia_mask + row) : 0u;
      ro[r] = in ? a.r[row] : 0.0f;
      po[r] = in && !FIRST ? a.p[row] : 0.0f;
      qo[r] = in && !FIRST ? a.q[row] : 0.0f;
      s[r] = UNIT ? ro[r] : 0.0f;
    }
#pragma unroll
    for (int d0 = 0; d0 < kDiaMax; d0 += C) {
      if (d0 >= a.dia_n) break;
      float v[R][C], g[R][C];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int row = min(i + r * T, last);
        const float* vs = a.val + (row >> 5) * sl + (row & 31);
#pragma unroll
        for (int j = 0; j < C; ++j)
          if (d0 + j < a.dia_n) {
            v[r][j] = __ldcs(vs + 32 * (d0 + j));
            g[r][j] = a.r[min(max(row + a.dia_off[d0 + j], 0), last)];
          }
      }
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < C; ++j)
          if (d0 + j < a.dia_n && ((m[r] >> (d0 + j)) & 1u)) s[r] = add(s[r], mul(v[r][j], g[r][j]));
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int row = i + r * T;
      if (row < a.n) pq += row_direction<FIRST>(a, row, ro[r], s[r], po[r], qo[r], beta);
    }
  }
  return pq;
}

template <bool DIA, bool UNIT>
__global__ void __launch_bounds__(kPT, DIA ? 2 : 1) inner_cg_kernel(PArgs a) {
  const int n = a.n;
  const int T = gridDim.x * kPT;
  const int t0 = blockIdx.x * kPT + threadIdx.x;
  // phase U: four rows per 16-byte access, two accesses per thread and
  // step, rows 4 * n4 .. n - 1 by the first threads
  const int n4 = n >> 2;
  const int tail = 4 * n4 + t0;
  const float4* q4 = reinterpret_cast<const float4*>(a.q);
  const float4* p4 = reinterpret_cast<const float4*>(a.p);
  const float4* w4 = reinterpret_cast<const float4*>(a.wdiag);
  float4* d4 = reinterpret_cast<float4*>(a.d);
  float4* r4 = reinterpret_cast<float4*>(a.r);
  const float4 one4 = make_float4(1.f, 1.f, 1.f, 1.f);
  unsigned epoch = 0;
  // k = 0 (reorthogonalize, :217-230, with d = 0 so r = r0): <r, r> and the
  // unscaled ||r0||^2 (the solve's ||b||, :194)
  double v0[2] = {0.0, 0.0};
  for (int i = t0; i < n; i += T) {
    const float ri = a.r[i];
    a.d[i] = 0.0f;
    const float rr = mul(ri, ri);
    v0[0] += static_cast<double>(rr);
    v0[1] += static_cast<double>(UNIT ? mul(a.wdiag[i], rr) : rr);
  }
  if (!grid_allreduce<2>(v0, a, 0, epoch)) return;
  const float bnorm = sqrtf(static_cast<float>(v0[1]));
  float rho = static_cast<float>(v0[0]);
  float beta = 0.0f;
  long long it = 0;
  int conv = 0;
  float rn = bnorm;
  if (bnorm == 0.0f) conv = 1;
  // phase S of one step (the first with p = r, q = A r) and <p, q>
  auto phase_s = [&](double (&pq)[1], bool first_step) -> bool {
    if (first_step) {
      if constexpr (DIA) pq[0] = phase_s_dia<UNIT, true>(a, t0, T, beta);
      else pq[0] = phase_s_sell<UNIT, true>(a, t0, T, beta);
    } else {
      if constexpr (DIA) pq[0] = phase_s_dia<UNIT, false>(a, t0, T, beta);
      else pq[0] = phase_s_sell<UNIT, false>(a, t0, T, beta);
    }
    return grid_allreduce<1>(pq, a, 1, epoch);
  };
  double pq[1] = {0.0};
  if (!conv && a.max_iters > 0) {
    // S: the product, the direction update and compute_step_size (:233-239)
    if (!phase_s(pq, true)) return;
    for (;;) {
      const float alpha = rho / static_cast<float>(pq[0]);
      // U: compute_new_solution, compute_new_residual, is_converged
      // (:242-276) and the next <r, z> (:279-284)
      double rr[2] = {0.0, 0.0};
      auto upd = [&](float pi, float qi, float di, float ro, float wi, float& dn, float& rnew) {
        dn = add(mul(alpha, pi), di);
        rnew = sub(ro, mul(alpha, qi));
        const float r2 = mul(rnew, rnew);
        rr[0] += static_cast<double>(r2);
        if (UNIT) rr[1] += static_cast<double>(mul(wi, r2));
      };
      auto upd4 = [&](float4 pv, float4 qv, float4 dv, float4 rv, float4 wv, float4& dn, float4& rw) {
        upd(pv.x, qv.x, dv.x, rv.x, wv.x, dn.x, rw.x);
        upd(pv.y, qv.y, dv.y, rv.y, wv.y, dn.y, rw.y);
        upd(pv.z, qv.z, dv.z, rv.z, wv.z, dn.z, rw.z);
        upd(pv.w, qv.w, dv.w, rv.w, wv.w, dn.w, rw.w);
      };
      int j = t0;
      for (; j + T < n4; j += 2 * T) {
        const int j1 = j + T;
        const float4 pv0 = p4[j], qv0 = q4[j], dv0 = d4[j], rv0 = r4[j];
        const float4 pv1 = p4[j1], qv1 = q4[j1], dv1 = d4[j1], rv1 = r4[j1];
        const float4 wv0 = UNIT ? w4[j] : one4, wv1 = UNIT ? w4[j1] : one4;
        float4 dn0, rw0, dn1, rw1;
        upd4(pv0, qv0, dv0, rv0, wv0, dn0, rw0);
        upd4(pv1, qv1, dv1, rv1, wv1, dn1, rw1);
        d4[j] = dn0;
        r4[j] = rw0;
        d4[j1] = dn1;
        r4[j1] = rw1;
      }
      if (j < n4) {
        float4 dn, rw;
        upd4(p4[j], q4[j], d4[j], r4[j], UNIT ? w4[j] : one4, dn, rw);
        d4[j] = dn;
        r4[j] = rw;
      }
      if (tail < n) {
        float dn, rw;
        upd(a.p[tail], a.q[tail], a.d[tail], a.r[tail], UNIT ? a.wdiag[tail] : 1.f, dn, rw);
        a.d[tail] = dn;
        a.r[tail] = rw;
      }
      if (!grid_allreduce<2>(rr, a, 0, epoch)) return;
      ++it;
      rn = sqrtf(static_cast<float>(UNIT ? rr[1] : rr[0]));
      conv = rn / bnorm < a.tol ? 1 : 0;
      if (conv || it >= a.max_iters) break;
      const float rho_new = static_cast<float>(rr[0]);
      beta = rho_new / rho;  // update_direction (:285-290), applied in phase S
      rho = rho_new;
      if (!phase_s(pq, false)) return;
    }
  }

  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.sync->iterations = it;
    a.sync->converged = conv;
    a.sync->rnorm = static_cast<double>(rn);
  }
}

const void* pick_kernel(bool dia, bool unit) {
  if (dia)
    return unit ? reinterpret_cast<const void*>(&inner_cg_kernel<true, true>)
                : reinterpret_cast<const void*>(&inner_cg_kernel<true, false>);
  return unit ? reinterpret_cast<const void*>(&inner_cg_kernel<false, true>)
              : reinterpret_cast<const void*>(&inner_cg_kernel<false, false>);
}

// ------------------------------------------------------------------
// Plain FP64 conjugate gradient (conjugate_gradient.hpp:122-312 with a
// Jacobi or identity left preconditioner, identity right, true residual at
// k = 0 only) as one cooperative launch, for systems small enough that the
// three kernels per step are bound by launch and reduction latency.  Each
// CTA owns a contiguous block of rows; per step, behind two grid-wide
// reductions:
//   1  p = D^-1 r + beta p for the CTA's rows into the other half of a
//      double buffer, and q = A p with every gathered p_j recomputed the
//      same way from r_j and the previous p_j (so no barrier is needed
//      between the direction update and the product), <p, q>
//                                               -> alpha = rz / <p, q>
//   2  x += alpha p, r -= alpha q, <r, r>, <r, D^-1 r>
//                                               -> the test, beta, rz
// with the arithmetic of the per-step kernels (OpCgDirection, EpiCgPq,
// OpCgUpdate: the same products, sums and roundings per element, a
// recomputed p_j has the bits its owner stores); only the order in which
// the dot products' partial sums meet differs.
// ------------------------------------------------------------------
struct Cg64Args {
  PArgs g;  // n, off, len, col (SELL-32), slots, sync, wait_ns, bias
  const double* val;
  const double* b;
  double* x;
  double* r;
  double* p0;  // direction, double-buffered: step k writes p[k & 1]
  double* p1;
  double* q;
  const double* invd;  // Jacobi: 1 / a_ii; null: identity
  double* hist;        // residual history, or null
  Scalars* sc;
};

// (A v)_i with v_j = f(j), each row summed in storage order
template <class Args, class F>
__device__ __forceinline__ double sell_row64(Args const& a, int i, F const& f) {
  const int len = __ldg(a.g.len + i);
  const int base = __ldg(a.g.off + (i >> 5)) + (i & 31);
  double sum = 0.0;
  int k = 0;
  for (; k + 4 <= len; k += 4) {
    double pr[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = base + 32 * (k + j);
      pr[j] = mul(__ldg(a.val + e), f(__ldg(a.g.col + e)));
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) sum = add(sum, pr[j]);
  }
  for (; k < len; ++k) {
    const int e = base + 32 * k;
    sum = add(sum, mul(__ldg(a.val + e), f(__ldg(a.g.col + e))));
  }
  return sum;
}

template <bool JAC>
__global__ void __launch_bounds__(kPT, 1) cg64_kernel(Cg64Args a) {
  unsigned epoch = 0;
  const int n = a.g.n;
  const int per = (((n + gridDim.x - 1) / gridDim.x) + 31) & ~31;
  const int r0 = min(n, static_cast<int>(blockIdx.x) * per), r1 = min(n, r0 + per);
  Scalars* sc = a.sc;
  const double bnorm = sc->bnorm, tol = sc->tol;
  const long long max_iters = sc->max_iters;
  const double* __restrict__ invd = a.invd;
  const double* x0 = a.x;
  // k = 0: r = b - A x, p = z = D^-1 r, rz = <r, z>   (EpiCgResid)
  double v1[1] = {0.0};
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const double ri = sub(a.b[i], sell_row64(a, i, [&](int j) { return x0[j]; }));
    a.r[i] = ri;
    const double zi = JAC ? mul(invd[i], ri) : ri;
    a.p0[i] = zi;
    v1[0] += mul(ri, zi);
  }
  if (!grid_allreduce<1>(v1, a.g, 0, epoch)) return;
  double rz = v1[0];
  long long it = 0;
  int conv = 0;
  double rn = 0.0, alpha = 0.0, beta = 0.0;
  int set = 1;
  while (it < max_iters) {
    // 1: p (for k > 0), q = A p, <p, q>          (OpCgDirection, EpiCgPq)
    const double* pold = (it & 1) ? a.p0 : a.p1;  // step it - 1 wrote p[(it - 1) & 1]
    double* pcur = (it & 1) ? a.p1 : a.p0;
    const double* __restrict__ rr_ = a.r;
    auto pnew = [&](int j) {
      const double zj = JAC ? mul(invd[j], rr_[j]) : rr_[j];
      return add(zj, mul(beta, pold[j]));
    };
    double pq[1] = {0.0};
    if (it == 0) {
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const double qi = sell_row64(a, i, [&](int j) { return a.p0[j]; });
        a.q[i] = qi;
        pq[0] += mul(a.p0[i], qi);
      }
    } else {
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const double pi = pnew(i);
        pcur[i] = pi;
        const double qi = sell_row64(a, i, pnew);
        a.q[i] = qi;
        pq[0] += mul(pi, qi);
      }
    }
    if (!grid_allreduce<1>(pq, a.g, set, epoch)) return;
    set ^= 1;
    alpha = rz / pq[0];
    // 2: x += alpha p, r -= alpha q, <r, r>, <r, D^-1 r>  (OpCgUpdate)
    double rr[2] = {0.0, 0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      a.x[i] = add(mul(alpha, pcur[i]), a.x[i]);
      const double ri = sub(a.r[i], mul(alpha, a.q[i]));
      a.r[i] = ri;
      rr[0] += mul(ri, ri);
      if (JAC) rr[1] += mul(ri, mul(invd[i], ri));
    }
    if (!grid_allreduce<2>(rr, a.g, set, epoch)) return;
    set ^= 1;
    ++it;
    rn = sqrt(rr[0]);
    if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[it - 1] = rn;
    conv = rn / bnorm < tol ? 1 : 0;
    if (conv || it >= max_iters) break;
    const double rz_new = JAC ? rr[1] : rr[0];
    beta = rz_new / rz;
    rz = rz_new;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->iters = it;
    sc->converged = conv;
    sc->done = 1;
    sc->rnorm = rn;
    sc->rz = rz;
    sc->alpha = alpha;
    sc->beta = beta;
    sc->hist_len = a.hist ? it : 0;
  }
}

// ------------------------------------------------------------------
// Plain FP64 BiCGSTAB (bicgstab.hpp:93-361 with identity or Jacobi on
// each side) as one cooperative launch for the same small systems.  Per
// step, behind three grid-wide reductions:
//   A  p = r + beta (p - omega v) and p_hat = M_R M_L p for the CTA's rows
//      into the other half of double buffers, v = A p_hat with every
//      gathered p_hat_j recomputed from r_j and the previous p_j, v_j;
//      <r_hat, v>                        -> alpha, or SK_BREAKDOWN at 0
//   B  s = r - alpha v, s_hat = M s, t = A s_hat (s_hat_j recomputed from
//      r_j, v_j); ||s||^2, <t, t>, <t, s> -> the half-step test, omega
//   C  x += alpha p_hat + omega s_hat, r = s - omega t; ||r||^2,
//      <r_hat, r>                        -> the full-step test, rho
// mirroring the per-step kernels (OpBiP, EpiBiV, OpBiS, OpBiHalfOrS,
// EpiBiT, OpBiUpdate): the same element arithmetic, iteration counting,
// history entries (one per half step), omega = 0 skip and breakdowns;
// only the order in which the dot products' partial sums meet differs.
// ------------------------------------------------------------------
struct Bi64Args {
  PArgs g;  // n, off, len, col (SELL-32), slots, sync, wait_ns, bias
  const double* val;
  const double* b;
  double* x;
  double* r;
  double* r_hat;
  double* p[2];
  double* v[2];
  double* p_hat;
  double* s;
  double* s_hat;
  double* t;
  const double* invl;  // Jacobi left: 1 / a_ii, or null
  const double* invr;  // Jacobi right, or null
  double* hist;
  Scalars* sc;
};

__global__ void __launch_bounds__(kPT, 1) bi64_kernel(Bi64Args a) {
  unsigned epoch = 0;
  const int n = a.g.n;
  const int per = (((n + gridDim.x - 1) / gridDim.x) + 31) & ~31;
  const int r0 = min(n, static_cast<int>(blockIdx.x) * per), r1 = min(n, r0 + per);
  Scalars* sc = a.sc;
  const double bnorm = sc->bnorm, tol = sc->tol;
  const long long max_iters = sc->max_iters;
  const double* __restrict__ invl = a.invl;
  const double* __restrict__ invr = a.invr;
  auto hat = [&](int j, double v) {  // M_R M_L v, in that order (OpBiP, OpBiHalfOrS)
    if (invl) v = mul(invl[j], v);
    if (invr) v = mul(invr[j], v);
    return v;
  };
  const double* x0 = a.x;
  // compute_initial_residual, r_hat = r, rho_new = <r, r>   (EpiBiResid)
  double v1[1] = {0.0};
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const double ri = sub(a.b[i], sell_row64(a, i, [&](int j) { return x0[j]; }));
    a.r[i] = ri;
    a.r_hat[i] = ri;
    a.p[0][i] = 0.0;
    a.v[0][i] = 0.0;
    v1[0] += mul(ri, ri);
  }
  if (!grid_allreduce<1>(v1, a.g, 0, epoch)) return;
  double rho_new = v1[0], rho = 1.0, alpha = 1.0, omega = 1.0;
  long long iters = 0, hist_len = 0;
  int converged = 0, status = 0;
  int set = 1;
  double last = 0.0;
  auto record = [&](double v) {
    if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[hist_len] = v;
    ++hist_len;
    last = v;
  };
  bool done = max_iters <= 0;
  if (!done && rho_new == 0.0) {
    converged = 1;
    done = true;
  }
  const long long max_steps = max_iters > 1 ? max_iters : 1;
  for (long long step = 0; !done && step < max_steps; ++step) {
    const int cur = static_cast<int>(step & 1);
    const double* __restrict__ pold = a.p[cur];
    const double* __restrict__ vold = a.v[cur];
    double* pnew = a.p[cur ^ 1];
    double* vnew = a.v[cur ^ 1];
    const double beta = (rho_new / rho) * (alpha / omega);
    const double* __restrict__ rr_ = a.r;
    auto p_of = [&](int j) { return add(rr_[j], mul(beta, sub(pold[j], mul(omega, vold[j])))); };
    // A: p, p_hat, v = A p_hat, <r_hat, v>
    double rv[1] = {0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const double pi = p_of(i);
      pnew[i] = pi;
      a.p_hat[i] = hat(i, pi);
      const double vi = sell_row64(a, i, [&](int j) { return hat(j, p_of(j)); });
      vnew[i] = vi;
      rv[0] += mul(a.r_hat[i], vi);
    }
    if (!grid_allreduce<1>(rv, a.g, set, epoch)) return;
    set ^= 1;
    ++iters;
    if (rv[0] == 0.0) {
      status = SK_BREAKDOWN;
      break;
    }
    alpha = rho_new / rv[0];
    // B: s, s_hat, t = A s_hat, ||s||^2, <t, t>, <t, s>
    const double* __restrict__ vn = vnew;
    auto s_of = [&](int j) { return sub(rr_[j], mul(alpha, vn[j])); };
    double st[3] = {0.0, 0.0, 0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const double si = s_of(i);
      a.s[i] = si;
      a.s_hat[i] = hat(i, si);
      const double ti = sell_row64(a, i, [&](int j) { return hat(j, s_of(j)); });
      a.t[i] = ti;
      st[0] += mul(si, si);
      st[1] += mul(ti, ti);
      st[2] += mul(ti, si);
    }
    if (!grid_allreduce<3>(st, a.g, set, epoch)) return;
    set ^= 1;
    const double sn = sqrt(st[0]);
    record(sn);
    if (sn / bnorm < tol) {  // half step converged: x += alpha p_hat (OpBiHalfOrS)
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) a.x[i] = add(a.x[i], mul(alpha, a.p_hat[i]));
      converged = 1;
      break;
    }
    ++iters;
    const double tt = st[1];
    omega = tt == 0.0 ? 0.0 : st[2] / tt;
    const bool skip = omega == 0.0;
    // C: x, r, ||r||^2, <r_hat, r>
    double rr[2] = {0.0, 0.0};
    if (!skip) {
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        a.x[i] = add(a.x[i], add(mul(alpha, a.p_hat[i]), mul(omega, a.s_hat[i])));
        const double ri = sub(a.s[i], mul(omega, a.t[i]));
        a.r[i] = ri;
        rr[0] += mul(ri, ri);
        rr[1] += mul(a.r_hat[i], ri);
      }
    }
    if (!grid_allreduce<2>(rr, a.g, set, epoch)) return;
    set ^= 1;
    if (!skip) {
      rho = rho_new;
      const double rn = sqrt(rr[0]);
      record(rn);
      if (rn / bnorm < tol) {
        converged = 1;
        break;
      }
      rho_new = rr[1];
    }
    if (iters >= max_iters) break;
    if (rho_new == 0.0) {
      status = SK_BREAKDOWN;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->iters = iters;
    sc->converged = converged;
    sc->status = status;
    sc->done = 1;
    sc->rho = rho;
    sc->rho_new = rho_new;
    sc->alpha = alpha;
    sc->omega = omega;
    sc->hist_len = a.hist ? hist_len : 0;
    sc->rnorm = last;
    sc->half = 0;
    sc->skip = 0;
  }
}

// ------------------------------------------------------------------
// Plain FP64 CGS (cgs.hpp:106-395 with identity or Jacobi on each side)
// as one cooperative launch for the same small systems.  Per step, behind
// two grid-wide reductions:
//   A  the previous step's direction update (u = r + beta q,
//      p = u + beta (q + beta p), skipped after rho_new = 0) for the
//      CTA's rows into the other half of a double-buffered p, and
//      q_hat = A M p with every gathered p_j recomputed from r_j, q_j and
//      the previous p_j; <r_hat, q_hat>               -> alpha
//   B  q = u - alpha q_hat, u_hat = M (u + q), x += alpha u_hat, and
//      r -= alpha A u_hat with every gathered u_hat_j recomputed from u_j
//      and q_hat_j; ||r||^2, <r_hat, r>   -> the test, rho, beta, skip
// mirroring the per-step kernels (OpLR, EpiCgsQhat, OpCgsQ, EpiCgsR,
// OpCgsDir): the same element arithmetic, iteration counting (two per
// step) and history; only the order in which the dot products' partial
// sums meet differs.
// ------------------------------------------------------------------
struct Cgs64Args {
  PArgs g;  // n, off, len, col (SELL-32), slots, sync, wait_ns, bias
  const double* val;
  const double* b;
  double* x;
  double* r;
  double* r_hat;
  double* p[2];
  double* u;
  double* q;
  double* q_hat;
  const double* invl;  // Jacobi left: 1 / a_ii, or null
  const double* invr;  // Jacobi right, or null
  double* hist;
  Scalars* sc;
};

__global__ void __launch_bounds__(kPT, 1) cgs64_kernel(Cgs64Args a) {
  unsigned epoch = 0;
  const int n = a.g.n;
  const int per = (((n + gridDim.x - 1) / gridDim.x) + 31) & ~31;
  const int r0 = min(n, static_cast<int>(blockIdx.x) * per), r1 = min(n, r0 + per);
  Scalars* sc = a.sc;
  const double bnorm = sc->bnorm, tol = sc->tol;
  const long long max_iters = sc->max_iters;
  const double* __restrict__ invl = a.invl;
  const double* __restrict__ invr = a.invr;
  auto hat = [&](int j, double v) {  // M_R M_L v, in that order (OpLR, OpCgsQ)
    if (invl) v = mul(invl[j], v);
    if (invr) v = mul(invr[j], v);
    return v;
  };
  const double* x0 = a.x;
  // compute_initial_residual: r = r_hat = p = u = b - A x, rho = <r, r>  (EpiCgsInit)
  double v1[1] = {0.0};
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const double ri = sub(a.b[i], sell_row64(a, i, [&](int j) { return x0[j]; }));
    a.r[i] = ri;
    a.r_hat[i] = ri;
    a.p[0][i] = ri;
    a.u[i] = ri;
    v1[0] += mul(ri, ri);
  }
  if (!grid_allreduce<1>(v1, a.g, 0, epoch)) return;
  double rho = v1[0], alpha = 0.0, beta = 0.0, last = 0.0;
  long long iters = 0, hist_len = 0;
  int converged = 0, skip = 0;
  int set = 1, cur = 0;
  bool upd = false;  // the previous step left a direction update to apply
  bool done = max_iters <= 0;
  while (!done) {
    const double* __restrict__ pold = a.p[cur];
    double* pnew = a.p[cur ^ 1];
    const double* __restrict__ rr_ = a.r;
    const double* __restrict__ qq_ = a.q;
    const bool up = upd;
    const double bt = beta;
    auto p_of = [&](int j) {  // OpCgsDir
      if (!up) return pold[j];
      const double uj = add(rr_[j], mul(bt, qq_[j]));
      return add(uj, mul(bt, add(qq_[j], mul(bt, pold[j]))));
    };
    // A: direction update, q_hat = A M p, <r_hat, q_hat>
    double rq[1] = {0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      if (up) {
        a.u[i] = add(rr_[i], mul(bt, qq_[i]));
        pnew[i] = p_of(i);
      }
      const double qh = sell_row64(a, i, [&](int j) { return hat(j, p_of(j)); });
      a.q_hat[i] = qh;
      rq[0] += mul(a.r_hat[i], qh);
    }
    if (!grid_allreduce<1>(rq, a.g, set, epoch)) return;
    set ^= 1;
    if (up) cur ^= 1;
    alpha = rho / rq[0];
    // B: q, u_hat, x, r -= alpha A u_hat, ||r||^2, <r_hat, r>
    const double* __restrict__ uu_ = a.u;
    const double* __restrict__ qh_ = a.q_hat;
    const double al = alpha;
    auto uhat_of = [&](int j) {  // OpCgsQ
      const double qj = sub(uu_[j], mul(al, qh_[j]));
      return hat(j, add(uu_[j], qj));
    };
    double rr[2] = {0.0, 0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const double ui = uu_[i];
      const double qi = sub(ui, mul(al, qh_[i]));
      const double uh = hat(i, add(ui, qi));
      a.x[i] = add(a.x[i], mul(al, uh));
      const double au = sell_row64(a, i, uhat_of);
      a.q[i] = qi;
      const double ri = sub(rr_[i], mul(al, au));
      a.r[i] = ri;
      rr[0] += mul(ri, ri);
      rr[1] += mul(a.r_hat[i], ri);
    }
    if (!grid_allreduce<2>(rr, a.g, set, epoch)) return;
    set ^= 1;
    // EpiCgsR
    iters += 2;
    const double rn = sqrt(rr[0]);
    if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[hist_len] = rn;
    ++hist_len;
    last = rn;
    if (rn / bnorm < tol) {
      converged = 1;
      break;
    }
    const double rho_new = rr[1];
    if (rho_new == 0.0) {
      skip = 1;
      upd = false;
    } else {
      skip = 0;
      beta = rho_new / rho;
      rho = rho_new;
      upd = true;
    }
    if (iters >= max_iters) done = true;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->iters = iters;
    sc->converged = converged;
    sc->done = 1;
    sc->rho = rho;
    sc->alpha = alpha;
    sc->beta = beta;
    sc->skip = skip;
    sc->hist_len = a.hist ? hist_len : 0;
    sc->rnorm = last;
  }
}

// ------------------------------------------------------------------
// Plain FP64 MINRES (minres.hpp:106-418 with identity or Jacobi on each
// side) as one cooperative launch for the same small systems.  Per step,
// behind two grid-wide reductions:
//   A  the previous step's update_solution and rotate_state for the CTA's
//      rows (d, x; z = q / beta, v_prev = v, v = w / beta), and
//      w = A z with every gathered z_j recomputed from q_j;
//      <z, w>                                              -> alpha
//   B  w -= alpha v + beta v_prev, q = M_R M_L w; <w, q> -> beta_new, the
//      Givens rotation, the test and the scalars of rotate_state
// mirroring the per-step kernels (EpiMinInit, OpMinScale, EpiMinW,
// OpMinLanczos, min_step_finalize, OpMinUpdate): the same element and
// scalar arithmetic, iteration counting and history; q holds what the
// per-step form writes into v_prev before the rotation.  Only the order in
// which the dot products' partial sums meet differs.
// ------------------------------------------------------------------
struct Min64Args {
  PArgs g;  // n, off, len, col (SELL-32), slots, sync, wait_ns, bias
  const double* val;
  const double* b;
  double* x;
  double* v;
  double* vp;
  double* z;
  double* w;
  double* q;
  double* d;
  double* dp;
  const double* invl;  // Jacobi left: 1 / a_ii, or null
  const double* invr;  // Jacobi right, or null
  double* hist;
  Scalars* sc;
};

__global__ void __launch_bounds__(kPT, 1) min64_kernel(Min64Args a) {
  unsigned epoch = 0;
  const int n = a.g.n;
  const int per = (((n + gridDim.x - 1) / gridDim.x) + 31) & ~31;
  const int r0 = min(n, static_cast<int>(blockIdx.x) * per), r1 = min(n, r0 + per);
  Scalars* sc = a.sc;
  const double bnorm = sc->bnorm, tol = sc->tol;
  const long long max_iters = sc->max_iters;
  const double* __restrict__ invl = a.invl;
  const double* __restrict__ invr = a.invr;
  auto hat = [&](int j, double v) {  // M_R M_L v, in that order
    if (invl) v = mul(invl[j], v);
    if (invr) v = mul(invr[j], v);
    return v;
  };
  const double* x0 = a.x;
  // compute_initial_residual: v = b - A x, z = M v, beta = sqrt(<v, z>)
  double v1[1] = {0.0};
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const double vi = sub(a.b[i], sell_row64(a, i, [&](int j) { return x0[j]; }));
    const double zi = hat(i, vi);
    a.v[i] = vi;
    a.z[i] = zi;
    a.vp[i] = 0.0;
    a.d[i] = 0.0;
    a.dp[i] = 0.0;
    v1[0] += mul(vi, zi);
  }
  if (!grid_allreduce<1>(v1, a.g, 0, epoch)) return;
  int set = 1;
  double beta = sqrt(v1[0]);
  double alpha = 0.0, eps = 0.0, delta = 0.0, rho = 0.0, phi = 0.0, phi_bar = beta;
  double cs_prev = 1.0, sn_prev = 0.0, cs = 1.0, sn = 0.0, cs_new = 0.0, sn_new = 0.0, inv_bn = 0.0;
  long long iters = 0, hist_len = 0;
  int converged = 0;
  double last = 0.0;
  bool done = false;
  if (beta == 0.0) {
    converged = 1;
    done = true;
  } else {
    inv_bn = dvd(1.0, beta);
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {  // OpMinScale
      a.v[i] = mul(a.v[i], inv_bn);
      a.z[i] = mul(a.z[i], inv_bn);
    }
    double none[1] = {0.0};  // the scaled z is gathered by the first product
    if (!grid_allreduce<1>(none, a.g, set, epoch)) return;
    set ^= 1;
  }
  if (max_iters <= 0) done = true;
  bool pending = false, rotate = false;
  // update_solution and rotate_state of the step just taken, for row i
  auto update_row = [&](int i) {
    const double dn = dvd(sub(sub(a.z[i], mul(delta, a.d[i])), mul(eps, a.dp[i])), rho);
    a.dp[i] = a.d[i];
    a.d[i] = dn;
    a.x[i] = add(a.x[i], mul(phi, dn));
    if (rotate) {
      a.z[i] = mul(a.q[i], inv_bn);
      a.vp[i] = a.v[i];
      a.v[i] = mul(a.w[i], inv_bn);
    } else {
      a.vp[i] = a.q[i];
    }
  };
  while (!done) {
    // A: the pending update, w = A z, <z, w>
    const bool up = pending, rot = rotate;
    const double ib = inv_bn;
    const double* __restrict__ qq = a.q;
    const double* zz = a.z;
    double zw[1] = {0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      if (up) update_row(i);
      const double wi = sell_row64(a, i, [&](int j) { return up && rot ? mul(qq[j], ib) : zz[j]; });
      a.w[i] = wi;
      zw[0] += mul(a.z[i], wi);
    }
    if (!grid_allreduce<1>(zw, a.g, set, epoch)) return;
    set ^= 1;
    pending = false;
    alpha = zw[0];
    // B: the Lanczos vector, q = M w, <w, q>
    double wq[1] = {0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const double wi = sub(a.w[i], add(mul(alpha, a.v[i]), mul(beta, a.vp[i])));
      const double qi = hat(i, wi);
      a.w[i] = wi;
      a.q[i] = qi;
      wq[0] += mul(wi, qi);
    }
    if (!grid_allreduce<1>(wq, a.g, set, epoch)) return;
    set ^= 1;
    // min_step_finalize
    const double beta_new = sqrt(wq[0]);
    eps = mul(sn_prev, beta);
    const double delta_1 = mul(cs_prev, beta);
    const double dl = add(mul(cs, delta_1), mul(sn, alpha));
    const double rho_bar = add(mul(-sn, delta_1), mul(cs, alpha));
    const double rh = sqrt(add(mul(rho_bar, rho_bar), mul(beta_new, beta_new)));
    if (rh != 0.0) {
      cs_new = dvd(rho_bar, rh);
      sn_new = dvd(beta_new, rh);
      phi = mul(cs_new, phi_bar);
      phi_bar = mul(-sn_new, phi_bar);
      rho = rh;
      delta = dl;
    }
    pending = true;
    const double res = fabs(phi_bar);
    if (a.hist && blockIdx.x == 0 && threadIdx.x == 0) a.hist[hist_len] = res;
    ++hist_len;
    last = res;
    const bool conv = res / bnorm < tol;
    converged = conv ? 1 : 0;
    iters += 1;
    rotate = !conv && beta_new != 0.0;
    if (rotate) {
      inv_bn = dvd(1.0, beta_new);
      cs_prev = cs;
      sn_prev = sn;
      cs = cs_new;
      sn = sn_new;
      beta = beta_new;
    }
    if (conv || iters >= max_iters) done = true;
  }
  if (pending)
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) update_row(i);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->iters = iters;
    sc->converged = converged;
    sc->done = 1;
    sc->hist_len = a.hist ? hist_len : 0;
    sc->rnorm = last;
  }
}

// CTAs of the cooperative grid (0: the kernel does not fit).
int coop_grid(sk_matrix A, const void* k) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kPT, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * A->sm_count;
}

// ------------------------------------------------------------------
// The scaled copies of S = D^-1/2 A D^-1/2, built from the FP64 CSR arrays
// on the first Jacobi inner solve that needs them.
// ------------------------------------------------------------------

// isq_i = 1 / sqrt(a_ii) and a_ii as float; counts the rows whose diagonal
// entry is absent or not positive (S is then not formed).
__global__ void sym_diag_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci,
                                const double* __restrict__ v, double* __restrict__ isq,
                                float* __restrict__ dg, unsigned long long* bad) {
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<i64>(gridDim.x) * blockDim.x) {
    double a = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) a = v[k];
    if (!(a > 0.0)) {
      atomicAdd(bad, 1ull);
      a = 1.0;
    }
    isq[i] = __ddiv_rn(1.0, __dsqrt_rn(a));
    dg[i] = static_cast<float>(a);
  }
}

__device__ __forceinline__ float sym_value(double a, double isq_i, double isq_j) {
  return static_cast<float>(__dmul_rn(__dmul_rn(a, isq_i), isq_j));
}

// Off-diagonal entries of each row, and the largest count of each 32-row
// slice (one warp per slice; the grid covers whole slices).
__global__ void sym_sell_count_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci,
                                      int* __restrict__ slice_w) {
  const i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  int cnt = 0;
  if (i < n) {
    cnt = rp[i + 1] - rp[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) --cnt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt = max(cnt, __shfl_xor_sync(0xffffffffu, cnt, o));
  if ((threadIdx.x & 31) == 0 && i < n) slice_w[i >> 5] = cnt;
}

__global__ void sym_sell_fill_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci,
                                     const double* __restrict__ v, const double* __restrict__ isq,
                                     const int* __restrict__ off, int* __restrict__ col,
                                     float* __restrict__ val, unsigned char* __restrict__ len) {
  for (i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<i64>(gridDim.x) * blockDim.x) {
    const i64 base = off[i >> 5] + (i & 31);
    const double si = isq[i];
    int k = 0;
    for (int e = rp[i]; e < rp[i + 1]; ++e) {
      const int c = ci[e];
      if (c == i) continue;
      col[base + 32 * k] = c;
      val[base + 32 * k] = sym_value(v[e], si, isq[c]);
      ++k;
    }
    len[i] = static_cast<unsigned char>(k);
  }
}

struct SymOffsets {
  int n;
  int off[kDiaMax];
};

__global__ void sym_dia_fill_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci,
                                    const double* __restrict__ v, const double* __restrict__ isq, SymOffsets o,
                                    float* __restrict__ planes, unsigned short* __restrict__ mask) {
  for (i64 r = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<i64>(gridDim.x) * blockDim.x) {
    unsigned m = 0;
    const double sr = isq[r];
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
      const int c = ci[k];
      if (c == r) continue;
      const int off = c - static_cast<int>(r);
      int d = 0;
      while (d + 1 < o.n && o.off[d] != off) ++d;  // every off-diagonal offset is in the set
      planes[((r >> 5) * o.n + d) * 32 + (r & 31)] = sym_value(v[k], sr, isq[c]);
      m |= 1u << d;
    }
    mask[r] = static_cast<unsigned short>(m);
  }
}

sk_status sym_prepare_diag(sk_matrix A, cudaStream_t st) {
  auto& C = A->csr;
  if (C.sym_diag_state) return SK_OK;
  const i64 n = A->nrow;
  void *isq = nullptr, *dg = nullptr, *bad = nullptr;
  sk_status s;
  if ((s = dev_alloc(A, &isq, (n + 64) * 8)) != SK_OK) return s;
  if ((s = dev_alloc(A, &dg, (n + 64) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &bad, 8)) != SK_OK) return s;
  SK_CUDA(cudaMemsetAsync(bad, 0, 8, st));
  SK_LAUNCH(sym_diag_kernel, grid_for(n), kThreads, 0, st, n, C.row_ptr, C.col_ind,
            static_cast<const double*>(C.vals), static_cast<double*>(isq), static_cast<float*>(dg),
            static_cast<unsigned long long*>(bad));
  unsigned long long nb = 0;
  SK_CUDA(cudaMemcpyAsync(&nb, bad, 8, cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  C.sym_isq = static_cast<double*>(isq);
  C.sym_diag = static_cast<float*>(dg);
  C.sym_diag_state = nb ? -1 : 1;
  return SK_OK;
}

sk_status sym_prepare_sell(sk_matrix A, cudaStream_t st) {
  auto& C = A->csr;
  const i64 n = A->nrow;
  const i64 nslices = (n + 31) / 32;
  void* wdev = nullptr;
  sk_status s;
  SK_CUDA(cudaMalloc(&wdev, (nslices + 1) * sizeof(int)));
  SK_LAUNCH(sym_sell_count_kernel, ceil_div(nslices * 32, kThreads), kThreads, 0, st, n, C.row_ptr, C.col_ind,
            static_cast<int*>(wdev));
  std::vector<int> w(static_cast<size_t>(nslices));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(w.data(), wdev, nslices * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(wdev);
  if (e != cudaSuccess) return cuda_fail(e, "scaled SELL row counts");
  std::vector<int> off(static_cast<size_t>(nslices) + 1, 0);
  i64 total = 0;
  for (i64 k = 0; k < nslices; ++k) {
    if (w[static_cast<size_t>(k)] > 255) {
      C.sym_sell_state = -1;
      return SK_OK;
    }
    off[static_cast<size_t>(k)] = static_cast<int>(total);
    total += 32 * static_cast<i64>(w[static_cast<size_t>(k)]);
    if (total > (i64(1) << 31) - 64) {
      C.sym_sell_state = -1;
      return SK_OK;
    }
  }
  off[static_cast<size_t>(nslices)] = static_cast<int>(total);
  if (total > A->nnz + A->nnz / 4 + 64) {  // skewed rows: more than a quarter of padding
    C.sym_sell_state = -1;
    return SK_OK;
  }
  void *col = nullptr, *val = nullptr, *len = nullptr;
  if ((s = dev_alloc(A, &col, (total + 64) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &val, (total + 64) * 4)) != SK_OK) return s;
  if ((s = dev_alloc(A, &len, n + 64)) != SK_OK) return s;
  SK_CUDA(cudaMemsetAsync(col, 0, (total + 64) * 4, st));
  SK_CUDA(cudaMemsetAsync(val, 0, (total + 64) * 4, st));
  if ((s = upload_vector(A, off, &C.sym_off, st)) != SK_OK) return s;
  SK_LAUNCH(sym_sell_fill_kernel, grid_for(n), kThreads, 0, st, n, C.row_ptr, C.col_ind,
            static_cast<const double*>(C.vals), C.sym_isq, C.sym_off, static_cast<int*>(col),
            static_cast<float*>(val), static_cast<unsigned char*>(len));
  SK_CUDA(cudaGetLastError());
  SK_CUDA(cudaStreamSynchronize(st));
  C.sym_col = static_cast<int*>(col);
  C.sym_val = static_cast<float*>(val);
  C.sym_len = static_cast<unsigned char*>(len);
  C.sym_sell_state = 1;
  return SK_OK;
}

// The scaled diagonal planes of the pattern's off-diagonal offsets (the
// handle's own diagonal copy need not exist).
sk_status sym_prepare_dia(sk_matrix A, cudaStream_t st) {
  auto& C = A->csr;
  const i64 n = A->nrow;
  std::vector<int> offs;
  sk_status s0 = dia_pattern(A, &offs);
  if (s0 != SK_OK) return s0;
  SymOffsets o{};
  for (int k : offs)
    if (k != 0) o.off[o.n++] = k;
  if (o.n == 0) {
    C.sym_dia_state = -1;
    return SK_OK;
  }
  const i64 len = (n + 31) / 32 * 32 * o.n;
  void *planes = nullptr, *mask = nullptr;
  sk_status s;
  if ((s = dev_alloc(A, &planes, len * 4 + 64)) != SK_OK) return s;
  if ((s = dev_alloc(A, &mask, (n + 64) * 2)) != SK_OK) return s;
  SK_CUDA(cudaMemsetAsync(planes, 0, len * 4 + 64, st));
  SK_LAUNCH(sym_dia_fill_kernel, grid_for(n), kThreads, 0, st, n, C.row_ptr, C.col_ind,
            static_cast<const double*>(C.vals), C.sym_isq, o, static_cast<float*>(planes),
            static_cast<unsigned short*>(mask));
  SK_CUDA(cudaGetLastError());
  SK_CUDA(cudaStreamSynchronize(st));
  C.sym_dval = static_cast<float*>(planes);
  C.sym_dmask = static_cast<unsigned short*>(mask);
  C.sym_dn = o.n;
  for (int k = 0; k < o.n; ++k) C.sym_doff[k] = o.off[k];
  C.sym_dia_state = 1;
  return SK_OK;
}

// The layout the persistent solve reads: for the unscaled solve the
// handle's diagonal copy when it has FP32 planes, else its SELL-32 copy;
// for the scaled solve the scaled planes when the pattern has them, else
// the scaled SELL-32 copy.
bool use_dia(sk_matrix A, bool scaled) {
  return scaled ? A->csr.sym_dia_state > 0 : A->csr.dia_n > 0 && A->csr.dia_vals32;
}

}  // namespace

sk_status inner_sym_prepare(sk_matrix A, cudaStream_t st, bool* ok) {
  *ok = false;
  if (!A || A->format != SK_CSR || A->dtype != SK_F64 || A->nrow <= 0) return SK_OK;
  sk_status s = sym_prepare_diag(A, st);
  if (s != SK_OK || A->csr.sym_diag_state < 0) return s;
  if (!A->csr.sym_dia_state && (s = sym_prepare_dia(A, st)) != SK_OK) return s;
  if (A->csr.sym_dia_state < 0 && !A->csr.sym_sell_state && (s = sym_prepare_sell(A, st)) != SK_OK) return s;
  *ok = A->csr.sym_dia_state > 0 || A->csr.sym_sell_state > 0;
  return SK_OK;
}

const double* inner_sym_isq(sk_matrix A) { return A->csr.sym_isq; }

bool inner_persistent_ok(sk_matrix A, bool scaled) {
  if (!A || A->format != SK_CSR || A->nrow <= 0) return false;
  const auto& C = A->csr;
  if (scaled ? !(C.sym_diag_state > 0 && (C.sym_dia_state > 0 || C.sym_sell_state > 0))
             : !(use_dia(A, false) || (C.sell && C.sell_vals32)))
    return false;
  if (A->nrow > INT_MAX / 4) return false;
  int coop = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, A->device) != cudaSuccess || !coop) return false;
  return coop_grid(A, pick_kernel(use_dia(A, scaled), scaled)) > 0;
}

size_t inner_persistent_scratch(sk_matrix A) {
  return sizeof(SyncWords) + static_cast<size_t>(2) * kPT * kSlot * sizeof(double) + 256;
}

sk_status inner_cg_persistent(sk_matrix A, bool scaled, float* r, float* d, float* p, float* q, void* scratch,
                              double tol, long long max_iters, cudaStream_t st, InnerResult* out) {
  *out = InnerResult{};
  const auto& C = A->csr;
  SK_CHECK(!scaled || C.sym_diag_state > 0, SK_NOT_SUPPORTED,
           "scaled inner solve: D^-1/2 A D^-1/2 is not formed (a diagonal entry is absent or not positive)");
  SK_CHECK(inner_persistent_ok(A, scaled), SK_NOT_SUPPORTED,
           scaled ? "persistent scaled inner solve: the scaled copy is not built"
                  : "persistent inner solve needs a CSR handle with FP32 SELL values or an FP32 diagonal copy");
  const bool dia = use_dia(A, scaled);
  const void* k = pick_kernel(dia, scaled);
  int grid = coop_grid(A, k);
  SK_CHECK(grid > 0, SK_NOT_SUPPORTED, "persistent inner solve does not fit on the device");
  grid = std::min(grid, kPT);  // a CTA sums the grid's slots one per thread
  const int need = ceil_div(A->nrow, kPT);
  if (grid > need) grid = need;
  SyncWords* sync = static_cast<SyncWords*>(scratch);
  double* slots = reinterpret_cast<double*>(static_cast<char*>(scratch) + 256);
  SK_CUDA(cudaMemsetAsync(sync, 0, sizeof(SyncWords), st));
  PArgs a{};
  a.n = static_cast<int>(A->nrow);
  if (dia && scaled) {
    a.val = C.sym_dval;
    a.dia_n = C.sym_dn;
    a.dia_mask = C.sym_dmask;
    for (int j = 0; j < kDiaMax; ++j) a.dia_off[j] = C.sym_doff[j];
  } else if (dia) {
    a.val = C.dia_vals32;
    a.dia_n = C.dia_n;
    a.dia_mask = C.dia_mask;
    for (int j = 0; j < kDiaMax; ++j) a.dia_off[j] = C.dia_off[j];
  } else if (scaled) {
    a.off = C.sym_off;
    a.len = C.sym_len;
    a.col = C.sym_col;
    a.val = C.sym_val;
  } else {
    a.off = C.sell_off;
    a.len = C.sell_len;
    a.col = C.sell_col;
    a.val = C.sell_vals32;
  }
  a.wdiag = scaled ? C.sym_diag : nullptr;
  a.r = r;
  a.d = d;
  a.p = p;
  a.q = q;
  a.slots = slots;
  a.sync = sync;
  a.tol = static_cast<float>(tol);
  a.max_iters = max_iters;
  a.wait_ns = wait_limit_ns();
  a.bias = wait_target_bias();
  void* params[] = {&a};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  SK_CUDA(cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kPT), params, 0, st));
  SyncWords h{};
  SK_CUDA(cudaMemcpyAsync(&h, sync, sizeof(h), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  if (h.err) return fail(SK_TIMEOUT, "persistent inner solve: a grid barrier wait ran out");
  out->iterations = h.iterations;
  out->converged = h.converged;
  out->rnorm = h.rnorm;
  return SK_OK;
}

bool cg64_persistent_ok(sk_matrix A) {
  if (!A || A->format != SK_CSR || A->dtype != SK_F64 || !A->csr.sell || A->nrow <= 0) return false;
  if (A->nrow > kCg64MaxRows || summation_sequential()) return false;
  int coop = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, A->device) != cudaSuccess || !coop) return false;
  return coop_grid(A, reinterpret_cast<const void*>(&cg64_kernel<true>)) > 0 &&
         coop_grid(A, reinterpret_cast<const void*>(&cg64_kernel<false>)) > 0;
}

sk_status cg64_persistent(sk_matrix A, const double* b, double* x, double* r, double* p0, double* p1, double* q,
                          const double* invd, double* hist, Scalars* sc, void* scratch, cudaStream_t st) {
  SK_CHECK(cg64_persistent_ok(A), SK_NOT_SUPPORTED, "persistent CG needs a small FP64 CSR handle with SELL-32");
  const auto& C = A->csr;
  const void* k = invd ? reinterpret_cast<const void*>(&cg64_kernel<true>)
                       : reinterpret_cast<const void*>(&cg64_kernel<false>);
  int grid = std::min(A->sm_count, kPT);  // one CTA per SM (cg64_persistent_ok: at least one fits)
  const int need = ceil_div(A->nrow, 32);
  if (grid > need) grid = need;
  SyncWords* sync = static_cast<SyncWords*>(scratch);
  double* slots = reinterpret_cast<double*>(static_cast<char*>(scratch) + 256);
  SK_CUDA(cudaMemsetAsync(sync, 0, sizeof(SyncWords), st));
  Cg64Args a{};
  a.g.n = static_cast<int>(A->nrow);
  a.g.off = C.sell_off;
  a.g.len = C.sell_len;
  a.g.col = C.sell_col;
  a.g.slots = slots;
  a.g.sync = sync;
  a.g.wait_ns = wait_limit_ns();
  a.g.bias = wait_target_bias();
  a.val = static_cast<const double*>(C.sell_vals);
  a.b = b;
  a.x = x;
  a.r = r;
  a.p0 = p0;
  a.p1 = p1;
  a.q = q;
  a.invd = invd;
  a.hist = hist;
  a.sc = sc;
  void* params[] = {&a};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  SK_CUDA(cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kPT), params, 0, st));
  int err = 0;
  SK_CUDA(cudaMemcpyAsync(&err, &sync->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  if (err) return fail(SK_TIMEOUT, "persistent CG: a grid barrier wait ran out");
  return SK_OK;
}

bool bi64_persistent_ok(sk_matrix A) {
  if (!cg64_persistent_ok(A)) return false;
  return coop_grid(A, reinterpret_cast<const void*>(&bi64_kernel)) > 0;
}

sk_status bi64_persistent(sk_matrix A, const double* b, double* x, double* const* vec, const double* invl,
                          const double* invr, double* hist, Scalars* sc, void* scratch, cudaStream_t st) {
  SK_CHECK(bi64_persistent_ok(A), SK_NOT_SUPPORTED, "persistent BiCGSTAB needs a small FP64 CSR handle with SELL-32");
  const auto& C = A->csr;
  int grid = std::min(A->sm_count, kPT);
  const int need = ceil_div(A->nrow, 32);
  if (grid > need) grid = need;
  SyncWords* sync = static_cast<SyncWords*>(scratch);
  double* slots = reinterpret_cast<double*>(static_cast<char*>(scratch) + 256);
  SK_CUDA(cudaMemsetAsync(sync, 0, sizeof(SyncWords), st));
  Bi64Args a{};
  a.g.n = static_cast<int>(A->nrow);
  a.g.off = C.sell_off;
  a.g.len = C.sell_len;
  a.g.col = C.sell_col;
  a.g.slots = slots;
  a.g.sync = sync;
  a.g.wait_ns = wait_limit_ns();
  a.g.bias = wait_target_bias();
  a.val = static_cast<const double*>(C.sell_vals);
  a.b = b;
  a.x = x;
  a.r = vec[0];
  a.r_hat = vec[1];
  a.p[0] = vec[2];
  a.p[1] = vec[3];
  a.v[0] = vec[4];
  a.v[1] = vec[5];
  a.p_hat = vec[6];
  a.s = vec[7];
  a.s_hat = vec[8];
  a.t = vec[9];
  a.invl = invl;
  a.invr = invr;
  a.hist = hist;
  a.sc = sc;
  void* params[] = {&a};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  SK_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&bi64_kernel), dim3(grid), dim3(kPT), params, 0,
                                      st));
  int err = 0;
  SK_CUDA(cudaMemcpyAsync(&err, &sync->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  if (err) return fail(SK_TIMEOUT, "persistent BiCGSTAB: a grid barrier wait ran out");
  return SK_OK;
}

bool cgs64_persistent_ok(sk_matrix A) {
  if (!cg64_persistent_ok(A)) return false;
  return coop_grid(A, reinterpret_cast<const void*>(&cgs64_kernel)) > 0;
}

sk_status cgs64_persistent(sk_matrix A, const double* b, double* x, double* const* vec, const double* invl,
                           const double* invr, double* hist, Scalars* sc, void* scratch, cudaStream_t st) {
  SK_CHECK(cgs64_persistent_ok(A), SK_NOT_SUPPORTED, "persistent CGS needs a small FP64 CSR handle with SELL-32");
  const auto& C = A->csr;
  int grid = std::min(A->sm_count, kPT);
  const int need = ceil_div(A->nrow, 32);
  if (grid > need) grid = need;
  SyncWords* sync = static_cast<SyncWords*>(scratch);
  double* slots = reinterpret_cast<double*>(static_cast<char*>(scratch) + 256);
  SK_CUDA(cudaMemsetAsync(sync, 0, sizeof(SyncWords), st));
  Cgs64Args a{};
  a.g.n = static_cast<int>(A->nrow);
  a.g.off = C.sell_off;
  a.g.len = C.sell_len;
  a.g.col = C.sell_col;
  a.g.slots = slots;
  a.g.sync = sync;
  a.g.wait_ns = wait_limit_ns();
  a.g.bias = wait_target_bias();
  a.val = static_cast<const double*>(C.sell_vals);
  a.b = b;
  a.x = x;
  a.r = vec[0];
  a.r_hat = vec[1];
  a.p[0] = vec[2];
  a.p[1] = vec[3];
  a.u = vec[4];
  a.q = vec[5];
  a.q_hat = vec[6];
  a.invl = invl;
  a.invr = invr;
  a.hist = hist;
  a.sc = sc;
  void* params[] = {&a};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  SK_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&cgs64_kernel), dim3(grid), dim3(kPT), params, 0,
                                      st));
  int err = 0;
  SK_CUDA(cudaMemcpyAsync(&err, &sync->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  if (err) return fail(SK_TIMEOUT, "persistent CGS: a grid barrier wait ran out");
  return SK_OK;
}

bool min64_persistent_ok(sk_matrix A) {
  if (!cg64_persistent_ok(A)) return false;
  return coop_grid(A, reinterpret_cast<const void*>(&min64_kernel)) > 0;
}

sk_status min64_persistent(sk_matrix A, const double* b, double* x, double* const* vec, const double* invl,
                           const double* invr, double* hist, Scalars* sc, void* scratch, cudaStream_t st) {
  SK_CHECK(min64_persistent_ok(A), SK_NOT_SUPPORTED, "persistent MINRES needs a small FP64 CSR handle with SELL-32");
  const auto& C = A->csr;
  int grid = std::min(A->sm_count, kPT);
  const int need = ceil_div(A->nrow, 32);
  if (grid > need) grid = need;
  SyncWords* sync = static_cast<SyncWords*>(scratch);
  double* slots = reinterpret_cast<double*>(static_cast<char*>(scratch) + 256);
  SK_CUDA(cudaMemsetAsync(sync, 0, sizeof(SyncWords), st));
  Min64Args a{};
  a.g.n = static_cast<int>(A->nrow);
  a.g.off = C.sell_off;
  a.g.len = C.sell_len;
  a.g.col = C.sell_col;
  a.g.slots = slots;
  a.g.sync = sync;
  a.g.wait_ns = wait_limit_ns();
  a.g.bias = wait_target_bias();
  a.val = static_cast<const double*>(C.sell_vals);
  a.b = b;
  a.x = x;
  a.v = vec[0];
  a.vp = vec[1];
  a.z = vec[2];
  a.w = vec[3];
  a.q = vec[4];
  a.d = vec[5];
  a.dp = vec[6];
  a.invl = invl;
  a.invr = invr;
  a.hist = hist;
  a.sc = sc;
  void* params[] = {&a};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  SK_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&min64_kernel), dim3(grid), dim3(kPT), params, 0,
                                      st));
  int err = 0;
  SK_CUDA(cudaMemcpyAsync(&err, &sync->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  if (err) return fail(SK_TIMEOUT, "persistent MINRES: a grid barrier wait ran out");
  return SK_OK;
}

}  // namespace sk
