// sk_mixed.cu -- the FP32 inner solve of the mixed-precision solver as one
// persistent cooperative launch.
//
// No reference counterpart as a whole: the iteration is the reference's
// conjugate gradient (conjugate_gradient.hpp:122-312, Jacobi or identity
// left preconditioner, true residual only at k = 0) in FP32, exactly as the
// per-step path of sk_solvers.cu runs it, but without a kernel boundary per
// step.  One CTA per SM (two over the diagonal copy) stays resident for
// the whole solve; each iteration
// is three phases separated by grid barriers:
//
//   A  q = A p (SELL-32 rows, or the rows of the diagonal copy, each summed
//      in storage order) and <p, q>                               -> alpha
//   B  d += alpha p, r -= alpha q, <r, r> and <r, D^-1 r>          -> test, beta
//   C  p = D^-1 r + beta p
//
// The dot products are reduced deterministically: each CTA publishes its
// partial in a slot before the barrier, and after it every CTA sums all the
// slots in the same fixed order, so every CTA holds the same scalars and
// takes the same convergence decision.  Barrier waits are bounded in time;
// a wait that runs out sets an error word that makes every other CTA leave
// at its next wait, and the host reports SK_TIMEOUT.
//
// The vectors (r, d, p, q and the inverse diagonal, 5 x 4 B per row) stay
// in L2 (a persisting window set by the caller) while the matrix streams
// through it with evict-first loads.
#include <climits>

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
  const int* off;
  const unsigned char* len;
  const int* col;
  const float* val;  // SELL-32 values, or the FP32 values of the diagonal copy
  int dia_n;         // diagonal copy: diagonals, row masks and offsets
  const unsigned short* dia_mask;
  int dia_off[kDiaMax];
  const float* inv_d;
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

// Phase A: q = A p over this thread's rows t0, t0 + T, ... with each row
// summed from 0 in storage order (sparse_blas.hpp:25-28, the order of the
// per-step FP32 product).  Three rows are in flight per thread: the slots
// of row k+2 stream from HBM while the gathers of row k+1 return and row k
// is summed, so neither the matrix stream nor the gathers wait on each
// other.  Returns this thread's share of <p, q>.
__device__ __forceinline__ double phase_spmv(PArgs const& a, int t0, int T) {
  double pq = 0.0;
  // row a: summed this step; row b: slots arrived, gathers issued this
  // step; row c: slots issued this step
  int ia = t0, la, basea, lb, bb, lc, bc;
  float va[kPU], ga[kPU], pa = 0.0f;
  int cb[kPU];
  float vb[kPU];
  row_meta(a, ia, la, basea);
  row_fetch(a, la, basea, 0, cb, vb);
#pragma unroll
  for (int j = 0; j < kPU; ++j) {
    va[j] = vb[j];
    ga[j] = (j < la) ? a.p[cb[j]] : 0.0f;
  }
  if (ia < a.n) pa = a.p[ia];
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
    // gathers of row b
    float gb[kPU];
#pragma unroll
    for (int j = 0; j < kPU; ++j)
      if (j < lb) gb[j] = a.p[cb[j]];
    const int ib = ia + T;
    const float pb = ib < a.n ? a.p[ib] : 0.0f;
    // sum of row a
    float sum = 0.0f;
#pragma unroll
    for (int j = 0; j < kPU; ++j)
      if (j < la) sum = add(sum, mul(va[j], ga[j]));
    for (int k = kPU; k < la; k += kPU) {  // rows longer than kPU slots
      int c[kPU];
      float v[kPU], g[kPU];
      row_fetch(a, la, basea, k, c, v);
#pragma unroll
      for (int j = 0; j < kPU; ++j)
        if (k + j < la) g[j] = a.p[c[j]];
#pragma unroll
      for (int j = 0; j < kPU; ++j)
        if (k + j < la) sum = add(sum, mul(v[j], g[j]));
    }
    a.q[ia] = sum;
    pq += static_cast<double>(mul(pa, sum));
    // rotate a <- b <- c <- d
    ia = ib;
    la = lb;
    basea = bb;
    pa = pb;
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

// Phase A over the diagonal copy.  The values of a warp's rows for one
// diagonal are one 32-value segment and the reads of p at row + off[d] are
// contiguous, so no load depends on another: each thread issues the value
// and p loads of kDiaRows rows for kDiaGroup diagonals at a time without
// waiting for the rows' masks (a diagonal a row does not store reads a zero
// value and a clamped p, and the mask leaves both out of the sum).  The
// kernel runs 2 CTAs per SM here (this phase needs few registers), which
// hides the load latency better than the deeper register pipeline of the
// SELL phase at one CTA per SM.  Each row is summed from 0 over its stored
// diagonals in ascending column order (its CSR order).  Returns this
// thread's share of <p, q>.
constexpr int kDiaRows = 2;
constexpr int kDiaGroup = 4;

__device__ __forceinline__ double phase_spmv_dia(PArgs const& a, int t0, int T) {
  constexpr int R = kDiaRows, C = kDiaGroup;
  double pq = 0.0;
  const int last = a.n - 1;
  const long long sl = 32 * a.dia_n;
  for (int i = t0; i < a.n; i += R * T) {
    unsigned m[R];
    float s[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int row = i + r * T;
      m[r] = row < a.n ? __ldcs(a.dia_mask + row) : 0u;
      s[r] = 0.0f;
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
            g[r][j] = a.p[min(max(row + a.dia_off[d0 + j], 0), last)];
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
      if (row < a.n) {
        a.q[row] = s[r];
        pq += static_cast<double>(mul(a.p[row], s[r]));
      }
    }
  }
  return pq;
}

template <bool JAC, bool DIA>
__global__ void __launch_bounds__(kPT, DIA ? 2 : 1) inner_cg_kernel(PArgs a) {
  const int n = a.n;
  const int T = gridDim.x * kPT;
  const int t0 = blockIdx.x * kPT + threadIdx.x;
  // element-wise phases: four rows per 16-byte access, two accesses per
  // thread and step, rows 4 * n4 .. n - 1 by the first threads
  const int n4 = n >> 2;
  const int tail = 4 * n4 + t0;
  const float4* q4 = reinterpret_cast<const float4*>(a.q);
  const float4* z4 = reinterpret_cast<const float4*>(a.inv_d);
  float4* p4 = reinterpret_cast<float4*>(a.p);
  float4* d4 = reinterpret_cast<float4*>(a.d);
  float4* r4 = reinterpret_cast<float4*>(a.r);
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  unsigned epoch = 0;
  // k = 0 (reorthogonalize, :217-230, with d = 0 so r = r0): z = M r,
  // p = z, rz = <r, z>; and ||r0|| (the solve's ||b||, :194).
  double v0[2] = {0.0, 0.0};
  for (int i = t0; i < n; i += T) {
    const float ri = a.r[i];
    const float zi = JAC ? mul(a.inv_d[i], ri) : ri;
    a.d[i] = 0.0f;
    a.p[i] = zi;
    v0[0] += static_cast<double>(mul(ri, zi));
    v0[1] += static_cast<double>(mul(ri, ri));
  }
  if (!grid_allreduce<2>(v0, a, 0, epoch)) return;
  const float bnorm = sqrtf(static_cast<float>(v0[1]));
  float rz = static_cast<float>(v0[0]);
  long long it = 0;
  int conv = 0;
  float rn = bnorm;
  if (bnorm == 0.0f) conv = 1;
  while (!conv && it < a.max_iters) {
    // A: compute_step_size (:233-239)
    double pq[1];
    if constexpr (DIA) pq[0] = phase_spmv_dia(a, t0, T);
    else pq[0] = phase_spmv(a, t0, T);
    if (!grid_allreduce<1>(pq, a, 1, epoch)) return;
    const float alpha = rz / static_cast<float>(pq[0]);
    // B: compute_new_solution, compute_new_residual, is_converged
    // (:242-276) and the new <r, z> (:279-284)
    double rr[2] = {0.0, 0.0};
    auto upd = [&](float pi, float qi, float di, float ro, float zi, float& dn, float& rnew) {
      dn = add(mul(alpha, pi), di);
      rnew = sub(ro, mul(alpha, qi));
      rr[0] += static_cast<double>(mul(rnew, rnew));
      if (JAC) rr[1] += static_cast<double>(mul(rnew, mul(zi, rnew)));
    };
    auto upd4 = [&](float4 pv, float4 qv, float4 dv, float4 rv, float4 zv, float4& dn, float4& rw) {
      upd(pv.x, qv.x, dv.x, rv.x, zv.x, dn.x, rw.x);
      upd(pv.y, qv.y, dv.y, rv.y, zv.y, dn.y, rw.y);
      upd(pv.z, qv.z, dv.z, rv.z, zv.z, dn.z, rw.z);
      upd(pv.w, qv.w, dv.w, rv.w, zv.w, dn.w, rw.w);
    };
    int j = t0;
    for (; j + T < n4; j += 2 * T) {
      const int j1 = j + T;
      const float4 pv0 = p4[j], qv0 = q4[j], dv0 = d4[j], rv0 = r4[j];
      const float4 pv1 = p4[j1], qv1 = q4[j1], dv1 = d4[j1], rv1 = r4[j1];
      const float4 zv0 = JAC ? z4[j] : zero4, zv1 = JAC ? z4[j1] : zero4;
      float4 dn0, rw0, dn1, rw1;
      upd4(pv0, qv0, dv0, rv0, zv0, dn0, rw0);
      upd4(pv1, qv1, dv1, rv1, zv1, dn1, rw1);
      d4[j] = dn0;
      r4[j] = rw0;
      d4[j1] = dn1;
      r4[j1] = rw1;
    }
    if (j < n4) {
      float4 dn, rw;
      upd4(p4[j], q4[j], d4[j], r4[j], JAC ? z4[j] : zero4, dn, rw);
      d4[j] = dn;
      r4[j] = rw;
    }
    if (tail < n) {
      float dn, rw;
      upd(a.p[tail], a.q[tail], a.d[tail], a.r[tail], JAC ? a.inv_d[tail] : 0.f, dn, rw);
      a.d[tail] = dn;
      a.r[tail] = rw;
    }
    if (!grid_allreduce<2>(rr, a, 0, epoch)) return;
    ++it;
    rn = sqrtf(static_cast<float>(rr[0]));
    conv = rn / bnorm < a.tol ? 1 : 0;
    if (conv || it >= a.max_iters) break;
    const float rz_new = static_cast<float>(JAC ? rr[1] : rr[0]);
    const float beta = rz_new / rz;
    rz = rz_new;
    // C: update_direction (:285-290)
    auto dir = [&](float ri, float zi, float pi) { return add(JAC ? mul(zi, ri) : ri, mul(beta, pi)); };
    auto dir4 = [&](float4 rv, float4 zv, float4 pv) {
      return make_float4(dir(rv.x, zv.x, pv.x), dir(rv.y, zv.y, pv.y), dir(rv.z, zv.z, pv.z),
                         dir(rv.w, zv.w, pv.w));
    };
    j = t0;
    for (; j + T < n4; j += 2 * T) {
      const int j1 = j + T;
      const float4 rv0 = r4[j], pv0 = p4[j], rv1 = r4[j1], pv1 = p4[j1];
      const float4 zv0 = JAC ? z4[j] : zero4, zv1 = JAC ? z4[j1] : zero4;
      p4[j] = dir4(rv0, zv0, pv0);
      p4[j1] = dir4(rv1, zv1, pv1);
    }
    if (j < n4) p4[j] = dir4(r4[j], JAC ? z4[j] : zero4, p4[j]);
    if (tail < n) a.p[tail] = dir(a.r[tail], JAC ? a.inv_d[tail] : 0.f, a.p[tail]);
    if (!grid_barrier(a.sync, epoch, a.wait_ns, a.bias)) return;
  }

  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.sync->iterations = it;
    a.sync->converged = conv;
    a.sync->rnorm = static_cast<double>(rn);
  }
}

// The handle's diagonal copy when it has FP32 values, else its SELL copy.
bool use_dia(sk_matrix A) { return A->csr.dia_n > 0 && A->csr.dia_vals32; }

const void* pick_kernel(bool jac, bool dia) {
  if (dia)
    return jac ? reinterpret_cast<const void*>(&inner_cg_kernel<true, true>)
               : reinterpret_cast<const void*>(&inner_cg_kernel<false, true>);
  return jac ? reinterpret_cast<const void*>(&inner_cg_kernel<true, false>)
             : reinterpret_cast<const void*>(&inner_cg_kernel<false, false>);
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

}  // namespace

bool inner_persistent_ok(sk_matrix A) {
  if (!A || A->format != SK_CSR || A->nrow <= 0) return false;
  if (!use_dia(A) && !(A->csr.sell && A->csr.sell_vals32)) return false;
  if (A->nrow > INT_MAX / 4) return false;
  int coop = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, A->device) != cudaSuccess || !coop) return false;
  return coop_grid(A, pick_kernel(true, use_dia(A))) > 0 && coop_grid(A, pick_kernel(false, use_dia(A))) > 0;
}

size_t inner_persistent_scratch(sk_matrix A) {
  return sizeof(SyncWords) + static_cast<size_t>(2) * kPT * kSlot * sizeof(double) + 256;
}

sk_status inner_cg_persistent(sk_matrix A, const float* inv_d, float* r, float* d, float* p, float* q,
                              void* scratch, double tol, long long max_iters, cudaStream_t st,
                              InnerResult* out) {
  *out = InnerResult{};
  SK_CHECK(inner_persistent_ok(A), SK_NOT_SUPPORTED,
           "persistent inner solve needs a CSR handle with FP32 SELL values or an FP32 diagonal copy");
  const bool dia = use_dia(A);
  const void* k = pick_kernel(inv_d != nullptr, dia);
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
  if (dia) {
    a.val = A->csr.dia_vals32;
    a.dia_n = A->csr.dia_n;
    a.dia_mask = A->csr.dia_mask;
    for (int d = 0; d < kDiaMax; ++d) a.dia_off[d] = A->csr.dia_off[d];
  } else {
    a.off = A->csr.sell_off;
    a.len = A->csr.sell_len;
    a.col = A->csr.sell_col;
    a.val = A->csr.sell_vals32;
  }
  a.inv_d = inv_d;
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

}  // namespace sk
