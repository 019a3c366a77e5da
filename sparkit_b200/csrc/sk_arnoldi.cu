// sk_arnoldi.cu -- the modified Gram-Schmidt of one Arnoldi step of
// GMRES(m) / FGMRES(m) as one cooperative launch.
//
// The reference orthogonalizes w = A z_j against v_0 .. v_j one vector at
// a time (fgmres.hpp:259-281, gmres.hpp:259-281): h_ij = <v_i, w>, w -= h_ij
// v_i, and then h_{j+1,j} = ||w||, v_{j+1} = w / h_{j+1,j} (:283-285,
// scale_vector :403-408).  As separate launches that is j + 1 passes each
// reading and writing w.  Here each CTA keeps its rows of w in shared
// memory for the whole step, so w is read once and written once, each v_i
// is read once, and each h is one grid-wide sum behind a bounded grid
// barrier.  The arithmetic of every element is that of the per-vector
// kernels (OpFgMgs, OpFgScale: w - h v in the value type, dot terms summed
// in double); only the order in which the dot products' partial sums meet
// differs.
#include <algorithm>
#include <climits>

#include "sk_arnoldi.cuh"

namespace sk {
namespace {

constexpr int kAT = 512;  // threads per CTA (two CTAs per SM where w fits)
constexpr int kAW = kAT / 32;

__device__ __forceinline__ unsigned long long arn_ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long arn_now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier number `epoch` (from 1) of this launch: passed when the arrival
// counter reaches epoch * gridDim.x (+ bias, which only the timeout tests
// set).  False when a wait ran out here or in another CTA (the error word
// is set); the caller then returns.
__device__ bool arn_barrier(ArnoldiSync* s, unsigned& epoch, unsigned long long wait_ns, unsigned bias) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    epoch += 1;
    const unsigned long long target = static_cast<unsigned long long>(epoch) * gridDim.x + bias;
    asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u64 [%0], 1;" ::"l"(&s->arrived) : "memory");
    unsigned long long t0 = 0;
    for (unsigned spins = 0; arn_ld_acquire(&s->arrived) < target; ++spins) {
      if ((spins & 255u) == 255u) {
        if (*reinterpret_cast<volatile int*>(&s->err) != 0) {
          ok = 0;
          break;
        }
        const unsigned long long t = arn_now_ns();
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

__device__ __forceinline__ double arn_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The grid-wide sum of v, the same bits in every thread of every CTA: a
// block tree, one slot per CTA, a barrier, then every CTA sums the slots in
// CTA order with the same tree.  Consecutive sums alternate slot sets.
__device__ bool arn_allreduce(double& v, double* slots, int set, ArnoldiSync* s, unsigned& epoch,
                              unsigned long long wait_ns, unsigned bias) {
  __shared__ double s_part[kAW];
  __shared__ double s_tot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  v = arn_warp_sum(v);
  if (lane == 0) s_part[warp] = v;
  __syncthreads();
  double* slot = slots + static_cast<size_t>(set) * gridDim.x;
  if (warp == 0) {
    double t = arn_warp_sum(lane < kAW ? s_part[lane] : 0.0);
    if (lane == 0) slot[blockIdx.x] = t;
  }
  if (!arn_barrier(s, epoch, wait_ns, bias)) return false;
  double t = threadIdx.x < gridDim.x ? __ldcg(slot + threadIdx.x) : 0.0;
  t = arn_warp_sum(t);
  if (lane == 0) s_part[warp] = t;
  __syncthreads();
  if (warp == 0) {
    t = arn_warp_sum(lane < kAW ? s_part[lane] : 0.0);
    if (lane == 0) s_tot = t;
  }
  __syncthreads();
  v = s_tot;
  return true;
}

template <typename T>
__global__ void __launch_bounds__(kAT, 2) arnoldi_mgs_kernel(ArnoldiArgs<T> a) {
  extern __shared__ __align__(16) unsigned char arn_smem[];
  T* wt = reinterpret_cast<T*>(arn_smem);
  if (solve_done(a.sc)) return;  // the same flag for every CTA
  const i64 r0 = static_cast<i64>(blockIdx.x) * a.rows_per_cta;
  const i64 r1 = a.n < r0 + a.rows_per_cta ? a.n : r0 + a.rows_per_cta;
  const int cnt = r1 > r0 ? static_cast<int>(r1 - r0) : 0;
  for (int k = threadIdx.x; k < cnt; k += kAT) wt[k] = a.w[r0 + k];
  __syncthreads();
  unsigned epoch = 0;
  double hd = *a.hcol;  // h_{0j}, from the product's epilogue
  for (int i = 0; i <= a.j; ++i) {
    // w -= h_ij v_i; then h_{i+1,j} = <v_{i+1}, w>, or ||w|| at i = j
    const T h = static_cast<T>(hd);
    const T* vi = a.V + static_cast<i64>(i) * a.ldv + r0;
    const T* vn = i < a.j ? a.V + static_cast<i64>(i + 1) * a.ldv + r0 : nullptr;
    double red = 0.0;
    for (int k = threadIdx.x; k < cnt; k += kAT) {
      const T wk = sub(wt[k], mul(h, vi[k]));
      wt[k] = wk;
      red += static_cast<double>(mul(vn ? vn[k] : wk, wk));
    }
    if (!arn_allreduce(red, a.slots, i & 1, a.sync, epoch, a.wait_ns, a.bias)) return;
    const T d = static_cast<T>(red);
    const T hn = vn ? d : sqrt(d);
    hd = static_cast<double>(hn);
    if (blockIdx.x == 0 && threadIdx.x == 0) a.hcol[i + 1] = hd;
  }
  // v_{j+1} = w / h_{j+1,j}, skipped when h_{j+1,j} is not positive
  const T h = static_cast<T>(hd);
  const bool scale = h > T(0);
  const T f = a.divide ? h : T(1) / h;
  for (int k = threadIdx.x; k < cnt; k += kAT) {
    const T wk = wt[k];
    a.w[r0 + k] = scale ? (a.divide ? dvd(wk, f) : mul(wk, f)) : wk;
  }
}

template <typename T>
int arnoldi_grid(const sk_matrix_s* A, i64 n, size_t* smem_out, i64* rows_out) {
  if (n <= 0 || n > INT_MAX) return 0;
  int coop = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, A->device) != cudaSuccess || !coop) return 0;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, A->device) != cudaSuccess) return 0;
  // two CTAs per SM when both fit (twice the warps and half the rows per
  // thread to hide the loads of each basis vector), else one
  for (int per : {2, 1}) {
    const int grid = static_cast<int>(std::min<i64>(static_cast<i64>(per) * A->sm_count, (n + kAT - 1) / kAT));
    const i64 rows = (n + grid - 1) / grid;
    const size_t smem = static_cast<size_t>(rows) * sizeof(T);
    if (smem + 2048 > static_cast<size_t>(optin) || grid > kAT) continue;  // w does not fit on chip
    // The attribute is process-wide: it is always set to the largest size
    // any plan can use, so a plan made on another thread never lowers it
    // below this plan's size between this call and the launch.
    if (cudaFuncSetAttribute(arnoldi_mgs_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - 2048) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, arnoldi_mgs_kernel<T>, kAT, smem) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (per_sm < 1 || grid > per_sm * A->sm_count) continue;
    *smem_out = smem;
    *rows_out = rows;
    return grid;
  }
  return 0;
}

}  // namespace

template <typename T>
bool arnoldi_plan(const sk_matrix_s* A, i64 n, ArnoldiPlan* p) {
  *p = ArnoldiPlan{};
  p->grid = arnoldi_grid<T>(A, n, &p->smem, &p->rows_per_cta);
  return p->grid > 0;
}

template <typename T>
sk_status arnoldi_launch(const ArnoldiPlan& p, ArnoldiArgs<T> a, cudaStream_t st) {
  a.rows_per_cta = p.rows_per_cta;
  a.wait_ns = wait_limit_ns();
  a.bias = wait_target_bias();
  // the step's barriers count from 0; the error word stays for the solve
  SK_CUDA(cudaMemsetAsync(&a.sync->arrived, 0, sizeof(unsigned long long), st));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(p.grid));
  cfg.blockDim = dim3(kAT);
  cfg.dynamicSmemBytes = p.smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  SK_CUDA(cudaLaunchKernelEx(&cfg, arnoldi_mgs_kernel<T>, a));
  return SK_OK;
}

template bool arnoldi_plan<double>(const sk_matrix_s*, i64, ArnoldiPlan*);
template bool arnoldi_plan<float>(const sk_matrix_s*, i64, ArnoldiPlan*);
template sk_status arnoldi_launch<double>(const ArnoldiPlan&, ArnoldiArgs<double>, cudaStream_t);
template sk_status arnoldi_launch<float>(const ArnoldiPlan&, ArnoldiArgs<float>, cudaStream_t);

}  // namespace sk
