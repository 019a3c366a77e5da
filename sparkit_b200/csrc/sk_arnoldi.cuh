// sk_arnoldi.cuh -- the modified Gram-Schmidt of one GMRES / FGMRES Arnoldi
// step as one cooperative launch (sk_arnoldi.cu).
#pragma once

#include "sk_kernels.cuh"

namespace sk {

// Barrier words of the launch: `arrived` is zeroed before every launch; a
// barrier wait that runs out sets `err`, which stays set for the solve.
struct ArnoldiSync {
  unsigned long long arrived;
  int err;
  int pad;
};

// w (= v_{j+1}) holds A z_j and hcol[0] = h_{0j} (the product's epilogue);
// the launch writes hcol[1 .. j+1] and leaves v_{j+1} = w / h_{j+1,j}.
// slots: 2 * grid doubles.
template <typename T>
struct ArnoldiArgs {
  i64 n;
  T* w;
  const T* V;
  i64 ldv;
  int j;
  double* hcol;
  bool divide;  // GMRES divides by h, FGMRES multiplies by 1 / h
  const Scalars* sc;
  ArnoldiSync* sync;
  double* slots;
  i64 rows_per_cta;             // set by arnoldi_launch
  unsigned long long wait_ns;   // bound of each barrier wait, set by arnoldi_launch
  unsigned bias;                // extra arrivals a barrier waits for (timeout tests)
};

struct ArnoldiPlan {
  int grid = 0;
  size_t smem = 0;
  i64 rows_per_cta = 0;
};

// Whether the step fits: a cooperative grid of at most one CTA per SM whose
// CTAs hold their rows of w in shared memory.
template <typename T>
bool arnoldi_plan(const sk_matrix_s* A, i64 n, ArnoldiPlan* p);

// Enqueues the step on st (capturable: a memset of the barrier counter and
// a cooperative kernel launch).
template <typename T>
sk_status arnoldi_launch(const ArnoldiPlan& p, ArnoldiArgs<T> a, cudaStream_t st);

}  // namespace sk
