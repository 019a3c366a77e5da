// sk_solvers.cu -- conjugate gradient, BiCGSTAB and FGMRES(m) on the
// device.  The whole iteration stays on the GPU: scalars (alpha, beta,
// rho, ...) live in device memory and are produced by the finalize step of
// the fused kernel that computes them; a converged or exhausted solve sets
// a `done` flag that turns every later kernel into a no-op.  The host
// enqueues iterations in chunks and reads the flag back once per chunk
// (CG, BiCGSTAB) or once per restart cycle (FGMRES).
//
// Each solver follows its reference template step for step (cited per
// kernel), with the reference's element-wise arithmetic order; only the
// dot products are summed in a different (fixed, deterministic) order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <type_traits>
#include <vector>

#include "sk_arnoldi.cuh"
#include "sk_learned.cuh"
#include "sk_vec.cuh"
#include "sk_mixed.cuh"

namespace sk {

void precond_apply_dispatch(const sk_precond_s* M, sk_dtype dt, i64 n, const void* r, void* z,
                            RedWs ws, const Scalars* sc, cudaStream_t st);

enum { PK_IDENTITY = 0, PK_JACOBI = 1, PK_OTHER = 2 };

// The dtype of a solve's vectors (an FP64 handle runs FP32 vectors in the
// mixed-precision solvers).
template <typename T>
constexpr sk_dtype kVecType = sizeof(T) == 8 ? SK_F64 : SK_F32;

inline int prec_kind(const sk_precond_s* M) {
  if (!M) return PK_IDENTITY;
  return M->kind == 1 ? PK_JACOBI : PK_OTHER;
}

// ------------------------------------------------------------------
// Step chunks as CUDA graphs.  Once a solve has run its first chunks
// directly, each later chunk of `len` steps (the same launches with the
// same arguments every time: the kernels read their scalars from device
// memory and turn into no-ops once the solve is done) is captured once and
// then replayed, one graph launch per chunk instead of one host launch per
// kernel.  Preconditioners whose apply does host work (the learned network,
// the two-level form) keep the direct launches.
// ------------------------------------------------------------------
struct StepGraph {
  cudaGraphExec_t exec = nullptr;
  i64 len = 0;
  i64 launches = 0;
  StepGraph() = default;
  StepGraph(StepGraph const&) = delete;
  StepGraph& operator=(StepGraph const&) = delete;
  ~StepGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
  // Enqueues `n_steps` steps on gs through the graph (captured on first use
  // or when the chunk length changes); enqueue(n) issues n steps on gs.
  template <class F>
  sk_status replay(cudaStream_t gs, i64 n_steps, F const& enqueue) {
    if (!exec || len != n_steps) {
      if (exec) cudaGraphExecDestroy(exec);
      exec = nullptr;
      const i64 before = g_launches.load();
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        enqueue(n_steps);
        e = cudaStreamEndCapture(gs, &g);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        exec = nullptr;
        return cuda_fail(e, "solver step capture");
      }
      launches = g_launches.load() - before;
      g_launches.fetch_sub(launches);  // counted at each replay instead
      len = n_steps;
    }
    g_launches.fetch_add(launches);
    SK_CUDA(cudaGraphLaunch(exec, gs));
    return SK_OK;
  }
};

// Whether a preconditioner's apply is device launches only (none, Jacobi,
// Chebyshev), so that its steps can be captured.
inline bool capturable(const sk_precond_s* M) { return !M || M->kind == 1 || M->kind == 2; }

// The stream a solve with captured chunks runs on: the caller's, unless it
// is a default stream (the legacy stream cannot be captured), in which case
// the caller's stream is drained and the handle's own stream is used.  The
// solve's last host read synchronizes that stream, so the caller sees the
// results in order.
static sk_status solve_stream(sk_matrix A, cudaStream_t st, cudaStream_t* gs) {
  *gs = st;
  if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread) {
    SK_CUDA(cudaStreamSynchronize(st));
    *gs = A->stream;
  }
  return SK_OK;
}

// ------------------------------------------------------------------
// Workspace carved out of the handle's grow-only buffer.
// ------------------------------------------------------------------
struct Carver {
  char* base;
  size_t off = 0;
  template <typename P>
  P* take(size_t bytes) {
    off = (off + 255) & ~size_t(255);
    P* p = reinterpret_cast<P*>(base + off);
    off += bytes;
    return p;
  }
};

static sk_status ensure_ws(sk_matrix A, size_t bytes) {
  if (A->ws_bytes >= bytes) return SK_OK;
  if (A->ws) {
    cudaStreamSynchronize(A->stream);
    cudaFree(A->ws);
    A->ws = nullptr;
    A->ws_bytes = 0;
  }
  SK_CUDA(cudaMalloc(&A->ws, bytes));
  A->ws_bytes = bytes;
  return SK_OK;
}

struct SolveCommon {
  Scalars* sc;
  RedWs ws;
  double* hist;
  size_t used;
};

// Reserves scalars, the reduction slots and the history buffer, then
// `nvec` n-vectors of `vb` bytes each plus `extra` bytes.
static size_t common_bytes(sk_matrix A, i64 nvec, size_t vb, size_t extra, i64 hist_cap) {
  const int cap = std::max(spmv_grid(A), vec_grid(A->nrow));
  return 4096 + sizeof(Scalars) + 256 + static_cast<size_t>(cap) * kMaxRed * 8 +
         static_cast<size_t>(hist_cap + 8) * 8 + static_cast<size_t>(nvec) * (vb + 256) + extra + 1024;
}

// Terms of the sequential summation order: kMaxRed per row.
static size_t seq_bytes(sk_matrix A) { return static_cast<size_t>(kMaxRed) * (A->nrow + 8) * 8 + 256; }

// Carves from `base` when given (the caller sized it with common_bytes),
// else from the handle's grow-only workspace.
static sk_status carve_common(sk_matrix A, cudaStream_t st, i64 nvec, size_t vb, size_t extra,
                              i64 hist_cap, SolveCommon* c, std::vector<char*>* vecs,
                              char** extra_ptr, char* base = nullptr) {
  const int cap = std::max(spmv_grid(A), vec_grid(A->nrow));
  // the sequential order applies to the solves that use the handle's own
  // workspace (the reference's solvers), not to a caller-sized region
  const bool seq = !base && summation_sequential();
  if (!base) {
    sk_status s = ensure_ws(A, common_bytes(A, nvec, vb, extra, hist_cap) + (seq ? seq_bytes(A) : 0));
    if (s != SK_OK) return s;
    base = static_cast<char*>(A->ws);
  }
  Carver cv{base};
  c->sc = cv.take<Scalars>(sizeof(Scalars));
  c->ws.counter = cv.take<unsigned>(sizeof(unsigned) * 4);
  c->ws.partials = cv.take<double>(static_cast<size_t>(cap) * kMaxRed * 8);
  c->ws.capacity = cap;
  c->hist = cv.take<double>(static_cast<size_t>(hist_cap + 8) * 8);
  for (i64 k = 0; k < nvec; ++k) vecs->push_back(cv.take<char>(vb));
  if (extra_ptr) *extra_ptr = cv.take<char>(extra);
  if (seq) {
    c->ws.seq = cv.take<double>(seq_bytes(A));
    c->ws.seq_ld = A->nrow + 8;
    c->ws.seq_n = A->nrow;
    c->ws.seq_f32 = A->dtype == SK_F32 ? 1 : 0;
  }
  c->used = cv.off;
  SK_CUDA(cudaMemsetAsync(c->sc, 0, sizeof(Scalars), st));
  SK_CUDA(cudaMemsetAsync(c->ws.counter, 0, sizeof(unsigned) * 4, st));
  return SK_OK;
}

static sk_status finish_summary(SolveCommon const& c, cudaStream_t st, sk_summary* out,
                                double* history_host) {
  Scalars h;
  SK_CUDA(cudaMemcpyAsync(&h, c.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  out->residual_norm = h.rnorm;
  out->computed_iterations = h.iters;
  out->converged = h.converged;
  out->status = h.status;
  out->history_length = h.hist_on ? h.hist_len : 0;
  if (history_host && h.hist_on && h.hist_len > 0)
    SK_CUDA(cudaMemcpy(history_host, c.hist, h.hist_len * sizeof(double), cudaMemcpyDeviceToHost));
  return SK_OK;
}

static sk_status read_scalars(Scalars const* d, Scalars* h, cudaStream_t st) {
  SK_CUDA(cudaMemcpyAsync(h, d, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
  SK_CUDA(cudaStreamSynchronize(st));
  return SK_OK;
}

// Writes initial scalars from the host.
static sk_status put_scalars(Scalars* d, Scalars const& h, cudaStream_t st) {
  SK_CUDA(cudaMemcpyAsync(d, &h, sizeof(Scalars), cudaMemcpyHostToDevice, st));
  return SK_OK;
}

__device__ __forceinline__ void record(Scalars* sc, double* hist, double v) {
  sc->rnorm = v;
  if (sc->hist_on) hist[sc->hist_len++] = v;
}

// ||b|| (conjugate_gradient.hpp:194, bicgstab.hpp:160, fgmres.hpp:168)
template <typename T>
struct OpNormB {
  static constexpr int kNR = 1;
  const T* b;
  Scalars* sc;
  struct In { T b; };
  __device__ bool prepare(const Scalars*) { return true; }
  __device__ In load(i64 i) const { return {b[i]}; }
  __device__ void apply(i64, In const& v, double* red) const { red[0] += static_cast<double>(mul(v.b, v.b)); }
  __device__ void finalize(const double* t) const {
    sc->bnorm = static_cast<double>(sqrt(static_cast<T>(t[0])));
  }
};

template <typename T>
static sk_status norm_b(const T* b, i64 n, SolveCommon const& c, cudaStream_t st, double* bnorm) {
  launch_vec(n, OpNormB<T>{b, c.sc}, c.ws, nullptr, st);
  SK_CUDA(cudaGetLastError());
  Scalars h;
  sk_status s = read_scalars(c.sc, &h, st);
  if (s != SK_OK) return s;
  *bnorm = h.bnorm;
  return SK_OK;
}

// ==================================================================
// Conjugate gradient, conjugate_gradient.hpp:122-312
// ==================================================================

// reorthogonalize (:217-230): r = b - A x; z = M_L r; rz = <r, z>; p = z.
// The identity and Jacobi left preconditioners are fused into the epilogue.
template <typename T, int LK>
struct EpiCgResid {
  static constexpr int kNR = LK == PK_OTHER ? 0 : 1;
  const T* b;
  T* r;
  T* p;
  const T* inv_d;
  Scalars* sc;
  __device__ void operator()(int row, T ax, double* red) const {
    const T ri = sub(b[row], ax);
    r[row] = ri;
    if constexpr (LK == PK_IDENTITY) {
      p[row] = ri;
      red[0] += static_cast<double>(mul(ri, ri));
    } else if constexpr (LK == PK_JACOBI) {
      const T zi = mul(inv_d[row], ri);
      p[row] = zi;
      red[0] += static_cast<double>(mul(ri, zi));
    }
  }
  __device__ void finalize(const double* t) const {
    if constexpr (kNR > 0) sc->rz = static_cast<double>(static_cast<T>(t[0]));
  }
};

// rz = <r, z>; p = z  (left preconditioner applied separately)
template <typename T>
struct OpCgReorthDot {
  static constexpr int kNR = 1;
  const T* r;
  const T* z;
  T* p;
  Scalars* sc;
  struct In { T r, z; };
  __device__ bool prepare(const Scalars* s) { return !solve_done(s); }
  __device__ In load(i64 i) const { return {r[i], z[i]}; }
  __device__ void apply(i64 i, In const& v, double* red) const {
    p[i] = v.z;
    red[0] += static_cast<double>(mul(v.r, v.z));
  }
  __device__ void finalize(const double* t) const { sc->rz = static_cast<double>(static_cast<T>(t[0])); }
};

// compute_step_size (:233-239): q = A p_hat; alpha = rz / <p, q>.
template <typename T>
struct EpiCgPq {
  static constexpr int kNR = 1;
  T* q;
  const T* p;
  Scalars* sc;
  __device__ void operator()(int row, T v, double* red) const {
    q[row] = v;
    red[0] += static_cast<double>(mul(p[row], v));
  }
  __device__ void finalize(const double* t) const {
    sc->alpha = static_cast<double>(static_cast<T>(sc->rz) / static_cast<T>(t[0]));
  }
};

// compute_new_solution (:242-249), compute_new_residual (:252-259),
// is_converged (:262-276), and for identity / Jacobi left preconditioners
// the <r, z> of update_direction (:279-284).
template <typename T, int LK>
struct OpCgUpdate {
  static constexpr int kNR = LK == PK_JACOBI ? 2 : 1;
  T* x;
  T* r;
  const T* hatp;
  const T* q;
  const T* inv_d;
  Scalars* sc;
  double* hist;
  T alpha;
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    alpha = static_cast<T>(s->alpha);
    return true;
  }
  struct In { T x, h, r, q, d; };
  __device__ In load(i64 i) const {
    return {x[i], hatp[i], r[i], q[i], LK == PK_JACOBI ? inv_d[i] : T(0)};
  }
  __device__ void apply(i64 i, In const& v, double* red) const {
    x[i] = add(mul(alpha, v.h), v.x);
    const T ri = sub(v.r, mul(alpha, v.q));
    r[i] = ri;
    red[0] += static_cast<double>(mul(ri, ri));
    if constexpr (LK == PK_JACOBI) red[1] += static_cast<double>(mul(ri, mul(v.d, ri)));
  }
  __device__ void finalize(const double* t) const {
    sc->iters += 1;
    const T rn = sqrt(static_cast<T>(t[0]));
    record(sc, hist, static_cast<double>(rn));
    const bool conv = rn / static_cast<T>(sc->bnorm) < static_cast<T>(sc->tol);
    sc->converged = conv ? 1 : 0;
    if (conv || sc->iters >= sc->max_iters) sc->done = 1;
    if (LK != PK_OTHER && !conv) {
      const T rz_new = static_cast<T>(LK == PK_JACOBI ? t[1] : t[0]);
      sc->beta = static_cast<double>(rz_new / static_cast<T>(sc->rz));
      sc->rz = static_cast<double>(rz_new);
    }
  }
};

// update_direction with a separately applied left preconditioner:
// beta = <r, z>_new / rz.
template <typename T>
struct OpCgBeta {
  static constexpr int kNR = 1;
  const T* r;
  const T* z;
  Scalars* sc;
  struct In { T r, z; };
  __device__ bool prepare(const Scalars* s) { return !solve_done(s); }
  __device__ In load(i64 i) const { return {r[i], z[i]}; }
  __device__ void apply(i64, In const& v, double* red) const { red[0] += static_cast<double>(mul(v.r, v.z)); }
  __device__ void finalize(const double* t) const {
    const T rz_new = static_cast<T>(t[0]);
    sc->beta = static_cast<double>(rz_new / static_cast<T>(sc->rz));
    sc->rz = static_cast<double>(rz_new);
  }
};

// p = z + beta p (:285-290), z recomputed in registers for identity/Jacobi.
template <typename T, int LK>
struct OpCgDirection {
  static constexpr int kNR = 0;
  T* p;
  const T* r;
  const T* z;
  const T* inv_d;
  T beta;
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    beta = static_cast<T>(s->beta);
    return true;
  }
  struct In { T z, p; };
  __device__ In load(i64 i) const {
    T zi;
    if constexpr (LK == PK_IDENTITY) zi = r[i];
    else if constexpr (LK == PK_JACOBI) zi = mul(inv_d[i], r[i]);
    else zi = z[i];
    return {zi, p[i]};
  }
  __device__ void apply(i64 i, In const& v, double*) const { p[i] = add(v.z, mul(beta, v.p)); }
  __device__ void finalize(const double*) const {}
};

// One CG iteration.  `vals` (may be null) replaces the handle's values:
// the mixed-precision solver runs T = float over the FP32 value copy of an
// FP64 handle; its preconditioner is then identity or an FP32 Jacobi.
template <typename T, int LK>
static void cg_iteration(sk_matrix A, const sk_precond_s* L, const sk_precond_s* R, bool reorth,
                         const T* b, T* x, T* r, T* z, T* p, T* hatp, T* q, SolveCommon const& c,
                         cudaStream_t st, const T* vals) {
  const i64 n = A->nrow;
  const sk_dtype dt = sizeof(T) == 8 ? SK_F64 : SK_F32;
  const T* invL = L && L->kind == 1 ? static_cast<const T*>(L->inv_diag) : nullptr;
  if (reorth) {
    launch_spmv<T>(A, x, EpiCgResid<T, LK>{b, r, p, invL, c.sc}, c.ws, c.sc, st, vals);
    if constexpr (LK == PK_OTHER) {
      precond_apply_dispatch(L, dt, n, r, z, c.ws, c.sc, st);
      launch_vec(n, OpCgReorthDot<T>{r, z, p, c.sc}, c.ws, c.sc, st);
    }
  }
  const T* ph = p;
  if (R) {
    precond_apply_dispatch(R, dt, n, p, hatp, c.ws, c.sc, st);
    ph = hatp;
  }
  launch_spmv<T>(A, ph, EpiCgPq<T>{q, p, c.sc}, c.ws, c.sc, st, vals);
  launch_vec(n, OpCgUpdate<T, LK>{x, r, ph, q, invL, c.sc, c.hist, T(0)}, c.ws, c.sc, st);
  if constexpr (LK == PK_OTHER) {
    precond_apply_dispatch(L, dt, n, r, z, c.ws, c.sc, st);
    launch_vec(n, OpCgBeta<T>{r, z, c.sc}, c.ws, c.sc, st);
  }
  launch_vec(n, OpCgDirection<T, LK>{p, r, z, invL, T(0)}, c.ws, c.sc, st);
}

template <typename T>
static sk_status cg_solve(sk_matrix A, sk_precond L, sk_precond R, const T* b, T* x,
                          const sk_cg_config* cfg, sk_summary* out, double* history_host,
                          cudaStream_t st, const T* vals = nullptr, char* ws_base = nullptr) {
  Range range_("sk conjugate_gradient");
  const i64 n = A->nrow;
  const size_t vb = static_cast<size_t>(n + 8) * sizeof(T);
  SolveCommon c;
  std::vector<char*> v;
  const i64 hist_cap = cfg->collect_residuals ? cfg->max_iterations : 0;
  // small FP64 systems with a Jacobi or identity left preconditioner and
  // no restart before the last step: the whole solve in one cooperative
  // launch (sk_mixed.cu), where three kernels per step would be bound by
  // launch and reduction latency
  const bool cg64 = std::is_same<T, double>::value && !vals && !ws_base && !R &&
                    (!L || L->kind == 1) && cfg->restart_iterations >= cfg->max_iterations &&
                    cg64_persistent_ok(A);
  const size_t pextra = cg64 ? (inner_persistent_scratch(A) + 511) & ~size_t(511) : 0;
  char* pscratch = nullptr;
  sk_status s = carve_common(A, st, 5, vb, pextra, hist_cap, &c, &v, cg64 ? &pscratch : nullptr, ws_base);
  if (s != SK_OK) return s;
  T *r = (T*)v[0], *z = (T*)v[1], *p = (T*)v[2], *hatp = (T*)v[3], *q = (T*)v[4];
  *out = sk_summary{};
  double bnorm = 0;
  if ((s = norm_b<T>(b, n, c, st, &bnorm)) != SK_OK) return s;
  if (bnorm == 0.0) {  // :195-199
    SK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), st));
    SK_CUDA(cudaStreamSynchronize(st));
    out->converged = 1;
    return SK_OK;
  }
  Scalars h{};
  h.bnorm = bnorm;
  h.tol = cfg->tolerance;
  h.max_iters = cfg->max_iterations;
  h.hist_on = cfg->collect_residuals ? 1 : 0;
  if ((s = put_scalars(c.sc, h, st)) != SK_OK) return s;
  const int lk = prec_kind(L);
  if constexpr (std::is_same<T, double>::value) {
    if (cg64) {
      const double* invd = L ? static_cast<const double*>(L->inv_diag) : nullptr;
      if ((s = cg64_persistent(A, b, x, r, p, hatp, q, invd, cfg->collect_residuals ? c.hist : nullptr, c.sc,
                               pscratch, st)) != SK_OK)
        return s;
      return finish_summary(c, st, out, history_host);
    }
  }
  const bool graphs = capturable(L) && capturable(R);
  if (graphs && (s = solve_stream(A, st, &st)) != SK_OK) return s;
  auto steps = [&](i64 k0, i64 cnt) {
    for (i64 j = 0; j < cnt; ++j) {
      const bool reorth = ((k0 + j) % cfg->restart_iterations) == 0;
      if (lk == PK_IDENTITY)
        cg_iteration<T, PK_IDENTITY>(A, L, R, reorth, b, x, r, z, p, hatp, q, c, st, vals);
      else if (lk == PK_JACOBI)
        cg_iteration<T, PK_JACOBI>(A, L, R, reorth, b, x, r, z, p, hatp, q, c, st, vals);
      else
        cg_iteration<T, PK_OTHER>(A, L, R, reorth, b, x, r, z, p, hatp, q, c, st, vals);
    }
  };
  StepGraph sg;
  constexpr i64 kMaxChunk = 64;
  i64 k = 0, chunk = 8;
  while (k < cfg->max_iterations) {
    const i64 todo = std::min(chunk, cfg->max_iterations - k);
    // a chunk without a true-residual step (k % restart_iterations == 0)
    // repeats the same launches and is replayed from its graph
    const i64 next_reorth = (k + cfg->restart_iterations - 1) / cfg->restart_iterations * cfg->restart_iterations;
    if (graphs && todo == kMaxChunk && next_reorth >= k + todo) {
      if ((s = sg.replay(st, todo, [&](i64 cnt) { steps(k, cnt); })) != SK_OK) return s;
    } else {
      steps(k, todo);
    }
    k += todo;
    SK_CUDA(cudaGetLastError());
    if ((s = read_scalars(c.sc, &h, st)) != SK_OK) return s;
    if (h.done) break;
    chunk = std::min<i64>(chunk * 2, kMaxChunk);
  }
  return finish_summary(c, st, out, history_host);
}

// ==================================================================
// BiCGSTAB, bicgstab.hpp:93-361
// ==================================================================

// compute_initial_residual (:186-194), initialize_shadow_residual (:197),
// and the first rho_new = <r_hat, r> (:203).
template <typename T>
struct EpiBiResid {
  static constexpr int kNR = 1;
  const T* b;
  T* r;
  T* r_hat;
  Scalars* sc;
  __device__ void operator()(int row, T ax, double* red) const {
    const T ri = sub(b[row], ax);
    r[row] = ri;
    r_hat[row] = ri;
    red[0] += static_cast<double>(mul(ri, ri));
  }
  __device__ void finalize(const double* t) const {
    sc->rho_new = static_cast<double>(static_cast<T>(t[0]));
    sc->rho = sc->alpha = sc->omega = 1.0;
    if (sc->max_iters <= 0) {
      sc->done = 1;
    } else if (static_cast<T>(sc->rho_new) == T(0)) {
      // rho_0 = <r_0, r_0> = 0: the initial guess solves the system.  The
      // reference returns from every step here without using budget and
      // spins forever (:203-204); this solve ends converged with 0
      // iterations, as FGMRES does for a zero initial residual.
      sc->converged = 1;
      sc->done = 1;
    }
  }
};

// update_search_direction (:233-238) and, for identity / Jacobi
// preconditioners, apply_preconditioner_to_p (:241-244) in registers.
template <typename T, int LK, int RK>
struct OpBiP {
  static constexpr int kNR = 0;
  T* p;
  const T* r;
  const T* v;
  T* p_hat;
  const T* invL;
  const T* invR;
  T beta, omega;
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    const T rho_new = static_cast<T>(s->rho_new);
    omega = static_cast<T>(s->omega);
    beta = (rho_new / static_cast<T>(s->rho)) * (static_cast<T>(s->alpha) / omega);
    return true;
  }
  struct In { T r, p, v, dl, dr; };
  __device__ In load(i64 i) const {
    return {r[i], p[i], v[i], LK == PK_JACOBI ? invL[i] : T(0), RK == PK_JACOBI ? invR[i] : T(0)};
  }
  __device__ void apply(i64 i, In const& q, double*) const {
    const T pi = add(q.r, mul(beta, sub(q.p, mul(omega, q.v))));
    p[i] = pi;
    if constexpr (LK != PK_OTHER && RK != PK_OTHER) {
      T t = pi;
      if constexpr (LK == PK_JACOBI) t = mul(q.dl, t);
      if constexpr (RK == PK_JACOBI) t = mul(q.dr, t);
      p_hat[i] = t;
    }
  }
  __device__ void finalize(const double*) const {}
};

// compute_v (:247-250) and alpha = rho_new / <r_hat, v> (:211).
template <typename T>
struct EpiBiV {
  static constexpr int kNR = 1;
  T* v;
  const T* r_hat;
  Scalars* sc;
  __device__ void operator()(int row, T val, double* red) const {
    v[row] = val;
    red[0] += static_cast<double>(mul(r_hat[row], val));
  }
  __device__ void finalize(const double* t) const {
    sc->iters += 1;
    const T rv = static_cast<T>(t[0]);
    if (rv == T(0)) {
      // <r_hat, v> = 0: the reference divides by it (:211) and runs the
      // rest of its budget on infinities and NaNs, ending unconverged; this
      // solve ends unconverged here with SK_BREAKDOWN.
      sc->status = SK_BREAKDOWN;
      sc->done = 1;
      return;
    }
    sc->alpha = static_cast<double>(static_cast<T>(sc->rho_new) / rv);
  }
};

// compute_s (:253-258) and check_half_step_convergence (:261-268).
template <typename T>
struct OpBiS {
  static constexpr int kNR = 1;
  T* s;
  const T* r;
  const T* v;
  Scalars* sc;
  double* hist;
  T alpha;
  __device__ bool prepare(const Scalars* st) {
    if (solve_done(st)) return false;
    alpha = static_cast<T>(st->alpha);
    return true;
  }
  struct In { T r, v; };
  __device__ In load(i64 i) const { return {r[i], v[i]}; }
  __device__ void apply(i64 i, In const& q, double* red) const {
    const T si = sub(q.r, mul(alpha, q.v));
    s[i] = si;
    red[0] += static_cast<double>(mul(si, si));
  }
  __device__ void finalize(const double* t) const {
    const T sn = sqrt(static_cast<T>(t[0]));
    record(sc, hist, static_cast<double>(sn));
    if (sn / static_cast<T>(sc->bnorm) < static_cast<T>(sc->tol)) {
      sc->half = 1;
      sc->converged = 1;
      sc->done = 1;
    }
  }
};

// Either update_solution_half_step (:270-278) when the half step
// converged, or apply_preconditioner_to_s (:281-284) for identity / Jacobi.
template <typename T, int LK, int RK>
struct OpBiHalfOrS {
  static constexpr int kNR = 1;  // only to get a finalize that clears `half`
  T* x;
  const T* p_hat;
  const T* s;
  T* s_hat;
  const T* invL;
  const T* invR;
  Scalars* sc;
  T alpha;
  int mode;  // 1 = half-step x update, 2 = s_hat
  __device__ bool prepare(const Scalars* st) {
    if (st->half) {
      mode = 1;
      alpha = static_cast<T>(st->alpha);
      return true;
    }
    if (solve_done(st)) return false;
    mode = 2;
    return LK != PK_OTHER && RK != PK_OTHER;
  }
  struct In { T a, b, dl, dr; };
  __device__ In load(i64 i) const {
    if (mode == 1) return {x[i], p_hat[i], T(0), T(0)};
    return {s[i], T(0), LK == PK_JACOBI ? invL[i] : T(0), RK == PK_JACOBI ? invR[i] : T(0)};
  }
  __device__ void apply(i64 i, In const& q, double*) const {
    if (mode == 1) {
      x[i] = add(q.a, mul(alpha, q.b));
    } else if constexpr (LK != PK_OTHER && RK != PK_OTHER) {
      T t = q.a;
      if constexpr (LK == PK_JACOBI) t = mul(q.dl, t);
      if constexpr (RK == PK_JACOBI) t = mul(q.dr, t);
      s_hat[i] = t;
    }
  }
  __device__ void finalize(const double*) const {
    if (mode == 1) sc->half = 0;
  }
};

// compute_t (:287-290) and compute_omega (:293-297).
template <typename T>
struct EpiBiT {
  static constexpr int kNR = 2;
  T* t;
  const T* s;
  Scalars* sc;
  __device__ void operator()(int row, T val, double* red) const {
    t[row] = val;
    red[0] += static_cast<double>(mul(val, val));
    red[1] += static_cast<double>(mul(val, s[row]));
  }
  __device__ void finalize(const double* tot) const {
    sc->iters += 1;
    const T tt = static_cast<T>(tot[0]);
    const T om = tt == T(0) ? T(0) : static_cast<T>(tot[1]) / tt;
    sc->omega = static_cast<double>(om);
    if (om == T(0)) {  // :223, step ends without the full update
      sc->skip = 1;
    }
  }
};

// update_solution_full_step (:300-306), update_residual (:309-314),
// rho = rho_new (:227), check_full_step_convergence (:317-324), and the
// next step's rho_new = <r_hat, r> (:203) with its zero check (:204).
template <typename T>
struct OpBiUpdate {
  static constexpr int kNR = 2;
  T* x;
  T* r;
  const T* r_hat;
  const T* p_hat;
  const T* s_hat;
  const T* s;
  const T* t;
  Scalars* sc;
  double* hist;
  T alpha, omega;
  int skip;
  __device__ bool prepare(const Scalars* st) {
    if (solve_done(st)) return false;
    alpha = static_cast<T>(st->alpha);
    omega = static_cast<T>(st->omega);
    skip = st->skip;
    return true;
  }
  struct In { T x, ph, sh, s, t, rh; };
  __device__ In load(i64 i) const {
    if (skip) return {};
    return {x[i], p_hat[i], s_hat[i], s[i], t[i], r_hat[i]};
  }
  __device__ void apply(i64 i, In const& q, double* red) const {
    if (skip) return;
    x[i] = add(q.x, add(mul(alpha, q.ph), mul(omega, q.sh)));
    const T ri = sub(q.s, mul(omega, q.t));
    r[i] = ri;
    red[0] += static_cast<double>(mul(ri, ri));
    red[1] += static_cast<double>(mul(q.rh, ri));
  }
  __device__ void finalize(const double* tot) const {
    if (skip) {
      sc->skip = 0;
    } else {
      sc->rho = sc->rho_new;
      const T rn = sqrt(static_cast<T>(tot[0]));
      record(sc, hist, static_cast<double>(rn));
      if (rn / static_cast<T>(sc->bnorm) < static_cast<T>(sc->tol)) {
        sc->converged = 1;
        sc->done = 1;
        return;
      }
      sc->rho_new = static_cast<double>(static_cast<T>(tot[1]));
    }
    if (sc->iters >= sc->max_iters) {
      sc->done = 1;
    } else if (static_cast<T>(sc->rho_new) == T(0)) {
      sc->status = SK_BREAKDOWN;
      sc->done = 1;
    }
  }
};

template <typename T, int LK, int RK>
static void bicgstab_step(sk_matrix A, const sk_precond_s* L, const sk_precond_s* R, T* x, T* r,
                          T* r_hat, T* p, T* v, T* s, T* t, T* p_hat, T* s_hat, T* tmp,
                          SolveCommon const& c, cudaStream_t st) {
  const i64 n = A->nrow;
  const T* invL = L && L->kind == 1 ? static_cast<const T*>(L->inv_diag) : nullptr;
  const T* invR = R && R->kind == 1 ? static_cast<const T*>(R->inv_diag) : nullptr;
  constexpr bool fused = LK != PK_OTHER && RK != PK_OTHER;
  launch_vec(n, OpBiP<T, LK, RK>{p, r, v, p_hat, invL, invR, T(0), T(0)}, c.ws, c.sc, st);
  if constexpr (!fused) {
    precond_apply_dispatch(L, A->dtype, n, p, tmp, c.ws, c.sc, st);
    precond_apply_dispatch(R, A->dtype, n, tmp, p_hat, c.ws, c.sc, st);
  }
  launch_spmv<T>(A, p_hat, EpiBiV<T>{v, r_hat, c.sc}, c.ws, c.sc, st);
  launch_vec(n, OpBiS<T>{s, r, v, c.sc, c.hist, T(0)}, c.ws, c.sc, st);
  launch_vec(n, OpBiHalfOrS<T, LK, RK>{x, p_hat, s, s_hat, invL, invR, c.sc, T(0), 0}, c.ws,
             c.sc, st);
  if constexpr (!fused) {
    precond_apply_dispatch(L, A->dtype, n, s, tmp, c.ws, c.sc, st);
    precond_apply_dispatch(R, A->dtype, n, tmp, s_hat, c.ws, c.sc, st);
  }
  launch_spmv<T>(A, s_hat, EpiBiT<T>{t, s, c.sc}, c.ws, c.sc, st);
  launch_vec(n, OpBiUpdate<T>{x, r, r_hat, p_hat, s_hat, s, t, c.sc, c.hist, T(0), T(0), 0}, c.ws,
             c.sc, st);
}

template <typename T>
static sk_status bicgstab_solve(sk_matrix A, sk_precond L, sk_precond R, const T* b, T* x,
                                const sk_bicgstab_config* cfg, sk_summary* out,
                                double* history_host, cudaStream_t st) {
  Range range_("sk bicgstab");
  const i64 n = A->nrow;
  const size_t vb = static_cast<size_t>(n + 8) * sizeof(T);
  SolveCommon c;
  std::vector<char*> vv;
  const i64 hist_cap = cfg->collect_residuals ? cfg->max_iterations + 2 : 0;
  // FP64 with identity / Jacobi sides on a small SELL handle: the whole
  // solve in one cooperative launch (sk_mixed.cu)
  const bool bi64 = std::is_same<T, double>::value && (!L || L->kind == 1) && (!R || R->kind == 1) &&
                    bi64_persistent_ok(A);
  const size_t pextra = bi64 ? (inner_persistent_scratch(A) + 511) & ~size_t(511) : 0;
  char* pscratch = nullptr;
  sk_status s = carve_common(A, st, bi64 ? 10 : 9, vb, pextra, hist_cap, &c, &vv, bi64 ? &pscratch : nullptr);
  if (s != SK_OK) return s;
  T *r = (T*)vv[0], *r_hat = (T*)vv[1], *p = (T*)vv[2], *v = (T*)vv[3], *sv = (T*)vv[4],
    *t = (T*)vv[5], *p_hat = (T*)vv[6], *s_hat = (T*)vv[7], *tmp = (T*)vv[8];
  *out = sk_summary{};
  double bnorm = 0;
  if ((s = norm_b<T>(b, n, c, st, &bnorm)) != SK_OK) return s;
  if (bnorm == 0.0) {  // :161-165
    SK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), st));
    SK_CUDA(cudaStreamSynchronize(st));
    out->converged = 1;
    return SK_OK;
  }
  Scalars h{};
  h.bnorm = bnorm;
  h.tol = cfg->tolerance;
  h.max_iters = cfg->max_iterations;
  h.hist_on = cfg->collect_residuals ? 1 : 0;
  if ((s = put_scalars(c.sc, h, st)) != SK_OK) return s;
  if constexpr (std::is_same<T, double>::value) {
    if (bi64) {
      double* vec[10] = {r, r_hat, p, tmp, v, (double*)vv[9], p_hat, sv, s_hat, t};
      const double* invl = L ? static_cast<const double*>(L->inv_diag) : nullptr;
      const double* invr = R ? static_cast<const double*>(R->inv_diag) : nullptr;
      if ((s = bi64_persistent(A, b, x, vec, invl, invr, cfg->collect_residuals ? c.hist : nullptr, c.sc, pscratch,
                               st)) != SK_OK)
        return s;
      return finish_summary(c, st, out, history_host);
    }
  }
  SK_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), st));  // :173-174
  SK_CUDA(cudaMemsetAsync(v, 0, n * sizeof(T), st));
  launch_spmv<T>(A, x, EpiBiResid<T>{b, r, r_hat, c.sc}, c.ws, nullptr, st);
  const int lk = prec_kind(L), rk = prec_kind(R);
  const bool graphs = capturable(L) && capturable(R);
  if (graphs && (s = solve_stream(A, st, &st)) != SK_OK) return s;
  auto steps_of = [&](i64 cnt) {
    for (i64 j = 0; j < cnt; ++j) {
#define SK_BI_STEP(LKV, RKV)                                                                  \
  bicgstab_step<T, LKV, RKV>(A, L, R, x, r, r_hat, p, v, sv, t, p_hat, s_hat, tmp, c, st)
      if (lk == PK_IDENTITY && rk == PK_IDENTITY) SK_BI_STEP(PK_IDENTITY, PK_IDENTITY);
      else if (lk == PK_JACOBI && rk == PK_IDENTITY) SK_BI_STEP(PK_JACOBI, PK_IDENTITY);
      else if (lk == PK_IDENTITY && rk == PK_JACOBI) SK_BI_STEP(PK_IDENTITY, PK_JACOBI);
      else if (lk == PK_JACOBI && rk == PK_JACOBI) SK_BI_STEP(PK_JACOBI, PK_JACOBI);
      else SK_BI_STEP(PK_OTHER, PK_OTHER);
#undef SK_BI_STEP
    }
  };
  StepGraph sg;
  constexpr i64 kMaxChunk = 32;
  i64 steps = 0, chunk = 4;
  while (steps < std::max<i64>(cfg->max_iterations, 1)) {
    if (graphs && chunk == kMaxChunk) {
      if ((s = sg.replay(st, chunk, steps_of)) != SK_OK) return s;
    } else {
      steps_of(chunk);
    }
    steps += chunk;
    SK_CUDA(cudaGetLastError());
    if ((s = read_scalars(c.sc, &h, st)) != SK_OK) return s;
    if (h.done && !h.half) break;
    chunk = std::min<i64>(chunk * 2, kMaxChunk);
  }
  return finish_summary(c, st, out, history_host);
}

// ==================================================================
// FGMRES(m), fgmres.hpp:96-428
// ==================================================================

struct FgSmall {  // device arrays of one restart cycle
  double* H;   // (m+1) x m, column-major, leading dimension m+1
  double* cs;
  double* sn;
  double* g;   // m+1
  double* y;   // m
  double* zero;  // a constant 0 (the h of an MGS pass that only takes a dot)
};

// GMRES(m) (gmres.hpp:106-396) runs the FGMRES cycle with these changes:
// the left preconditioner M_L on the initial residual and on A z_j
// (:221-222, :253-254), and normalisation by division (:230, :278) where
// fgmres.hpp multiplies by the reciprocal.  A Jacobi M_L is fused into the
// product's epilogue; any other goes through the work vector `tmp`.
template <typename T>
struct GmLeft {
  const sk_precond_s* L = nullptr;  // null: identity (FGMRES)
  const T* linv = nullptr;          // Jacobi M_L: its inverse diagonal
  T* tmp = nullptr;                 // other M_L: the vector before it
  bool divide = false;              // GMRES normalisation
};

template <typename T>
__device__ void fg_init_finalize(T beta, FgSmall const& sm, int m, Scalars* sc, bool divide) {
  for (int i = 0; i < (m + 1) * m; ++i) sm.H[i] = 0.0;
  for (int i = 0; i < m; ++i) sm.cs[i] = sm.sn[i] = 0.0;
  for (int i = 0; i <= m; ++i) sm.g[i] = 0.0;
  *sm.zero = 0.0;
  sm.g[0] = static_cast<double>(beta);
  sc->beta_cycle = static_cast<double>(beta);
  sc->jfinal = 0;
  sc->done = 0;
  sc->beta0 = 0;
  if (beta == T(0)) {
    sc->beta0 = 1;
    sc->converged = 1;
    sc->done = 1;
    sc->rnorm = 0.0;
  } else {
    sc->aux = divide ? static_cast<double>(beta) : static_cast<double>(T(1) / beta);
  }
}

// compute_initial_residual (:207-224) and clear_hessenberg (:227-231).
// A zero beta (the reference divides by it) ends the solve as converged.
template <typename T>
struct EpiFgInit {
  static constexpr int kNR = 1;
  const T* b;
  T* v0;
  Scalars* sc;
  FgSmall sm;
  int m;
  const T* linv;  // Jacobi M_L (GMRES), else null
  bool divide;
  __device__ void operator()(int row, T ax, double* red) const {
    T vi = sub(b[row], ax);
    if (linv) vi = mul(linv[row], vi);
    v0[row] = vi;
    red[0] += static_cast<double>(mul(vi, vi));
  }
  __device__ void finalize(const double* t) const {
    fg_init_finalize<T>(sqrt(static_cast<T>(t[0])), sm, m, sc, divide);
  }
};

// tmp = b - A x (GMRES with a general M_L, before it is applied)
template <typename T>
struct EpiGmResid {
  static constexpr int kNR = 0;
  const T* b;
  T* t;
  __device__ void operator()(int row, T ax, double*) const { t[row] = sub(b[row], ax); }
  __device__ void finalize(const double*) const {}
};

// beta = ||v0|| after a general M_L, and the cycle's initialisation.
template <typename T>
struct OpGmInitNorm {
  static constexpr int kNR = 1;
  const T* v0;
  Scalars* sc;
  FgSmall sm;
  int m;
  bool divide;
  struct In { T v; };
  __device__ bool prepare(const Scalars*) { return true; }
  __device__ In load(i64 i) const { return {v0[i]}; }
  __device__ void apply(i64, In const& q, double* red) const { red[0] += static_cast<double>(mul(q.v, q.v)); }
  __device__ void finalize(const double* t) const {
    fg_init_finalize<T>(sqrt(static_cast<T>(t[0])), sm, m, sc, divide);
  }
};

// scale_vector (:403-408): v *= factor, factor = 1/beta or 1/h (from aux
// or from H), skipped when the factor's norm is not positive.
template <typename T>
struct OpFgScale {
  static constexpr int kNR = 0;
  T* v;
  const double* hsrc;  // null: factor = aux; else factor = 1 / *hsrc if > 0
  T f;
  bool divide;         // GMRES: v /= beta or v /= h (gmres.hpp:230, :278)
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    if (!hsrc) {
      f = static_cast<T>(s->aux);
      return true;
    }
    const T h = static_cast<T>(*hsrc);
    if (!(h > T(0))) return false;  // :283
    f = divide ? h : T(1) / h;
    return true;
  }
  struct In { T v; };
  __device__ In load(i64 i) const { return {v[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const { v[i] = divide ? dvd(q.v, f) : mul(q.v, f); }
  __device__ void finalize(const double*) const {}
};

// arnoldi_step (:247-256): w = A z_j into V_{j+1}; first MGS dot h_{0j}.
template <typename T>
struct EpiFgW {
  static constexpr int kNR = 1;
  T* w;
  const T* v0;
  double* h_out;
  const T* linv;  // Jacobi M_L (GMRES): w = M_L A z_j
  __device__ void operator()(int row, T val, double* red) const {
    if (linv) val = mul(linv[row], val);
    w[row] = val;
    red[0] += static_cast<double>(mul(v0[row], val));
  }
  __device__ void finalize(const double* t) const { *h_out = static_cast<double>(static_cast<T>(t[0])); }
};

// orthogonalize (:259-273) step i: w -= h_ij v_i, then the next dot
// h_{i+1,j} = <v_{i+1}, w>, or for i = j the norm h_{j+1,j} (:276-281).
template <typename T>
struct OpFgMgs {
  static constexpr int kNR = 1;
  T* w;
  const T* vi;
  const T* vnext;  // null at i = j
  const double* h_in;
  double* h_out;
  T h;
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    h = static_cast<T>(*h_in);
    return true;
  }
  struct In { T w, vi, vn; };
  __device__ In load(i64 k) const { return {w[k], vi[k], vnext ? vnext[k] : T(0)}; }
  __device__ void apply(i64 k, In const& q, double* red) const {
    const T wk = sub(q.w, mul(h, q.vi));
    w[k] = wk;
    red[0] += static_cast<double>(mul(vnext ? q.vn : wk, wk));
  }
  __device__ void finalize(const double* t) const {
    const T d = static_cast<T>(t[0]);
    *h_out = static_cast<double>(vnext ? d : sqrt(d));
  }
};

// Columns of up to this many rotations are rotated in thread-local arrays.
constexpr int kFgLocal = 64;

// apply_givens_rotations (:287-337), record_residual (:340-346),
// check_convergence (:349-356), in the value type T.
template <typename T>
struct FgGivens {
  Scalars* sc;
  double* hist;
  FgSmall sm;
  int j, m;
  // The same steps with every operand (the column, the earlier rotations,
  // g_j, g_j+1 and the solve's scalars) loaded in one batch, so that the
  // single thread waits on memory once instead of once per rotation.
  __device__ void local_path() const {
    const int um1 = m + 1;
    const int done = sc->done, hon = sc->hist_on;
    const long long it = sc->iters, hl = sc->hist_len;
    const double bnorm = sc->bnorm, tol = sc->tol;
    double hc[kFgLocal + 2], cv[kFgLocal], sv[kFgLocal];
    for (int i = 0; i <= j + 1; ++i) hc[i] = sm.H[i + j * um1];
    for (int i = 0; i < j; ++i) {
      cv[i] = sm.cs[i];
      sv[i] = sm.sn[i];
    }
    const double g0 = sm.g[j], g1 = sm.g[j + 1];
    if (done) return;
    for (int i = 0; i < j; ++i) {
      const T cs = static_cast<T>(cv[i]), sn = static_cast<T>(sv[i]);
      const T hij = static_cast<T>(hc[i]), hi1 = static_cast<T>(hc[i + 1]);
      const T temp = add(mul(cs, hij), mul(sn, hi1));
      hc[i + 1] = static_cast<double>(add(mul(-sn, hij), mul(cs, hi1)));
      hc[i] = static_cast<double>(temp);
    }
    const T a = static_cast<T>(hc[j]), bb = static_cast<T>(hc[j + 1]);
    T cs, sn;
    if (bb == T(0)) {
      cs = T(1);
      sn = T(0);
    } else if (a == T(0)) {
      cs = T(0);
      sn = T(1);
    } else {
      const T rr = sqrt(add(mul(a, a), mul(bb, bb)));
      cs = dvd(a, rr);
      sn = dvd(bb, rr);
    }
    sm.cs[j] = static_cast<double>(cs);
    sm.sn[j] = static_cast<double>(sn);
    hc[j] = static_cast<double>(add(mul(cs, a), mul(sn, bb)));
    hc[j + 1] = 0.0;
    for (int i = 0; i <= j + 1; ++i) sm.H[i + j * um1] = hc[i];
    const T gj = static_cast<T>(g0), gj1 = static_cast<T>(g1);
    const T temp = add(mul(cs, gj), mul(sn, gj1));
    const double gn = static_cast<double>(add(mul(-sn, gj), mul(cs, gj1)));
    sm.g[j + 1] = gn;
    sm.g[j] = static_cast<double>(temp);
    sc->iters = it + 1;
    sc->jfinal = j;
    const T absres = fabs(static_cast<T>(gn));
    sc->rnorm = static_cast<double>(absres);  // record()
    if (hon) {
      hist[hl] = static_cast<double>(absres);
      sc->hist_len = hl + 1;
    }
    if (absres / static_cast<T>(bnorm) < static_cast<T>(tol)) {
      sc->converged = 1;
      sc->done = 1;
    }
  }
  __device__ void operator()() const {
    if (j < kFgLocal) {
      local_path();
      return;
    }
    if (sc->done) return;
    const int um1 = m + 1;
    auto H = [&](int r, int c) -> double& { return sm.H[r + c * um1]; };
    for (int i = 0; i < j; ++i) {
      const T cs = static_cast<T>(sm.cs[i]), sn = static_cast<T>(sm.sn[i]);
      const T hij = static_cast<T>(H(i, j)), hi1 = static_cast<T>(H(i + 1, j));
      const T temp = add(mul(cs, hij), mul(sn, hi1));
      H(i + 1, j) = static_cast<double>(add(mul(-sn, hij), mul(cs, hi1)));
      H(i, j) = static_cast<double>(temp);
    }
    const T a = static_cast<T>(H(j, j)), bb = static_cast<T>(H(j + 1, j));
    T cs, sn;
    if (bb == T(0)) {
      cs = T(1);
      sn = T(0);
    } else if (a == T(0)) {
      cs = T(0);
      sn = T(1);
    } else {
      const T rr = sqrt(add(mul(a, a), mul(bb, bb)));
      cs = dvd(a, rr);
      sn = dvd(bb, rr);
    }
    sm.cs[j] = static_cast<double>(cs);
    sm.sn[j] = static_cast<double>(sn);
    H(j, j) = static_cast<double>(add(mul(cs, a), mul(sn, bb)));
    H(j + 1, j) = 0.0;
    const T gj = static_cast<T>(sm.g[j]), gj1 = static_cast<T>(sm.g[j + 1]);
    const T temp = add(mul(cs, gj), mul(sn, gj1));
    sm.g[j + 1] = static_cast<double>(add(mul(-sn, gj), mul(cs, gj1)));
    sm.g[j] = static_cast<double>(temp);
    sc->iters += 1;
    sc->jfinal = j;
    const T absres = fabs(static_cast<T>(sm.g[j + 1]));
    record(sc, hist, static_cast<double>(absres));
    if (absres / static_cast<T>(sc->bnorm) < static_cast<T>(sc->tol)) {
      sc->converged = 1;
      sc->done = 1;
    }
  }
};

// back_substitute (:365-379).
template <typename T>
struct FgBackSub {
  Scalars* sc;
  FgSmall sm;
  int m;
  __device__ void operator()() const {
    if (sc->beta0) return;
    const int um1 = m + 1;
    const int nj = static_cast<int>(sc->jfinal) + 1;
    for (int ii = nj; ii > 0; --ii) {
      const int i = ii - 1;
      T yi = static_cast<T>(sm.g[i]);
      for (int k = i + 1; k < nj; ++k)
        yi = sub(yi, mul(static_cast<T>(sm.H[i + k * um1]), static_cast<T>(sm.y[k])));
      yi = dvd(yi, static_cast<T>(sm.H[i + i * um1]));
      sm.y[i] = static_cast<double>(yi);
    }
  }
};

// update_solution (:382-394): x_i += sum_k Z_k[i] y_k, summed in k order.
template <typename T>
struct OpFgUpdateX {
  static constexpr int kNR = 0;
  T* x;
  const T* Z;
  i64 ldz;
  const double* y;
  int nj;
  __device__ bool prepare(const Scalars* s) {
    if (s->beta0) return false;
    nj = static_cast<int>(s->jfinal) + 1;
    return true;
  }
  struct In { T x; };
  __device__ In load(i64 i) const { return {x[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const {
    T sum = T(0);
    for (int k = 0; k < nj; ++k) sum = add(sum, mul(Z[k * ldz + i], static_cast<T>(y[k])));
    x[i] = add(q.x, sum);
  }
  __device__ void finalize(const double*) const {}
};

// With `fallback` non-null, a restart cycle whose residual estimate ends
// above stall_ratio times the cycle's starting residual switches the
// preconditioner to `fallback` for the rest of the solve; *switched_at
// receives the first cycle run with it (-1: never switched).
//
// With `left` non-null this is GMRES(m) (gmres.hpp:106-396): `left` is M_L
// and M is M_R; the cycle applies M_L and normalises by division.
template <typename T>
static sk_status fgmres_solve(sk_matrix A, sk_precond M, const T* b, T* x,
                              const sk_fgmres_config* cfg, sk_summary* out, double* history_host,
                              cudaStream_t st, sk_precond fallback = nullptr, double stall_ratio = 0.0,
                              int64_t* switched_at = nullptr, sk_precond left = nullptr, bool gmres = false,
                              const T* vals = nullptr, bool hess64 = false) {
  Range range_("sk fgmres");
  const i64 n = A->nrow;
  const int m = static_cast<int>(cfg->restart_dimension);
  SK_CHECK(m >= 1 && m <= 4096, SK_INVALID_ARG, "restart_dimension must be in [1, 4096]");
  const i64 ld = n + 8 + 32;  // leading dimension of V and Z, 256-byte rounded below
  const i64 ldv = (ld * static_cast<i64>(sizeof(T)) + 255) / 256 * 256 / static_cast<i64>(sizeof(T));
  const bool alias_z = (M == nullptr);  // identity: Z_j = V_j
  GmLeft<T> gl;
  gl.L = left;
  gl.divide = gmres;
  if (left && left->kind == 1) gl.linv = static_cast<const T*>(left->inv_diag);
  const bool general_left = left && left->kind != 1;
  const i64 nvecs = (m + 1) + (alias_z ? 0 : m) + (general_left ? 1 : 0);
  const size_t small_bytes = static_cast<size_t>((m + 1) * m + 4 * (m + 2) + 4) * 8;
  SolveCommon c;
  std::vector<char*> vv;
  char* extra = nullptr;
  const i64 hist_cap = cfg->collect_residuals ? cfg->max_iterations : 0;
  // the Arnoldi step's barrier words and reduction slots (2 x grid <= 2 x 512)
  const size_t arn_bytes = 256 + 2 * 512 * sizeof(double);
  sk_status s = carve_common(A, st, 0, 0,
                             static_cast<size_t>(nvecs) * ldv * sizeof(T) + small_bytes + arn_bytes + 1024,
                             hist_cap, &c, &vv, &extra);
  if (s != SK_OK) return s;
  T* V = reinterpret_cast<T*>(extra);
  T* Z = alias_z ? V : V + (m + 1) * ldv;
  FgSmall sm;
  double* smallp = reinterpret_cast<double*>(
      (reinterpret_cast<uintptr_t>(V + nvecs * ldv) + 255) & ~uintptr_t(255));
  sm.H = smallp;
  sm.cs = sm.H + (m + 1) * m;
  sm.sn = sm.cs + (m + 2);
  sm.g = sm.sn + (m + 2);
  sm.y = sm.g + (m + 2);
  sm.zero = sm.y + (m + 2);
  if (general_left) gl.tmp = V + ((m + 1) + (alias_z ? 0 : m)) * ldv;  // after V and Z
  // Modified Gram-Schmidt of each Arnoldi step as one cooperative launch
  // when w fits on chip (sk_arnoldi.cu), else one launch per basis vector.
  ArnoldiPlan aplan;
  const bool arnoldi_fused = !c.ws.seq && arnoldi_plan<T>(A, n, &aplan);
  auto* arn_sync = reinterpret_cast<ArnoldiSync*>(
      (reinterpret_cast<uintptr_t>(smallp) + small_bytes + 255) & ~uintptr_t(255));
  double* arn_slots = reinterpret_cast<double*>(reinterpret_cast<char*>(arn_sync) + 256);
  sk_status arn_status = SK_OK;
  if (arnoldi_fused) SK_CUDA(cudaMemsetAsync(arn_sync, 0, sizeof(ArnoldiSync), st));
  *out = sk_summary{};
  double bnorm = 0;
  if ((s = norm_b<T>(b, n, c, st, &bnorm)) != SK_OK) return s;
  if (bnorm == 0.0) {  // :169-173
    SK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), st));
    SK_CUDA(cudaStreamSynchronize(st));
    out->converged = 1;
    return SK_OK;
  }
  Scalars h{};
  h.bnorm = bnorm;
  h.tol = cfg->tolerance;
  h.max_iters = cfg->max_iterations;
  h.hist_on = cfg->collect_residuals ? 1 : 0;
  if ((s = put_scalars(c.sc, h, st)) != SK_OK) return s;
  const int um1 = m + 1;
  if (switched_at) *switched_at = -1;
  // One restart cycle (compute_initial_residual .. update_solution) as a
  // fixed sequence of launches: every pointer is the same from cycle to
  // cycle, and a converged solve turns the remaining kernels into no-ops.
  auto enqueue_cycle = [&](cudaStream_t q, int m_eff, sk_precond P) {
    if (general_left) {  // r0 = b - A x; v0 = M_L r0; beta = ||v0|| (:214-224)
      launch_spmv<T>(A, x, EpiGmResid<T>{b, gl.tmp}, c.ws, nullptr, q, vals);
      precond_apply_dispatch(gl.L, kVecType<T>, n, gl.tmp, V, c.ws, nullptr, q);
      launch_vec(n, OpGmInitNorm<T>{V, c.sc, sm, m, gl.divide}, c.ws, nullptr, q);
    } else {
      launch_spmv<T>(A, x, EpiFgInit<T>{b, V, c.sc, sm, m, gl.linv, gl.divide}, c.ws, nullptr, q, vals);
    }
    launch_vec(n, OpFgScale<T>{V, nullptr, T(0), gl.divide}, c.ws, c.sc, q);
    for (int j = 0; j < m_eff; ++j) {
      T* Vj = V + j * ldv;
      T* Vj1 = V + (j + 1) * ldv;
      T* Zj = Z + j * ldv;
      if (!alias_z) precond_apply_dispatch(P, kVecType<T>, n, Vj, Zj, c.ws, c.sc, q);
      if (general_left) {  // v_{j+1} = M_L A z_j, then h_0j = <v_0, v_{j+1}>
        launch_spmv<T>(A, Zj, EpiStore<T>{gl.tmp}, c.ws, c.sc, q, vals);
        precond_apply_dispatch(gl.L, kVecType<T>, n, gl.tmp, Vj1, c.ws, c.sc, q);
        launch_vec(n, OpFgMgs<T>{Vj1, V, V, sm.zero, sm.H + j * um1, T(0)}, c.ws, c.sc, q);
      } else {
        launch_spmv<T>(A, Zj, EpiFgW<T>{Vj1, V, sm.H + j * um1, gl.linv}, c.ws, c.sc, q, vals);
      }
      if (arnoldi_fused) {
        const sk_status as = arnoldi_launch<T>(
            aplan, ArnoldiArgs<T>{n, Vj1, V, ldv, j, sm.H + j * um1, gl.divide, c.sc, arn_sync, arn_slots, 0}, q);
        if (as != SK_OK && arn_status == SK_OK) arn_status = as;
      } else {
        for (int i = 0; i <= j; ++i) {
          const T* vnext = i < j ? V + (i + 1) * ldv : nullptr;
          launch_vec(n, OpFgMgs<T>{Vj1, V + i * ldv, vnext, sm.H + i + j * um1, sm.H + (i + 1) + j * um1, T(0)},
                     c.ws, c.sc, q);
        }
        launch_vec(n, OpFgScale<T>{Vj1, sm.H + (j + 1) + j * um1, T(0), gl.divide}, c.ws, c.sc, q);
      }
      g_launches.fetch_add(1, std::memory_order_relaxed);
      if (hess64)  // the least-squares problem in FP64 around FP32 vectors
        scalar_kernel<<<1, 1, 0, q>>>(FgGivens<double>{c.sc, c.hist, sm, j, m});
      else
        scalar_kernel<<<1, 1, 0, q>>>(FgGivens<T>{c.sc, c.hist, sm, j, m});
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (hess64)
      scalar_kernel<<<1, 1, 0, q>>>(FgBackSub<double>{c.sc, sm, m});
    else
      scalar_kernel<<<1, 1, 0, q>>>(FgBackSub<T>{c.sc, sm, m});
    launch_vec(n, OpFgUpdateX<T>{x, Z, ldv, sm.y, 0}, c.ws, c.sc, q);
  };
  // Solves expected to run several cycles replay each cycle as a CUDA graph
  // (one launch per cycle instead of ~m^2 / 2), captured on a created stream
  // (the legacy stream cannot be captured; the caller's stream is drained
  // first and this call returns after its last host read).
  const bool graphs = cfg->max_iterations >= 3 * static_cast<i64>(m) && n >= 1;
  cudaStream_t gs = st;
  if (graphs && (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread)) {
    SK_CUDA(cudaStreamSynchronize(st));
    gs = A->stream;
  }
  struct Exec { cudaGraphExec_t exec = nullptr; i64 launches = 0; };
  std::map<int, Exec> execs;  // by m_eff
  auto drop_graphs = [&]() {
    for (auto& kv : execs) cudaGraphExecDestroy(kv.second.exec);
    execs.clear();
  };
  int64_t cycle = 0;
  while (h.iters < cfg->max_iterations && !h.converged) {
    const int m_eff = static_cast<int>(std::min<i64>(m, cfg->max_iterations - h.iters));  // :241-244
    if (graphs) {
      auto it = execs.find(m_eff);
      if (it == execs.end()) {
        for (const sk_precond_s* P : {static_cast<const sk_precond_s*>(M), static_cast<const sk_precond_s*>(left)}) {
          const sk_precond_s* net_prec = P && P->kind == 4 ? P->smoother : P;
          if (net_prec && net_prec->kind == 3 && (s = learned_prepare(net_prec)) != SK_OK) {
            drop_graphs();
            return s;
          }
        }
        const i64 before = g_launches.load();
        cudaGraph_t g = nullptr;
        Exec e;
        cudaError_t ce = cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) {
          enqueue_cycle(gs, m_eff, M);
          ce = cudaStreamEndCapture(gs, &g);
        }
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e.exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
          drop_graphs();
          return cuda_fail(ce, "FGMRES cycle capture");
        }
        e.launches = g_launches.load() - before;
        g_launches.fetch_sub(e.launches);  // counted at each replay instead
        it = execs.emplace(m_eff, e).first;
      }
      g_launches.fetch_add(it->second.launches);
      cudaError_t ce = cudaGraphLaunch(it->second.exec, gs);
      if (ce != cudaSuccess) {
        drop_graphs();
        return cuda_fail(ce, "cudaGraphLaunch");
      }
    } else {
      enqueue_cycle(gs, m_eff, M);
    }
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess || arn_status != SK_OK) {
      drop_graphs();
      return le != cudaSuccess ? cuda_fail(le, "FGMRES cycle") : arn_status;
    }
    if ((s = read_scalars(c.sc, &h, gs)) != SK_OK) {
      drop_graphs();
      return s;
    }
    if (arnoldi_fused) {
      int err = 0;
      SK_CUDA(cudaMemcpy(&err, &arn_sync->err, sizeof(int), cudaMemcpyDeviceToHost));
      if (err) {
        drop_graphs();
        return fail(SK_TIMEOUT, "FGMRES Arnoldi step: a grid barrier wait ran out");
      }
    }
    ++cycle;
    if (fallback && M != fallback && !h.converged && h.rnorm > stall_ratio * h.beta_cycle) {
      M = fallback;
      drop_graphs();
      if (switched_at) *switched_at = cycle;
    }
  }
  drop_graphs();
  st = gs;
  return finish_summary(c, st, out, history_host);
}

// ==================================================================
// Preconditioner pair of CGS and MINRES: out = M_R (M_L in), applied in
// that order as cgs.hpp:235-239 / minres.hpp:190-191 do.  Identity and
// Jacobi on both sides fuse into one element-wise pass.
// ==================================================================
template <typename T>
struct OpLR {
  static constexpr int kNR = 0;
  const T* invl;  // null: identity
  const T* invr;
  const T* in;
  T* out;
  struct In { T v, l, r; };
  __device__ bool prepare(const Scalars* sc) { return !solve_done(sc); }
  __device__ In load(i64 i) const { return {in[i], invl ? invl[i] : T(0), invr ? invr[i] : T(0)}; }
  __device__ void apply(i64 i, In const& q, double*) const {
    T v = q.v;
    if (invl) v = mul(q.l, v);
    if (invr) v = mul(q.r, v);
    out[i] = v;
  }
  __device__ void finalize(const double*) const {}
};

template <typename T>
struct LRPair {
  const sk_precond_s* L;
  const sk_precond_s* R;
  const T* invl = nullptr;
  const T* invr = nullptr;
  bool fused = false;  // both sides identity or Jacobi
  LRPair(const sk_precond_s* l, const sk_precond_s* r) : L(l), R(r) {
    const bool lf = !l || l->kind == 1, rf = !r || r->kind == 1;
    fused = lf && rf;
    if (l && l->kind == 1) invl = static_cast<const T*>(l->inv_diag);
    if (r && r->kind == 1) invr = static_cast<const T*>(r->inv_diag);
  }
};

template <typename T>
static void apply_lr(LRPair<T> const& lr, i64 n, const T* in, T* tmp, T* out, SolveCommon const& c,
                     cudaStream_t st) {
  const sk_dtype dt = sizeof(T) == 8 ? SK_F64 : SK_F32;
  if (lr.fused) {
    launch_vec(n, OpLR<T>{lr.invl, lr.invr, in, out}, c.ws, c.sc, st);
    return;
  }
  precond_apply_dispatch(lr.L, dt, n, in, tmp, c.ws, c.sc, st);
  precond_apply_dispatch(lr.R, dt, n, tmp, out, c.ws, c.sc, st);
}

// ==================================================================
// CGS, cgs.hpp:106-395
// ==================================================================

// compute_initial_residual (:191-198), initialize_shadow_residual and
// initialize_search_directions (:201-209), rho = <r_hat, r> (:178).
template <typename T>
struct EpiCgsInit {
  static constexpr int kNR = 1;
  const T* b;
  T *r, *r_hat, *p, *u;
  Scalars* sc;
  __device__ void operator()(int row, T ax, double* red) const {
    const T ri = sub(b[row], ax);
    r[row] = r_hat[row] = p[row] = u[row] = ri;
    red[0] += static_cast<double>(mul(ri, ri));
  }
  __device__ void finalize(const double* t) const { sc->rho = static_cast<double>(static_cast<T>(t[0])); }
};

// compute_q_hat's product (:235-239) and compute_alpha (:242-244)
template <typename T>
struct EpiCgsQhat {
  static constexpr int kNR = 1;
  T* q_hat;
  const T* r_hat;
  Scalars* sc;
  __device__ void operator()(int row, T v, double* red) const {
    q_hat[row] = v;
    red[0] += static_cast<double>(mul(r_hat[row], v));
  }
  __device__ void finalize(const double* t) const {
    sc->alpha = static_cast<double>(static_cast<T>(sc->rho) / static_cast<T>(t[0]));
  }
};

// compute_q (:247-252), compute_u_hat (:255-260); with a fusable
// preconditioner pair also apply_preconditioner_to_u_hat (:263-266) and
// update_solution (:269-275).
template <typename T>
struct OpCgsQ {
  static constexpr int kNR = 0;
  const T* u;
  const T* q_hat;
  T* q;
  T* u_hat;   // written when not fused
  T* p_hat;   // fused: p_hat = M_R M_L u_hat, x += alpha p_hat
  T* x;
  const T* invl;
  const T* invr;
  bool fused;
  T alpha;
  struct In { T u, qh, x, l, r; };
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    alpha = static_cast<T>(s->alpha);
    return true;
  }
  __device__ In load(i64 i) const {
    return {u[i], q_hat[i], fused ? x[i] : T(0), fused && invl ? invl[i] : T(0), fused && invr ? invr[i] : T(0)};
  }
  __device__ void apply(i64 i, In const& v, double*) const {
    const T qi = sub(v.u, mul(alpha, v.qh));
    q[i] = qi;
    T uh = add(v.u, qi);
    if (!fused) {
      u_hat[i] = uh;
      return;
    }
    if (invl) uh = mul(v.l, uh);
    if (invr) uh = mul(v.r, uh);
    p_hat[i] = uh;
    x[i] = add(v.x, mul(alpha, uh));
  }
  __device__ void finalize(const double*) const {}
};

// update_solution (:269-275) after a general preconditioner pair
template <typename T>
struct OpCgsX {
  static constexpr int kNR = 0;
  T* x;
  const T* p_hat;
  T alpha;
  struct In { T x, p; };
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    alpha = static_cast<T>(s->alpha);
    return true;
  }
  __device__ In load(i64 i) const { return {x[i], p_hat[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const { x[i] = add(v.x, mul(alpha, v.p)); }
  __device__ void finalize(const double*) const {}
};

// compute_residual_update (:278-284), check_convergence (:287-298), and
// rho_new = <r_hat, r> with its zero test and beta (:224-231).
template <typename T>
struct EpiCgsR {
  static constexpr int kNR = 2;
  T* r;
  const T* r_hat;
  Scalars* sc;
  double* hist;
  __device__ void operator()(int row, T ax, double* red) const {
    const T ri = sub(r[row], mul(static_cast<T>(sc->alpha), ax));
    r[row] = ri;
    red[0] += static_cast<double>(mul(ri, ri));
    red[1] += static_cast<double>(mul(r_hat[row], ri));
  }
  __device__ void finalize(const double* t) const {
    sc->iters += 2;
    const T rn = sqrt(static_cast<T>(t[0]));
    record(sc, hist, static_cast<double>(rn));
    if (rn / static_cast<T>(sc->bnorm) < static_cast<T>(sc->tol)) {
      sc->converged = 1;
      sc->done = 1;
      return;
    }
    const T rho_new = static_cast<T>(t[1]);
    if (rho_new == T(0)) {
      sc->skip = 1;
    } else {
      sc->skip = 0;
      sc->beta = static_cast<double>(rho_new / static_cast<T>(sc->rho));
      sc->rho = static_cast<double>(rho_new);
    }
    if (sc->iters >= sc->max_iters) sc->done = 1;
  }
};

// update_search_directions (:301-309)
template <typename T>
struct OpCgsDir {
  static constexpr int kNR = 0;
  const T* r;
  const T* q;
  T* u;
  T* p;
  T beta;
  struct In { T r, q, p; };
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s) || s->skip) return false;
    beta = static_cast<T>(s->beta);
    return true;
  }
  __device__ In load(i64 i) const { return {r[i], q[i], p[i]}; }
  __device__ void apply(i64 i, In const& v, double*) const {
    const T ui = add(v.r, mul(beta, v.q));
    u[i] = ui;
    p[i] = add(ui, mul(beta, add(v.q, mul(beta, v.p))));
  }
  __device__ void finalize(const double*) const {}
};

template <typename T>
static sk_status cgs_solve(sk_matrix A, sk_precond L, sk_precond R, const T* b, T* x, const sk_cgs_config* cfg,
                           sk_summary* out, double* history_host, cudaStream_t st) {
  Range range_("sk cgs");
  const i64 n = A->nrow;
  const size_t vb = static_cast<size_t>(n + 8) * sizeof(T);
  SolveCommon c;
  std::vector<char*> vv;
  const i64 hist_cap = cfg->collect_residuals ? cfg->max_iterations / 2 + 4 : 0;
  // FP64 with identity / Jacobi sides on a small SELL handle: the whole
  // solve in one cooperative launch (sk_mixed.cu)
  const bool c64 = std::is_same<T, double>::value && (!L || L->kind == 1) && (!R || R->kind == 1) &&
                   cgs64_persistent_ok(A);
  const size_t pextra = c64 ? (inner_persistent_scratch(A) + 511) & ~size_t(511) : 0;
  char* pscratch = nullptr;
  sk_status s = carve_common(A, st, 9, vb, pextra, hist_cap, &c, &vv, c64 ? &pscratch : nullptr);
  if (s != SK_OK) return s;
  T *r = (T*)vv[0], *r_hat = (T*)vv[1], *p = (T*)vv[2], *u = (T*)vv[3], *q = (T*)vv[4], *q_hat = (T*)vv[5],
    *u_hat = (T*)vv[6], *p_hat = (T*)vv[7], *tmp = (T*)vv[8];
  *out = sk_summary{};
  double bnorm = 0;
  if ((s = norm_b<T>(b, n, c, st, &bnorm)) != SK_OK) return s;
  if (bnorm == 0.0) {  // :168-172
    SK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), st));
    SK_CUDA(cudaStreamSynchronize(st));
    out->converged = 1;
    return SK_OK;
  }
  Scalars h{};
  h.bnorm = bnorm;
  h.tol = cfg->tolerance;
  h.max_iters = cfg->max_iterations;
  h.hist_on = cfg->collect_residuals ? 1 : 0;
  h.done = cfg->max_iterations <= 0 ? 1 : 0;
  if ((s = put_scalars(c.sc, h, st)) != SK_OK) return s;
  if constexpr (std::is_same<T, double>::value) {
    if (c64) {
      double* vec[7] = {r, r_hat, p, tmp, u, q, q_hat};
      const double* invl = L ? static_cast<const double*>(L->inv_diag) : nullptr;
      const double* invr = R ? static_cast<const double*>(R->inv_diag) : nullptr;
      if ((s = cgs64_persistent(A, b, x, vec, invl, invr, cfg->collect_residuals ? c.hist : nullptr, c.sc, pscratch,
                                st)) != SK_OK)
        return s;
      return finish_summary(c, st, out, history_host);
    }
  }
  launch_spmv<T>(A, x, EpiCgsInit<T>{b, r, r_hat, p, u, c.sc}, c.ws, nullptr, st);
  const LRPair<T> lr(L, R);
  const bool graphs = capturable(L) && capturable(R);
  if (graphs && (s = solve_stream(A, st, &st)) != SK_OK) return s;
  auto steps_of = [&](i64 cnt) {
    for (i64 j = 0; j < cnt; ++j) {  // cgs_step (:212-232)
      apply_lr<T>(lr, n, p, tmp, p_hat, c, st);
      launch_spmv<T>(A, p_hat, EpiCgsQhat<T>{q_hat, r_hat, c.sc}, c.ws, c.sc, st);
      launch_vec(n, OpCgsQ<T>{u, q_hat, q, u_hat, p_hat, x, lr.invl, lr.invr, lr.fused, T(0)}, c.ws, c.sc, st);
      if (!lr.fused) {
        apply_lr<T>(lr, n, u_hat, tmp, p_hat, c, st);
        launch_vec(n, OpCgsX<T>{x, p_hat, T(0)}, c.ws, c.sc, st);
      }
      launch_spmv<T>(A, p_hat, EpiCgsR<T>{r, r_hat, c.sc, c.hist}, c.ws, c.sc, st);
      launch_vec(n, OpCgsDir<T>{r, q, u, p, T(0)}, c.ws, c.sc, st);
    }
  };
  StepGraph sg;
  constexpr i64 kMaxChunk = 32;
  i64 chunk = 4;
  while (!h.done) {
    if (graphs && chunk == kMaxChunk) {
      if ((s = sg.replay(st, chunk, steps_of)) != SK_OK) return s;
    } else {
      steps_of(chunk);
    }
    SK_CUDA(cudaGetLastError());
    if ((s = read_scalars(c.sc, &h, st)) != SK_OK) return s;
    chunk = std::min<i64>(chunk * 2, kMaxChunk);
  }
  return finish_summary(c, st, out, history_host);
}

// ==================================================================
// MINRES, minres.hpp:106-418
// ==================================================================

struct MinScalars {  // the solver's recurrence scalars, in T (stored as double)
  double alpha, beta, eps, delta, rho, phi, phi_bar, cs_prev, sn_prev, cs, sn, cs_new, sn_new, inv_bn;
  int rotate;   // this step rotates the Lanczos vectors (:230-233)
  int pending;  // update_solution of the step just run is still to be applied
};

// compute_initial_residual (:184-217): v = b - A x; z = M_R M_L v
// (fused pair) and beta = sqrt(<v, z>).
template <typename T>
__device__ void min_init_finalize(T beta, Scalars* sc, MinScalars* ms) {
  if (beta == T(0)) {
    sc->converged = 1;
    sc->done = 1;
    return;
  }
  ms->beta = static_cast<double>(beta);
  ms->inv_bn = static_cast<double>(T(1) / beta);
  ms->phi_bar = static_cast<double>(beta);
  ms->cs_prev = 1.0;
  ms->sn_prev = 0.0;
  ms->cs = 1.0;
  ms->sn = 0.0;
}

template <typename T>
struct EpiMinInit {
  static constexpr int kNR = 1;
  const T* b;
  T* v;
  T* z;  // fused pair: z = M_R M_L v
  const T* invl;
  const T* invr;
  bool fused;
  Scalars* sc;
  MinScalars* ms;
  __device__ void operator()(int row, T ax, double* red) const {
    const T vi = sub(b[row], ax);
    v[row] = vi;
    if (!fused) return;
    T zi = vi;
    if (invl) zi = mul(invl[row], zi);
    if (invr) zi = mul(invr[row], zi);
    z[row] = zi;
    red[0] += static_cast<double>(mul(vi, zi));
  }
  __device__ void finalize(const double* t) const {
    if (fused) min_init_finalize<T>(sqrt(static_cast<T>(t[0])), sc, ms);
  }
};

// beta = sqrt(<v, z>) after a general preconditioner pair
template <typename T>
struct OpMinInitDot {
  static constexpr int kNR = 1;
  const T* v;
  const T* z;
  Scalars* sc;
  MinScalars* ms;
  struct In { T v, z; };
  __device__ bool prepare(const Scalars*) { return true; }
  __device__ In load(i64 i) const { return {v[i], z[i]}; }
  __device__ void apply(i64, In const& q, double* red) const { red[0] += static_cast<double>(mul(q.v, q.z)); }
  __device__ void finalize(const double* t) const { min_init_finalize<T>(sqrt(static_cast<T>(t[0])), sc, ms); }
};

// v *= 1 / beta, z *= 1 / beta (:207-214)
template <typename T>
struct OpMinScale {
  static constexpr int kNR = 0;
  T* v;
  T* z;
  const MinScalars* ms;
  T f;
  struct In { T v, z; };
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    f = static_cast<T>(ms->inv_bn);
    return true;
  }
  __device__ In load(i64 i) const { return {v[i], z[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const {
    v[i] = mul(q.v, f);
    z[i] = mul(q.z, f);
  }
  __device__ void finalize(const double*) const {}
};

// lanczos_step's product w = A z and alpha = <z, w> (:237-241)
template <typename T>
struct EpiMinW {
  static constexpr int kNR = 1;
  T* w;
  const T* z;
  MinScalars* ms;
  __device__ void operator()(int row, T val, double* red) const {
    w[row] = val;
    red[0] += static_cast<double>(mul(z[row], val));
  }
  __device__ void finalize(const double* t) const { ms->alpha = static_cast<double>(static_cast<T>(t[0])); }
};

// apply_givens_rotations (:265-286), check_convergence (:300-309), the
// step count (:231) and the scalar half of rotate_state (:320-324), from
// beta_new; the vector half runs in OpMinUpdate.
template <typename T>
__device__ void min_step_finalize(T beta_new, Scalars* sc, MinScalars* ms, double* hist) {
  const T beta = static_cast<T>(ms->beta), alpha = static_cast<T>(ms->alpha);
  const T cs_prev = static_cast<T>(ms->cs_prev), sn_prev = static_cast<T>(ms->sn_prev);
  const T cs = static_cast<T>(ms->cs), sn = static_cast<T>(ms->sn);
  ms->eps = static_cast<double>(mul(sn_prev, beta));
  const T delta_1 = mul(cs_prev, beta);
  const T delta = add(mul(cs, delta_1), mul(sn, alpha));
  const T rho_bar = add(mul(-sn, delta_1), mul(cs, alpha));
  const T rho = sqrt(add(mul(rho_bar, rho_bar), mul(beta_new, beta_new)));
  if (rho != T(0)) {  // else rho, delta and phi keep the previous step's values
    const T cs_new = dvd(rho_bar, rho), sn_new = dvd(beta_new, rho);
    const T phi_bar = static_cast<T>(ms->phi_bar);
    ms->cs_new = static_cast<double>(cs_new);
    ms->sn_new = static_cast<double>(sn_new);
    ms->phi = static_cast<double>(mul(cs_new, phi_bar));
    ms->phi_bar = static_cast<double>(mul(-sn_new, phi_bar));
    ms->rho = static_cast<double>(rho);
    ms->delta = static_cast<double>(delta);
  }
  ms->pending = 1;
  const T res = fabs(static_cast<T>(ms->phi_bar));
  record(sc, hist, static_cast<double>(res));
  const bool conv = res / static_cast<T>(sc->bnorm) < static_cast<T>(sc->tol);
  sc->converged = conv ? 1 : 0;
  sc->iters += 1;
  ms->rotate = (!conv && beta_new != T(0)) ? 1 : 0;
  if (ms->rotate) {
    ms->inv_bn = static_cast<double>(T(1) / beta_new);
    ms->cs_prev = ms->cs;
    ms->sn_prev = ms->sn;
    ms->cs = ms->cs_new;
    ms->sn = ms->sn_new;
    ms->beta = static_cast<double>(beta_new);
  }
  if (conv || sc->iters >= sc->max_iters) sc->done = 1;
}

// w -= alpha v + beta v_prev (:244-246); with a fusable pair also
// precondition_lanczos (:250-262): v_prev = M_R M_L w, beta_new.
template <typename T>
struct OpMinLanczos {
  static constexpr int kNR = 1;
  T* w;
  const T* v;
  T* vp;
  const T* invl;
  const T* invr;
  bool fused;
  Scalars* sc;
  MinScalars* ms;
  double* hist;
  T alpha, beta;
  struct In { T w, v, vp, l, r; };
  __device__ bool prepare(const Scalars* s) {
    if (solve_done(s)) return false;
    alpha = static_cast<T>(ms->alpha);
    beta = static_cast<T>(ms->beta);
    return true;
  }
  __device__ In load(i64 i) const {
    return {w[i], v[i], vp[i], fused && invl ? invl[i] : T(0), fused && invr ? invr[i] : T(0)};
  }
  __device__ void apply(i64 i, In const& q, double* red) const {
    const T wi = sub(q.w, add(mul(alpha, q.v), mul(beta, q.vp)));
    w[i] = wi;
    if (!fused) return;
    T zi = wi;
    if (invl) zi = mul(q.l, zi);
    if (invr) zi = mul(q.r, zi);
    vp[i] = zi;
    red[0] += static_cast<double>(mul(wi, zi));
  }
  __device__ void finalize(const double* t) const {
    if (fused) min_step_finalize<T>(sqrt(static_cast<T>(t[0])), sc, ms, hist);
  }
};

// beta_new = sqrt(<w, v_prev>) after a general preconditioner pair
template <typename T>
struct OpMinDot {
  static constexpr int kNR = 1;
  const T* w;
  const T* vp;
  Scalars* sc;
  MinScalars* ms;
  double* hist;
  struct In { T w, vp; };
  __device__ bool prepare(const Scalars* s) { return !solve_done(s); }
  __device__ In load(i64 i) const { return {w[i], vp[i]}; }
  __device__ void apply(i64, In const& q, double* red) const { red[0] += static_cast<double>(mul(q.w, q.vp)); }
  __device__ void finalize(const double* t) const { min_step_finalize<T>(sqrt(static_cast<T>(t[0])), sc, ms, hist); }
};

// update_solution (:288-297) and the vector half of rotate_state
// (:311-319).  Runs for the step just taken even when it converged (the
// reference updates x before it tests), hence its own `pending` gate,
// cleared by its finalize.
template <typename T>
struct OpMinUpdate {
  static constexpr int kNR = 1;
  T *d, *dp, *x, *z, *v, *vp;
  const T* w;
  MinScalars* ms;
  T delta, eps, rho, phi, inv_bn;
  int rotate;
  struct In { T d, dp, x, z, v, vp, w; };
  __device__ bool prepare(const Scalars*) {
    if (!*reinterpret_cast<const volatile int*>(&ms->pending)) return false;
    delta = static_cast<T>(ms->delta);
    eps = static_cast<T>(ms->eps);
    rho = static_cast<T>(ms->rho);
    phi = static_cast<T>(ms->phi);
    inv_bn = static_cast<T>(ms->inv_bn);
    rotate = ms->rotate;
    return true;
  }
  __device__ In load(i64 i) const { return {d[i], dp[i], x[i], z[i], v[i], vp[i], rotate ? w[i] : T(0)}; }
  __device__ void apply(i64 i, In const& q, double* red) const {
    const T dn = dvd(sub(sub(q.z, mul(delta, q.d)), mul(eps, q.dp)), rho);
    d[i] = dn;
    dp[i] = q.d;
    x[i] = add(q.x, mul(phi, dn));
    if (rotate) {
      z[i] = mul(q.vp, inv_bn);
      vp[i] = q.v;
      v[i] = mul(q.w, inv_bn);
    }
    red[0] += 0.0;
  }
  __device__ void finalize(const double*) const { ms->pending = 0; }
};

template <typename T>
static sk_status minres_solve(sk_matrix A, sk_precond L, sk_precond R, const T* b, T* x,
                              const sk_minres_config* cfg, sk_summary* out, double* history_host,
                              cudaStream_t st) {
  Range range_("sk minres");
  const i64 n = A->nrow;
  const size_t vb = static_cast<size_t>(n + 8) * sizeof(T);
  SolveCommon c;
  std::vector<char*> vv;
  char* extra = nullptr;
  const i64 hist_cap = cfg->collect_residuals ? cfg->max_iterations + 2 : 0;
  // FP64 with identity / Jacobi sides on a small SELL handle: the whole
  // solve in one cooperative launch (sk_mixed.cu)
  const bool m64 = std::is_same<T, double>::value && (!L || L->kind == 1) && (!R || R->kind == 1) &&
                   min64_persistent_ok(A);
  const size_t pextra = m64 ? (inner_persistent_scratch(A) + 511) & ~size_t(511) : 0;
  sk_status s = carve_common(A, st, 7, vb, sizeof(MinScalars) + 512 + pextra, hist_cap, &c, &vv, &extra);
  if (s != SK_OK) return s;
  T *vp = (T*)vv[0], *v = (T*)vv[1], *z = (T*)vv[2], *w = (T*)vv[3], *tmp = (T*)vv[4], *dp = (T*)vv[5],
    *d = (T*)vv[6];
  MinScalars* ms = reinterpret_cast<MinScalars*>(extra);
  *out = sk_summary{};
  double bnorm = 0;
  if ((s = norm_b<T>(b, n, c, st, &bnorm)) != SK_OK) return s;
  if (bnorm == 0.0) {  // :170-174
    SK_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), st));
    SK_CUDA(cudaStreamSynchronize(st));
    out->converged = 1;
    return SK_OK;
  }
  Scalars h{};
  h.bnorm = bnorm;
  h.tol = cfg->tolerance;
  h.max_iters = cfg->max_iterations;
  h.hist_on = cfg->collect_residuals ? 1 : 0;
  if ((s = put_scalars(c.sc, h, st)) != SK_OK) return s;
  if constexpr (std::is_same<T, double>::value) {
    if (m64) {
      double* vec[7] = {v, vp, z, w, tmp, d, dp};
      const double* invl = L ? static_cast<const double*>(L->inv_diag) : nullptr;
      const double* invr = R ? static_cast<const double*>(R->inv_diag) : nullptr;
      char* pscratch = extra + ((sizeof(MinScalars) + 255) & ~size_t(255)) + 256;
      if ((s = min64_persistent(A, b, x, vec, invl, invr, cfg->collect_residuals ? c.hist : nullptr, c.sc, pscratch,
                                st)) != SK_OK)
        return s;
      return finish_summary(c, st, out, history_host);
    }
  }
  SK_CUDA(cudaMemsetAsync(ms, 0, sizeof(MinScalars), st));
  for (T* vec : {vp, d, dp}) SK_CUDA(cudaMemsetAsync(vec, 0, n * sizeof(T), st));  // :144-158
  const LRPair<T> lr(L, R);
  launch_spmv<T>(A, x, EpiMinInit<T>{b, v, z, lr.invl, lr.invr, lr.fused, c.sc, ms}, c.ws, nullptr, st);
  if (!lr.fused) {
    apply_lr<T>(lr, n, v, tmp, z, c, st);
    launch_vec(n, OpMinInitDot<T>{v, z, c.sc, ms}, c.ws, nullptr, st);
  }
  launch_vec(n, OpMinScale<T>{v, z, ms, T(0)}, c.ws, c.sc, st);
  SK_CUDA(cudaGetLastError());
  if ((s = read_scalars(c.sc, &h, st)) != SK_OK) return s;
  if (!h.done && cfg->max_iterations <= 0) h.done = 1;
  const bool graphs = capturable(L) && capturable(R);
  if (graphs && (s = solve_stream(A, st, &st)) != SK_OK) return s;
  auto steps_of = [&](i64 cnt) {
    for (i64 j = 0; j < cnt; ++j) {  // minres_step (:225-234)
      launch_spmv<T>(A, z, EpiMinW<T>{w, z, ms}, c.ws, c.sc, st);
      launch_vec(n, OpMinLanczos<T>{w, v, vp, lr.invl, lr.invr, lr.fused, c.sc, ms, c.hist, T(0), T(0)}, c.ws,
                 c.sc, st);
      if (!lr.fused) {
        apply_lr<T>(lr, n, w, tmp, vp, c, st);
        launch_vec(n, OpMinDot<T>{w, vp, c.sc, ms, c.hist}, c.ws, c.sc, st);
      }
      launch_vec(n, OpMinUpdate<T>{d, dp, x, z, v, vp, w, ms, T(0), T(0), T(0), T(0), T(0), 0}, c.ws, nullptr, st);
    }
  };
  StepGraph sg;
  constexpr i64 kMaxChunk = 32;
  i64 chunk = 4;
  while (!h.done) {
    if (graphs && chunk == kMaxChunk) {
      if ((s = sg.replay(st, chunk, steps_of)) != SK_OK) return s;
    } else {
      steps_of(chunk);
    }
    SK_CUDA(cudaGetLastError());
    if ((s = read_scalars(c.sc, &h, st)) != SK_OK) return s;
    chunk = std::min<i64>(chunk * 2, kMaxChunk);
  }
  return finish_summary(c, st, out, history_host);
}

// Keeps [base, base + bytes) resident in L2 for the kernels of stream `st`
// while it lives: a persisting access-policy window on the stream and a
// persisting set-aside of the same size (both settings of this process's
// context only; the previous limit is restored and the persisting lines are
// released on release()).  Sizes above the device's maximum shrink the hit
// ratio accordingly.  A null stream disables it.
struct L2Window {
  cudaStream_t st = nullptr;
  size_t prev_limit = 0;
  bool on = false;
  L2Window(cudaStream_t s, void* base, size_t bytes) {
    if (!s || bytes == 0) return;
    int dev = 0, maxp = 0, maxw = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, dev);
    cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, dev);
    if (maxp <= 0 || maxw <= 0) return;
    if (cudaDeviceGetLimit(&prev_limit, cudaLimitPersistingL2CacheSize) != cudaSuccess) return;
    const size_t want = std::min<size_t>(bytes, static_cast<size_t>(maxw));
    const size_t setaside = std::min<size_t>(want, static_cast<size_t>(maxp));
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, setaside) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    cudaStreamAttrValue attr{};
    attr.accessPolicyWindow.base_ptr = base;
    attr.accessPolicyWindow.num_bytes = want;
    attr.accessPolicyWindow.hitRatio = static_cast<float>(std::min(1.0, double(setaside) / double(want)));
    attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    if (cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &attr) != cudaSuccess) {
      cudaGetLastError();
      cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, prev_limit);
      return;
    }
    st = s;
    on = true;
  }
  void release() {
    if (!on) return;
    cudaStreamAttrValue attr{};
    attr.accessPolicyWindow.num_bytes = 0;
    cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &attr);
    cudaStreamSynchronize(st);
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, prev_limit);
    on = false;
  }
  ~L2Window() { release(); }
};

// ==================================================================
// Mixed precision: FP32 Jacobi-CG inside FP64 iterative refinement.
// No reference counterpart (the reference runs one precision per solve);
// its inner solver is conjugate_gradient.hpp:122-312 instantiated for float
// on the FP32 copy of the matrix values, and the outer loop keeps the
// residual r = b - A x, the solution update and the stopping test in FP64.
// ==================================================================

// r = b - A x in FP64 with ||r||^2.
struct EpiResid64 {
  static constexpr int kNR = 1;
  const double* b;
  double* r;
  Scalars* sc;
  __device__ void operator()(int row, double ax, double* red) const {
    const double ri = __dsub_rn(b[row], ax);
    r[row] = ri;
    red[0] += ri * ri;
  }
  __device__ void finalize(const double* t) const { sc->rnorm = sqrt(t[0]); }
};

// inner right-hand side: r32 = r / ||r||, and the inner guess d = 0
struct OpScaleDown {
  static constexpr int kNR = 0;
  const double* r;
  float* r32;
  float* d32;
  double inv;
  __device__ bool prepare(const Scalars* s) {
    inv = 1.0 / s->rnorm;
    return true;
  }
  struct In { double r; };
  __device__ In load(i64 i) const { return {r[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const {
    r32[i] = static_cast<float>(q.r * inv);
    d32[i] = 0.0f;
  }
  __device__ void finalize(const double*) const {}
};

// The scaled inner right-hand side of the Jacobi inner solve on
// S = D^-1/2 A D^-1/2: r32 = D^-1/2 r / ||r||, and the inner guess 0.
struct OpScaleDownSym {
  static constexpr int kNR = 0;
  const double* r;
  const double* isq;
  float* r32;
  float* d32;
  double inv;
  __device__ bool prepare(const Scalars* s) {
    inv = 1.0 / s->rnorm;
    return true;
  }
  struct In { double r, s; };
  __device__ In load(i64 i) const { return {r[i], isq[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const {
    r32[i] = static_cast<float>(q.r * q.s * inv);
    d32[i] = 0.0f;
  }
  __device__ void finalize(const double*) const {}
};

// x += ||r|| D^-1/2 y (the scaled inner solution y back in A's variables)
struct OpRefineSym {
  static constexpr int kNR = 0;
  double* x;
  const float* d32;
  const double* isq;
  double scale;
  __device__ bool prepare(const Scalars* s) {
    scale = s->rnorm;
    return true;
  }
  struct In { double x, s; float d; };
  __device__ In load(i64 i) const { return {x[i], isq[i], d32[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const {
    x[i] = q.x + scale * (q.s * static_cast<double>(q.d));
  }
  __device__ void finalize(const double*) const {}
};

// x += ||r|| d
struct OpRefine {
  static constexpr int kNR = 0;
  double* x;
  const float* d32;
  double scale;
  __device__ bool prepare(const Scalars* s) {
    scale = s->rnorm;
    return true;
  }
  struct In { double x; float d; };
  __device__ In load(i64 i) const { return {x[i], d32[i]}; }
  __device__ void apply(i64 i, In const& q, double*) const { x[i] = q.x + scale * static_cast<double>(q.d); }
  __device__ void finalize(const double*) const {}
};

// FP32 Jacobi for the inner solves: the FP64 inverse diagonal (jacobi.hpp:
// 27-35 on the FP64 values) rounded to float; exact zeros are counted.
__global__ void inv_diag32_kernel(i64 n, const int* __restrict__ rp, const int* __restrict__ ci,
                                  const double* __restrict__ v, float* __restrict__ inv32,
                                  unsigned long long* zeros) {
  const i64 i = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int lo = rp[i], hi = rp[i + 1];
  const int end = hi;
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (ci[mid] < i) lo = mid + 1; else hi = mid;
  }
  const double d = (lo < end && ci[lo] == i) ? v[lo] : 0.0;
  if (d == 0.0) atomicAdd(zeros, 1ull);
  inv32[i] = d == 0.0 ? 0.0f : static_cast<float>(__ddiv_rn(1.0, d));
}

static sk_status mixed_cg_solve(sk_matrix A, bool jacobi, const double* b, double* x,
                                const sk_mixed_config* cfg, sk_mixed_summary* out, double* history,
                                cudaStream_t st) {
  Range range_("sk mixed_cg");
  const i64 n = A->nrow;
  *out = sk_mixed_summary{};
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point t0) {
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  };
  const auto t_setup = clk::now();
  if (!f32_values(A)) {
    sk_status s0 = sk_matrix_add_f32_values(A);
    if (s0 != SK_OK) return s0;
  }
  // One workspace for the whole solve (allocated on the first call, reused
  // after; the FP32 Jacobi is built once per handle):
  //   [ inner FP32 CG region | d32 | inv32 ]  <- kept resident in L2
  //   [ r32 | r64 | outer scalars, counters, reduction slots ]
  // The inner solve runs as one persistent launch (sk_mixed.cu) when the
  // handle allows it, else as one kernel per CG step (cg_solve<float>).
  bool persistent = false;
  if (cfg->inner_kernel == 0 && jacobi) {
    // the persistent Jacobi inner solve runs on S = D^-1/2 A D^-1/2 (formed
    // once per handle); without it, the per-step inner solve is used
    bool sym_ok = false;
    sk_status s0 = inner_sym_prepare(A, st, &sym_ok);
    if (s0 != SK_OK) return s0;
    persistent = sym_ok && inner_persistent_ok(A, true);
  } else if (cfg->inner_kernel == 0) {
    persistent = inner_persistent_ok(A, false);
  }
  const double* isq = persistent && jacobi ? inner_sym_isq(A) : nullptr;
  out->inner_kernel = persistent ? 0 : 1;
  const int cap = spmv_grid(A);
  // persistent form: p, q and the inner residual in the first three
  // vectors of the inner region
  const size_t pstride = static_cast<size_t>((n + 8 + 63) / 64 * 64);
  const size_t inner_bytes =
      (std::max(common_bytes(A, 5, static_cast<size_t>(n + 8) * 4, 0, 0), 3 * pstride * 4) + 255) & ~size_t(255);
  const size_t pscratch_bytes = (inner_persistent_scratch(A) + 255) & ~size_t(255);
  const size_t need = inner_bytes + 4096 + static_cast<size_t>(n + 64) * (8 + 4 + 4 + 4) + 4096 +
                      static_cast<size_t>(cap) * kMaxRed * 8 + 1024 + pscratch_bytes + 256;
  const bool fresh = A->ws2_bytes < need;  // reused after the first call
  if (fresh) {
    if (A->ws2) {
      cudaStreamSynchronize(st);
      cudaFree(A->ws2);
      A->ws2 = nullptr;
    }
    SK_CUDA(cudaMalloc(&A->ws2, need));
    A->ws2_bytes = need;
  }
  char* inner_base = static_cast<char*>(A->ws2);
  Carver cv{inner_base};
  cv.off = inner_bytes;
  float* d32 = cv.take<float>(static_cast<size_t>(n + 8) * 4);
  float* inv32 = cv.take<float>(static_cast<size_t>(n + 8) * 4);
  const size_t resident_bytes = cv.off;
  float* r32 = cv.take<float>(static_cast<size_t>(n + 8) * 4);
  double* r = cv.take<double>(static_cast<size_t>(n + 8) * 8);
  Scalars* so = cv.take<Scalars>(sizeof(Scalars));
  unsigned* cnt = cv.take<unsigned>(16);
  double* partials = cv.take<double>(static_cast<size_t>(cap) * kMaxRed * 8);
  void* pscratch = cv.take<char>(pscratch_bytes);
  float* pv = reinterpret_cast<float*>(inner_base);
  float* qv = pv + pstride;
  float* rv = qv + pstride;
  SK_CUDA(cudaMemsetAsync(so, 0, sizeof(Scalars), st));
  SK_CUDA(cudaMemsetAsync(cnt, 0, 16, st));
  sk_precond_s jac32{};
  if (jacobi) {
    // built once per handle (ws2 keeps it): no allocation on later calls
    if (fresh || !A->mixed_jacobi_ready) {
      unsigned long long* zeros = reinterpret_cast<unsigned long long*>(cnt + 2);
      SK_CUDA(cudaMemsetAsync(zeros, 0, 8, st));
      SK_LAUNCH(inv_diag32_kernel, ceil_div(n, kThreads), kThreads, 0, st, n, A->csr.row_ptr, A->csr.col_ind,
                static_cast<const double*>(A->csr.vals), inv32, zeros);
      unsigned long long nz = 0;
      SK_CUDA(cudaMemcpyAsync(&nz, zeros, 8, cudaMemcpyDeviceToHost, st));
      SK_CUDA(cudaStreamSynchronize(st));
      if (nz) return fail(SK_ZERO_DIAGONAL, "jacobi: zero diagonal entry");
      A->mixed_jacobi_ready = true;
    }
    jac32.kind = 1;
    jac32.A = A;
    jac32.dtype = SK_F32;
    jac32.n = n;
    jac32.inv_diag = inv32;
  }
  RedWs ws{partials, cnt, cap};
  double bnorm = 0;
  {
    // ||b|| in FP64
    launch_vec(n, OpNormB<double>{b, so}, ws, nullptr, st);
    Scalars h;
    sk_status s1 = read_scalars(so, &h, st);
    if (s1 != SK_OK) return s1;
    bnorm = h.bnorm;
  }
  out->setup_ms = ms_since(t_setup);
  sk_status status = SK_OK;
  if (bnorm == 0.0) {
    SK_CUDA(cudaMemsetAsync(x, 0, n * 8, st));
    out->converged = 1;
  } else {
    sk_cg_config icfg{cfg->inner_tolerance, cfg->max_inner, cfg->max_inner, 0};
    for (i64 outer = 0;; ++outer) {
      auto t_outer = clk::now();
      launch_spmv<double>(A, x, EpiResid64{b, r, so}, ws, nullptr, st);
      Scalars h;
      status = read_scalars(so, &h, st);
      out->outer_ms += ms_since(t_outer);
      if (status != SK_OK) break;
      out->residual_norm = h.rnorm;
      if (history && cfg->collect_residuals) history[outer] = h.rnorm;
      out->outer_iterations = outer;
      if (h.rnorm / bnorm < cfg->tolerance) {
        out->converged = 1;
        break;
      }
      if (outer >= cfg->max_outer) break;
      if (isq)
        launch_vec(n, OpScaleDownSym{r, isq, rv, d32, 0.0}, ws, so, st);
      else
        launch_vec(n, OpScaleDown{r, persistent ? rv : r32, d32, 0.0}, ws, so, st);
      // The last step needs only the remaining factor tol ||b|| / ||r||: its
      // inner tolerance is tightened to half of that when that is below the
      // configured one (floor 1e-7, about what FP32 CG can resolve), so that
      // the refinement ends one step earlier instead of overshooting.
      const double needed = cfg->tolerance * bnorm / h.rnorm;
      icfg.tolerance = cfg->inner_tolerance;
      if (cfg->adaptive_last_step && 0.5 * needed < cfg->inner_tolerance)
        icfg.tolerance = std::max(0.5 * needed, 1e-7);
      sk_summary is{};
      auto t_inner = clk::now();
      Range inner_range("sk mixed_cg inner FP32 solve");
      L2Window win(cfg->l2_window ? st : nullptr, inner_base, resident_bytes);
      if (persistent) {
        InnerResult ir;
        status = inner_cg_persistent(A, jacobi, rv, d32, pv, qv, pscratch, icfg.tolerance, icfg.max_iterations, st,
                                     &ir);
        is.computed_iterations = ir.iterations;
        is.converged = ir.converged;
      } else {
        status = cg_solve<float>(A, jacobi ? &jac32 : nullptr, nullptr, r32, d32, &icfg, &is, nullptr, st,
                                 f32_values(A), inner_base);
      }
      win.release();
      out->inner_ms += ms_since(t_inner);
      if (status != SK_OK) break;
      out->inner_iterations += is.computed_iterations;
      t_outer = clk::now();
      if (isq)
        launch_vec(n, OpRefineSym{x, d32, isq, 0.0}, ws, so, st);
      else
        launch_vec(n, OpRefine{x, d32, 0.0}, ws, so, st);
      out->outer_ms += ms_since(t_outer);
    }
  }
  SK_CUDA(cudaStreamSynchronize(st));
  return status;
}

// Mixed-precision FGMRES(m): FP64 iterative refinement around an FP32
// FGMRES(m) inner solve.  FP64 stays in the outer residual r = b - A x
// (EpiResid64), the solution update x += ||r|| d (OpRefine) and the inner
// solve's Hessenberg least-squares problem (Givens rotations and back
// substitution, FgGivens<double> / FgBackSub<double>); the inner basis
// vectors, the products (the handle's FP32 values) and the Gram-Schmidt
// sums run in FP32 (fgmres.hpp:96-428 in FP32 otherwise).  M is applied in
// FP32 (Jacobi, Chebyshev) or, for a two-level preconditioner, in FP64
// between a widening and a narrowing pass.
static sk_status mixed_fgmres_solve(sk_matrix A, sk_precond M, const double* b, double* x,
                                    const sk_mixed_fgmres_config* cfg, sk_mixed_summary* out, double* history,
                                    cudaStream_t st) {
  Range range_("sk mixed_fgmres");
  const i64 n = A->nrow;
  *out = sk_mixed_summary{};
  out->inner_kernel = 1;
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point t0) {
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  };
  const auto t_setup = clk::now();
  sk_status s = SK_OK;
  if (!f32_values(A) && (s = sk_matrix_add_f32_values(A)) != SK_OK) return s;
  if ((s = precond_prepare_f32(M, st)) != SK_OK) return s;
  // the outer vectors in the second workspace (shared with the mixed CG,
  // whose FP32 Jacobi there is rebuilt on its next call)
  const int cap = spmv_grid(A);
  const size_t need = 4096 + static_cast<size_t>(n + 64) * (8 + 4 + 4) + 4096 +
                      static_cast<size_t>(std::max(cap, vec_grid(n))) * kMaxRed * 8 + 2048;
  if (A->ws2_bytes < need) {
    if (A->ws2) {
      cudaStreamSynchronize(st);
      cudaFree(A->ws2);
      A->ws2 = nullptr;
    }
    SK_CUDA(cudaMalloc(&A->ws2, need));
    A->ws2_bytes = need;
  }
  A->mixed_jacobi_ready = false;
  Carver cv{static_cast<char*>(A->ws2)};
  double* r = cv.take<double>(static_cast<size_t>(n + 8) * 8);
  float* r32 = cv.take<float>(static_cast<size_t>(n + 8) * 4);
  float* d32 = cv.take<float>(static_cast<size_t>(n + 8) * 4);
  Scalars* so = cv.take<Scalars>(sizeof(Scalars));
  unsigned* cnt = cv.take<unsigned>(16);
  double* partials = cv.take<double>(static_cast<size_t>(std::max(cap, vec_grid(n))) * kMaxRed * 8);
  SK_CUDA(cudaMemsetAsync(so, 0, sizeof(Scalars), st));
  SK_CUDA(cudaMemsetAsync(cnt, 0, 16, st));
  RedWs ws{partials, cnt, std::max(cap, vec_grid(n))};
  double bnorm = 0;
  {
    launch_vec(n, OpNormB<double>{b, so}, ws, nullptr, st);
    Scalars h;
    if ((s = read_scalars(so, &h, st)) != SK_OK) return s;
    bnorm = h.bnorm;
  }
  out->setup_ms = ms_since(t_setup);
  if (bnorm == 0.0) {
    SK_CUDA(cudaMemsetAsync(x, 0, n * 8, st));
    SK_CUDA(cudaStreamSynchronize(st));
    out->converged = 1;
    return SK_OK;
  }
  sk_fgmres_config icfg{cfg->inner_tolerance, cfg->restart_dimension, cfg->max_inner, 0};
  for (i64 outer = 0;; ++outer) {
    auto t_outer = clk::now();
    launch_spmv<double>(A, x, EpiResid64{b, r, so}, ws, nullptr, st);
    Scalars h;
    s = read_scalars(so, &h, st);
    out->outer_ms += ms_since(t_outer);
    if (s != SK_OK) break;
    out->residual_norm = h.rnorm;
    if (history && cfg->collect_residuals) history[outer] = h.rnorm;
    out->outer_iterations = outer;
    if (h.rnorm / bnorm < cfg->tolerance) {
      out->converged = 1;
      break;
    }
    if (outer >= cfg->max_outer) break;
    launch_vec(n, OpScaleDown{r, r32, d32, 0.0}, ws, so, st);
    // the last step needs only the remaining factor tol ||b|| / ||r||
    // (floor 1e-6, about what FP32 FGMRES resolves)
    const double needed = cfg->tolerance * bnorm / h.rnorm;
    icfg.tolerance = cfg->inner_tolerance;
    if (cfg->adaptive_last_step && 0.5 * needed < cfg->inner_tolerance)
      icfg.tolerance = std::max(0.5 * needed, 1e-6);
    sk_summary is{};
    auto t_inner = clk::now();
    Range inner_range("sk mixed_fgmres inner FP32 solve");
    s = fgmres_solve<float>(A, M, r32, d32, &icfg, &is, nullptr, st, nullptr, 0.0, nullptr, nullptr, false,
                            f32_values(A), true);
    out->inner_ms += ms_since(t_inner);
    if (s != SK_OK) break;
    out->inner_iterations += is.computed_iterations;
    t_outer = clk::now();
    launch_vec(n, OpRefine{x, d32, 0.0}, ws, so, st);
    out->outer_ms += ms_since(t_outer);
  }
  SK_CUDA(cudaStreamSynchronize(st));
  return s;
}

}  // namespace sk

using namespace sk;

namespace {

sk_status check_solver_args(sk_matrix A, sk_precond L, sk_precond R, const void* b, void* x) {
  SK_CHECK(A, SK_INVALID_ARG, "null matrix handle");
  SK_CHECK(A->nrow == A->ncol, SK_INVALID_ARG, "solvers need a square matrix");
  SK_CHECK(A->nrow == 0 || (b && x), SK_INVALID_ARG, "null b or x");
  for (sk_precond M : {L, R})
    if (M) {
      SK_CHECK(M->dtype == A->dtype, SK_INVALID_ARG, "preconditioner dtype differs from the matrix");
      SK_CHECK(M->n == A->nrow, SK_INVALID_ARG, "preconditioner size differs from the matrix");
    }
  return SK_OK;
}

template <typename Cfg, typename F>
sk_status host_wrapper(sk_matrix A, const void* b_host, void* x_host, F&& solve_dev) {
  SK_CHECK(A, SK_INVALID_ARG, "null matrix handle");
  const size_t V = A->dtype == SK_F64 ? 8 : 4;
  const size_t bytes = static_cast<size_t>(A->nrow) * V;
  void* bx = nullptr;
  SK_CUDA(cudaMalloc(&bx, 2 * bytes + 512));
  char* bd = static_cast<char*>(bx);
  char* xd = bd + ((bytes + 255) & ~size_t(255));
  cudaError_t e = cudaMemcpyAsync(bd, b_host, bytes, cudaMemcpyHostToDevice, A->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(xd, x_host, bytes, cudaMemcpyHostToDevice, A->stream);
  if (e != cudaSuccess) {
    cudaFree(bx);
    return cuda_fail(e, "copy in");
  }
  sk_status s = solve_dev(bd, xd);
  if (s == SK_OK) {
    e = cudaMemcpyAsync(x_host, xd, bytes, cudaMemcpyDeviceToHost, A->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
    if (e != cudaSuccess) s = cuda_fail(e, "copy out");
  }
  cudaFree(bx);
  return s;
}

}  // namespace

extern "C" {

sk_status sk_cg_solve(sk_matrix A, sk_precond left, sk_precond right, const void* b_dev, void* x_dev,
                      const sk_cg_config* cfg, sk_summary* out, double* history_host, sk_stream s) {
  sk_status st = check_solver_args(A, left, right, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  SK_CHECK(cfg->restart_iterations > 0, SK_INVALID_ARG,
           "restart_iterations must be positive (the reference takes k % restart_iterations)");
  SK_CHECK(cfg->max_iterations >= 0, SK_INVALID_ARG, "negative max_iterations");
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64)
    return cg_solve<double>(A, left, right, static_cast<const double*>(b_dev), static_cast<double*>(x_dev),
                            cfg, out, history_host, cs);
  return cg_solve<float>(A, left, right, static_cast<const float*>(b_dev), static_cast<float*>(x_dev), cfg,
                         out, history_host, cs);
}

sk_status sk_bicgstab_solve(sk_matrix A, sk_precond left, sk_precond right, const void* b_dev,
                            void* x_dev, const sk_bicgstab_config* cfg, sk_summary* out,
                            double* history_host, sk_stream s) {
  sk_status st = check_solver_args(A, left, right, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  SK_CHECK(cfg->max_iterations >= 0, SK_INVALID_ARG, "negative max_iterations");
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64)
    return bicgstab_solve<double>(A, left, right, static_cast<const double*>(b_dev),
                                  static_cast<double*>(x_dev), cfg, out, history_host, cs);
  return bicgstab_solve<float>(A, left, right, static_cast<const float*>(b_dev), static_cast<float*>(x_dev),
                               cfg, out, history_host, cs);
}

sk_status sk_fgmres_solve(sk_matrix A, sk_precond M, const void* b_dev, void* x_dev,
                          const sk_fgmres_config* cfg, sk_summary* out, double* history_host,
                          sk_stream s) {
  sk_status st = check_solver_args(A, M, nullptr, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  SK_CHECK(cfg->max_iterations >= 0, SK_INVALID_ARG, "negative max_iterations");
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64)
    return fgmres_solve<double>(A, M, static_cast<const double*>(b_dev), static_cast<double*>(x_dev), cfg,
                                out, history_host, cs);
  return fgmres_solve<float>(A, M, static_cast<const float*>(b_dev), static_cast<float*>(x_dev), cfg, out,
                             history_host, cs);
}

sk_status sk_gmres_solve(sk_matrix A, sk_precond left, sk_precond right, const void* b_dev, void* x_dev,
                         const sk_gmres_config* cfg, sk_summary* out, double* history_host, sk_stream s) {
  sk_status st = check_solver_args(A, left, right, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  SK_CHECK(cfg->max_iterations >= 0, SK_INVALID_ARG, "negative max_iterations");
  const sk_fgmres_config fc{cfg->tolerance, cfg->restart_dimension, cfg->max_iterations, cfg->collect_residuals};
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64)
    st = fgmres_solve<double>(A, right, static_cast<const double*>(b_dev), static_cast<double*>(x_dev), &fc, out,
                              history_host, cs, nullptr, 0.0, nullptr, left, true);
  else
    st = fgmres_solve<float>(A, right, static_cast<const float*>(b_dev), static_cast<float*>(x_dev), &fc, out,
                             history_host, cs, nullptr, 0.0, nullptr, left, true);
  if (st != SK_OK) return st;
  for (sk_precond P : {left, right}) {
    const sk_precond_s* net_prec = P && P->kind == 4 ? P->smoother : P;
    if (net_prec && net_prec->kind == 3) {
      sk_status ns = sk_net_status(net_prec->net);
      if (ns != SK_OK) return ns;
    }
  }
  return SK_OK;
}

sk_status sk_cgs_solve(sk_matrix A, sk_precond left, sk_precond right, const void* b_dev, void* x_dev,
                       const sk_cgs_config* cfg, sk_summary* out, double* history_host, sk_stream s) {
  sk_status st = check_solver_args(A, left, right, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64)
    return cgs_solve<double>(A, left, right, static_cast<const double*>(b_dev), static_cast<double*>(x_dev), cfg,
                             out, history_host, cs);
  return cgs_solve<float>(A, left, right, static_cast<const float*>(b_dev), static_cast<float*>(x_dev), cfg, out,
                          history_host, cs);
}

sk_status sk_minres_solve(sk_matrix A, sk_precond left, sk_precond right, const void* b_dev, void* x_dev,
                          const sk_minres_config* cfg, sk_summary* out, double* history_host, sk_stream s) {
  sk_status st = check_solver_args(A, left, right, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  cudaStream_t cs = pick_stream(A, s);
  if (A->dtype == SK_F64)
    return minres_solve<double>(A, left, right, static_cast<const double*>(b_dev), static_cast<double*>(x_dev),
                                cfg, out, history_host, cs);
  return minres_solve<float>(A, left, right, static_cast<const float*>(b_dev), static_cast<float*>(x_dev), cfg, out,
                             history_host, cs);
}

sk_status sk_fgmres_fallback_solve(sk_matrix A, sk_precond M, sk_precond fallback, const double* b_dev,
                                   double* x_dev, const sk_fgmres_config* cfg, double stall_ratio,
                                   sk_summary* out, double* history_host, int64_t* switched_at, sk_stream s) {
  sk_status st = check_solver_args(A, M, fallback, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out && M, SK_INVALID_ARG, "null config, summary or preconditioner");
  SK_CHECK(A->dtype == SK_F64, SK_INVALID_ARG, "the fallback driver solves in FP64");
  SK_CHECK(cfg->max_iterations >= 0, SK_INVALID_ARG, "negative max_iterations");
  cudaStream_t cs = pick_stream(A, s);
  st = fgmres_solve<double>(A, M, b_dev, x_dev, cfg, out, history_host, cs, fallback, stall_ratio, switched_at);
  if (st != SK_OK) return st;
  if (M->kind == 3) return sk_net_status(M->net);
  if (M->kind == 4 && M->smoother && M->smoother->kind == 3) return sk_net_status(M->smoother->net);
  return SK_OK;
}

sk_status sk_cg_solve_host(sk_matrix A, sk_precond left, sk_precond right, const void* b_host,
                           void* x_host, const sk_cg_config* cfg, sk_summary* out, double* history_host) {
  return host_wrapper<sk_cg_config>(A, b_host, x_host, [&](void* bd, void* xd) {
    return sk_cg_solve(A, left, right, bd, xd, cfg, out, history_host, A->stream);
  });
}

sk_status sk_bicgstab_solve_host(sk_matrix A, sk_precond left, sk_precond right, const void* b_host,
                                 void* x_host, const sk_bicgstab_config* cfg, sk_summary* out,
                                 double* history_host) {
  return host_wrapper<sk_bicgstab_config>(A, b_host, x_host, [&](void* bd, void* xd) {
    return sk_bicgstab_solve(A, left, right, bd, xd, cfg, out, history_host, A->stream);
  });
}

sk_status sk_gmres_solve_host(sk_matrix A, sk_precond left, sk_precond right, const void* b_host, void* x_host,
                              const sk_gmres_config* cfg, sk_summary* out, double* history_host) {
  return host_wrapper<sk_gmres_config>(A, b_host, x_host, [&](void* bd, void* xd) {
    return sk_gmres_solve(A, left, right, bd, xd, cfg, out, history_host, A->stream);
  });
}

sk_status sk_cgs_solve_host(sk_matrix A, sk_precond left, sk_precond right, const void* b_host, void* x_host,
                            const sk_cgs_config* cfg, sk_summary* out, double* history_host) {
  return host_wrapper<sk_cgs_config>(A, b_host, x_host, [&](void* bd, void* xd) {
    return sk_cgs_solve(A, left, right, bd, xd, cfg, out, history_host, A->stream);
  });
}

sk_status sk_minres_solve_host(sk_matrix A, sk_precond left, sk_precond right, const void* b_host, void* x_host,
                               const sk_minres_config* cfg, sk_summary* out, double* history_host) {
  return host_wrapper<sk_minres_config>(A, b_host, x_host, [&](void* bd, void* xd) {
    return sk_minres_solve(A, left, right, bd, xd, cfg, out, history_host, A->stream);
  });
}

sk_status sk_fgmres_solve_host(sk_matrix A, sk_precond M, const void* b_host, void* x_host,
                               const sk_fgmres_config* cfg, sk_summary* out, double* history_host) {
  return host_wrapper<sk_fgmres_config>(A, b_host, x_host, [&](void* bd, void* xd) {
    return sk_fgmres_solve(A, M, bd, xd, cfg, out, history_host, A->stream);
  });
}

}  // extern "C"

extern "C" sk_status sk_mixed_cg_solve(sk_matrix A, int32_t jacobi, const double* b_dev, double* x_dev,
                                       const sk_mixed_config* cfg, sk_mixed_summary* out, double* history_host,
                                       sk_stream s) {
  sk_status st = check_solver_args(A, nullptr, nullptr, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  SK_CHECK(A->dtype == SK_F64 && A->format == SK_CSR, SK_INVALID_ARG,
           "the mixed-precision solver needs an FP64 CSR handle");
  SK_CHECK(cfg->max_outer >= 0 && cfg->max_inner > 0, SK_INVALID_ARG, "bad iteration limits");
  // The solve runs on the handle's own stream (an access-policy window needs
  // a created stream), ordered after the caller's stream.
  SK_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(s)));
  return mixed_cg_solve(A, jacobi != 0, b_dev, x_dev, cfg, out, history_host, A->stream);
}

extern "C" sk_status sk_mixed_fgmres_solve(sk_matrix A, sk_precond M, const double* b_dev, double* x_dev,
                                           const sk_mixed_fgmres_config* cfg, sk_mixed_summary* out,
                                           double* history_host, sk_stream s) {
  sk_status st = check_solver_args(A, M, nullptr, b_dev, x_dev);
  if (st != SK_OK) return st;
  SK_CHECK(cfg && out, SK_INVALID_ARG, "null config or summary");
  SK_CHECK(A->dtype == SK_F64 && A->format == SK_CSR, SK_INVALID_ARG,
           "the mixed-precision solver needs an FP64 CSR handle");
  SK_CHECK(cfg->max_outer >= 0 && cfg->max_inner > 0, SK_INVALID_ARG, "bad iteration limits");
  SK_CHECK(cfg->restart_dimension >= 1 && cfg->restart_dimension <= 4096, SK_INVALID_ARG,
           "restart_dimension must be in [1, 4096]");
  SK_CHECK(!M || M->kind != 3, SK_NOT_SUPPORTED,
           "the learned preconditioner has no FP32 apply (use it as a two-level smoother)");
  SK_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(s)));
  return mixed_fgmres_solve(A, M, b_dev, x_dev, cfg, out, history_host, A->stream);
}
