// sk_internal.cuh -- shared definitions of the sm_100a library: device
// matrix layouts, status plumbing, launch accounting and the deterministic
// grid-wide reduction used by every fused kernel.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sparkit_b200.h"

#include <nvtx3/nvToolsExt.h>

namespace sk {

using i64 = std::int64_t;

constexpr int kThreads = 256;    // CTA size of the streaming kernels
constexpr int kTileNnz = 2048;   // CSR: stored entries staged per CTA
constexpr int kRowsMax = 256;    // CSR: rows per CTA (one per thread)
constexpr int kBsrTileVals = 4096;  // BSR: block values staged per CTA
constexpr int kMaxRed = 4;       // fused reductions carried per kernel
constexpr int kSellMaxRow = 64;  // CSR rows up to this length use SELL-32
constexpr int kDiaMax = 16;      // diagonals of the diagonal copy of a CSR handle
constexpr int kPanelSmem = 220 * 1024;  // dynamic shared memory of a column-panel CTA (at most)
constexpr int kPanelStages = 3;           // chunk stages in flight per column-panel CTA
constexpr int kPanelChunkEntries = 1536;  // entries per chunk (a multiple of 8)
constexpr int kPanelChunkSlices = 48;     // slices (or slice pieces) per chunk
constexpr int kHybLong = 32;     // rows longer than this take a warp in the split product

// ------------------------------------------------------------------
// Status plumbing
// ------------------------------------------------------------------
void set_error(std::string const& msg);
sk_status fail(sk_status st, std::string const& msg);
sk_status cuda_fail(cudaError_t e, char const* what);

#define SK_CUDA(call)                                                    \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) return ::sk::cuda_fail(e_, #call);            \
  } while (0)

#define SK_CHECK(cond, st, msg)                                          \
  do {                                                                   \
    if (!(cond)) return ::sk::fail((st), (msg));                         \
  } while (0)

// A named NVTX range (solver phases in a profiler's timeline); NVTX is
// header-only and costs nothing unless a tool is attached.
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(Range const&) = delete;
  Range& operator=(Range const&) = delete;
};

// Bound of every grid-barrier wait of the persistent kernels, in ns, and the
// extra arrivals each barrier waits for (0, or 1 when sk_debug_set_wait
// makes the barriers unmeetable to test the timeout path).
unsigned long long wait_limit_ns();
unsigned wait_target_bias();

// Every kernel launch of the library goes through SK_LAUNCH so that
// sk_launch_count() can account for them.
extern std::atomic<i64> g_launches;
#define SK_LAUNCH(kernel, grid, block, smem, stream, ...)                \
  do {                                                                   \
    ::sk::g_launches.fetch_add(1, std::memory_order_relaxed);            \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);          \
  } while (0)

// ------------------------------------------------------------------
// Device layouts
// ------------------------------------------------------------------

// CSR: int32 indices; arrays padded by 4 entries so that the 16-byte
// vector loads of a tile's last group stay inside the allocation.
// part[nparts+1] are the first rows of the row blocks one CTA handles.
struct Csr {
  int* row_ptr = nullptr;
  int* col_ind = nullptr;
  void* vals = nullptr;
  float* vals32 = nullptr;  // optional FP32 copy of FP64 values
  int2* tiles = nullptr;  // nparts + 1 of {first row, first entry}
  unsigned char* lanes = nullptr;  // per tile: 1 = one thread per row
  int nparts = 0;
  // SELL-32 copy used by the product when every row is short: slice s holds
  // rows 32s..32s+31, padded to the slice's longest row and stored slot by
  // slot (entry k of row 32s+l at sell_off[s] + 32k + l), so that a warp
  // reads each slot of its 32 rows as one contiguous segment.
  bool sell = false;
  int* sell_col = nullptr;
  void* sell_vals = nullptr;
  float* sell_vals32 = nullptr;
  int* sell_off = nullptr;             // nslices + 1 entry offsets
  unsigned char* sell_len = nullptr;   // entries per row
  i64 sell_entries = 0;                // padded size
  // Split product for skewed rows (when SELL-32 is refused and rows longer
  // than kHybLong entries hold most of the entries): the long rows, by
  // decreasing length, one warp each; the short rows, in row order, one
  // thread each.  A share hyb_long_frac of the kernel's one wave of CTAs
  // takes the long rows.
  bool hyb = false;
  int* hyb_short = nullptr;
  int* hyb_long = nullptr;
  int hyb_nshort = 0, hyb_nlong = 0;
  double hyb_long_frac = 0.0;
  // Column-panel copy (sk_matrix_add_panels, sk_panel.cu): every row summed
  // in the reference's order whatever its length.  The rows are cut into pn_blocks
  // row blocks of about equal entries, one CTA each; the columns into
  // pn_panels panels of pn_width columns.  A CTA walks the panels in
  // order, holding panel k of x in shared memory (double-buffered) and a
  // running sum per row of its block, so that a row's entries are still
  // added one after another in ascending column order from 0 (the bits of
  // sparse_blas.hpp:25-28) while every gather of x reads shared memory.
  // The entries of block b in panel k form segments (one per row that has
  // entries there), sorted by decreasing length and packed 32 to a slice,
  // a lane each.  Slot j of a slice holds entry j of the lanes whose
  // segment is longer than j (lanes 0 .. c_j - 1), right after slot j - 1,
  // without padding.  A panel's slices are cut into chunks of at most
  // kPanelChunkEntries entries and kPanelChunkSlices slices (at least one
  // chunk per panel, possibly empty); a slice with more entries than that
  // is cut by slots into pieces that go to successive chunks.  A chunk is copied whole into a shared-memory stage by
  // the bulk-copy engine: its values and 16-bit column offsets (from a
  // multiple of 8 entries) and its table (pn_meta: the pieces' entry
  // offsets, padded to 4 words, then 32 segment words per piece, local row
  // | length << 16, 0 for none).  pn_chunk[c] = {first entry, entries
  // rounded up to 8, first meta word, meta words}; pn_chunk_kn[c] = panel
  // | pieces << 16.
  bool panel = false;
  int pn_blocks = 0, pn_panels = 0, pn_width = 0, pn_smem = 0, pn_stage_bytes = 0;
  int* pn_row0 = nullptr;        // pn_blocks + 1 first rows
  int* pn_chunk_ptr = nullptr;   // pn_blocks + 1 first chunks
  int4* pn_chunk = nullptr;
  int* pn_chunk_kn = nullptr;
  unsigned* pn_meta = nullptr;
  unsigned short* pn_col = nullptr;
  void* pn_vals = nullptr;
  int* pn_err = nullptr;         // set by a stage wait that ran out
  i64 pn_entries = 0;            // stored entries, chunk starts rounded up to 8
  // Diagonal copy (sk_matrix_add_diagonals) of a handle whose entries lie
  // on at most kDiaMax diagonals c - r = off[d] and whose rows hold their
  // columns in ascending order, slice-major like the SELL-32 copy: A(r, r +
  // off[d]) at ((r / 32) * dia_n + d) * 32 + r % 32, so that the values a
  // warp reads for its 32 rows are dia_n consecutive 32-value segments.
  // Bit d of mask[r] says whether row r stores that entry.  The product
  // sums a row's stored entries in ascending column order, the CSR order.
  int dia_n = 0;
  int dia_off[kDiaMax] = {};
  i64 dia_len = 0;  // values in the copy: ceil(nrow / 32) * 32 * dia_n
  void* dia_vals = nullptr;
  float* dia_vals32 = nullptr;
  unsigned short* dia_mask = nullptr;
  // Symmetrically scaled FP32 copies for the Jacobi inner solve of the
  // mixed solver (sk_mixed.cu): S = D^-1/2 A D^-1/2 without its unit
  // diagonal, in the SELL-32 layout (sym_off, sym_len, sym_col, sym_val) or
  // as diagonal planes without the main one (sym_dn planes at sym_doff,
  // values sym_dval, row masks sym_dmask, laid out like the diagonal copy).
  // sym_isq = 1 / sqrt(a_ii) (FP64), sym_diag = a_ii (FP32).  State: 0 not
  // built, 1 built, -1 not possible (a diagonal entry absent or not
  // positive, or no SELL-32 / diagonal copy to derive it from).
  int sym_sell_state = 0, sym_dia_state = 0, sym_diag_state = 0;
  int* sym_off = nullptr;
  unsigned char* sym_len = nullptr;
  int* sym_col = nullptr;
  float* sym_val = nullptr;
  int sym_dn = 0;
  int sym_doff[kDiaMax] = {};
  float* sym_dval = nullptr;
  unsigned short* sym_dmask = nullptr;
  double* sym_isq = nullptr;
  float* sym_diag = nullptr;
};

// ELLPACK: slot-major (column-major) copy of the reference's row-major
// layout: entry k of row i at k * ld + i; rowlen[i] = entries before the
// first -1 sentinel.
struct Ell {
  int* col = nullptr;
  void* vals = nullptr;
  int* rowlen = nullptr;
  i64 width = 0;
  i64 ld = 0;  // slot stride (nrow rounded up, kept off powers of two)
};

// Jagged diagonal: the reference layout with int32 indices; plen[i] is the
// number of diagonals that reach permuted position i.
struct Jad {
  int* perm = nullptr;
  int* jdiag = nullptr;
  int* col = nullptr;
  void* vals = nullptr;
  int* plen = nullptr;
  i64 njd = 0;
};

// BSR: block CSR; part[] as for CSR but over block rows.
struct Bsr {
  int* row_ptr = nullptr;
  int* col = nullptr;
  void* vals = nullptr;
  int* part = nullptr;
  int nparts = 0;
  i64 br = 0, bc = 0, nbr = 0, nbr_mult = 0, nblocks = 0;
  // Sliced copy for 2x2 and 3x3 blocks with at most kSellMaxRow blocks per
  // block row: slice s holds block rows 32s..32s+31 padded to the slice's
  // longest; block k of block row 32s+l has its column at sell_off[s] +
  // 32k + l and its element e at (sell_off[s] + 32k) * br * bc + 32e + l.
  bool sell = false;
  int* sell_col = nullptr;
  void* sell_vals = nullptr;
  int* sell_off = nullptr;
  unsigned char* sell_len = nullptr;
  i64 sell_blocks = 0;
};

// Plan of the pipelined host-buffer product (sk_spmv_host), built on the
// first call: row chunks, the prefix of x each chunk reads, and the copy
// streams and events.
struct HostPipe;
void destroy_host_pipe(HostPipe* p);

}  // namespace sk

struct sk_matrix_s {
  sk_format format;
  sk_dtype dtype;
  int device = 0;
  int sm_count = 148;
  sk::i64 nrow = 0, ncol = 0, nnz = 0;
  sk::Csr csr;
  sk::Ell ell;
  sk::Jad jad;
  sk::Bsr bsr;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocations;
  sk::i64 device_bytes = 0;
  void* io = nullptr;  // x and y buffers of the host-pointer calls
  sk::HostPipe* pipe = nullptr;  // chunk plan of sk_spmv_host
  // Grow-only workspace of the solver calls on this handle.
  void* ws = nullptr;
  size_t ws_bytes = 0;
  void* ws2 = nullptr;  // second workspace (outer loop of the mixed solver)
  size_t ws2_bytes = 0;
  bool mixed_jacobi_ready = false;  // FP32 inverse diagonal held in ws2
  double build_ms = 0;  // device time of the kernels that built the handle on the device
  sk::i64 spmv_bytes() const;
};

struct sk_net_s;

struct sk_precond_s {
  int kind;  // 1 = Jacobi, 2 = Chebyshev, 3 = learned network, 4 = two-level
  sk_matrix A;
  sk_dtype dtype;
  sk::i64 n;
  void* inv_diag = nullptr;  // Jacobi (dtype)
  std::vector<double> coeffs;  // Chebyshev, host copy (double)
  double lambda_min = 0, lambda_max = 0;
  sk::i64 degree = 0;
  void* work = nullptr;  // Chebyshev: 3 n-vectors
  float* inv_diag32 = nullptr;  // FP32 copy for mixed precision
  // learned (kind 3): the network and the matrix's coefficient planes on
  // its grid_nx x grid_ny grid (d, w, e, s, n, 1/d; float)
  sk_net_s* net = nullptr;
  float* coef = nullptr;
  void* xfeat = nullptr;  // BF16 [grid][8]: the fixed input channels (w, e, s, n over d)
  sk::i64 grid_nx = 0, grid_ny = 0;
  // two-level (kind 4): smoother (not owned), agg x agg aggregates of the
  // grid, the dense inverse of the Galerkin coarse operator (coarse_n^2,
  // stored in FP32) and FP64 work vectors
  sk_precond_s* smoother = nullptr;
  sk::i64 agg = 0, coarse_n = 0;
  int post = 0, coarse_first = 0;
  float* coarse_inv = nullptr;  // FP32, row-major nc x nc
  double* tbuf = nullptr;
  double* tbuf2 = nullptr;
  double* rc = nullptr;
  double* zc = nullptr;
  // FP64 staging of an FP32 apply of a two-level preconditioner (the
  // mixed-precision FGMRES): r widened in, z narrowed out
  double* cvt_in = nullptr;
  double* cvt_out = nullptr;
};

namespace sk {

// The FP32 value copy in the layout the product kernel reads.
inline const float* f32_values(const sk_matrix_s* A) {
  return A->csr.dia_n ? A->csr.dia_vals32 : A->csr.sell ? A->csr.sell_vals32 : A->csr.vals32;
}

cudaStream_t pick_stream(sk_matrix A, sk_stream s);

// Makes the FP32 copies an FP32 apply of a preconditioner of an FP64 handle
// reads (the inverse diagonal as float, the handle's FP32 values);
// SK_NOT_SUPPORTED for a preconditioner without an FP32 apply.
sk_status precond_prepare_f32(sk_precond_s* M, cudaStream_t st);
sk_status dev_alloc(sk_matrix A, void** p, size_t bytes);

// Grid-wide deterministic reduction workspace: one slot of kMaxRed doubles
// per CTA plus an arrival counter.  The last CTA to arrive sums the slots in
// CTA order, so the result does not depend on scheduling.
//
// In the sequential summation order (sk_set_summation_order), `seq` holds
// each element's terms instead (term j of element i at seq[j * seq_ld + i],
// i < seq_n), and the last CTA sums them in element order, one warp per
// reduction, in the value type (seq_f32: float), as std::inner_product does.
struct RedWs {
  double* partials = nullptr;
  unsigned* counter = nullptr;
  int capacity = 0;  // CTAs
  double* seq = nullptr;
  i64 seq_ld = 0;
  i64 seq_n = 0;
  int seq_f32 = 0;
};

// Whether the solvers sum their dot products in the reference's sequential
// order (sk_set_summation_order); read once at the start of each solve.
bool summation_sequential();

// Solver scalars resident on the device for a whole solve.  Written only
// by the finalize step of a fused kernel (one thread of the last CTA) or by
// a single-thread kernel; read by every later kernel of the solve.
struct Scalars {
  double bnorm;     // ||b||
  double rz;        // CG: <r, z>
  double alpha;
  double beta;
  double omega;
  double rho;       // BiCGSTAB: rho of the last full step
  double rho_new;   // BiCGSTAB: <r_hat, r> for the next step
  double rnorm;     // last residual norm recorded
  double tol;
  double aux;       // FGMRES: 1 / beta or 1 / h_{j+1,j}
  double beta_cycle;  // FGMRES: ||r|| at the start of the current cycle
  long long iters;
  long long hist_len;
  long long max_iters;
  long long jfinal; // FGMRES: last Arnoldi step of the cycle
  int converged;
  int done;         // later kernels of the solve (or cycle) are no-ops
  int status;
  int half;         // BiCGSTAB: half-step convergence, x update pending
  int skip;         // BiCGSTAB: omega == 0, skip the full-step update
  int beta0;        // FGMRES: initial residual exactly zero
  int hist_on;
  int pad;
};
inline int ceil_div(i64 a, i64 b) { return static_cast<int>((a + b - 1) / b); }

// ------------------------------------------------------------------
// Handle construction, shared by the uploads of host arrays (sk_core.cu)
// and the conversions on the device (sk_convert.cu)
// ------------------------------------------------------------------
constexpr i64 kChunk = i64(1) << 23;  // staging elements per host copy step

inline size_t vbytes(sk_dtype dt) { return dt == SK_F64 ? 8 : 4; }

// Grid of a grid-stride kernel over n elements: at most 32 CTAs per SM.
int grid_for(i64 n);

// A new handle of format f on the current device, with its own stream.
sk_status new_handle(sk_matrix* out, sk_format f, sk_dtype dt, i64 nrow, i64 ncol);
void destroy_handle(sk_matrix A);

// Destroys a half-built handle when its constructor returns early.
struct HandleGuard {
  sk_matrix* slot;
  bool ok = false;
  ~HandleGuard() {
    if (!ok && slot && *slot) {
      destroy_handle(*slot);
      *slot = nullptr;
    }
  }
};

template <typename V>
sk_status upload_vector(sk_matrix A, const std::vector<V>& h, V** dev, cudaStream_t st) {
  void* p = nullptr;
  sk_status s = dev_alloc(A, &p, h.size() * sizeof(V) + 64);
  if (s != SK_OK) return s;
  *dev = static_cast<V*>(p);
  if (!h.empty()) SK_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, st));
  return SK_OK;
}

// The product's tables of a CSR handle whose row_ptr / col_ind / vals are
// already on the device, from the host copy of its row pointers.
sk_status csr_finish(sk_matrix A, const int64_t* row_ptr, cudaStream_t st);

// FP32 planes of the diagonal copy of an FP64 handle (no-op without one).
sk_status build_dia_f32(sk_matrix A);
// The column-panel copy of a CSR handle (host row pointers); a no-op when
// the handle does not qualify (sk_matrix_add_panels).
sk_status build_panel(sk_matrix A, const int64_t* rp, cudaStream_t st);
// The sorted diagonal offsets c - r of a CSR handle whose pattern fits the
// diagonal copy (at most kDiaMax diagonals, columns ascending in every row,
// planes at most half empty); empty when it does not.
sk_status dia_pattern(sk_matrix A, std::vector<int>* offsets);

// BSR block-row partition of the product kernel (host row pointers) and
// the sliced copy of 2x2 / 3x3 handles.
void bsr_partition(const int64_t* rp, i64 nbr, i64 br, i64 bsz, std::vector<int>& part);
sk_status build_bsr_sell(sk_matrix A, const int64_t* rp, cudaStream_t st);

}  // namespace sk
