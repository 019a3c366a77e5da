// sk_panel.cu -- the column-panel copy of a large skewed CSR handle.
//
// The product of a CSR matrix whose rows are too long for SELL-32 and
// whose columns are spread over an x far larger than the L1 (a Zipf-like
// random matrix) is bound by the gathers of x: every entry costs one
// lane's private L1/L2 request.  The panel copy turns those gathers into
// shared-memory reads.  Each CTA owns a block of rows; it walks the column
// panels in order with panel k of x staged in shared memory and a running
// sum per row, and adds each row's entries of panel k to the row's sum.
// Panels are visited in ascending column order and a row's entries within
// a panel in storage order, so every row is still summed entry after entry
// from 0 in ascending column order, as sparse_blas.hpp:25-28 sums it.
//
// The copy holds, per entry, the value and a 16-bit column offset within
// the panel, grouped by (row block, panel) into 32-lane slices of row
// segments sorted by decreasing length; slot j of a slice stores entry j
// of the segments longer than j, contiguously, so nothing is padded.  The
// slices of a (block, panel) are cut into chunks small enough for a
// shared-memory stage; each chunk (values, columns and its slice table) is
// contiguous and 16-byte aligned, so the product moves it with three bulk
// copies.  Built on the host from the row pointers and a host copy of the
// column indices; the values are scattered on the device.
#include <algorithm>
#include <climits>
#include <thread>
#include <vector>

#include "sk_internal.cuh"

namespace sk {

namespace {

__global__ void panel_scatter_kernel(i64 nnz, const int* __restrict__ ci, const int* __restrict__ dst, int width,
                                     unsigned short* __restrict__ pcol) {
  for (i64 e = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; e < nnz;
       e += static_cast<i64>(gridDim.x) * blockDim.x) {
    const int c = ci[e];
    pcol[dst[e]] = static_cast<unsigned short>(c % width);
  }
}

template <typename T>
__global__ void panel_values_kernel(i64 nnz, const T* __restrict__ v, const int* __restrict__ dst,
                                    T* __restrict__ pv) {
  for (i64 e = blockIdx.x * static_cast<i64>(blockDim.x) + threadIdx.x; e < nnz;
       e += static_cast<i64>(gridDim.x) * blockDim.x)
    pv[dst[e]] = v[e];
}

struct Seg {
  int k;      // panel
  int row;    // local row
  int start;  // first entry (CSR index)
  int len;
};

// A slice, or the slots [ja, jb) of one (a slice with more entries than a
// stage is cut by slots into pieces that go to successive chunks, so that
// each lane still adds its entries in order).
struct Piece {
  int seg;  // first segment of the slice (sorted order)
  int cnt;  // segments in the slice
  int ja, jb;
  int entries;
};

struct ChunkPlan {
  int k;
  std::vector<Piece> pieces;
  int entries;
};

struct BlockPlan {
  std::vector<Seg> segs;  // sorted by (panel, decreasing length, row)
  std::vector<ChunkPlan> chunks;
  i64 entries = 0;     // chunk entries rounded up to 8, summed
  i64 meta_words = 0;  // chunk slice tables, summed
  bool ok = true;      // columns ascending in every row
};

inline i64 round_up(i64 v, i64 m) { return (v + m - 1) / m * m; }
// Slice table of a chunk: the slices' entry offsets, padded to 4 words,
// then 32 segment words per slice.
inline i64 meta_words_of(i64 ns) { return round_up(ns, 4) + 32 * ns; }

}  // namespace

// Bytes of one chunk stage in shared memory: values, columns, slice table.
int panel_stage_bytes(sk_dtype dt) {
  const i64 V = static_cast<i64>(vbytes(dt));
  return static_cast<int>(round_up(kPanelChunkEntries * V + kPanelChunkEntries * 2 +
                                       meta_words_of(kPanelChunkSlices) * 4, 16));
}

sk_status build_panel(sk_matrix A, const int64_t* rp, cudaStream_t st_) {
  auto& C = A->csr;
  const i64 n = A->nrow, nnz = A->nnz, ncol = A->ncol;
  const i64 V = static_cast<i64>(vbytes(A->dtype));
  if (n == 0 || nnz == 0 || nnz > INT_MAX - (i64(1) << 24)) return SK_OK;
  const i64 stage = panel_stage_bytes(A->dtype);
  // Row blocks: about equal entries, one per SM, and at most kMaxRows rows
  // (the running sums live in shared memory, a local row in 16 bits).
  // When the row limit cuts more blocks than SMs, the entries are spread
  // over whole waves of blocks instead.
  const i64 kMaxRows = std::min<i64>(65535, (kPanelSmem / 3) / V);
  std::vector<int> row0;
  for (i64 waves = 1;; ++waves) {
    const i64 slots = waves * A->sm_count;
    const i64 target = (nnz + slots - 1) / slots;
    row0.assign(1, 0);
    i64 r = 0;
    while (r < n) {
      const i64 r_begin = r;
      i64 acc = 0;
      while (r < n && r - r_begin < kMaxRows && (acc < target || r == r_begin)) {
        acc += rp[r + 1] - rp[r];
        ++r;
      }
      row0.push_back(static_cast<int>(r));
    }
    if (static_cast<i64>(row0.size()) - 1 <= slots) break;
    if (waves == 4) return SK_OK;  // too many short rows for the running sums
  }
  const int nb = static_cast<int>(row0.size()) - 1;
  i64 rows_max = 0;
  for (int b = 0; b < nb; ++b) rows_max = std::max<i64>(rows_max, row0[b + 1] - row0[b]);
  const i64 run_bytes = round_up(rows_max * V, 16);
  i64 width = (kPanelSmem - run_bytes - kPanelStages * stage - 64) / (2 * V);
  width = std::min<i64>(width, 65532) / 4 * 4;
  if (width < 1024) return SK_OK;
  const i64 np = (ncol + width - 1) / width;
  if (np > 65535 || static_cast<i64>(nb) * np > INT_MAX / 4) return SK_OK;
  // Host copy of the column indices.
  std::vector<int> col(static_cast<size_t>(nnz));
  SK_CUDA(cudaMemcpyAsync(col.data(), C.col_ind, nnz * sizeof(int), cudaMemcpyDeviceToHost, st_));
  SK_CUDA(cudaStreamSynchronize(st_));
  // Pass 1 (blocks in parallel): each block's segments, sorted, and its
  // chunks.
  std::vector<BlockPlan> plan(static_cast<size_t>(nb));
  const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  auto pass1 = [&](int b) {
    BlockPlan& P = plan[static_cast<size_t>(b)];
    for (i64 r = row0[b]; r < row0[b + 1] && P.ok; ++r) {
      const int local = static_cast<int>(r - row0[b]);
      i64 e = rp[r];
      const i64 end = rp[r + 1];
      for (i64 q = e + 1; q < end; ++q)
        if (col[static_cast<size_t>(q)] <= col[static_cast<size_t>(q - 1)]) P.ok = false;
      while (e < end) {
        const int k = static_cast<int>(col[static_cast<size_t>(e)] / width);
        i64 f = e + 1;
        while (f < end && col[static_cast<size_t>(f)] / width == k) ++f;
        P.segs.push_back({k, local, static_cast<int>(e), static_cast<int>(f - e)});
        e = f;
      }
    }
    if (!P.ok) return;
    std::stable_sort(P.segs.begin(), P.segs.end(), [](Seg const& a, Seg const& c) {
      return a.k != c.k ? a.k < c.k : a.len > c.len;
    });
    size_t i = 0;
    for (int k = 0; k < np; ++k) {
      size_t j = i;
      while (j < P.segs.size() && P.segs[j].k == k) ++j;
      ChunkPlan ch{k, {}, 0};
      auto add_piece = [&](Piece const& pc) {
        if (!ch.pieces.empty() && (ch.entries + pc.entries > kPanelChunkEntries ||
                                   static_cast<int>(ch.pieces.size()) == kPanelChunkSlices || pc.ja > 0)) {
          P.chunks.push_back(std::move(ch));
          ch = ChunkPlan{k, {}, 0};
        }
        ch.pieces.push_back(pc);
        ch.entries += pc.entries;
      };
      // slices of 32 segments from i (lengths non-increasing); a slice with
      // more entries than a stage is cut by slots into pieces that start
      // new chunks
      for (size_t s = i; s < j; s += 32) {
        const int cnt = static_cast<int>(std::min<size_t>(32, j - s));
        const Seg* sg = P.segs.data() + s;
        const int maxlen = sg[0].len;
        auto entries_of = [&](int ja, int jb) {
          int e = 0;
          for (int l = 0; l < cnt; ++l) e += std::max(0, std::min(sg[l].len, jb) - ja);
          return e;
        };
        for (int ja = 0; ja < maxlen;) {
          int jb = maxlen;
          if (entries_of(ja, jb) > kPanelChunkEntries) {  // the most slots that fit a stage
            jb = ja + 1;
            while (jb < maxlen && entries_of(ja, jb + 1) <= kPanelChunkEntries) ++jb;
          }
          add_piece(Piece{static_cast<int>(s), cnt, ja, jb, entries_of(ja, jb)});
          ja = jb;
        }
      }
      P.chunks.push_back(std::move(ch));  // every panel has a chunk, possibly empty
      i = j;
    }
    for (auto const& ch : P.chunks) {
      P.entries += round_up(ch.entries, 8);
      P.meta_words += meta_words_of(static_cast<i64>(ch.pieces.size()));
    }
  };
  auto run_parallel = [&](auto const& fn) {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < hw; ++t)
      pool.emplace_back([&, t] {
        for (int b = static_cast<int>(t); b < nb; b += static_cast<int>(hw)) fn(b);
      });
    for (auto& th : pool) th.join();
  };
  run_parallel(pass1);
  for (int b = 0; b < nb; ++b)
    if (!plan[static_cast<size_t>(b)].ok) return SK_OK;
  // Prefix sums over the blocks.
  std::vector<i64> chunk_base(static_cast<size_t>(nb) + 1, 0), entry_base(static_cast<size_t>(nb) + 1, 0),
      meta_base(static_cast<size_t>(nb) + 1, 0);
  for (int b = 0; b < nb; ++b) {
    const BlockPlan& P = plan[static_cast<size_t>(b)];
    chunk_base[static_cast<size_t>(b) + 1] = chunk_base[static_cast<size_t>(b)] + static_cast<i64>(P.chunks.size());
    entry_base[static_cast<size_t>(b) + 1] = entry_base[static_cast<size_t>(b)] + P.entries;
    meta_base[static_cast<size_t>(b) + 1] = meta_base[static_cast<size_t>(b)] + P.meta_words;
  }
  const i64 nchunks = chunk_base[static_cast<size_t>(nb)], total = entry_base[static_cast<size_t>(nb)],
            mwords = meta_base[static_cast<size_t>(nb)];
  if (total > INT_MAX - 64 || mwords > INT_MAX - 64 || nchunks > INT_MAX - 1) return SK_OK;
  // Pass 2: chunk tables, slice tables and the destination of every entry.
  std::vector<int> chunk_ptr(static_cast<size_t>(nb) + 1);
  std::vector<int4> chunk(static_cast<size_t>(nchunks));
  std::vector<int> chunk_kn(static_cast<size_t>(nchunks));
  std::vector<unsigned> meta(static_cast<size_t>(mwords), 0u);
  std::vector<int> dst(static_cast<size_t>(nnz));
  auto pass2 = [&](int b) {
    const BlockPlan& P = plan[static_cast<size_t>(b)];
    i64 c = chunk_base[static_cast<size_t>(b)];
    i64 e0 = entry_base[static_cast<size_t>(b)];
    i64 m0 = meta_base[static_cast<size_t>(b)];
    chunk_ptr[static_cast<size_t>(b)] = static_cast<int>(c);
    for (auto const& ch : P.chunks) {
      const int ns = static_cast<int>(ch.pieces.size());
      const i64 mw = meta_words_of(ns);
      chunk[static_cast<size_t>(c)] = make_int4(static_cast<int>(e0), static_cast<int>(round_up(ch.entries, 8)),
                                                static_cast<int>(m0), static_cast<int>(mw));
      chunk_kn[static_cast<size_t>(c)] = ch.k | (ns << 16);
      unsigned* rel = meta.data() + m0;
      unsigned* segw = rel + round_up(ns, 4);
      int off = 0;  // entry offset in the chunk
      for (int t = 0; t < ns; ++t) {
        const Piece& pc = ch.pieces[static_cast<size_t>(t)];
        rel[t] = static_cast<unsigned>(off);
        const Seg* sg = P.segs.data() + pc.seg;
        for (int l = 0; l < pc.cnt; ++l) {
          const int len = std::max(0, std::min(sg[l].len, pc.jb) - pc.ja);
          segw[32 * t + l] = len ? static_cast<unsigned>(sg[l].row) | (static_cast<unsigned>(len) << 16) : 0u;
        }
        // slot j holds entry j of lanes 0 .. c_j - 1 (the segments longer
        // than j), stored after slot j - 1
        int live = pc.cnt;
        for (int j = pc.ja; j < pc.jb && live > 0; ++j) {
          while (live > 0 && sg[live - 1].len <= j) --live;
          for (int l = 0; l < live; ++l)
            dst[static_cast<size_t>(sg[l].start) + static_cast<size_t>(j)] = static_cast<int>(e0 + off + l);
          off += live;
        }
      }
      e0 += round_up(ch.entries, 8);
      m0 += mw;
      ++c;
    }
  };
  run_parallel(pass2);
  chunk_ptr[static_cast<size_t>(nb)] = static_cast<int>(nchunks);
  // Upload and scatter.
  sk_status st;
  void *pcol = nullptr, *pval = nullptr, *perr = nullptr, *ddst = nullptr;
  if ((st = dev_alloc(A, &pcol, (total + 64) * 2)) != SK_OK) return st;
  if ((st = dev_alloc(A, &pval, (total + 64) * V)) != SK_OK) return st;
  if ((st = dev_alloc(A, &perr, 16)) != SK_OK) return st;
  SK_CUDA(cudaMemsetAsync(pcol, 0, (total + 64) * 2, st_));
  SK_CUDA(cudaMemsetAsync(pval, 0, (total + 64) * V, st_));
  SK_CUDA(cudaMemsetAsync(perr, 0, 16, st_));
  if ((st = upload_vector(A, row0, &C.pn_row0, st_)) != SK_OK) return st;
  if ((st = upload_vector(A, chunk_ptr, &C.pn_chunk_ptr, st_)) != SK_OK) return st;
  if ((st = upload_vector(A, chunk, &C.pn_chunk, st_)) != SK_OK) return st;
  if ((st = upload_vector(A, chunk_kn, &C.pn_chunk_kn, st_)) != SK_OK) return st;
  if ((st = upload_vector(A, meta, &C.pn_meta, st_)) != SK_OK) return st;
  SK_CUDA(cudaMalloc(&ddst, nnz * sizeof(int)));
  cudaError_t e = cudaMemcpyAsync(ddst, dst.data(), nnz * sizeof(int), cudaMemcpyHostToDevice, st_);
  if (e == cudaSuccess) {
    SK_LAUNCH(panel_scatter_kernel, grid_for(nnz), kThreads, 0, st_, nnz, C.col_ind, static_cast<const int*>(ddst),
              static_cast<int>(width), static_cast<unsigned short*>(pcol));
    if (A->dtype == SK_F64)
      SK_LAUNCH(panel_values_kernel<double>, grid_for(nnz), kThreads, 0, st_, nnz,
                static_cast<const double*>(C.vals), static_cast<const int*>(ddst), static_cast<double*>(pval));
    else
      SK_LAUNCH(panel_values_kernel<float>, grid_for(nnz), kThreads, 0, st_, nnz,
                static_cast<const float*>(C.vals), static_cast<const int*>(ddst), static_cast<float*>(pval));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  cudaFree(ddst);
  if (e != cudaSuccess) return cuda_fail(e, "panel copy");
  C.pn_col = static_cast<unsigned short*>(pcol);
  C.pn_vals = pval;
  C.pn_err = static_cast<int*>(perr);
  C.pn_entries = total;
  C.pn_blocks = nb;
  C.pn_panels = static_cast<int>(np);
  C.pn_width = static_cast<int>(width);
  C.pn_stage_bytes = static_cast<int>(stage);
  C.pn_smem = static_cast<int>(run_bytes + 2 * width * V + kPanelStages * stage);
  C.panel = true;
  return SK_OK;
}

}  // namespace sk

using namespace sk;

extern "C" sk_status sk_matrix_add_panels(sk_matrix A, int* built) {
  SK_CHECK(A && built, SK_INVALID_ARG, "null argument");
  *built = 0;
  SK_CHECK(A->format == SK_CSR, SK_NOT_SUPPORTED, "the column-panel copy is for CSR handles");
  if (A->csr.panel) {
    *built = 1;
    return SK_OK;
  }
  if (A->csr.sell || A->csr.dia_n || A->nrow == 0) return SK_OK;  // already summed in the reference's order
  std::vector<int> rp32(static_cast<size_t>(A->nrow) + 1);
  SK_CUDA(cudaMemcpyAsync(rp32.data(), A->csr.row_ptr, rp32.size() * sizeof(int), cudaMemcpyDeviceToHost,
                          A->stream));
  SK_CUDA(cudaStreamSynchronize(A->stream));
  std::vector<int64_t> rp(rp32.begin(), rp32.end());
  sk_status st = build_panel(A, rp.data(), A->stream);
  if (st != SK_OK) return st;
  *built = A->csr.panel ? 1 : 0;
  return SK_OK;
}
