"""Seeded matrix generators: the reference's own test matrices (restated
from sparkit/data/matgen.hpp so that parity tests use the same inputs
without the reference present) and the synthetic workloads of the
benchmark (Dirichlet Laplacians, the 3x3-block vector Laplacian, the
Zipf-row random matrix).

All builders return a formats.Compressed_row_matrix with sorted, unique
columns per row and int64 indices.
"""
import numpy as np

from .formats import Compressed_row_matrix


def _stencil_csr(n_rows, cand_cols, cand_vals, valid, dtype):
    """CSR from per-row candidate columns (already in increasing order)."""
    counts = valid.sum(axis=1).astype(np.int64)
    rp = np.zeros(n_rows + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    cols = cand_cols[valid]
    vals = cand_vals[valid].astype(dtype)
    return Compressed_row_matrix((n_rows, n_rows), rp, cols, vals)


# ------------------------------------------------------------------
# Matrices of the reference's tests (matgen.hpp)
# ------------------------------------------------------------------

def tridiagonal_matrix(n, sub, diag, sup, dtype=np.float64):
    """matgen.hpp:104-117."""
    i = np.arange(n, dtype=np.int64)
    cand = np.stack([i - 1, i, i + 1], axis=1)
    vals = np.broadcast_to(np.array([sub, diag, sup], dtype=np.float64), cand.shape)
    valid = (cand >= 0) & (cand < n)
    return _stencil_csr(n, cand, vals, valid, dtype)


def poisson_2d(nx, ny=None, shift=0.0, dtype=np.float64):
    """Graph Laplacian of an nx x ny grid, diagonal = neighbour count + shift
    (matgen.hpp:175-264).  poisson_2d(grid, shift) in the reference is
    poisson_2d(grid, grid, shift)."""
    if ny is None:
        ny = nx
    n = nx * ny
    node = np.arange(n, dtype=np.int64)
    r, c = node // nx, node % nx
    # the reference pushes W, E, S, N then the diagonal; CSR sorts them to
    # S, W, diag, E, N
    cand = np.stack([node - nx, node - 1, node, node + 1, node + nx], axis=1)
    valid = np.stack([r > 0, c > 0, np.ones(n, bool), c + 1 < nx, r + 1 < ny], axis=1)
    degree = valid.sum(axis=1) - 1
    vals = np.stack([-np.ones(n), -np.ones(n), degree.astype(np.float64) + shift,
                     -np.ones(n), -np.ones(n)], axis=1)
    return _stencil_csr(n, cand, vals, valid, dtype)


def convdiff_centered_2d(nx, ny, diffusion, cx, cy, shift=0.0, dtype=np.float64):
    """Centred convection-diffusion, matgen.hpp:341-391."""
    n = nx * ny
    node = np.arange(n, dtype=np.int64)
    r, c = node // nx, node % nx
    cand = np.stack([node - nx, node - 1, node, node + 1, node + nx], axis=1)
    valid = np.stack([r > 0, c > 0, np.ones(n, bool), c + 1 < nx, r + 1 < ny], axis=1)
    degree = (valid.sum(axis=1) - 1).astype(np.float64)
    vals = np.stack([np.full(n, -(diffusion + cy)), np.full(n, -(diffusion + cx)),
                     degree * diffusion + shift,
                     np.full(n, -(diffusion - cx)), np.full(n, -(diffusion - cy))], axis=1)
    return _stencil_csr(n, cand, vals, valid, dtype)


def convection_diffusion_2d(nx, ny, diffusion, cx, cy, dtype=np.float64):
    """First-order upwind convection-diffusion, matgen.hpp:276-330."""
    n = nx * ny
    node = np.arange(n, dtype=np.int64)
    r, c = node // nx, node % nx
    cand = np.stack([node - nx, node - 1, node, node + 1, node + nx], axis=1)
    valid = np.stack([r > 0, c > 0, np.ones(n, bool), c + 1 < nx, r + 1 < ny], axis=1)
    off = np.stack([np.full(n, -diffusion - cy), np.full(n, -diffusion - cx), np.zeros(n),
                    np.full(n, -diffusion), np.full(n, -diffusion)], axis=1)
    # the reference accumulates the diagonal as diag -= val in the order
    # W, E, S, N
    diag = np.zeros(n)
    for col in (1, 3, 0, 4):
        diag = np.where(valid[:, col], diag - off[:, col], diag)
    vals = off.copy()
    vals[:, 2] = diag
    return _stencil_csr(n, cand, vals, valid, dtype)


def nonsymmetric_sample(dtype=np.float64):
    """The hard-coded 4x4 of matgen.hpp:147-166."""
    rows = [0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3]
    cols = [0, 1, 2, 0, 1, 3, 0, 2, 3, 1, 2, 3]
    vals = [4, -1, 0.5, -0.5, 4, -1, 0.3, 4, -0.8, -0.6, 0.2, 4]
    return Compressed_row_matrix.from_entries((4, 4), rows, cols, vals, dtype=dtype)


# ------------------------------------------------------------------
# Benchmark workloads
# ------------------------------------------------------------------

def laplacian_2d_dirichlet(nx, ny=None, dtype=np.float64):
    """5-point Dirichlet Laplacian: 4 on the diagonal everywhere, -1 to
    in-grid neighbours (n = nx * ny)."""
    if ny is None:
        ny = nx
    n = nx * ny
    node = np.arange(n, dtype=np.int64)
    r, c = node // nx, node % nx
    cand = np.stack([node - nx, node - 1, node, node + 1, node + nx], axis=1)
    valid = np.stack([r > 0, c > 0, np.ones(n, bool), c + 1 < nx, r + 1 < ny], axis=1)
    vals = np.tile(np.array([-1.0, -1.0, 4.0, -1.0, -1.0]), (n, 1))
    return _stencil_csr(n, cand, vals, valid, dtype)


def laplacian_3d_dirichlet(nx, ny=None, nz=None, dtype=np.float64, diag=6.0):
    """7-point Dirichlet Laplacian on nx x ny x nz (diagonal 6)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    n = nx * ny * nz
    node = np.arange(n, dtype=np.int64)
    i = node % nx
    j = (node // nx) % ny
    k = node // (nx * ny)
    pl = nx * ny
    cand = np.stack([node - pl, node - nx, node - 1, node, node + 1, node + nx, node + pl], axis=1)
    valid = np.stack([k > 0, j > 0, i > 0, np.ones(n, bool), i + 1 < nx, j + 1 < ny, k + 1 < nz], axis=1)
    vals = np.tile(np.array([-1.0, -1.0, -1.0, diag, -1.0, -1.0, -1.0]), (n, 1))
    return _stencil_csr(n, cand, vals, valid, dtype)


def vector_laplacian_3d_bsr_csr(nx, seed=0, coupling=0.1, dtype=np.float64):
    """Scalar CSR of the 3-component vector Laplacian: every block is
    L_ij * I_3, and each diagonal block gets a dense 3x3 coupling with
    off-diagonal entries U[-coupling, coupling] (seeded).  Converted with
    to_block_sparse_row(., 3, 3) this is the BSR workload."""
    L = laplacian_3d_dirichlet(nx, dtype=np.float64)
    n = L.shape()[0]
    rng = np.random.default_rng(seed)
    coup = rng.uniform(-coupling, coupling, size=(n, 3, 3))
    lens = L.row_lengths()
    brow = np.repeat(np.arange(n, dtype=np.int64), lens)
    bcol = L.col_ind()
    bval = L.values()
    is_diag = brow == bcol
    # per block row: entries (3 scalar rows) x (blocks) x (3 columns)
    nb = bcol.size
    blk = np.zeros((nb, 3, 3))
    blk[:, [0, 1, 2], [0, 1, 2]] = bval[:, None]
    d_idx = np.nonzero(is_diag)[0]
    cpl = coup[brow[d_idx]]
    for a in range(3):
        for b in range(3):
            if a != b:
                blk[d_idx, a, b] = cpl[:, a, b]
    # scalar CSR: row 3I+a holds, block by block, columns 3J+b
    rows = (3 * brow[:, None, None] + np.arange(3)[None, :, None]).repeat(3, axis=2)
    cols = (3 * bcol[:, None, None] + np.arange(3)[None, None, :]).repeat(3, axis=1)
    rows, cols, vals = rows.ravel(), cols.ravel(), blk.ravel()
    keep = vals != 0.0
    return Compressed_row_matrix.from_entries((3 * n, 3 * n), rows[keep], cols[keep], vals[keep], dtype=dtype)


def zipf_random(n, s=1.5, cap=2048, seed=0, dtype=np.float64):
    """n x n random matrix: row lengths min(Zipf(s), cap), columns uniform
    in [0, n) (duplicates within a row dropped), values N(0, 1)."""
    rng = np.random.default_rng(seed)
    lens = np.minimum(rng.zipf(s, size=n), cap).astype(np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = rng.integers(0, n, size=rows.size, dtype=np.int64)
    vals = rng.standard_normal(rows.size)
    return Compressed_row_matrix.from_entries((n, n), rows, cols, vals, dtype=dtype)


def uniform_vector(n, seed=0, dtype=np.float64):
    """x ~ U[-1, 1], seeded."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=n).astype(dtype)


def vector_laplacian_3d_bsr(nx, seed=0, coupling=0.1, dtype=np.float64):
    """The same 3-component vector Laplacian as vector_laplacian_3d_bsr_csr,
    built directly as a 3x3 Block_sparse_row_matrix (no scalar CSR pass):
    block (I, J) = L_IJ * I_3, plus a dense U[-coupling, coupling] coupling
    (seeded, per block row) off the diagonal of every diagonal block."""
    from .formats import Block_sparse_row_matrix
    L = laplacian_3d_dirichlet(nx, dtype=np.float64)
    n = L.shape()[0]
    rng = np.random.default_rng(seed)
    coup = rng.uniform(-coupling, coupling, size=(n, 3, 3))
    lens = L.row_lengths()
    brow = np.repeat(np.arange(n, dtype=np.int64), lens)
    bcol = L.col_ind()
    blk = np.zeros((bcol.size, 3, 3), dtype=np.float64)
    blk[:, [0, 1, 2], [0, 1, 2]] = L.values()[:, None]
    d_idx = np.nonzero(brow == bcol)[0]
    off = ~np.eye(3, dtype=bool)
    blk[d_idx] = np.where(off[None], coup[brow[d_idx]], blk[d_idx])
    return Block_sparse_row_matrix((3 * n, 3 * n), 3, 3, L.row_ptr(), bcol, blk.reshape(-1).astype(dtype))


def gaussian_random_field(shape, sigma, corr_len, seed=0):
    """Stationary Gaussian random field on a periodic grid: white noise
    filtered in Fourier space by exp(-|k|^2 corr_len^2 / 2) (a Gaussian
    covariance of length corr_len cells), shifted to mean 0 and scaled to
    standard deviation sigma."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    ks = np.meshgrid(*[2 * np.pi * np.fft.fftfreq(s) for s in shape], indexing="ij")
    k2 = sum(k * k for k in ks)
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-0.5 * k2 * corr_len * corr_len)))
    g -= g.mean()
    g *= sigma / g.std()
    return g


def diffusion_3d_grf(n, sigma=2.0, corr_len=8.0, seed=0, dtype=np.float64):
    """7-point finite-volume diffusion on an n^3 grid with cell coefficients
    k = exp(g), g a Gaussian random field (sigma, corr_len cells).  Interior
    faces take the harmonic mean of their two cells, boundary faces the cell
    value (homogeneous Dirichlet): A_ii = sum of the cell's six face
    coefficients, A_ij = -k_face.  SPD."""
    g = gaussian_random_field((n, n, n), sigma, corr_len, seed)
    kc = np.exp(g).reshape(-1)  # index = i + n*(j + n*k)
    N = n ** 3
    node = np.arange(N, dtype=np.int64)
    i = node % n
    j = (node // n) % n
    kk = node // (n * n)
    pl = n * n
    offs = (-pl, -n, -1, 1, n, pl)
    inside = (kk > 0, j > 0, i > 0, i + 1 < n, j + 1 < n, kk + 1 < n)
    face = []
    for off, ok in zip(offs, inside):
        nb = np.where(ok, node + off, node)
        kf = np.where(ok, 2.0 * kc * kc[nb] / (kc + kc[nb]), kc)
        face.append(kf)
    diag = sum(face)
    cand = np.stack([node - pl, node - n, node - 1, node, node + 1, node + n, node + pl], axis=1)
    valid = np.stack([inside[0], inside[1], inside[2], np.ones(N, bool), inside[3], inside[4], inside[5]], axis=1)
    vals = np.stack([-face[0], -face[1], -face[2], diag, -face[3], -face[4], -face[5]], axis=1)
    return _stencil_csr(N, cand, vals, valid, dtype)


def convdiff_2d_grf(n, sigma=1.0, corr_len=None, peclet=None, pe_range=(1.0, 100.0), seed=0,
                    dtype=np.float64):
    """2-D convection-diffusion on an n x n grid (row y * n + x),
    finite-volume with first-order upwind convection and homogeneous
    Dirichlet boundaries (the variable-coefficient generalisation of
    matgen.hpp:276-330, whose constant-coefficient form has no boundary
    terms).

    * Diffusion k = exp(g) per cell, g a Gaussian random field (sigma,
      correlation length corr_len cells, default n / 32); interior faces take
      the harmonic mean of their two cells, boundary faces the cell value.
    * Velocity from a seeded stream function psi on the cell corners (a
      Gaussian random field of correlation length n / 8 times
      sin(pi i / n) sin(pi j / n), so that it vanishes on the boundary):
      u = d psi / dy on vertical faces, v = -d psi / dx on horizontal faces,
      which is exactly divergence-free discretely and has no flow through
      the boundary.
    * Scale: the median cell Peclet number |u_f| / k_f over the interior
      faces is `peclet`, drawn log-uniformly from pe_range when None.

    Row P: A_PP = sum_f k_f + sum_f max(F_f, 0), A_PQ = -k_f + min(F_f, 0)
    with F_f the outward flux through face f.  Returns (A, info) with the
    Peclet target and the coefficient fields."""
    rng = np.random.default_rng(seed)
    if corr_len is None:
        corr_len = max(n / 32.0, 1.0)
    g = gaussian_random_field((n, n), sigma, corr_len, seed=int(rng.integers(1 << 31)))
    kc = np.exp(g)  # [y, x]
    psi = gaussian_random_field((n + 1, n + 1), 1.0, max(n / 8.0, 1.0), seed=int(rng.integers(1 << 31)))
    w = np.sin(np.pi * np.arange(n + 1) / n)
    psi = psi * w[:, None] * w[None, :]  # psi[b, a] at corner (x = a, y = b)
    # vertical face between cells (x-1, y) and (x, y): x = 1..n-1 -> u[y, x]
    u = psi[1:, :] - psi[:-1, :]       # [n, n+1]: face at corner column a, cell row y
    v = -(psi[:, 1:] - psi[:, :-1])    # [n+1, n]: face at corner row b, cell column x
    kx = 2.0 * kc[:, :-1] * kc[:, 1:] / (kc[:, :-1] + kc[:, 1:])  # interior vertical faces [n, n-1]
    ky = 2.0 * kc[:-1, :] * kc[1:, :] / (kc[:-1, :] + kc[1:, :])  # interior horizontal faces [n-1, n]
    pe_faces = np.concatenate([np.abs(u[:, 1:-1]).ravel() / kx.ravel(), np.abs(v[1:-1, :]).ravel() / ky.ravel()])
    med = np.median(pe_faces)
    if peclet is None:
        peclet = float(np.exp(rng.uniform(np.log(pe_range[0]), np.log(pe_range[1]))))
    scale = peclet / med if med > 0 else 0.0
    u *= scale
    v *= scale
    N = n * n
    diag = np.zeros((n, n))
    offW = np.zeros((n, n))
    offE = np.zeros((n, n))
    offS = np.zeros((n, n))
    offN = np.zeros((n, n))
    # east faces of cells x = 0..n-2 (interior), flux out = u[:, x+1]
    Fe = u[:, 1:-1]
    diag[:, :-1] += kx + np.maximum(Fe, 0.0)
    offE[:, :-1] = -kx + np.minimum(Fe, 0.0)
    # west faces of cells x = 1..n-1, outward flux = -u[:, x]
    Fw = -u[:, 1:-1]
    diag[:, 1:] += kx + np.maximum(Fw, 0.0)
    offW[:, 1:] = -kx + np.minimum(Fw, 0.0)
    Fn = v[1:-1, :]
    diag[:-1, :] += ky + np.maximum(Fn, 0.0)
    offN[:-1, :] = -ky + np.minimum(Fn, 0.0)
    Fs = -v[1:-1, :]
    diag[1:, :] += ky + np.maximum(Fs, 0.0)
    offS[1:, :] = -ky + np.minimum(Fs, 0.0)
    # Dirichlet boundary faces: the cell coefficient
    diag[:, 0] += kc[:, 0]
    diag[:, -1] += kc[:, -1]
    diag[0, :] += kc[0, :]
    diag[-1, :] += kc[-1, :]
    node = np.arange(N, dtype=np.int64)
    r, c = node // n, node % n
    cand = np.stack([node - n, node - 1, node, node + 1, node + n], axis=1)
    valid = np.stack([r > 0, c > 0, np.ones(N, bool), c + 1 < n, r + 1 < n], axis=1)
    vals = np.stack([offS.ravel(), offW.ravel(), diag.ravel(), offE.ravel(), offN.ravel()], axis=1)
    A = _stencil_csr(N, cand, vals, valid, dtype)
    return A, {"peclet": peclet, "k": kc, "u": u, "v": v}


def batched_spd_systems(count=4096, nmin=1000, nmax=65536, shift=(0.0, 0.5), seed=0):
    """`count` independent SPD systems: each a 2-D 5-point or 3-D 7-point
    Dirichlet Laplacian (seeded coin) plus a diagonal shift U[shift], with
    n log-uniform in [nmin, nmax] rounded to a square or cubic grid.
    Returns (sys_offsets, row_ptr, col_ind, values, kinds) of the
    block-diagonal CSR matrix holding them (global row / column numbering,
    float32 values)."""
    rng = np.random.default_rng(seed)
    offs = [0]
    rps, cols, vals, kinds = [], [], [], []
    nnz_base = 0
    for _ in range(count):
        n_target = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        three_d = bool(rng.integers(0, 2))
        sft = rng.uniform(shift[0], shift[1])
        if three_d:
            g = max(2, int(round(n_target ** (1.0 / 3.0))))
            L = laplacian_3d_dirichlet(g, diag=6.0 + sft)
        else:
            g = max(2, int(round(n_target ** 0.5)))
            L = laplacian_2d_dirichlet(g)
            v = L.values().copy()
            rows = np.repeat(np.arange(L.shape()[0]), L.row_lengths())
            v[L.col_ind() == rows] += sft
            L = Compressed_row_matrix(L.shape(), L.row_ptr(), L.col_ind(), v)
        n = L.shape()[0]
        rps.append(L.row_ptr()[:-1] + nnz_base)
        cols.append(L.col_ind() + offs[-1])
        vals.append(L.values().astype(np.float32))
        nnz_base += L.size()
        offs.append(offs[-1] + n)
        kinds.append(3 if three_d else 2)
    row_ptr = np.concatenate(rps + [np.array([nnz_base], dtype=np.int64)])
    return (np.array(offs, dtype=np.int64), row_ptr, np.concatenate(cols), np.concatenate(vals),
            np.array(kinds, dtype=np.int8))
