"""The batched solver (one persistent launch, FP32 Jacobi-CG inside FP64
refinement per system) against the oracle's per-system FP64 Jacobi-CG: every
system reaches the FP64 tolerance on its true residual, with a comparable
number of CG iterations."""
import numpy as np
import pytest

from sparkit_b200 import _lib, gpu, matgen
from sparkit_b200.formats import Compressed_row_matrix

pytestmark = pytest.mark.gpu


def small_batch(count=48, seed=1):
    return matgen.batched_spd_systems(count, nmin=100, nmax=3000, seed=seed)


def system(offs, rp, ci, v, s):
    a, e = offs[s], offs[s + 1]
    rows = rp[a:e + 1] - rp[a]
    return Compressed_row_matrix((e - a, e - a), rows, ci[rp[a]:rp[e]] - a, v[rp[a]:rp[e]].astype(np.float64))


def test_batched_solves_every_system(gpu_lib, oracle):
    import torch
    offs, rp, ci, v, kinds = small_batch()
    B = gpu.Batch(offs, rp, ci, v)
    n = int(offs[-1])
    b = matgen.uniform_vector(n, seed=2)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    inner, outer, rel, conv = B.solve(bd, xd, gpu.Batch_config())
    x = xd.cpu().numpy()
    assert conv.all() and (rel < 1e-10).all()
    for s in range(len(offs) - 1):
        A = system(offs, rp, ci, v, s)
        a, e = offs[s], offs[s + 1]
        r = b[a:e] - oracle.spmv(A, x[a:e])
        assert np.linalg.norm(r) / np.linalg.norm(b[a:e]) < 1e-10, s
        if s % 8 == 0:
            _, sr = oracle.cg(A, b[a:e], np.zeros(e - a), 1e-10, 10 ** 6, 100000, left="jacobi")
            assert inner[s] <= 1.6 * sr["computed_iterations"] + 20, (s, inner[s], sr["computed_iterations"])


def test_autotune_and_graph_replay(gpu_lib):
    import torch
    offs, rp, ci, v, _ = small_batch(32, seed=3)
    B = gpu.Batch(offs, rp, ci, v)
    bd = torch.from_numpy(matgen.uniform_vector(int(offs[-1]), seed=4)).cuda()
    xd = torch.zeros_like(bd)
    g, t, ms = B.autotune(bd, xd, sample=16)
    assert g in (1, 2, 4, 8) and t in (256, 512, 1024) and (ms > 0).all()
    cfg = gpu.Batch_config(lanes_per_row=g, threads_per_cta=t)
    B.solve(bd, xd, cfg)
    x1 = xd.clone()
    xd.zero_()
    B.solve(bd, xd, cfg)  # replays the captured graph
    torch.cuda.synchronize()
    assert torch.equal(xd, x1)
    for lanes in (1, 4, 8):
        xd.zero_()
        _, _, rel, conv = B.solve(bd, xd, gpu.Batch_config(lanes_per_row=lanes, threads_per_cta=256))
        assert conv.all() and (rel < 1e-10).all()


def test_batch_rejects_coupled_systems(gpu_lib):
    offs = np.array([0, 2, 4], np.int64)
    rp = np.array([0, 1, 3, 4, 5], np.int64)
    ci = np.array([0, 1, 2, 2, 3], np.int64)  # row 1 reaches column 2 of the second system
    with pytest.raises(_lib.SkError):
        gpu.Batch(offs, rp, ci, np.ones(5, np.float32))
