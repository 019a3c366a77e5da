"""The learned FGMRES preconditioner on the GPU, through the C ABI:
coefficient planes, forward pass (tcgen05 and its mma.sync cross-check)
and parameter gradients against the CPU oracle, training, the fallback
driver, and what the trained network gains over Jacobi."""
import numpy as np
import pytest

from oracle.binding import grid_planes
from sparkit_b200 import gpu, matgen

pytestmark = pytest.mark.gpu

LAYERS = [(8, 16), (16, 32), (32, 64), (64, 64), (64, 64), (64, 32), (32, 16), (16, 16), (16, 1)]


def layer_slices():
    out, off = [], 0
    for ci, co in LAYERS:
        n = co * 9 * ci + co
        out.append(slice(off, off + n))
        off += n
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def rect_convdiff(nx, ny, seed):
    """Upwind convection-diffusion with constant coefficients on nx x ny,
    Dirichlet (diagonal 4 d + |cx| + |cy|)."""
    rng = np.random.default_rng(seed)
    d, cx, cy = 1.0, rng.uniform(-2, 2), rng.uniform(-2, 2)
    n = nx * ny
    node = np.arange(n)
    r, c = node // nx, node % nx
    cand = np.stack([node - nx, node - 1, node, node + 1, node + nx], axis=1)
    valid = np.stack([r > 0, c > 0, np.ones(n, bool), c + 1 < nx, r + 1 < ny], axis=1)
    vals = np.stack([np.full(n, -d - max(cy, 0)), np.full(n, -d - max(cx, 0)), np.full(n, 4 * d + abs(cx) + abs(cy)),
                     np.full(n, -d + min(cx, 0)), np.full(n, -d + min(cy, 0))], axis=1)
    return matgen._stencil_csr(n, cand, vals, valid, np.float64)


@pytest.mark.parametrize("nx,ny", [(64, 64), (48, 80), (256, 256), (320, 272), (392, 400), (512, 512)])
def test_planes_and_forward_match_oracle(gpu_lib, oracle, torch, nx, ny):
    """The network's apply against the oracle's forward pass.  At 392 x 400
    and 512^2 the full-resolution layers have more tiles than one wave of
    resident CTAs and take two tiles per CTA (at 392 the last CTA of each
    row has its second tile wholly outside the grid); every size runs the
    first layer with the vector channel computed in the kernel."""
    A = matgen.convdiff_2d_grf(nx, seed=11)[0] if nx == ny else rect_convdiff(nx, ny, 3)
    Ad = gpu.Device_matrix(A)
    net = gpu.Net(seed=5)
    M = gpu.learned_preconditioner(Ad, net, nx, ny)
    P = grid_planes(A, ny, nx)
    assert np.array_equal(M.planes(), P)
    params = net.params()
    v = np.random.default_rng(1).standard_normal(nx * ny)
    vd = torch.from_numpy(v).cuda()
    zt = torch.zeros_like(vd)
    M.apply(vd, zt)
    net.set_legacy_mma(True)
    zm = torch.zeros_like(vd)
    M.apply(vd, zm)
    net.set_legacy_mma(False)
    torch.cuda.synchronize()
    z_ref, _ = oracle.net_apply(params, v, P.reshape(-1), ny, nx, round_bf16=True)
    zt, zm = zt.cpu().numpy(), zm.cpu().numpy()
    assert np.isfinite(zt).all()
    assert rel(zm, z_ref) < 1e-2, rel(zm, z_ref)
    assert rel(zt, z_ref) < 1e-2, rel(zt, z_ref)
    # the two tensor-core paths see the same operands; they differ only in
    # FP32 accumulation order (and the BF16 roundings that follow from it)
    assert rel(zt, zm) < 1e-2


def test_gradient_matches_oracle(gpu_lib, oracle, torch):
    nx = ny = 64
    A = matgen.convdiff_2d_grf(nx, seed=12)[0]
    Ad = gpu.Device_matrix(A)
    pairs = gpu.Pairs(nx, ny, 8, 2)
    inst = pairs.add_instance(Ad)
    rng = np.random.default_rng(4)
    es, rs = [], []
    for k in range(3):
        e = rng.standard_normal(nx * ny)
        r = oracle.spmv(A, e)
        pairs.add(inst, torch.from_numpy(r).cuda(), torch.from_numpy(e).cuda())
        es.append(e.astype(np.float32).astype(np.float64))
        rs.append(r.astype(np.float32).astype(np.float64))
    net = gpu.Net(seed=9)
    params = net.params()
    idx = [2, 0]
    mu = 0.2
    loss, g = net.loss_grad(pairs, idx, mu)
    P = grid_planes(A, ny, nx).reshape(-1)
    coef = np.concatenate([P, P])
    r = np.concatenate([rs[i] for i in idx])
    e = np.concatenate([es[i] for i in idx])
    loss_ref, g_ref, _ = oracle.net_loss_grad(params, r, e, coef, 2, ny, nx, mu=mu, round_bf16=True)
    assert loss == pytest.approx(loss_ref, rel=1e-2)
    for l, sl in enumerate(layer_slices()):
        assert rel(g[sl], g_ref[sl]) < 3e-2, (l, rel(g[sl], g_ref[sl]))
    cos = float(np.dot(g, g_ref) / np.linalg.norm(g) / np.linalg.norm(g_ref))
    assert cos > 0.999


def test_training_harvest_and_gain_over_jacobi(gpu_lib, oracle, torch):
    """Harvest (residual, error) pairs from the plain Jacobi-FGMRES(30), train
    on the GPU, and compare FGMRES(30) on a held-out instance with and
    without the network: the plain solver does not reach 1e-8 in the budget
    (or needs at least twice the iterations); the learned one does."""
    n = 64
    pairs = gpu.Pairs(n, n, 400, 8)
    for seed in range(6):
        A = matgen.convdiff_2d_grf(n, pe_range=(1.0, 10.0), seed=100 + seed)[0]
        Ad = gpu.Device_matrix(A)
        inst = pairs.add_instance(Ad)
        xs = np.random.default_rng(seed).uniform(-1, 1, n * n)
        b = oracle.spmv(A, xs)
        got = pairs.harvest(inst, Ad, torch.from_numpy(b).cuda(), torch.from_numpy(xs).cuda(), restart=30,
                            cycles=40)
        assert got == 40
    assert len(pairs) == 240
    net = gpu.Net(seed=1)
    ts = net.train(pairs, gpu.Train_config(steps=600, batch=8, lr=2e-3, mu=1.0, seed=3))
    h = np.array(ts.loss_history)
    assert np.isfinite(h).all()
    assert h[-50:].mean() < 0.8 * h[:20].mean(), (h[:20].mean(), h[-50:].mean())
    A = matgen.convdiff_2d_grf(n, peclet=3.0, seed=999)[0]
    Ad = gpu.Device_matrix(A)
    b = np.random.default_rng(7).uniform(-1, 1, n * n)
    bd = torch.from_numpy(b).cuda()
    cfg = gpu.Fgmres_config(1e-8, 30, 3000)
    res = {}
    for name, M in (("jacobi", gpu.jacobi(Ad)), ("learned", gpu.learned_preconditioner(Ad, net, n, n))):
        xd = torch.zeros_like(bd)
        s = gpu.fgmres(bd, xd, cfg, gpu.spmv(Ad), M)
        torch.cuda.synchronize()
        x = xd.cpu().numpy()
        res[name] = (s.converged, s.computed_iterations, np.linalg.norm(b - oracle.spmv(A, x)) / np.linalg.norm(b))
    conv, its, true_rel = res["learned"]
    assert conv and true_rel < 1.5e-8, res
    assert (not res["jacobi"][0]) or res["jacobi"][1] >= 2 * its, res


def test_fallback_switches_on_stall(gpu_lib, oracle, torch):
    n = 64
    A = matgen.convdiff_2d_grf(n, seed=21)[0]
    Ad = gpu.Device_matrix(A)
    net = gpu.Net(seed=2)
    M = gpu.learned_preconditioner(Ad, net, n, n)
    J = gpu.jacobi(Ad)
    b = np.random.default_rng(8).uniform(-1, 1, n * n)
    bd = torch.from_numpy(b).cuda()
    cfg = gpu.Fgmres_config(1e-8, 30, 300)
    # a ratio of 0 counts every cycle as stalled: the second cycle runs on Jacobi
    xd = torch.zeros_like(bd)
    s, sw = gpu.fgmres_fallback(bd, xd, cfg, gpu.spmv(Ad), M, J, stall_ratio=0.0)
    torch.cuda.synchronize()
    assert sw == 1 and s.computed_iterations == 300
    x = xd.cpu().numpy()
    true = np.linalg.norm(b - oracle.spmv(A, x))
    assert np.isfinite(true) and true < np.linalg.norm(b)
    # a ratio above 1 never switches
    xd = torch.zeros_like(bd)
    s2, sw2 = gpu.fgmres_fallback(bd, xd, cfg, gpu.spmv(Ad), M, J, stall_ratio=1.5)
    assert sw2 == -1 and s2.computed_iterations == 300


def test_coarse_corrected_smoother_gain_at_128(gpu_lib, oracle, torch):
    """The network trained on coarse-corrected pairs, as the smoother of the
    two-level form (coarse correction first), on a held-out 128^2
    instance: FGMRES(30) reaches 1e-8 on the true residual in at most half
    the iterations of the two-level form with Jacobi, and in less time."""
    import time
    net, info = gpu.train_coarse_corrected_smoother(128, instances=40, held=4, cycles=30, steps=3000)
    assert info["held_out_loss_after"] < 0.5 * info["held_out_loss_before"], info
    g = 128
    A = matgen.convdiff_2d_grf(g, seed=777)[0]
    Ad = gpu.Device_matrix(A)
    b = np.random.default_rng(3).uniform(-1, 1, g * g)
    bd = torch.from_numpy(b).cuda()
    L = gpu.learned_preconditioner(Ad, net, g, g)
    forms = {"jacobi": gpu.twolevel(Ad, gpu.jacobi(Ad), g, g, 8),
             "learned": gpu.twolevel(Ad, L, g, g, 8, coarse_first=True)}
    res = {}
    for name, M in forms.items():
        for _ in range(2):  # the second run is timed
            xd = torch.zeros_like(bd)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s = gpu.fgmres(bd, xd, gpu.Fgmres_config(1e-8, 30, 3000), gpu.spmv(Ad), M)
            torch.cuda.synchronize()
            ms = (time.perf_counter() - t0) * 1e3
        rel = np.linalg.norm(b - oracle.spmv(A, xd.cpu().numpy())) / np.linalg.norm(b)
        res[name] = (s.converged, s.computed_iterations, rel, ms)
    assert res["jacobi"][0] and res["learned"][0], res
    assert res["learned"][2] < 1.5e-8, res
    assert 2 * res["learned"][1] <= res["jacobi"][1], res
    assert res["learned"][3] < res["jacobi"][3], res
