"""CPU checks of the learned-preconditioner oracle (oracle/sk_oracle_net.c):
its analytic gradient against central finite differences, and its
features and coefficient planes against plain numpy restatements."""
import numpy as np
import pytest

from oracle.binding import grid_planes
from sparkit_b200 import matgen

CIN = [8, 16, 32, 64, 64, 64, 32, 16, 16]
COUT = [16, 32, 64, 64, 64, 32, 16, 16, 1]


def he_params(seed):
    rng = np.random.default_rng(seed)
    p = []
    for ci, co in zip(CIN, COUT):
        p.append(rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)))
        p.append(rng.standard_normal(co) * 0.1)
    return np.concatenate(p).astype(np.float32)


def test_param_count(oracle):
    assert oracle.net_param_count() == sum(co * 9 * ci + co for ci, co in zip(CIN, COUT)) == 123713


def test_grid_planes_of_the_generator():
    A, _ = matgen.convdiff_2d_grf(16, seed=2)
    P = grid_planes(A, 16, 16)
    d = A.values()[A.col_ind() == np.repeat(np.arange(256), np.diff(A.row_ptr()))]
    assert np.array_equal(P[0], d.astype(np.float32))
    # west coefficient missing on the x = 0 column, north on the last row
    assert not P[1].reshape(16, 16)[:, 0].any() and not P[4].reshape(16, 16)[-1, :].any()
    assert np.array_equal(P[5], (1.0 / d).astype(np.float32))


def test_features(oracle):
    A, _ = matgen.convdiff_2d_grf(16, seed=4)
    P = grid_planes(A, 16, 16)
    r = np.random.default_rng(0).standard_normal(256)
    x, s = oracle.net_features(r, P.reshape(-1), 1, 16, 16, round_bf16=False)
    rt = r * P[5].astype(np.float64)
    assert s[0] == pytest.approx(np.sqrt(np.mean(rt * rt)), rel=1e-14)
    assert np.allclose(x[0, :, :, 0].ravel(), (rt / s[0]).astype(np.float32), rtol=0, atol=0)
    assert np.array_equal(x[0, :, :, 1].ravel(), (P[1] * P[5]).astype(np.float64))
    assert not x[0, :, :, 5:].any()


def test_gradient_matches_finite_differences(oracle):
    """Unrounded (double) oracle: analytic backward vs central differences."""
    H = W = 16
    B = 2
    A, _ = matgen.convdiff_2d_grf(W, seed=5)
    P = grid_planes(A, H, W).reshape(-1)
    coef = np.concatenate([P, P])
    params = he_params(1)
    rng = np.random.default_rng(2)
    r = rng.standard_normal(B * H * W)
    e = rng.standard_normal(B * H * W)
    mu = 0.3
    _, g, _ = oracle.net_loss_grad(params, r, e, coef, B, H, W, mu=mu, round_bf16=False)
    idx = rng.choice(params.size, 48, replace=False)
    worst = 0.0
    for i in idx:
        h = np.float32(1e-5 * max(1.0, abs(float(params[i]))))
        p1 = params.copy()
        p2 = params.copy()
        p1[i] += h
        p2[i] -= h
        hh = (np.float64(p1[i]) - np.float64(p2[i])) / 2
        l1 = oracle.net_loss_grad(p1, r, e, coef, B, H, W, mu, False, False)[0]
        l2 = oracle.net_loss_grad(p2, r, e, coef, B, H, W, mu, False, False)[0]
        worst = max(worst, abs((l1 - l2) / (2 * hh) - g[i]))
    assert worst < 1e-6 * max(1.0, np.abs(g).max())


def test_bf16_rounding_changes_little(oracle):
    """The BF16-rounded forward stays within a few percent of the unrounded one."""
    H = W = 16
    A, _ = matgen.convdiff_2d_grf(W, seed=6)
    P = grid_planes(A, H, W).reshape(-1)
    v = np.random.default_rng(3).standard_normal(H * W)
    params = he_params(7)
    z1, _ = oracle.net_apply(params, v, P, H, W, round_bf16=True)
    z0, _ = oracle.net_apply(params, v, P, H, W, round_bf16=False)
    assert np.linalg.norm(z1 - z0) <= 0.05 * np.linalg.norm(z0)


def test_adam_step(oracle):
    rng = np.random.default_rng(0)
    p = rng.standard_normal(100).astype(np.float32)
    m = np.zeros(100, np.float32)
    v = np.zeros(100, np.float32)
    g = rng.standard_normal(100).astype(np.float32)
    p0 = p.copy()
    oracle.adam(p, m, v, g, 1e-3, 0.9, 0.999, 1e-8, 1)
    # first step of Adam moves every parameter by lr against the gradient's sign
    assert np.allclose(p0 - p, 1e-3 * np.sign(g), rtol=1e-3)
