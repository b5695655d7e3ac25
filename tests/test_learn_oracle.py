"""The warm-start network's CPU oracle (oracle/warmstart.py), pinned without a
GPU: convolution against direct loops, dgrad / wgrad as exact adjoints, the
network gradient against central finite differences in float64, and BF16
rounding known answers."""
from __future__ import annotations

import numpy as np

import warmstart as ws


def test_bf16_rounding_known_answers():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -7, -2.5, 0.0, 3.140625], np.float32)
    # 1 + 2^-8 is a tie -> even (1.0); 1 + 3*2^-8 is a tie -> even (1 + 2^-6)
    want = np.array([1.0, 1.0, 1.0 + 2 ** -6, 1.0 + 2 ** -7, -2.5, 0.0, 3.140625])
    assert np.array_equal(ws.bf16(x), want)
    assert ws.bf16_bits(np.array([1.0], np.float32))[0] == 0x3F80


def test_conv3d_matches_direct_loops():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(3, 4, 5, 2))
    w = rng.normal(size=(27, 3, 2))
    b = rng.normal(size=3)
    y = ws.conv3d(x, w, b)
    nz, ny, nx = x.shape[:3]
    ref = np.zeros((nz, ny, nx, 3))
    for z in range(nz):
        for yy in range(ny):
            for xx in range(nx):
                acc = b.copy()
                for t, (dz, dy, dx) in enumerate(ws.taps()):
                    zz, y2, x2 = z + dz, yy + dy, xx + dx
                    if 0 <= zz < nz and 0 <= y2 < ny and 0 <= x2 < nx:
                        acc += w[t] @ x[zz, y2, x2]
                ref[z, yy, xx] = acc
    assert np.allclose(y, ref, rtol=1e-12, atol=1e-12)


def test_dgrad_and_wgrad_are_adjoints():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(4, 3, 5, 3))
    w = rng.normal(size=(27, 2, 3))
    g = rng.normal(size=(4, 3, 5, 2))
    lhs = (ws.conv3d(x, w) * g).sum()
    assert np.isclose(lhs, (x * ws.conv3d_dgrad(g, w)).sum(), rtol=1e-12)
    assert np.isclose(lhs, (w * ws.conv3d_wgrad(x, g)).sum(), rtol=1e-12)


def test_net_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    C, Wd, D = 2, 3, 3
    shapes = ws.layer_shapes(C, Wd, D)
    n = sum(27 * ci * co + co for ci, co in shapes)
    p = rng.normal(0, 0.2, n)
    x = rng.uniform(0, 1, (C, 3, 4, 4))
    t = rng.uniform(0, 1, (C, 3, 4, 4))
    loss, g, _ = ws.net_loss_grad(p, x, t, C, Wd, D, in_scale=1.7, bf16_emulation=False)
    idx = rng.choice(n, 40, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(n)
        e[i] = h
        lp, _, _ = ws.net_loss_grad(p + e, x, t, C, Wd, D, in_scale=1.7, bf16_emulation=False)
        lm, _, _ = ws.net_loss_grad(p - e, x, t, C, Wd, D, in_scale=1.7, bf16_emulation=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
    assert loss > 0


def test_tensor_loss_is_the_frobenius_error_of_the_direction_tensor():
    """The oracle's orientation term equals weight * ||sum_k d_k S_k S_k^T||_F^2
    summed over voxels (/ K voxels), and its gradient matches finite
    differences."""
    rng = np.random.default_rng(3)
    C, Wd, D = 3, 3, 2
    basis = rng.normal(0, 1, (C, 3))
    shapes = ws.layer_shapes(C, Wd, D)
    n = sum(27 * ci * co + co for ci, co in shapes)
    p = rng.normal(0, 0.2, n)
    x = rng.uniform(0, 1, (C, 3, 4, 4))
    t = rng.uniform(0, 1, (C, 3, 4, 4))
    w = 2.5
    l0, _, pred = ws.net_loss_grad(p, x, t, C, Wd, D, bf16_emulation=False)
    loss, g, _ = ws.net_loss_grad(p, x, t, C, Wd, D, bf16_emulation=False, tensor_basis=basis, tensor_weight=w)
    d = pred - t                                              # [C, nz, ny, nx]
    SS = np.einsum("ki,kj->kij", basis, basis)
    dT = np.einsum("kzyx,kij->zyxij", d, SS)
    assert abs(loss - (l0 + w * (dT ** 2).sum() / d.size)) <= 1e-12 * loss
    idx = rng.choice(n, 30, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(n)
        e[i] = h
        lp, _, _ = ws.net_loss_grad(p + e, x, t, C, Wd, D, bf16_emulation=False, tensor_basis=basis,
                                    tensor_weight=w)
        lm, _, _ = ws.net_loss_grad(p - e, x, t, C, Wd, D, bf16_emulation=False, tensor_basis=basis,
                                    tensor_weight=w)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
