"""The regularisers' CPU oracle (oracle/regularisers.py) by its own identities
(parity against the reference is unpinned: the reference's code is host
Eigen, absent here)."""
from __future__ import annotations

import numpy as np

import regularisers as rg


def test_tv_operator_is_the_masked_forward_difference():
    rng = np.random.default_rng(0)
    Z, Y, X = 4, 5, 6
    v = rng.normal(size=(Z, Y, X))
    F = rg.tv_operator(X, Y, Z)
    fx = (F @ v.ravel()).reshape(Z, Y, X, 3)
    want = np.zeros((Z, Y, X, 3))
    want[:-1, :-1, :-1, 0] = (v[:-1, :-1, 1:] - v[:-1, :-1, :-1])
    want[:-1, :-1, :-1, 1] = (v[:-1, 1:, :-1] - v[:-1, :-1, :-1])
    want[:-1, :-1, :-1, 2] = (v[1:, :-1, :-1] - v[:-1, :-1, :-1])
    assert np.allclose(fx, want)


def test_tv_without_penalty_returns_the_input():
    rng = np.random.default_rng(1)
    v = rng.uniform(0, 1, (5, 6, 7))
    out = rg.tv_minimize(v, 0.7, 0.0, 200)       # ADMM from y = u = 1 converges geometrically
    assert np.abs(out - v).max() < 1e-9


def test_tv_penalty_reduces_total_variation():
    rng = np.random.default_rng(2)
    v = rng.uniform(0, 1, (6, 6, 6))
    F = rg.tv_operator(6, 6, 6)
    tv = lambda a: np.abs(F @ a.ravel()).sum()
    out = rg.tv_minimize(v, 0.5, 0.2, 30)
    assert tv(out) < 0.5 * tv(v)
    assert abs(out.mean() - v.mean()) < 0.05


def test_quad_tensor_decomposes_back():
    """Q = R^T diag(m, m, 0) R: eigenvalues (0, m, m); the smallest
    eigenvector is row 2 of R, whose z component is the input cosine."""
    rng = np.random.default_rng(3)
    shape = (3, 4, 5)
    vox = rng.uniform(0.1, 1.0, (3,) + shape)
    coef = np.stack([rng.uniform(-3, 3, shape), rng.uniform(0.1, 0.95, shape)])
    v2, c2 = rg.quad_decompose(rg.quad_tensor(vox, coef))
    m = vox.sum(0)
    assert np.allclose(v2[0], m) and np.allclose(v2[1], m) and np.allclose(v2[2], 0, atol=1e-12)
    assert np.allclose(c2[1], coef[1])
