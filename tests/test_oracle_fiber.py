"""Pin the oracle's fiber-model restatement (forwardProjFiber,
backwardProjFiber with rayCastingFiber's frame) bit for bit against golden
vectors from the reference's own fiber.cu built for the host
(tests/golden/make_golden_fiber.py).  CPU only."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import Scan


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_fiber_small.npz"))


def _scan(g, K) -> Scan:
    sdd, sod, det, N, Nd, V = g[f"k{K}_geom"]
    return Scan(sdd=float(sdd), sod=float(sod), det=float(det), N=int(N), Nd=int(Nd), V=int(V), rot=g[f"k{K}_rot"],
                trans=g[f"k{K}_trans"], offset=g[f"k{K}_offset"], basis=g[f"k{K}_basis"])


@pytest.mark.parametrize("K", [3, 4])
@pytest.mark.parametrize("cond", [0, 1, 2])
@pytest.mark.parametrize("sign", [1, -1])
def test_fiber_projectors_bit_exact(oracle, g, K, cond, sign):
    """Views n > 0 (Rotate::CW) and n < 0 (Rotate::CCW, written to image |n|)."""
    s = _scan(g, K)
    N, Nd, V = s.N, s.Nd, s.V
    n = sign * (2 + 3 * cond)
    m = abs(n)
    tag = "" if sign > 0 else "_ccw"
    vol = g[f"k{K}_vol"].ravel()
    p = np.zeros(V * Nd * Nd, np.float32)
    oracle.fiber_forward_view(s, cond, n, vol.copy(), p)
    assert np.array_equal(p[m * Nd * Nd:(m + 1) * Nd * Nd], g[f"k{K}_fwd_c{cond}{tag}"])
    assert not p[:m * Nd * Nd].any() and not p[(m + 1) * Nd * Nd:].any()
    tmp = np.zeros(K * N * N, np.float32)
    fac = np.zeros(K * N * N, np.float32)
    oracle.fiber_backward_slab(s, cond, 4, n, g[f"k{K}_ratio"].ravel().copy(), vol.copy(), tmp, fac)
    assert np.array_equal(tmp, g[f"k{K}_bwd_c{cond}{tag}_tmp"])
    assert np.array_equal(fac, g[f"k{K}_bwd_c{cond}{tag}_fac"])


@pytest.mark.parametrize("K", [3, 4])
def test_fiber_forward_fp64_and_symmetries(oracle, g, K):
    """The FP32 restatement against the FP64 one (relative 1e-5 of the largest
    pixel), and two exact properties of forwardProjFiber's |ps| weight: the
    projection of -mu equals that of mu bit for bit, and scaling mu by a power
    of two scales the projection by it exactly."""
    s = _scan(g, K)
    Nd, V = s.Nd, s.V
    vol = g[f"k{K}_vol"].ravel()
    for cond in range(3):
        n = 1 + 2 * cond
        p32 = np.zeros(V * Nd * Nd, np.float32)
        oracle.fiber_forward_view(s, cond, n, vol.copy(), p32)
        p64 = np.zeros(V * Nd * Nd, np.float64)
        oracle.fiber_forward_view(s, cond, n, vol.astype(np.float64), p64, dt=np.float64)
        assert np.abs(p64).max() > 0
        assert np.abs(p32 - p64).max() <= 1e-5 * np.abs(p64).max()
        neg = np.zeros_like(p32)
        oracle.fiber_forward_view(s, cond, n, (-vol).copy(), neg)
        assert np.array_equal(neg, p32)
        dbl = np.zeros_like(p32)
        oracle.fiber_forward_view(s, cond, n, (4.0 * vol).astype(np.float32), dbl)
        assert np.array_equal(dbl, 4.0 * p32)


@pytest.mark.parametrize("i", [0, 1, 2, 3, 4])
def test_fiber_session_bit_exact(oracle, g, i):
    """Whole fiberModelReconstruct runs (two epochs, three subsets; MLEM / ART,
    CW / CCW, K = 3 / 4; case 4 with 7 views, so subsets revisit views and
    their forwards add onto the earlier ratio images) from 0.01: the oracle's
    driver gives the reference's
    volume (channel 0 updated, the others untouched) and last ratio images bit
    for bit; the loss sums agree to float accumulation order."""
    K, art, ccw = (int(v) for v in g[f"s{i}_case"])
    sdd, sod, det, N, Nd, V = g[f"s{i}_geom"]
    s = Scan(sdd=float(sdd), sod=float(sod), det=float(det), N=int(N), Nd=int(Nd), V=int(V), rot=g[f"s{i}_rot"],
             trans=g[f"s{i}_trans"], offset=g[f"s{i}_offset"], basis=g[f"s{i}_basis"])
    v0 = np.full((K, s.N, s.N, s.N), 0.01, np.float32)
    vol, ratio, losses = oracle.fiber_reconstruct(s, g[f"s{i}_sino"], v0, 2, 3, ccw, bool(art), 1e-2)
    assert np.array_equal(vol, g[f"s{i}_vol"])
    assert np.array_equal(ratio, g[f"s{i}_ratio"])
    assert np.array_equal(vol[1:], v0[1:]) and not np.array_equal(vol[0], v0[0])
    assert np.allclose(losses, g[f"s{i}_losses"], rtol=1e-5)
