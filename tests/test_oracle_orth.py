"""Pin the oracle's orientation-parametrised XTT restatement (forwardOrth,
backwardOrth, calcNormalVectorThreeDirec) bit for bit against golden vectors
from the reference's own ir.cu built for the host
(tests/golden/make_golden_orth.py).  CPU only."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import Scan


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_orth_small.npz"))


def _scan(g) -> Scan:
    sdd, sod, det, N, Nd, V = g["geom"]
    return Scan(sdd=float(sdd), sod=float(sod), det=float(det), N=int(N), Nd=int(Nd), V=int(V), rot=g["rot"],
                trans=g["trans"], offset=g["offset"], basis=g["basis"])


@pytest.mark.parametrize("cond", [0, 1, 2])
def test_forward_and_backward_orth_bit_exact(oracle, g, cond):
    s = _scan(g)
    N, Nd, V = s.N, s.Nd, s.V
    n = 2 + 3 * cond
    p = np.zeros(V * Nd * Nd, np.float32)
    oracle.forward_orth_view(s, cond, n, g["vol"].ravel().copy(), g["coef"].ravel().copy(), p)
    assert np.array_equal(p[n * Nd * Nd:(n + 1) * Nd * Nd], g[f"fwd_c{cond}"])
    tmp = np.zeros(3 * N * N, np.float32)
    fac = np.zeros(3 * N * N, np.float32)
    oracle.backward_orth_slab(s, cond, 5, n, g["ratio"].ravel().copy(), g["coef"].ravel().copy(), tmp, fac)
    assert np.array_equal(tmp, g[f"bwd_c{cond}_tmp"])
    assert np.array_equal(fac, g[f"bwd_c{cond}_fac"])


@pytest.mark.parametrize("rot", [0, 1, 2, 3])
def test_normal_three_bit_exact(oracle, g, rot):
    s = _scan(g)
    c = g["coef"].ravel().copy()
    loss = np.zeros(s.N ** 3, np.float32)
    oracle.normal_three(s, g["vol"].ravel().copy(), c, loss, rot)
    assert np.array_equal(c, g[f"nrm_r{rot}_coef"])
    assert np.array_equal(loss, g[f"nrm_r{rot}_loss"])
