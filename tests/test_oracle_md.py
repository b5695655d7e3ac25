"""Pin the oracle's main-direction restatements (forwardOrthByMD,
backwardOrthByMD, meanFiltFiberMD, calcMainDirection, calcMDWithEst,
updateEstimation) and coefficient-plane steps (meanFiltFiber,
calcNormalVectorThreeDirecWithEst, updateEstimationByCoef) bit for bit against golden vectors from the reference's own
ir.cu built for the host (tests/golden/make_golden_md.py).  CPU only."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import Scan


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_md_small.npz"))


def _scan(g) -> Scan:
    sdd, sod, det, N, Nd, V = g["geom"]
    return Scan(sdd=float(sdd), sod=float(sod), det=float(det), N=int(N), Nd=int(Nd), V=int(V), rot=g["rot"],
                trans=g["trans"], offset=g["offset"], basis=g["basis"])


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


@pytest.mark.parametrize("cond", [0, 1, 2])
def test_forward_and_backward_md_bit_exact(oracle, g, cond):
    s = _scan(g)
    N, Nd, V = s.N, s.Nd, s.V
    n = 1 + 3 * cond
    p = np.zeros(V * Nd * Nd, np.float32)
    fac = np.zeros(Nd * Nd, np.float32)
    oracle.forward_md_view(s, cond, n, g["vol"].ravel().copy(), g["md"].ravel().copy(), p, fac)
    assert same(p[n * Nd * Nd:(n + 1) * Nd * Nd], g[f"fwd_c{cond}"])
    assert same(fac, g[f"fwd_c{cond}_fac"])
    tmp = np.zeros(3 * N * N, np.float32)
    bf = np.zeros(3 * N * N, np.float32)
    oracle.backward_md_slab(s, cond, 5, n, g["ratio"].ravel().copy(), g["md"].ravel().copy(), tmp, bf)
    assert same(tmp, g[f"bwd_c{cond}_tmp"])
    assert same(bf, g[f"bwd_c{cond}_fac"])


def test_md_filter_bit_exact(oracle, g):
    s = _scan(g)
    out = g["md"].ravel().copy()
    for y in range(2, s.N - 2):
        oracle.md_filter_slab(s, y, g["md"].ravel().copy(), out, 1.0)
    assert same(out, g["filter"])


@pytest.mark.parametrize("it", [0, 1, 2, 3])
def test_main_direction_bit_exact(oracle, g, it):
    s = _scan(g)
    m = g["md"].ravel().copy()
    oracle.main_direction(s, g["vol"].ravel().copy(), m, it)
    assert same(m, g[f"main_it{it}"])


def test_md_with_estimate_and_update_bit_exact(oracle, g):
    s = _scan(g)
    m = g["md"].ravel().copy()
    oracle.md_with_estimate(s, g["vol"].ravel().copy(), m, g["est"].ravel().copy())
    assert same(m, g["with_est"])
    e = g["est"].ravel().copy()
    oracle.update_estimation(s, g["vol"].ravel().copy(), e, 2)
    assert same(e, g["update_est"])


def test_coefficient_steps_bit_exact(oracle, g):
    s = _scan(g)
    c = g["coef"].ravel().copy()
    loss = np.zeros(s.N ** 3, np.float32)
    oracle.normal_three_est(s, g["vol"].ravel().copy(), c, loss, g["est"].ravel().copy())
    assert same(c, g["nrm_est_coef"])
    assert same(loss, g["nrm_est_loss"])
    cf = g["coef"].ravel().copy()
    for y in range(1, s.N - 1):
        oracle.coef_filter_slab(s, y, g["coef"].ravel().copy(), g["vol"].ravel().copy(), cf, 1.0)
    assert same(cf, g["coef_filter"])
    e = g["est"].ravel().copy()
    oracle.update_estimation_coef(s, g["vol"].ravel().copy(), e, 3)
    assert same(e, g["update_est_coef"])
