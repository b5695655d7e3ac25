"""The oracle's FDK and orientation post-processing against the reference's
own kernels (CPU, no GPU): the fixture tests/golden/ref_fdk_small.npz was made
by tests/golden/make_golden_fdk.py from reconstruct/src/fdk.cu:13-170 and
direction/src/pca.cu:67-106 compiled for the host, driven by the restated
FDK::reconstruct loop (reconstruct.cu:1651-1724).  The FP32 oracle must match
bit for bit."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import Scan

FIX = os.path.join(ROOT, "tests", "golden", "ref_fdk_small.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(FIX)


def _scan(g) -> Scan:
    sdd, sod, det, N, Nd, V = g["fdk_geom"]
    return Scan(sdd=float(sdd), sod=float(sod), det=float(det), N=int(N), Nd=int(Nd), V=int(V), rot=g["fdk_rot"],
                trans=g["fdk_trans"], offset=g["fdk_offset"], basis=np.array([[0.0, 0.0, 1.0]], np.float32))


def test_oracle_fdk_weight_and_filter_bit_exact(oracle, gold):
    s = _scan(gold)
    assert np.array_equal(oracle.fdk_weight(s), gold["fdk_weight"])
    assert np.array_equal(oracle.fdk_filter(s, ramlak=False), gold["fdk_filter"])


@pytest.mark.parametrize("ccw", [0, 1])
def test_oracle_fdk_bit_exact(oracle, gold, ccw):
    """Whole FDK::reconstruct: filtered sinograms and volumes (axis 0's
    filtered block back-projected for every axis, as the reference)."""
    s = _scan(gold)
    vol, filt = oracle.fdk_reconstruct(s, gold["fdk_sino"], rotate_ccw=ccw, ramlak=False, block0=True)
    assert np.abs(gold[f"fdk_vol_{ccw}"]).max() > 0
    assert np.array_equal(filt, gold[f"fdk_filt_{ccw}"])
    assert np.array_equal(vol, gold[f"fdk_vol_{ccw}"])


def test_oracle_angle_bit_exact(oracle, gold):
    assert np.array_equal(oracle.angle_from_md(gold["pca_md"]), gold["pca_angle"])


def test_oracle_direction_normalization_bit_exact(oracle, gold):
    got = oracle.direction_normalization(gold["pca_md"])
    assert np.array_equal(got, gold["pca_norm"])
    assert (got == 0).any() and (got != 0).any()        # both branches of the 0.65 threshold
