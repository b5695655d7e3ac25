"""Host-side helpers of bench.py that need no GPU: the angular error between
per-voxel main directions (unsigned axes, masked voxels, zero vectors left
out) used by the time-to-residual comparison."""
from __future__ import annotations

import importlib.util
import math
import os

import pytest

from conftest import ROOT

torch = pytest.importorskip("torch")


def _bench():
    spec = importlib.util.spec_from_file_location("xr_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_angle_stats_unsigned_and_masked():
    b = _bench()
    N = 6
    ang = math.radians(25.0)
    md_a = torch.zeros(3, N, N, N)
    md_a[0] = 2.0                                   # lengths do not matter
    md_b = torch.zeros(3, N, N, N)
    md_b[0], md_b[1] = math.cos(ang), math.sin(ang)
    md_b[:, :3] *= -1                               # nor does the sign of an axis
    mask = torch.ones(N, N, N, dtype=torch.bool)
    mask[0] = False
    st = b.angle_stats(md_a, md_b, mask)
    assert st["voxels"] == (N - 1) * N * N
    for k in ("mean_deg", "median_deg", "p90_deg"):
        assert abs(st[k] - 25.0) < 1e-5             # FP32 inputs
    md_a[:, 1] = 0.0                                # empty voxels are left out
    assert b.angle_stats(md_a, md_b, mask)["voxels"] == (N - 2) * N * N
    assert b.angle_stats(md_a, md_b, torch.zeros(N, N, N, dtype=torch.bool)) == {"voxels": 0}
