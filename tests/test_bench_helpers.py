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


def test_issue_roofline_scales_the_captured_counts():
    """The bench's roofline of a projector kernel: the captured warp
    instructions per voxel-view times this launch's voxel-views, over the
    launch time, against 148 SMs x 4 schedulers x the SM clock; traffic scaled
    by the unit the capture names for reads and writes."""
    bench = _bench()
    figs = bench.profile_figures()
    assert figs is not None and "k_fwd_col<1,g,float>" in figs["kernels"]
    k = figs["kernels"]["k_fwd_col<1,g,float>"]
    per_vv = k["warp_inst_per_launch"] / k["voxel_views_per_launch"]
    r = bench.issue_roofline("k_fwd_col<1,g,float>", 2e-3, 1e9, 2e7, 1e6, 1965.0, 6452.2)
    assert r["bound"] == "issue"
    assert abs(r["achieved"] - per_vv * 1e9 / 2e-3 / 1e9) < 1e-6 * r["achieved"]
    assert abs(r["peak"] - 148 * 4 * 1965e6 / 1e9) < 1e-9
    exp_traffic = (k["dram_read_bytes_per_launch"] * 2e7 / k["voxels_per_launch"] +
                   k["dram_write_bytes_per_launch"] * 1e6 / k["pixel_views_per_launch"])
    assert abs(r["traffic"] - exp_traffic) < 1e-6 * exp_traffic
    assert r["frac"] > 0 and abs(r["frac"] - r["achieved"] / r["peak"]) <= 1e-12 * r["frac"]
    assert bench.issue_roofline("no_such_kernel", 1e-3, 1.0, 1.0, 1.0, 1965.0, 6452.2) is None


def test_l1_roofline_scales_the_captured_wavefronts():
    """The L1 data-pipe roofline: captured LSU wavefronts per voxel-view times
    this launch's voxel-views, over the launch time, against one wavefront per
    cycle on each of 148 SMs at the sampled clock."""
    bench = _bench()
    k = bench.profile_figures()["kernels"]["k_fwd_col<1,g,float>"]
    per_vv = k["l1_wavefronts_per_launch"] / k["voxel_views_per_launch"]
    r = bench.l1_roofline("k_fwd_col<1,g,float>", 2e-3, 1e9, 1965.0)
    assert r["bound"] == "l1"
    assert abs(r["achieved"] - per_vv * 1e9 / 2e-3 / 1e9) < 1e-6 * r["achieved"]
    assert abs(r["peak"] - 148 * 1965e6 / 1e9) < 1e-9
    assert 0 < r["frac"] == r["achieved"] / r["peak"]
    assert bench.l1_roofline("no_such_kernel", 1e-3, 1.0, 1965.0) is None
