"""The allocation-free forward splat, xr_dev_forward_proj_only_static.

Some callers cannot let a library call cudaMalloc: their device memory all
belongs to another allocator (a framework's caching pool that must account
for every byte), or their steady-state loop is not allowed to allocate.  This
entry point keeps its only scratch in a fixed array inside libxr, takes the
caller's device buffers, and must give the same projections as the regular
xr_forward_proj_only.  Collected last (file name) so a failure here leaves
every other test already run; it also passes alone in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_xr
from scans import three_axes

pytestmark = pytest.mark.gpu

TOL = 1e-5   # the projector tolerance of tests/test_gpu_parity.py
XR_ERR_ARG = 1


def _rel(a, b):
    return float(np.abs(a.astype(np.float64) - b).max() / np.abs(b).max())


def _static(L, ctx, d_vol, d_out, rotate, stream):
    return L.xr_dev_forward_proj_only_static(ctx._h, ctypes.c_void_p(d_vol.data_ptr()),
                                             ctypes.c_void_p(d_out.data_ptr()), rotate,
                                             ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("rotate", [0, 1], ids=["cw", "ccw"])
def test_static_forward_matches_regular_entry_point(rotate):
    """Two calls in a row on a context no other call has used (the static
    entry point runs the device and division checks itself), against the
    regular entry point on the same scan and rotation direction."""
    torch = pytest.importorskip("torch")
    xr = load_xr()
    L = xr.lib()
    rng = np.random.default_rng(31 + rotate)
    N, Nd, V, C = 28, 40, 24, 3
    args = (1000.0, 500.0, 2.0, N, Nd, V, three_axes(), rng.normal(0, 0.3, (C, 3)), rng.normal(0, 0.2, (C, 3)))
    ctx = xr.Context.create(*args)
    vol = rng.uniform(0, 1, (N, N, N)).astype(np.float32)

    d_vol = torch.from_numpy(vol).cuda()
    d_out = torch.empty((C, V, Nd, Nd), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    free = []
    got = []
    for call in range(2):                                  # two calls in a row share the scratch
        d_out.fill_(float("nan"))                          # the entry point must clear its output
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        st = _static(L, ctx, d_vol, d_out, rotate, stream)
        assert st == 0, L.xr_last_error(ctx._h)
        stream.synchronize()
        got.append(d_out.cpu().numpy())
    # The first call may load the module holding the fixed array (lazy module
    # loading); the second call must leave free device memory untouched.
    assert torch.cuda.mem_get_info()[0] >= free[1]

    ref = ctx.forward_proj_only(vol, rotate=rotate)        # existing entry point (host buffers)
    for call, g in enumerate(got):
        assert np.isfinite(g).all()
        assert _rel(g, ref) <= TOL, f"call {call}"
    ctx.close()


def test_static_forward_fills_the_scratch_exactly():
    """num_cond * num_proj == 4096: every slot of the fixed array is used
    (frames and view list at their limits)."""
    torch = pytest.importorskip("torch")
    xr = load_xr()
    L = xr.lib()
    rng = np.random.default_rng(32)
    N, Nd, V = 8, 12, 2048
    rot = three_axes()[:2]
    ctx = xr.Context.create(1000.0, 500.0, 2.0, N, Nd, V, rot)
    vol = rng.uniform(0, 1, (N, N, N)).astype(np.float32)
    ref = ctx.forward_proj_only(vol, rotate=1)
    d_vol = torch.from_numpy(vol).cuda()
    d_out = torch.full((2, V, Nd, Nd), float("nan"), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    st = _static(L, ctx, d_vol, d_out, 1, stream)
    assert st == 0, L.xr_last_error(ctx._h)
    stream.synchronize()
    assert _rel(d_out.cpu().numpy(), ref) <= TOL
    ctx.close()


def test_static_forward_refuses_stream_capture():
    """The frames come from host stack memory on every call, so a call on a
    capturing stream is refused (nothing is enqueued) and the capture still
    completes."""
    torch = pytest.importorskip("torch")
    xr = load_xr()
    L = xr.lib()
    N, Nd, V = 8, 12, 6
    ctx = xr.Context.create(1000.0, 500.0, 2.0, N, Nd, V, three_axes())
    d_vol = torch.ones((N, N, N), dtype=torch.float32, device="cuda")
    d_out = torch.zeros((3, V, Nd, Nd), dtype=torch.float32, device="cuda")
    side = torch.zeros(1, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        side.add_(1.0)
        st = _static(L, ctx, d_vol, d_out, 0, stream)
    assert st == XR_ERR_ARG
    assert b"captured" in L.xr_last_error(ctx._h)
    del g
    ctx.close()


def test_static_forward_rejects_oversized_scan():
    xr = load_xr()
    L = xr.lib()
    rot = np.tile(np.eye(3, dtype=np.float32).ravel(), (2, 1))
    ctx = xr.Context.create(1000.0, 500.0, 2.0, 8, 12, 2049, rot)   # 2 * 2049 > 4096 pairs
    st = L.xr_dev_forward_proj_only_static(ctx._h, ctypes.c_void_p(1), ctypes.c_void_p(1), 0, None)
    assert st == XR_ERR_ARG
    assert b"4096" in L.xr_last_error(ctx._h)
    ctx.close()
