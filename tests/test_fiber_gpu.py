"""The fiber model on the GPU (xr_dev_forward_fiber, xr_dev_session_begin_fiber,
xr_fiber_reconstruct) against the oracle's restatement of forwardProjFiber /
backwardProjFiber (fiber.cu:13-226), itself pinned bit for bit to the
reference's host build (tests/test_oracle_fiber.py), driven the way
fiberModelReconstruct (reconstruct.cu:1242-1371) drives them.

Tolerance 1e-5 of the largest value, as for the other projectors: the forward
splat sums its taps in another order (per-brick fixed-point tiles, then float
atomics per pixel)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_xr
from oracle import Scan
from scans import fiber_phantom, oblique_rot, three_axes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-5


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


class _DevFloats:
    """A float32 device buffer owned by libxr, seen through the CUDA array
    interface (read-only use: copied to the host at once)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (ptr, False),
                                         "version": 3, "strides": None}


def _device_array(ptr, shape):
    torch.cuda.synchronize()
    return torch.as_tensor(_DevFloats(ptr, shape), device="cuda").cpu().numpy()


def _case(rot, N, Nd, V, K, seed):
    rng = np.random.default_rng(seed)
    C = rot.shape[0]
    basis = np.eye(4, 3, dtype=np.float32)[:K]
    s = Scan(sdd=1000.0, sod=500.0, det=2.0, N=N, Nd=Nd, V=V, rot=rot, trans=rng.normal(0, 0.3, (C, 3)),
             offset=rng.normal(0, 0.2, (C, 3)), basis=basis)
    ctx = load_xr().Context.create(s.sdd, s.sod, s.det, N, Nd, V, s.rot, s.trans, s.offset, s.basis)
    return s, ctx


def _fiber_volume(N, K, seed):
    """Signed fiber vectors (mu_0, mu_1, mu_2) and, for K = 4, a positive
    isotropic term: ps then takes both signs across voxels and views."""
    rng = np.random.default_rng(seed)
    vol = rng.uniform(-1.0, 1.0, (K, N, N, N)).astype(np.float32)
    if K == 4:
        vol[3] = rng.uniform(0.0, 0.5, (N, N, N))
    return vol


def _oracle_forward(oracle, s, vol, rotation=1):
    out = np.zeros((s.C, s.V * s.Nd * s.Nd), np.float32)
    for c in range(s.C):
        for v in range(s.V):
            oracle.fiber_forward_view(s, c, rotation * v, vol.ravel(), out[c])
    return out.reshape(s.C, s.V, s.Nd, s.Nd)


def _oracle_session(oracle, s, sino, vol, epochs, batch, art, lam):
    """fiberModelReconstruct's epochs (reconstruct.cu:1296-1352) with the
    oracle kernels: per subset forwardProjFiber + projRatio / projSubtract over
    every axis, then per slab backwardProjFiber over every axis and view and
    voxelProduct / voxelPlus of channel 0 alone.  Returns (volume, ratio images)."""
    N, Nd, V, K = s.N, s.Nd, s.V, s.K
    sub_size = (V + batch - 1) // batch
    alpha = np.float32(lam / sub_size)
    vol = vol.reshape(K, -1).copy()
    orders = oracle.subset_orders(batch, epochs, True)
    proj = np.zeros((s.C, V * Nd * Nd), np.float32)
    for e in range(epochs):
        proj[:] = 0
        for sub in orders[e]:
            views = [(int(sub) + batch * j) % V for j in range(sub_size)]
            for c in range(s.C):
                for n in views:
                    oracle.fiber_forward_view(s, c, n, vol.ravel(), proj[c])
                    oracle.ratio(s, n, proj[c], sino[c].ravel(), art)
            for y in range(N):
                tmp = np.zeros(K * N * N, np.float32)
                fac = np.zeros(K * N * N, np.float32)
                for c in range(s.C):
                    for n in views:
                        oracle.fiber_backward_slab(s, c, y, n, proj[c], vol.ravel(), tmp, fac)
                v0 = vol[0].reshape(N, N, N)
                t0, f0 = tmp[:N * N].reshape(N, N), fac[:N * N].reshape(N, N)
                if art:
                    v0[:, y, :] = v0[:, y, :] + alpha * t0
                else:
                    with np.errstate(divide="ignore", invalid="ignore"):
                        upd = (v0[:, y, :] * t0) / f0
                    v0[:, y, :] = np.where(f0 == 0, np.float32(0), upd).astype(np.float32)
    return vol.reshape(K, N, N, N), proj.reshape(s.C, V, Nd, Nd)


@pytest.mark.parametrize("axes", ["grid", "oblique"])
@pytest.mark.parametrize("K", [3, 4])
def test_forward_fiber(oracle, axes, K):
    xr = load_xr()
    rot = three_axes() if axes == "grid" else np.concatenate([oblique_rot(71, 2), three_axes()[:1]])
    s, ctx = _case(rot, 16, 24, 10, K, 72)
    vol = _fiber_volume(16, K, 73)
    dv = torch.from_numpy(vol).cuda()
    for rotation, rotate in [(1, xr.Rotate.CW), (-1, xr.Rotate.CCW)]:
        out = torch.full((s.C, s.V, s.Nd, s.Nd), 7.0, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.dev_forward_fiber(dv.data_ptr(), out.data_ptr(), rotate)
        got = out.cpu().numpy()
        ref = _oracle_forward(oracle, s, vol, rotation)
        assert np.abs(ref).max() > 0
        assert rel_err(got, ref) <= TOL, (rotation, rel_err(got, ref))


@pytest.mark.parametrize("ratio_texture", [1, 0], ids=["texture_gather", "linear_loads"])
@pytest.mark.parametrize("method", ["MLEM", "ART"])
@pytest.mark.parametrize("K", [3, 4])
def test_fiber_session(oracle, method, K, ratio_texture):
    xr = load_xr()
    rot = np.concatenate([three_axes()[:2], oblique_rot(74, 1)])
    s, ctx = _case(rot, 12, 20, 9, K, 75)
    ctx.set_option(xr.Option.RATIO_TEXTURE, ratio_texture)
    truth = np.abs(_fiber_volume(12, K, 76))
    truth[:3] *= fiber_phantom(12, 3, 77, np.eye(3, dtype=np.float32))[:3] > 0
    sino = _oracle_forward(oracle, s, truth)
    v0 = np.full((K, 12, 12, 12), 0.01, np.float32)
    art = method == "ART"
    lam = 1e-2
    ref, ref_proj = _oracle_session(oracle, s, sino, v0, 2, 3, art, lam)
    db, dv = torch.from_numpy(sino).cuda(), torch.from_numpy(v0).cuda()
    torch.cuda.synchronize()
    ctx.dev_session_begin_fiber(db.data_ptr(), dv.data_ptr(), 2, 3, method=xr.Method[method], lam=lam)
    for _ in range(2):
        ctx.dev_session_epoch()
    ctx.dev_session_end(0, 0)
    got = dv.cpu().numpy()
    print(f"fiber session {method} K={K}: max rel {rel_err(got, ref):.2e}")
    assert not np.array_equal(ref[0], v0[0])
    assert np.array_equal(got[1:], v0[1:])             # only channel 0 is updated
    assert rel_err(got, ref) <= TOL


@pytest.mark.parametrize("method", ["MLEM", "ART"])
def test_fiber_session_views_revisited(oracle, method):
    """V % batch != 0 (V = 7, batch = 3): the last view of some subsets wraps
    around to a view an earlier subset of the same epoch already ratioed, and
    its forward adds onto that ratio image (reconstruct.cu:1302-1326).  The
    volume and the last ratio images are compared with the oracle."""
    xr = load_xr()
    s, ctx = _case(three_axes(), 12, 20, 7, 4, 80)
    truth = np.abs(_fiber_volume(12, 4, 81))
    sino = _oracle_forward(oracle, s, truth)
    v0 = np.full((4, 12, 12, 12), 0.01, np.float32)
    ref, ref_proj = _oracle_session(oracle, s, sino, v0, 2, 3, method == "ART", 1e-2)
    db, dv = torch.from_numpy(sino).cuda(), torch.from_numpy(v0).cuda()
    torch.cuda.synchronize()
    ctx.dev_session_begin_fiber(db.data_ptr(), dv.data_ptr(), 2, 3, method=xr.Method[method], lam=1e-2)
    for _ in range(2):
        ctx.dev_session_epoch()
    proj = _device_array(ctx.dev_session_proj(), (s.C, s.V, s.Nd, s.Nd))
    ctx.dev_session_end(0, 0)
    got = dv.cpu().numpy()
    assert rel_err(got, ref) <= TOL
    assert rel_err(proj, ref_proj) <= TOL


def test_fiber_reconstruct_host(oracle):
    """xr_fiber_reconstruct on host buffers: channels start at 0.01 whatever
    the caller passed, sino comes back as the last ratio images."""
    xr = load_xr()
    s, ctx = _case(three_axes(), 12, 20, 8, 4, 78)
    truth = np.abs(_fiber_volume(12, 4, 79))
    sino = _oracle_forward(oracle, s, truth)
    ref, ref_proj = _oracle_session(oracle, s, sino, np.full((4, 12, 12, 12), 0.01, np.float32), 3, 2, False, 0.0)
    vol, ratio, losses = ctx.fiber_reconstruct(sino, 3, 2, method=xr.Method.MLEM)
    assert rel_err(vol, ref) <= TOL
    assert rel_err(ratio, ref_proj) <= TOL
    assert losses.shape == (3,) and np.all(losses > 0)


def test_fiber_column_kernels_many_bricks(oracle):
    """40^3 x 4 on three grid-aligned axes (one grating along each of x, y,
    z): the column forms run several bricks per axis (16 x 16 x 8 forward,
    8^3 back, ragged at the volume's edge) and view chunks of the automatic
    size.  Forward of every view, then one MLEM epoch of 3 subsets, against
    the oracle."""
    xr = load_xr()
    s, ctx = _case(three_axes(), 40, 64, 24, 4, 82)
    truth = np.abs(_fiber_volume(40, 4, 83))
    dv = torch.from_numpy(truth).cuda()
    out = torch.empty((s.C, s.V, s.Nd, s.Nd), dtype=torch.float32, device="cuda")
    ctx.dev_forward_fiber(dv.data_ptr(), out.data_ptr(), xr.Rotate.CW)
    sino = _oracle_forward(oracle, s, truth)
    err = rel_err(out.cpu().numpy(), sino)
    print(f"fiber forward 40^3 x 4, 3 x 24 views: max rel {err:.2e}")
    assert err <= TOL
    v0 = np.full((4, 40, 40, 40), 0.01, np.float32)
    ref, ref_proj = _oracle_session(oracle, s, sino, v0, 1, 3, False, 0.0)
    db, dv = torch.from_numpy(sino).cuda(), torch.from_numpy(v0).cuda()
    torch.cuda.synchronize()
    ctx.dev_session_begin_fiber(db.data_ptr(), dv.data_ptr(), 1, 3, method=xr.Method.MLEM)
    ctx.dev_session_epoch()
    proj = _device_array(ctx.dev_session_proj(), (s.C, s.V, s.Nd, s.Nd))
    ctx.dev_session_end(0, 0)
    got = dv.cpu().numpy()
    print(f"fiber MLEM epoch 40^3: volume max rel {rel_err(got, ref):.2e}, ratio {rel_err(proj, ref_proj):.2e}")
    assert rel_err(got, ref) <= TOL
    assert rel_err(proj, ref_proj) <= TOL


def test_fiber_back_nan_in_ratio_images(oracle):
    """A NaN in the measured sinogram of the axis whose grating is along x:
    that axis's channel-0 weight is exactly zero, yet the reference's
    (0 * c) * r turns the voxels that tap the NaN pixel into NaN.  One subset
    of MLEM from mu = 0.01; the NaN voxels and the finite values both match
    the oracle."""
    xr = load_xr()
    s, ctx = _case(three_axes(), 16, 24, 6, 3, 84)
    truth = np.abs(_fiber_volume(16, 3, 85))
    sino = _oracle_forward(oracle, s, truth)
    assert int(np.argmax(np.abs(s.rot[1].reshape(3, 3)[:, 2]))) == 0   # axis 1: grating along x
    sino[1, 2, 12, 12] = np.nan
    v0 = np.full((3, 16, 16, 16), 0.01, np.float32)
    ref, _ = _oracle_session(oracle, s, sino, v0, 1, 1, False, 0.0)
    db, dv = torch.from_numpy(sino).cuda(), torch.from_numpy(v0).cuda()
    torch.cuda.synchronize()
    ctx.dev_session_begin_fiber(db.data_ptr(), dv.data_ptr(), 1, 1, method=xr.Method.MLEM)
    ctx.dev_session_epoch()
    ctx.dev_session_end(0, 0)
    got = dv.cpu().numpy()
    nan_ref = np.isnan(ref)
    assert nan_ref.sum() > 0
    assert np.array_equal(np.isnan(got), nan_ref)
    assert rel_err(np.where(nan_ref, 0, got), np.where(nan_ref, 0, ref)) <= TOL
