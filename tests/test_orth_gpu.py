"""Orientation-parametrised XTT on the GPU (xr_dev_forward_orth,
xr_dev_session_begin_orth, xr_orth_normal_update) against the oracle's
restatement of forwardOrth / backwardOrth / calcNormalVectorThreeDirec, itself
pinned bit for bit to the reference's host build (tests/test_oracle_orth.py).

Tolerance 1e-5 of the largest value, as for the other projectors: the float
sums run in another order, and the rotation's cos / sin are the device's."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_xr
from oracle import Scan
from scans import basis13, fiber_phantom, oblique_rot, three_axes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-5


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _case(rot, N, Nd, V, K, seed):
    rng = np.random.default_rng(seed)
    C = rot.shape[0]
    s = Scan(sdd=1000.0, sod=500.0, det=2.0, N=N, Nd=Nd, V=V, rot=rot, trans=rng.normal(0, 0.3, (C, 3)),
             offset=rng.normal(0, 0.2, (C, 3)), basis=basis13()[:K])
    ctx = load_xr().Context.create(s.sdd, s.sod, s.det, N, Nd, V, s.rot, s.trans, s.offset, s.basis)
    coef = np.stack([rng.uniform(-3.1, 3.1, (N, N, N)), rng.uniform(0.05, 0.99, (N, N, N))]).astype(np.float32)
    return s, ctx, coef


def _oracle_forward(oracle, s, vol, coef):
    out = np.zeros((s.C, s.V * s.Nd * s.Nd), np.float32)
    for c in range(s.C):
        for v in range(s.V):
            oracle.forward_orth_view(s, c, v, vol.ravel(), coef.ravel(), out[c])
    return out.reshape(s.C, s.V, s.Nd, s.Nd)


@pytest.mark.parametrize("axes", ["grid", "oblique"])
@pytest.mark.parametrize("K", [3, 13])
def test_forward_orth(oracle, axes, K):
    rot = three_axes() if axes == "grid" else np.concatenate([oblique_rot(51, 2), three_axes()[:1]])
    s, ctx, coef = _case(rot, 16, 24, 10, K, 52)
    vol = np.random.default_rng(53).uniform(0, 1, (K, 16, 16, 16)).astype(np.float32)
    dv, dc = torch.from_numpy(vol).cuda(), torch.from_numpy(coef).cuda()
    out = torch.zeros((s.C, s.V, s.Nd, s.Nd), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx.dev_forward_orth(dv.data_ptr(), dc.data_ptr(), out.data_ptr())
    got = out.cpu().numpy()
    ref = _oracle_forward(oracle, s, vol, coef)
    assert rel_err(got, ref) <= TOL


def _oracle_session(oracle, s, sino, vol, coef, epochs, batch, art, lam):
    """orthTwiceReconstruct's inner epochs (reconstruct.cu:1067-1127) with the
    oracle kernels: per subset forwardOrth + projRatio over every axis, then per
    slab backwardOrth over every axis and view, then voxelProduct / voxelPlus."""
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
                    oracle.forward_orth_view(s, c, n, vol.ravel(), coef.ravel(), proj[c])
                    oracle.ratio(s, n, proj[c], sino[c].ravel(), art)
            for y in range(N):
                tmp = np.zeros(K * N * N, np.float32)
                fac = np.zeros(K * N * N, np.float32)
                for c in range(s.C):
                    for n in views:
                        oracle.backward_orth_slab(s, c, y, n, proj[c], coef.ravel(), tmp, fac)
                v3 = vol.reshape(K, N, N, N)
                t3, f3 = tmp.reshape(K, N, N), fac.reshape(K, N, N)
                if art:
                    v3[:, :, y, :] = v3[:, :, y, :] + alpha * t3
                else:
                    with np.errstate(divide="ignore", invalid="ignore"):
                        upd = (v3[:, :, y, :] * t3) / f3
                    v3[:, :, y, :] = np.where(f3 == 0, np.float32(0), upd).astype(np.float32)
    return vol.reshape(K, N, N, N)


@pytest.mark.parametrize("method", ["MLEM", "ART"])
def test_orth_session(oracle, method):
    xr = load_xr()
    s, ctx, coef = _case(three_axes(), 12, 20, 8, 3, 54)
    truth = fiber_phantom(s.N, 3, 55, s.basis)
    sino = _oracle_forward(oracle, s, truth, coef)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.05, np.float32)
    art = method == "ART"
    lam = 1e-3
    ref = _oracle_session(oracle, s, sino, v0, coef, 2, 3, art, lam)
    ctx.set_option(xr.Option.XTT_SQRT, 0)
    db, dv, dc = (torch.from_numpy(a).cuda() for a in (sino, v0, coef))
    torch.cuda.synchronize()
    ctx.dev_session_begin_orth(db.data_ptr(), dv.data_ptr(), dc.data_ptr(), 2, 3, method=xr.Method[method], lam=lam)
    for _ in range(2):
        ctx.dev_session_epoch()
    ctx.dev_session_end(0, 0)
    got = dv.cpu().numpy()
    print(f"orth session {method}: max rel {rel_err(got, ref):.2e}")
    assert rel_err(got, ref) <= TOL


@pytest.mark.parametrize("rot", [0, 1, 2, 3])
def test_orth_normal_update(oracle, rot):
    s, ctx, coef = _case(three_axes(), 12, 20, 8, 3, 56)
    vol = np.random.default_rng(57).uniform(0.1, 1.0, (3, 12, 12, 12)).astype(np.float32)
    c_ref = coef.ravel().copy()
    l_ref = np.zeros(12 ** 3, np.float32)
    oracle.normal_three(s, vol.ravel().copy(), c_ref, l_ref, rot)
    dv, dc = torch.from_numpy(vol).cuda(), torch.from_numpy(coef).cuda()
    dl = torch.zeros(12 ** 3, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx.orth_normal_update(dv.data_ptr(), dc.data_ptr(), dl.data_ptr(), rot)
    c_got = dc.cpu().numpy().ravel()
    n3 = 12 ** 3
    # compare the direction (cos, sin of phi) and cos theta, not the wrapped angle
    unit = lambda c: np.stack([np.cos(c[:n3]), np.sin(c[:n3]), c[n3:]])
    assert np.abs(unit(c_got) - unit(c_ref)).max() <= 1e-4
    assert np.abs(dl.cpu().numpy() - l_ref).max() <= 1e-5


def test_orth_coefficient_steps(oracle):
    """calcNormalVectorThreeDirecWithEst, meanFiltFiber (two passes, border
    kept) and updateEstimationByCoef against the oracle."""
    s, ctx, coef = _case(three_axes(), 12, 20, 8, 3, 58)
    N = s.N
    rng = np.random.default_rng(59)
    vol = rng.uniform(0.1, 1.0, (3, N, N, N)).astype(np.float32)
    est = np.stack([rng.uniform(-1, 1, (N, N, N)), rng.uniform(0, 3.5, (N, N, N))]).astype(np.float32)
    dv, de = torch.from_numpy(vol).cuda(), torch.from_numpy(est).cuda()
    n3 = N ** 3
    unit = lambda c: np.stack([np.cos(c[:n3]), np.sin(c[:n3]), c[n3:]])
    # WithEst
    c_ref = coef.ravel().copy()
    l_ref = np.zeros(n3, np.float32)
    oracle.normal_three_est(s, vol.ravel().copy(), c_ref, l_ref, est.ravel().copy())
    dc = torch.from_numpy(coef).cuda()
    dl = torch.zeros(n3, dtype=torch.float32, device="cuda")
    ctx.orth_normal_update_est(dv.data_ptr(), dc.data_ptr(), dl.data_ptr(), de.data_ptr())
    assert np.abs(unit(dc.cpu().numpy().ravel()) - unit(c_ref)).max() <= 1e-4
    assert np.abs(dl.cpu().numpy() - l_ref).max() <= 1e-5
    # meanFiltFiber, two passes
    ref = coef.ravel().copy()
    for _ in range(2):
        out = ref.copy()
        for y in range(1, N - 1):
            oracle.coef_filter_slab(s, y, ref, vol.ravel().copy(), out, 1.0)
        ref = out
    dc = torch.from_numpy(coef).cuda()
    tmp = torch.empty_like(dc)
    ctx.orth_filter(dc.data_ptr(), tmp.data_ptr(), dv.data_ptr(), 1.0, 2)
    assert np.abs(unit(dc.cpu().numpy().ravel()) - unit(ref)).max() <= 1e-4
    # updateEstimationByCoef
    ref = est.ravel().copy()
    oracle.update_estimation_coef(s, vol.ravel().copy(), ref, 3)
    ctx.orth_update_estimation(dv.data_ptr(), de.data_ptr(), 3)
    got = de.cpu().numpy().ravel()
    assert np.array_equal(got[n3:], ref[n3:])
    assert np.abs(got[:n3] - ref[:n3]).max() <= 1e-6


def test_kept_sensitivity_follows_the_session_kind(oracle):
    """The per-subset sensitivity of a plain XTT MLEM session is kept on the
    context for the next session of the same subsets and rotation; a
    rotated-basis session in between computes its own into the same buffer,
    so the next plain session must compute it again.  Plain -> orth -> plain
    (CW) -> plain (CCW) on one context, each against the oracle."""
    xr = load_xr()
    s, ctx, coef = _case(three_axes(), 12, 20, 8, 13, 58)
    truth = fiber_phantom(s.N, 3, 59, s.basis)
    sino_plain = {rot: oracle.forward_all(s, truth, 1 if rot else 0, True) for rot in (0, 1)}
    sino_orth = _oracle_forward(oracle, s, truth, coef)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.05, np.float32)

    def plain(rot):
        ref, _, _ = oracle.xtt_reconstruct(s, sino_plain[rot], v0, 2, 3, rotate_ccw=rot)
        ctx.set_option(xr.Option.XTT_SQRT, 1)      # ends with voxelSqrt, as the oracle
        db, dv = torch.from_numpy(sino_plain[rot]).cuda(), torch.from_numpy(v0).cuda()
        torch.cuda.synchronize()
        ctx.dev_session_begin(db.data_ptr(), dv.data_ptr(), True, 2, 3, rotate=rot)
        for _ in range(2):
            ctx.dev_session_epoch()
        ctx.dev_session_end(0, 0)
        return rel_err(dv.cpu().numpy(), ref)

    assert plain(0) <= TOL
    ref = _oracle_session(oracle, s, sino_orth, v0, coef, 2, 3, False, 1e-3)
    ctx.set_option(xr.Option.XTT_SQRT, 0)      # the rotated-basis session's iterate
    db, dv, dc = (torch.from_numpy(a).cuda() for a in (sino_orth, v0, coef))
    torch.cuda.synchronize()
    ctx.dev_session_begin_orth(db.data_ptr(), dv.data_ptr(), dc.data_ptr(), 2, 3)
    for _ in range(2):
        ctx.dev_session_epoch()
    ctx.dev_session_end(0, 0)
    assert rel_err(dv.cpu().numpy(), ref) <= TOL
    assert plain(0) <= TOL          # recomputed after the orth session
    assert plain(0) <= TOL          # kept
    assert plain(1) <= TOL          # another rotation: recomputed
