"""Main-direction XTT on the GPU (xr_dev_forward_md, xr_dev_session_begin_md and
the circle-estimate steps xr_md_filter / _main_direction / _with_estimate /
_update_estimation) against the oracle's restatement of forwardOrthByMD,
backwardOrthByMD, meanFiltFiberMD, calcMainDirection, calcMDWithEst and
updateEstimation, itself pinned bit for bit to the reference's host build
(tests/test_oracle_md.py).

Tolerance 1e-5 of the largest value for the projectors and sessions (float
sums in another order, device square roots and divisions); the per-voxel
direction steps round their sign-deciding sums as the reference does and are
compared at 1e-5 of the largest component."""
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
    md = rng.normal(0, 1, (3, N, N, N)).astype(np.float32)
    md[:, 1, 2, 3] = 0.0                 # identity rotation
    md[:2, 4, 4, 4] = 0.0                # along z
    return s, ctx, md


def _oracle_forward(oracle, s, vol, md):
    """forwardOrthByMD then correlationProjByLength per view (reconstruct.cu:1495-1507)."""
    out = np.zeros((s.C, s.V * s.Nd * s.Nd), np.float32)
    for c in range(s.C):
        for v in range(s.V):
            fac = np.zeros(s.Nd * s.Nd, np.float32)
            oracle.forward_md_view(s, c, v, vol.ravel(), md.ravel(), out[c], fac)
            oracle.correlation(s, c, v, out[c], fac)
    return out.reshape(s.C, s.V, s.Nd, s.Nd)


@pytest.mark.parametrize("axes", ["grid", "oblique"])
@pytest.mark.parametrize("K", [3, 13])
def test_forward_md(oracle, axes, K):
    rot = three_axes() if axes == "grid" else np.concatenate([oblique_rot(71, 2), three_axes()[:1]])
    s, ctx, md = _case(rot, 16, 24, 10, K, 72)
    vol = np.random.default_rng(73).uniform(0, 1, (K, 16, 16, 16)).astype(np.float32)
    dv, dm = torch.from_numpy(vol).cuda(), torch.from_numpy(md).cuda()
    out = torch.zeros((s.C, s.V, s.Nd, s.Nd), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx.dev_forward_md(dv.data_ptr(), dm.data_ptr(), out.data_ptr())
    got = out.cpu().numpy()
    ref = _oracle_forward(oracle, s, vol, md)
    assert rel_err(got, ref) <= TOL


def _oracle_session(oracle, s, sino, vol, md, epochs, batch, art, lam):
    """circleEstReconstruct's inner epochs (reconstruct.cu:1486-1543) with the
    oracle kernels, in the XTT session's subset order."""
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
                    fac = np.zeros(Nd * Nd, np.float32)
                    oracle.forward_md_view(s, c, n, vol.ravel(), md.ravel(), proj[c], fac)
                    oracle.correlation(s, c, n, proj[c], fac)
                    oracle.ratio(s, n, proj[c], sino[c].ravel(), art)
            for y in range(N):
                tmp = np.zeros(K * N * N, np.float32)
                fac = np.zeros(K * N * N, np.float32)
                for c in range(s.C):
                    for n in views:
                        oracle.backward_md_slab(s, c, y, n, proj[c], md.ravel(), tmp, fac)
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
def test_md_session(oracle, method):
    xr = load_xr()
    s, ctx, md = _case(three_axes(), 12, 20, 8, 3, 74)
    truth = fiber_phantom(s.N, 3, 75, s.basis)
    sino = _oracle_forward(oracle, s, truth, md)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.1, np.float32)
    art = method == "ART"
    lam = 1e-3
    ref = _oracle_session(oracle, s, sino, v0, md, 2, 3, art, lam)
    ctx.set_option(xr.Option.XTT_SQRT, 0)
    db, dv, dm = (torch.from_numpy(a).cuda() for a in (sino, v0, md))
    torch.cuda.synchronize()
    ctx.dev_session_begin_md(db.data_ptr(), dv.data_ptr(), dm.data_ptr(), 2, 3, method=xr.Method[method], lam=lam)
    for _ in range(2):
        ctx.dev_session_epoch()
    ctx.dev_session_end(0, 0)
    got = dv.cpu().numpy()
    print(f"md session {method}: max rel {rel_err(got, ref):.2e}")
    assert rel_err(got, ref) <= TOL


def test_md_steps(oracle):
    s, ctx, md = _case(three_axes(), 12, 20, 8, 3, 76)
    N, N3 = s.N, s.N ** 3
    rng = np.random.default_rng(77)
    vol = rng.uniform(0.1, 1.0, (3, N, N, N)).astype(np.float32)
    est = np.stack([rng.uniform(0, 2, (N, N, N)), rng.uniform(0, 3.5, (N, N, N))]).astype(np.float32)
    dv = torch.from_numpy(vol).cuda()
    # meanFiltFiberMD, two passes (border kept)
    ref = md.ravel().copy()
    for _ in range(2):
        out = ref.copy()
        for y in range(2, N - 2):
            oracle.md_filter_slab(s, y, ref, out, 1.0)
        ref = out
    dm = torch.from_numpy(md).cuda()
    tmp = torch.empty_like(dm)
    ctx.md_filter(dm.data_ptr(), tmp.data_ptr(), 1.0, 2)
    assert rel_err(dm.cpu().numpy().ravel(), ref) <= TOL
    # calcMainDirection, every sign pattern
    for it in range(4):
        ref = md.ravel().copy()
        oracle.main_direction(s, vol.ravel().copy(), ref, it)
        dm = torch.from_numpy(md).cuda()
        ctx.md_main_direction(dv.data_ptr(), dm.data_ptr(), it)
        assert rel_err(dm.cpu().numpy().ravel(), ref) <= TOL, it
    # calcMDWithEst
    ref = md.ravel().copy()
    oracle.md_with_estimate(s, vol.ravel().copy(), ref, est.ravel().copy())
    dm, de = torch.from_numpy(md).cuda(), torch.from_numpy(est).cuda()
    ctx.md_with_estimate(dv.data_ptr(), dm.data_ptr(), de.data_ptr())
    assert rel_err(dm.cpu().numpy().ravel(), ref) <= TOL
    # updateEstimation
    ref = est.ravel().copy()
    oracle.update_estimation(s, vol.ravel().copy(), ref, 2)
    ctx.md_update_estimation(dv.data_ptr(), de.data_ptr(), 2)
    assert np.array_equal(de.cpu().numpy().ravel(), ref)
    # fillVolume
    f = torch.zeros(1000, dtype=torch.float32, device="cuda")
    ctx.dev_fill(f.data_ptr(), 1000, 0.1)
    assert np.all(f.cpu().numpy() == np.float32(0.1))
