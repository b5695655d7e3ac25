"""GPU parity: every sm_100a kernel path of libxr (called through the C ABI)
against the oracle — the FP32 restatement pinned bit-exact to the reference's
own ir.cu — on the same seeded inputs.

Tolerance (FP32): max |gpu - oracle| <= 1e-5 * max |oracle| for projections
and volumes ("max relative error <= 1e-5").  The per-voxel detector
coordinates and weights are bit-identical to the reference's; only the order
of float sums differs (the reference itself sums with float atomics in a
nondeterministic order), plus the XTT weight identity
(|B x S|^2 = |S|^2 - (B.S)^2), exact in real arithmetic.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_xr
from oracle import Scan
from scans import basis13, ellipsoid_phantom, fiber_phantom, three_axes

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def make(N, Nd, V, C=1, K=1, seed=0, shifts=True, sdd=1000.0, sod=500.0, det=2.0):
    rng = np.random.default_rng(seed)
    rot = three_axes()[:C] if C <= 3 else np.tile(np.eye(3, dtype=np.float32).ravel(), (C, 1))
    trans = rng.normal(0, 0.3, (C, 3)) if shifts else np.zeros((C, 3))
    off = rng.normal(0, 0.2, (C, 3)) if shifts else np.zeros((C, 3))
    basis = basis13()[:K] if K > 1 else np.array([[0, 0, 1.0]])
    s = Scan(sdd=sdd, sod=sod, det=det, N=N, Nd=Nd, V=V, rot=rot, trans=trans, offset=off, basis=basis)
    xr = load_xr()
    ctx = xr.Context.create(sdd, sod, det, N, Nd, V, s.rot, s.trans, s.offset, s.basis)
    return s, ctx


@pytest.mark.parametrize("axes_one_launch", [0, 1], ids=["launch_per_column_axis", "one_launch"])
@pytest.mark.parametrize("xtt", [False, True])
def test_forward_operator(oracle, xtt, axes_one_launch):
    """a1-a5: forward splat + chord-length normalisation, every axis/view; the
    three axes (column axes z, x, y) as one launch per column axis and as one
    launch for all (XR_OPT_AXES_ONE_LAUNCH)."""
    s, ctx = make(24, 36, 16, C=3, K=13 if xtt else 1, seed=1)
    ctx.set_option(load_xr().Option.AXES_ONE_LAUNCH, axes_one_launch)
    rng = np.random.default_rng(2)
    vol = rng.uniform(0, 1, (s.K if xtt else 1, s.N, s.N, s.N)).astype(np.float32)
    got = ctx.forward(vol, xtt)
    ref = oracle.forward_all(s, vol if xtt else vol[0], 0, xtt)
    assert rel_err(got, ref) <= TOL
    # Error against FP64: the reference's own FP32 arithmetic sits ~1e-4 from
    # the FP64 restatement (FP32 detector coordinates feed the weights); the
    # GPU result must sit at the same distance, not further.
    ref64 = oracle.forward_all(s, (vol if xtt else vol[0]).astype(np.float64), 0, xtt, dt=np.float64)
    e_gpu, e_ref = rel_err(got, ref64), rel_err(ref, ref64)
    print(f"forward xtt={xtt}: gpu vs FP64 {e_gpu:.3e}, reference FP32 vs FP64 {e_ref:.3e}")
    assert e_gpu <= e_ref + TOL


def test_forward_proj_only(oracle):
    """forwardProjOnly (reconstruct.cu:1890-1949): raw splat, no normaliser."""
    s, ctx = make(20, 28, 10, C=2, seed=3)
    vol = np.random.default_rng(4).uniform(0, 1, (s.N, s.N, s.N)).astype(np.float32)
    got = ctx.forward_proj_only(vol)
    ref = np.zeros((s.C, s.V * s.Nd * s.Nd), np.float32)
    f = np.zeros(s.Nd * s.Nd, np.float32)
    for c in range(s.C):
        for v in range(s.V):
            oracle.forward_view(s, c, v, vol.ravel(), ref[c], f, 0)
    assert rel_err(got.reshape(s.C, -1), ref) <= TOL


def test_forward_large_footprint_fallback(oracle):
    """Bricks whose footprint exceeds the 64 x 64 shared tile (source 50 mm from
    the centre of a 64^3 volume: 15 of 1536 brick-views, up to 7826 pixels)
    take the global-atomic path."""
    s, ctx = make(64, 160, 12, C=1, seed=5, sod=50.0, sdd=100.0, det=2.0)
    vol = np.random.default_rng(6).uniform(0, 1, (1, s.N, s.N, s.N)).astype(np.float32)
    got = ctx.forward(vol, False)
    ref = oracle.forward_all(s, vol[0], 0, False)
    assert rel_err(got, ref) <= TOL


@pytest.mark.parametrize("ratio_texture", [1, 0], ids=["texture_gather", "linear_loads"])
@pytest.mark.parametrize("method", ["MLEM", "ART"])
def test_ir_reconstruct_small(oracle, method, ratio_texture):
    """a6, a7, a9, a11: IR::reconstruct, 2 axes reconstructed independently,
    V % batch != 0 (the subset wrap-around revisits views); the back-projection
    gathering its taps from the layered ratio texture or loading them."""
    xr = load_xr()
    s, ctx = make(24, 36, 14, C=2, seed=7)
    ctx.set_option(xr.Option.RATIO_TEXTURE, ratio_texture)
    truth = ellipsoid_phantom(s.N, 5, 8)
    b = oracle.forward_all(s, truth, 0, False)
    v0 = np.ones((s.C, s.N, s.N, s.N), np.float32)
    art = method == "ART"
    got, gl = ctx.ir_reconstruct(b, v0, 3, 4, xr.Rotate.CW, xr.Method[method], 1e-2)
    ref, rl = oracle.ir_reconstruct(s, b, v0, 3, 4, art=art, lam=1e-2)
    assert rel_err(got, ref) <= TOL
    assert np.allclose(gl, rl, rtol=1e-4)


@pytest.mark.parametrize("variant", [(0, 1), (1, 1), (1, 0)],
                         ids=["launch_per_column_axis", "one_launch", "one_launch_linear_ratio_loads"])
@pytest.mark.parametrize("method", ["MLEM", "ART"])
def test_xtt_reconstruct_small(oracle, method, variant):
    """a4, a8, a9, a10, a11: XTT::reconstruct, 3 axes, K = 13, sqrt at the end;
    the returned ratio images are the reference's last ratio images.  The
    forward as one launch per column axis or one for all axes
    (XR_OPT_AXES_ONE_LAUNCH); the back-projection gathering its taps from the
    layered ratio texture or loading them from the linear images
    (XR_OPT_RATIO_TEXTURE)."""
    xr = load_xr()
    s, ctx = make(16, 24, 12, C=3, K=13, seed=9)
    ctx.set_option(xr.Option.AXES_ONE_LAUNCH, variant[0])
    ctx.set_option(xr.Option.RATIO_TEXTURE, variant[1])
    truth = fiber_phantom(s.N, 4, 10, s.basis)
    b = oracle.forward_all(s, truth, 0, True)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    art = method == "ART"
    mu, ratio, md, ev, gl = ctx.xtt_reconstruct(b, v0, 2, 5, xr.Rotate.CW, xr.Method[method], 1e-3)
    ref, rproj, rl = oracle.xtt_reconstruct(s, b, v0, 2, 5, art=art, lam=1e-3)
    assert rel_err(mu, ref) <= TOL
    assert rel_err(ratio, rproj) <= TOL
    assert np.allclose(gl, rl, rtol=1e-4)
    omd, oev = oracle.orientation(s.basis, ref)
    mask = np.abs(oev[1] - oev[0]) > 1e-3 * np.abs(oev).max()   # non-degenerate smallest eigenvalue
    assert np.allclose(md[:, mask], omd[:, mask], atol=1e-4 * np.abs(omd).max())


def test_c1_plain_mlem_64(oracle):
    """The plain cone-beam MLEM workload: 64^3, 8 ellipsoids (seed 1), 90
    views over 360 degrees, 96x96 detector, SOD 500 / SDD 1000 / 1 mm voxels,
    noiseless projections from the voxel-driven projector, 20 MLEM
    iterations from 1.0; result within 1e-5 of the reference's."""
    xr = load_xr()
    s, ctx = make(64, 96, 90, C=1, seed=0, shifts=False)
    truth = ellipsoid_phantom(64, 8, 1)
    b = oracle.forward_all(s, truth, 0, False)
    v0 = np.ones((1, 64, 64, 64), np.float32)
    got, gl = ctx.ir_reconstruct(b, v0, 20, 1, xr.Rotate.CW, xr.Method.MLEM, 1e-2)
    ref, rl = oracle.ir_reconstruct(s, b, v0, 20, 1, art=False)
    err = rel_err(got, ref)
    m = np.abs(ref) > 1e-3 * np.abs(ref).max()
    elem = float((np.abs(got - ref)[m] / np.abs(ref)[m]).max())
    print(f"C1 MLEM: max|d|/max|ref| = {err:.3e}, masked elementwise max rel = {elem:.3e}")
    assert err <= TOL
    # The reference sums |b - p| of 90 x 96^2 pixels into ONE float
    # (ir.cu:1623), which loses ~1e-3 of the total; libxr sums in FP64.
    assert np.allclose(gl, rl, rtol=2e-3)


@pytest.mark.parametrize("filt", ["REFERENCE", "RAMLAK"])
def test_fdk(oracle, filt):
    """a13: FDK weight + row convolution + weighted back-projection."""
    xr = load_xr()
    s, ctx = make(24, 40, 24, C=1, seed=11)
    truth = ellipsoid_phantom(s.N, 5, 12)
    b = oracle.forward_all(s, truth, 0, False)
    got, gf = ctx.fdk_reconstruct(b, xr.Rotate.CW, xr.Filter[filt])
    ref, rf = oracle.fdk_reconstruct(s, b, 0, ramlak=filt == "RAMLAK", block0=True)
    assert rel_err(gf, rf) <= TOL
    assert rel_err(got, ref) <= TOL


def test_fdk_axis_blocks(oracle):
    """The reference back-projects axis 0's filtered block for every axis
    (reconstruct.cu:1708); XR_OPT_FDK_AXIS_BLOCKS=1 uses each axis's own."""
    xr = load_xr()
    s, ctx = make(16, 28, 12, C=2, seed=13)
    b = np.random.default_rng(14).uniform(0, 1, (s.C, s.V, s.Nd, s.Nd)).astype(np.float32)
    got, _ = ctx.fdk_reconstruct(b)
    ref, _ = oracle.fdk_reconstruct(s, b, 0, block0=True)
    assert rel_err(got, ref) <= TOL
    ctx.set_option(xr.Option.FDK_AXIS_BLOCKS, 1)
    got2, _ = ctx.fdk_reconstruct(b)
    ref2, _ = oracle.fdk_reconstruct(s, b, 0, block0=False)
    assert rel_err(got2, ref2) <= TOL


def test_fdk_every_column_axis_and_oblique(oracle):
    """FDK back-projection on axes rotating about z, x and y (the column form
    for each column axis, y as the column axis included, where the
    (sod / (sod + o_y))^2 weight varies along the column) and one oblique
    axis (the per-voxel form), each axis with its own filtered block."""
    from scans import oblique_rot
    xr = load_xr()
    rng = np.random.default_rng(17)
    rot = np.concatenate([three_axes(), oblique_rot(18, 1)])
    C = rot.shape[0]
    s = Scan(sdd=1000.0, sod=500.0, det=2.0, N=20, Nd=32, V=16, rot=rot, trans=rng.normal(0, 0.3, (C, 3)),
             offset=rng.normal(0, 0.2, (C, 3)), basis=np.array([[0, 0, 1.0]]))
    ctx = xr.Context.create(s.sdd, s.sod, s.det, s.N, s.Nd, s.V, s.rot, s.trans, s.offset, s.basis)
    ctx.set_option(xr.Option.FDK_AXIS_BLOCKS, 1)
    b = rng.uniform(0, 1, (C, s.V, s.Nd, s.Nd)).astype(np.float32)
    ref, rf = oracle.fdk_reconstruct(s, b, 0, block0=False)
    vols = []
    for tex in (1, 0):   # taps gathered from the layered texture, or loaded
        ctx.set_option(xr.Option.RATIO_TEXTURE, tex)
        got, gf = ctx.fdk_reconstruct(b)
        assert rel_err(gf, rf) <= TOL
        for c in range(C):
            assert rel_err(got[c], ref[c]) <= TOL, (tex, c)
        vols.append(got)
    assert np.array_equal(vols[0], vols[1])   # the same taps, the same sums
    ctx.close()


def test_orientation(oracle):
    """a12: per-voxel FP64 eigen step vs the oracle (FP64 Jacobi)."""
    s, ctx = make(12, 16, 4, C=1, K=13, seed=15)
    mu = np.random.default_rng(16).uniform(0, 1, (13, 12, 12, 12)).astype(np.float32)
    mu[:, 0, 0, :] = 0.0                                  # empty voxels
    md, ev = ctx.orientation(mu)
    omd, oev = oracle.orientation(s.basis, mu)
    assert np.allclose(md, omd, atol=1e-5)
    ok = np.isfinite(oev)
    assert np.allclose(ev[ok], oev[ok], atol=1e-5)


def test_angle_and_normalization(oracle):
    """calcAngleFromMD / directionNormalization (pca.cu:67-106) against the
    oracle, itself pinned bit for bit to the reference's pca.cu
    (tests/test_oracle_fdk.py): the normalisation bit for bit (lengths and
    quotients rounded op by op, so the 0.65 threshold decides alike); the
    angles within 4e-7 rad (the device atan2f against glibc's, a few ulp)."""
    s, ctx = make(8, 12, 4, seed=17)
    md = np.random.default_rng(18).normal(0, 0.6, (3, 8, 8, 8)).astype(np.float32)
    md[:, 0, 0, :3] = 0.0
    ang = ctx.angle_from_md(md)
    ref = oracle.angle_from_md(md)
    assert np.abs(ang.astype(np.float64) - ref).max() <= 4e-7
    nm = ctx.direction_normalization(md)
    assert np.array_equal(nm, oracle.direction_normalization(md))


def test_residual_fp64(oracle):
    s, ctx = make(20, 28, 10, C=2, K=13, seed=19)
    rng = np.random.default_rng(20)
    vol = rng.uniform(0, 1, (13, 20, 20, 20)).astype(np.float32)
    b = oracle.forward_all(s, vol, 0, True) * np.float32(1.01)
    r, l1 = ctx.residual(vol, b, True)
    # FP64 sums over the FP32 operator A (the reference's arithmetic)
    p = oracle.forward_all(s, vol, 0, True).astype(np.float64)
    rr = np.sqrt(((p - b) ** 2).sum() / (b.astype(np.float64) ** 2).sum())
    assert abs(r - rr) <= 1e-5 * rr
    assert abs(l1 - np.abs(p - b).sum()) <= 1e-5 * l1


def test_session_api_matches_host_call(oracle):
    """The device-buffer session (begin / epoch / end) drives the same XTT
    path as xr_xtt_reconstruct."""
    torch = pytest.importorskip("torch")
    xr = load_xr()
    s, ctx = make(16, 24, 12, C=3, K=13, seed=21)
    truth = fiber_phantom(s.N, 3, 22, s.basis)
    b = oracle.forward_all(s, truth, 0, True)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    mu_h, _, md_h, _, _ = ctx.xtt_reconstruct(b, v0, 2, 3)
    db = torch.from_numpy(b).cuda()
    dv = torch.from_numpy(v0).cuda()
    dmd = torch.zeros((3, s.N, s.N, s.N), device="cuda")
    torch.cuda.synchronize()
    ctx.dev_session_begin(db.data_ptr(), dv.data_ptr(), True, 2, 3)
    for _ in range(2):
        ctx.dev_session_epoch()
    ctx.dev_session_end(dmd.data_ptr(), 0)
    assert rel_err(dv.cpu().numpy(), mu_h) <= TOL
    assert rel_err(dmd.cpu().numpy(), md_h) <= 1e-4


def test_host_call_slab_tail_matches_session(oracle):
    """xr_xtt_reconstruct back-projects its last subset in z-slabs, each slab
    then voxelSqrt'ed, its orientation computed and its planes downloaded while
    the next slab runs.  At N = 70 (9 brick rows of 8: 5 slabs, the last
    ragged) the volume, the main directions and the eigenvalues equal the
    device session's, which applies voxelSqrt and the orientation to the
    whole volume at its end."""
    torch = pytest.importorskip("torch")
    xr = load_xr()
    s, ctx = make(70, 96, 10, C=3, K=13, seed=23)
    truth = np.random.default_rng(24).uniform(0, 1, (s.K, s.N, s.N, s.N)).astype(np.float32)
    db = torch.from_numpy(truth).cuda()
    b = torch.empty((s.C, s.V, s.Nd, s.Nd), dtype=torch.float32, device="cuda")
    ctx.dev_forward(db.data_ptr(), b.data_ptr(), True)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    mu_h, _, md_h, ev_h, _ = ctx.xtt_reconstruct(b.cpu().numpy(), v0, 1, 2)
    dv = torch.from_numpy(v0).cuda()
    dmd = torch.zeros((3, s.N, s.N, s.N), device="cuda")
    dev = torch.zeros((3, s.N, s.N, s.N), device="cuda")
    torch.cuda.synchronize()
    ctx.dev_session_begin(b.data_ptr(), dv.data_ptr(), True, 1, 2)
    ctx.dev_session_epoch()
    ctx.dev_session_end(dmd.data_ptr(), dev.data_ptr())
    md_d, ev_d = dmd.cpu().numpy(), dev.cpu().numpy()
    assert rel_err(mu_h, dv.cpu().numpy()) <= TOL
    assert rel_err(ev_h, ev_d) <= 1e-4
    mask = np.abs(ev_d[1] - ev_d[0]) > 1e-3 * np.abs(ev_d).max()   # non-degenerate smallest eigenvalue
    assert mask.sum() > 0
    assert np.allclose(md_h[:, mask], md_d[:, mask], atol=1e-4 * np.abs(md_d).max())
    ctx.close()


def test_art_zero_step_is_identity(oracle):
    """ART with lambda = 0 (voxelPlus, ir.cu:1682-1693) leaves mu bit-for-bit
    unchanged whatever the residual images hold."""
    xr = load_xr()
    s, ctx = make(16, 24, 12, C=1, seed=23)
    b = np.random.default_rng(24).uniform(0, 1, (1, s.V, s.Nd, s.Nd)).astype(np.float32)
    v0 = np.random.default_rng(25).uniform(0, 1, (1, 16, 16, 16)).astype(np.float32)
    a, _ = ctx.ir_reconstruct(b, v0, 1, 2, xr.Rotate.CW, xr.Method.ART, 0.0)
    assert np.array_equal(a, v0)


def test_errors_on_device():
    xr = load_xr()
    rot = np.eye(3, dtype=np.float32).ravel()
    b20 = np.tile(basis13(), (2, 1))[:20]
    ctx = xr.Context.create(1000, 500, 2, 8, 12, 4, rot, basis=b20)
    with pytest.raises(xr.XRError) as e:                       # K > 16 on the XTT path
        ctx.forward(np.ones((20, 8, 8, 8), np.float32), xtt=True)
    assert e.value.status == 1
    ctx2 = xr.Context.create(1000, 500, 2, 8, 12, 4, rot)
    with pytest.raises(xr.XRError):                            # batch > V
        ctx2.ir_reconstruct(np.zeros((1, 4, 12, 12)), np.ones((1, 8, 8, 8)), 1, 5)


def _oblique_rot(seed, n):
    """Rotation matrices in general position (not grid-aligned), like the
    reference's measured presets (settings.json "matrixRot")."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, c, d = q
        out.append([a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c),
                    2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b),
                    2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d])
    return np.array(out, np.float32)


def _make_rot(rot, N, Nd, V, K, seed, sdd=1000.0, sod=500.0, det=2.0):
    rng = np.random.default_rng(seed)
    C = rot.shape[0]
    basis = basis13()[:K] if K > 1 else np.array([[0, 0, 1.0]])
    s = Scan(sdd=sdd, sod=sod, det=det, N=N, Nd=Nd, V=V, rot=rot, trans=rng.normal(0, 0.3, (C, 3)),
             offset=rng.normal(0, 0.2, (C, 3)), basis=basis)
    xr = load_xr()
    ctx = xr.Context.create(sdd, sod, det, N, Nd, V, s.rot, s.trans, s.offset, s.basis)
    return s, ctx


@pytest.mark.parametrize("xtt", [False, True])
def test_forward_oblique_axes_odd_pitch(oracle, xtt):
    """General (non grid-aligned) rotation axes take the general kernels; a
    detector pitch that is not a power of two exercises the verified exact
    division by the pitch (the reference's oilpan preset: 0.0581777777 mm)."""
    rot = np.concatenate([_oblique_rot(41, 2), three_axes()[:1]])
    s, ctx = _make_rot(rot, 20, 30, 12, 13 if xtt else 1, 42, sdd=1819.6, sod=1316.5, det=0.0581777777)
    vol = np.random.default_rng(43).uniform(0, 1, (s.K if xtt else 1, s.N, s.N, s.N)).astype(np.float32)
    got = ctx.forward(vol, xtt)
    ref = oracle.forward_all(s, vol if xtt else vol[0], 0, xtt)
    assert rel_err(got, ref) <= TOL


@pytest.mark.parametrize("method", ["MLEM", "ART"])
def test_xtt_mixed_axes(oracle, method):
    """XTT with one grid-aligned and one oblique axis: column forward for the
    first, general kernels for the rest of the path."""
    xr = load_xr()
    rot = np.concatenate([three_axes()[:1], _oblique_rot(44, 1)])
    s, ctx = _make_rot(rot, 16, 24, 10, 13, 45)
    truth = fiber_phantom(s.N, 3, 46, s.basis)
    b = oracle.forward_all(s, truth, 0, True)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    mu, ratio, _, _, gl = ctx.xtt_reconstruct(b, v0, 2, 3, xr.Rotate.CW, xr.Method[method], 1e-3)
    ref, rproj, rl = oracle.xtt_reconstruct(s, b, v0, 2, 3, art=method == "ART", lam=1e-3)
    assert rel_err(mu, ref) <= TOL
    assert rel_err(ratio, rproj) <= TOL


def test_ir_oblique_axis_odd_pitch(oracle):
    xr = load_xr()
    s, ctx = _make_rot(_oblique_rot(47, 1), 20, 30, 12, 1, 48, sdd=1819.6, sod=1316.5, det=0.0581777777)
    truth = ellipsoid_phantom(s.N, 4, 49)
    b = oracle.forward_all(s, truth, 0, False)
    v0 = np.ones((1, s.N, s.N, s.N), np.float32)
    got, _ = ctx.ir_reconstruct(b, v0, 2, 3)
    ref, _ = oracle.ir_reconstruct(s, b, v0, 2, 3)
    assert rel_err(got, ref) <= TOL


def test_ccw_rotation(oracle):
    """Rotate::CCW (n = -view): the reference indexes correlationProjByLength
    with the signed n, which writes before the buffer; the restatement and
    libxr both use |n| and agree."""
    xr = load_xr()
    s, ctx = make(16, 24, 10, C=2, seed=50)
    vol = np.random.default_rng(51).uniform(0, 1, (s.N, s.N, s.N)).astype(np.float32)
    got = ctx.forward(vol[None], False, xr.Rotate.CCW)
    ref = oracle.forward_all(s, vol, 1, False)
    assert rel_err(got, ref) <= TOL


def _bf16_round(a):
    """Round float32 to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("storage", [1, 2])
def test_storage_forward_is_rounded_input(oracle, storage):
    """16-bit storage only rounds the stored volume: the forward of a BF16 /
    FP16 volume equals the FP32 forward of the rounded volume."""
    xr = load_xr()
    s, ctx = make(20, 30, 10, C=3, K=13, seed=60)
    vol = np.random.default_rng(61).uniform(0, 1, (13, 20, 20, 20)).astype(np.float32)
    ctx.set_option(xr.Option.STORAGE, storage)
    got = ctx.forward(vol, True)
    rounded = _bf16_round(vol) if storage == 1 else vol.astype(np.float16).astype(np.float32)
    ref = oracle.forward_all(s, rounded, 0, True)
    assert rel_err(got, ref) <= TOL


@pytest.mark.parametrize("storage,bound", [(0, 1e-3), (1, 3e-2), (2, 5e-3)])
def test_storage_xtt_error_vs_fp64(oracle, storage, bound):
    """XTT OS-EM with FP32 / BF16 / FP16 storage of volume and sinogram (FP32
    arithmetic): the error of each against the FP64 oracle is stated and
    bounded (max |d| / max |ref| over the reconstructed coefficients)."""
    xr = load_xr()
    s, ctx = make(16, 24, 12, C=3, K=13, seed=62, shifts=False)
    truth = fiber_phantom(s.N, 4, 63, s.basis)
    b = oracle.forward_all(s, truth, 0, True)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    ctx.set_option(xr.Option.STORAGE, storage)
    mu, _, _, _, _ = ctx.xtt_reconstruct(b, v0, 3, 3, orientation=False)
    ref64, _, _ = oracle.xtt_reconstruct(s, b.astype(np.float64), v0.astype(np.float64), 3, 3, dt=np.float64)
    err = rel_err(mu, ref64)
    print(f"XTT storage={['f32', 'bf16', 'f16'][storage]}: max|d|/max|ref| vs FP64 = {err:.3e}")
    assert err <= bound


@pytest.mark.parametrize("xtt", [True, False])
def test_graph_epochs_match_direct(oracle, xtt):
    """XR_OPT_GRAPHS: epochs replayed from CUDA graphs (one per subset order)
    give the same reconstruction as directly launched epochs."""
    torch = pytest.importorskip("torch")
    xr = load_xr()
    s, ctx = make(16, 24, 12, C=3, K=13 if xtt else 1, seed=70)
    if xtt:
        truth = fiber_phantom(s.N, 3, 71, s.basis)
        v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    else:
        truth = ellipsoid_phantom(s.N, 4, 71)
        v0 = np.ones((s.C, s.N, s.N, s.N), np.float32)
    b = oracle.forward_all(s, truth, 0, xtt)
    outs = []
    for graphs in (0, 1):
        ctx.set_option(xr.Option.GRAPHS, graphs)
        db = torch.from_numpy(b).cuda()
        dv = torch.from_numpy(v0).cuda()
        torch.cuda.synchronize()
        ctx.dev_session_begin(db.data_ptr(), dv.data_ptr(), xtt, 4, 3)
        for _ in range(4):
            ctx.dev_session_epoch()
        ctx.dev_session_end(0, 0)
        outs.append(dv.cpu().numpy())
    assert rel_err(outs[1], outs[0]) <= TOL


def test_bf16_stochastic_rounding_is_unbiased(oracle):
    """BF16 volumes with FP32 data and XTT ART steps far below half a BF16
    unit (relative 2^-9): nearest rounding drops the updates (the iteration
    stalls: almost no voxel changes), stochastic rounding (the default,
    XR_OPT_ROUNDING = 1) applies them in expectation: regressed on the FP32
    updates, its updates have slope 1, directly launched or replayed from a
    CUDA graph.  (The draw hashes the FP32 value, whose last bits vary with
    the order of the forward's float atomics, so runs agree statistically,
    not bit for bit.)"""
    torch = pytest.importorskip("torch")
    xr = load_xr()
    s, ctx = make(24, 36, 12, C=3, K=13, seed=80, shifts=False)
    truth = fiber_phantom(s.N, 5, 81, s.basis)
    db = torch.from_numpy(oracle.forward_all(s, truth, 0, True)).cuda()
    mu0 = np.random.default_rng(82).uniform(0.25, 0.75, (s.K, s.N, s.N, s.N)).astype(np.float32)
    mu0 = torch.from_numpy(mu0).to(torch.bfloat16).float().numpy()          # exactly representable

    def run(storage, rounding, graphs, lam):
        ctx.set_option(xr.Option.STORAGE, storage)
        ctx.set_option(xr.Option.SINO_STORAGE, 0)
        ctx.set_option(xr.Option.ROUNDING, rounding)
        ctx.set_option(xr.Option.GRAPHS, graphs)
        ctx.set_option(xr.Option.XTT_SQRT, 0)  # keep the iterate (no final voxelSqrt)
        dv = torch.from_numpy(mu0).cuda().to(torch.float32 if storage == 0 else torch.bfloat16)
        torch.cuda.synchronize()
        ctx.dev_session_begin(db.data_ptr(), dv.data_ptr(), True, 1, 2, method=xr.Method.ART, lam=lam)
        ctx.dev_session_epoch()
        ctx.dev_session_end(0, 0)
        return dv.float().cpu().numpy().astype(np.float64) - mu0

    probe = run(0, 1, 0, 1e-2)
    lam = 1e-2 * 2e-4 / np.median(np.abs(probe) / mu0)                   # median step 2e-4 of the value
    d32 = run(0, 1, 0, lam)
    d_near = run(1, 0, 0, lam)
    d_sr = run(1, 1, 0, lam)
    d_sr_g = run(1, 1, 1, lam)
    ctx.set_option(xr.Option.GRAPHS, 0)
    slope = lambda d: float((d * d32).sum() / (d32 * d32).sum())
    changed = lambda d: float((np.abs(d) > 1e-6 * mu0).mean())
    print(f"lambda {lam:.3e}: slope nearest {slope(d_near):.3f} (changed {changed(d_near):.3f}), "
          f"stochastic {slope(d_sr):.3f} (changed {changed(d_sr):.3f})")
    assert abs(slope(d_sr) - 1.0) <= 0.15
    assert abs(slope(d_sr_g) - 1.0) <= 0.15
    assert abs(slope(d_near)) <= 0.3
