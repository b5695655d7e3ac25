"""GPU parity at the configured sizes of the XTT kernels the bench times.

* XTT plain (128^3 volume, K = 13, 3 sample-rotation axes x 120 views,
  192^2 detector, 12 seeded fiber cylinders): the normalised forward
  operator (forwardProjXTT + correlationProjByLength, ir.cu:1533-1603,
  1753-1804) and one whole XTT::reconstruct epoch (MLEM, 5 subsets,
  reconstruct.cu:799-927, voxelSqrt at the end) through the host-buffer entry
  point, against the oracle.  At this size the column kernels run many bricks
  per axis, view chunks of the automatic size and the CTA's fixed-point tile
  shift over a real phantom's dynamic range.  The oracle runs its (axis, view)
  pairs and y slabs in parallel, bit-identical to its serial order.
* Bricks whose footprint overflows the shared detector tile at a larger N
  (strong magnification), XTT, against the oracle.
* The full XTT size (256^3 x 13, 3 x 180 views, 384^2 detector), where the
  oracle would take too long: properties that hold to float summation order.
  Linearity of the forward operator, A(x + 2y) = A(x) + 2 A(y); and the
  adjoint pair of the un-normalised XTT forward splat F and the XTT
  back-projection B (ir.cu:1807-1850):
  <N (.) F x, r> = vs * ratio * sum_k <x_k, B_k(N (.) r)>, with N the
  per-pixel chord normaliser (so A = N (.) F); B comes from one OS-ART epoch
  with one subset (step 1) from mu = 0, where the update is mu = B(b).

Tolerance: max |gpu - oracle| <= 1e-5 * max |oracle| (the projector bar of the
other parity tests); inner products and linearity to 1e-5 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_xr
from oracle import Scan
from scans import basis13, fiber_phantom, three_axes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-5


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _xtt_case(N, Nd, V, **geom):
    sdd, sod, det = geom.get("sdd", 1000.0), geom.get("sod", 500.0), geom.get("det", 2.0)
    s = Scan(sdd=sdd, sod=sod, det=det, N=N, Nd=Nd, V=V, rot=three_axes(), trans=np.zeros((3, 3)),
             offset=np.zeros((3, 3)), basis=basis13())
    ctx = load_xr().Context.create(sdd, sod, det, N, Nd, V, s.rot, s.trans, s.offset, s.basis)
    return s, ctx


@pytest.fixture(scope="module")
def c3(oracle):
    """The XTT plain configuration, its phantom and b = A mu_true (oracle)."""
    s, ctx = _xtt_case(128, 192, 120)
    truth = fiber_phantom(128, 12, 3, s.basis)
    b = oracle.forward_all(s, truth, 0, True)
    yield s, ctx, truth, b
    ctx.close()


def test_c3_xtt_forward_operator(c3):
    s, ctx, truth, b = c3
    got = ctx.forward(truth, True)
    assert np.abs(b).max() > 0
    err = rel_err(got, b)
    print(f"XTT forward 128^3 x 13, 3 x 120 views, 192^2: max rel {err:.2e}")
    assert err <= TOL


def test_c3_xtt_epoch(c3, oracle):
    """One XTT::reconstruct epoch (MLEM, 5 subsets) from mu = 0.01 through
    xr_xtt_reconstruct; volume after voxelSqrt, last ratio images, loss."""
    xr = load_xr()
    s, ctx, truth, b = c3
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    mu, ratio, md, ev, gl = ctx.xtt_reconstruct(b, v0, 1, 5, xr.Rotate.CW, xr.Method.MLEM, 1e-2,
                                                orientation=False)
    ref, rproj, rl = oracle.xtt_reconstruct(s, b, v0, 1, 5)
    e_mu, e_ratio = rel_err(mu, ref), rel_err(ratio, rproj)
    print(f"XTT epoch 128^3 x 13: volume max rel {e_mu:.2e}, ratio images {e_ratio:.2e}, "
          f"loss {gl[0]:.6e} vs {rl[0]:.6e}")
    assert e_mu <= TOL
    assert e_ratio <= TOL
    # The FP32 oracle adds the 13.3 M terms |b - p| into one float, as the
    # reference's single loss accumulator does (ir.cu:1623): at ~5e7 that sum
    # drops every term below half an ulp (2) and ends ~2 % low.  libxr sums
    # in FP64, so its loss is compared with the FP64 oracle's.
    _, _, rl64 = oracle.xtt_reconstruct(s, b.astype(np.float64), v0.astype(np.float64), 1, 5, dt=np.float64)
    print(f"loss: libxr {gl[0]:.9e}, FP64 oracle {rl64[0]:.9e}, FP32 oracle {rl[0]:.9e}")
    assert np.allclose(gl, rl64, rtol=1e-4)


def test_xtt_tile_overflow_large_n(oracle):
    """Source 50 mm from the centre of a 64^3 volume (SDD 100, vs 1 mm): the
    bricks that pass near the source have footprints beyond the 64 x 64 shared
    tile (15 of 1536 brick-views, up to 7826 pixels) and take the
    global-atomic path, beside bricks that fit."""
    s, ctx = _xtt_case(64, 160, 12, sdd=100.0, sod=50.0, det=2.0)
    vol = np.random.default_rng(41).uniform(0, 1, (s.K, s.N, s.N, s.N)).astype(np.float32)
    got = ctx.forward(vol, True)
    ref = oracle.forward_all(s, vol, 0, True)
    err = rel_err(got, ref)
    print(f"XTT forward, tile overflow at 64^3: max rel {err:.2e}")
    assert err <= TOL
    ctx.close()


@pytest.fixture(scope="module")
def c5():
    """The full XTT size on the device, FP32: N 256, K 13, 3 x 180, 384^2."""
    s, ctx = _xtt_case(256, 384, 180)
    yield s, ctx
    ctx.close()
    torch.cuda.empty_cache()


def _forward(ctx, s, vol):
    out = torch.empty((s.C, s.V, s.Nd, s.Nd), dtype=torch.float32, device="cuda")
    ctx.dev_forward(vol.data_ptr(), out.data_ptr(), True)
    torch.cuda.synchronize()
    return out


def test_c5_forward_linearity(c5):
    s, ctx = c5
    g = torch.Generator(device="cuda").manual_seed(51)
    shape = (s.K, s.N, s.N, s.N)
    x = torch.rand(shape, generator=g, device="cuda")
    y = torch.rand(shape, generator=g, device="cuda")
    ax, ay = _forward(ctx, s, x), _forward(ctx, s, y)
    axy = _forward(ctx, s, x + 2 * y)
    lhs, rhs = axy.double(), ax.double() + 2 * ay.double()
    err = float((lhs - rhs).abs().max() / lhs.abs().max())
    print(f"XTT forward 256^3 x 13 linearity: max rel {err:.2e}")
    assert float(lhs.abs().max()) > 0
    assert err <= TOL


def test_c5_forward_back_adjoint(c5):
    xr = load_xr()
    s, ctx = c5
    g = torch.Generator(device="cuda").manual_seed(52)
    x = torch.rand((s.K, s.N, s.N, s.N), generator=g, device="cuda")
    r = torch.rand((s.C, s.V, s.Nd, s.Nd), generator=g, device="cuda") + 0.5
    ax = _forward(ctx, s, x)                                        # N (.) F x
    # the normaliser N: normalised over raw plain splat of a volume of ones
    ones = np.ones((s.N, s.N, s.N), np.float32)
    raw = torch.from_numpy(ctx.forward_proj_only(ones)).cuda()     # ratio * (sum of weights)
    nrm_plain = torch.empty_like(raw)
    d_ones = torch.from_numpy(ones).cuda()
    ctx.dev_forward(d_ones.data_ptr(), nrm_plain.data_ptr(), False)
    torch.cuda.synchronize()
    norm = torch.where(raw > 0, nrm_plain / raw.clamp_min(1e-30), torch.zeros_like(raw))
    del raw, nrm_plain, d_ones
    b = (norm * r).contiguous()
    # B(b): one OS-ART epoch, one subset (subsetSize = V, lambda = V: step 1)
    # from mu = 0; the forward of mu = 0 is 0, so the ratio step passes b
    mu = torch.zeros((s.K, s.N, s.N, s.N), dtype=torch.float32, device="cuda")
    ctx.set_option(xr.Option.XTT_SQRT, 0)
    ctx.dev_session_begin(b.data_ptr(), mu.data_ptr(), True, 1, 1, method=xr.Method.ART, lam=float(s.V))
    ctx.dev_session_epoch()
    ctx.dev_session_end(0, 0)
    ctx.set_option(xr.Option.XTT_SQRT, 1)
    torch.cuda.synchronize()
    scale = ctx.vs * 1.0          # vs * ratio; ratio = vs^2 / (det * sod / sdd)^2 = 1 here
    lhs = float((ax.double() * r.double()).sum())
    rhs = scale * float((x.double() * mu.double()).sum())
    err = abs(lhs - rhs) / abs(lhs)
    print(f"XTT 256^3 x 13 adjoint pair: <A x, r> {lhs:.9e}, <x, B(N r)> {rhs:.9e}, rel {err:.2e}")
    assert lhs > 0
    assert err <= TOL
