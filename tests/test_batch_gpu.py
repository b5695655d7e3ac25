"""Several uneven specimens in one batch (xr_batch_*): each specimen's result
equals its own session's, with and without the multi-specimen CUDA graph and
after the autotuner (views per CTA and forward launch shape); with BF16 storage, each specimen's error
against the FP64 oracle is stated and bounded."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_xr
from oracle import Scan
from scans import basis13, fiber_phantom, three_axes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-5
SPECIMENS = [(16, 24, 12, 31), (20, 30, 16, 32), (24, 36, 10, 33)]   # (N, Nd, V, seed)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _specimens(oracle):
    xr = load_xr()
    out = []
    for N, Nd, V, seed in SPECIMENS:
        s = Scan(sdd=1000.0, sod=500.0, det=2.0, N=N, Nd=Nd, V=V, rot=three_axes(), trans=np.zeros((3, 3)),
                 offset=np.zeros((3, 3)), basis=basis13())
        ctx = xr.Context.create(1000.0, 500.0, 2.0, N, Nd, V, s.rot, None, None, s.basis)
        truth = fiber_phantom(N, 4, seed, s.basis)
        b = oracle.forward_all(s, truth, 0, True)
        out.append((s, ctx, b))
    return out


def _alone(ctx, b, epochs, subsets):
    db = torch.from_numpy(b).cuda()
    dv = torch.full((13,) + (ctx.N,) * 3, 0.01, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx.dev_session_begin(db.data_ptr(), dv.data_ptr(), True, epochs, subsets)
    for _ in range(epochs):
        ctx.dev_session_epoch()
    ctx.dev_session_end(0, 0)
    return dv.cpu().numpy()


@pytest.mark.parametrize("graphs", [0, 1])
def test_batch_equals_individual_sessions(oracle, graphs):
    xr = load_xr()
    spec = _specimens(oracle)
    ref = [_alone(ctx, b, 4, 3) for _, ctx, b in spec]
    for _, ctx, _ in spec:
        ctx.set_option(xr.Option.GRAPHS, graphs)
    batch = xr.Batch([ctx for _, ctx, _ in spec])
    dbs = [torch.from_numpy(b).cuda() for _, _, b in spec]
    dvs = [torch.full((13,) + (ctx.N,) * 3, 0.01, dtype=torch.float32, device="cuda") for _, ctx, _ in spec]
    torch.cuda.synchronize()
    batch.session_begin([d.data_ptr() for d in dbs], [d.data_ptr() for d in dvs], True, 4, 3)
    losses = [batch.epoch() for _ in range(4)]
    batch.session_end()
    assert all(np.all(np.isfinite(l)) and np.all(l > 0) for l in losses)
    for r, dv in zip(ref, dvs):
        assert rel_err(dv.cpu().numpy(), r) <= TOL
    batch.close()


def ctx_shape(ctx, shapes, spec):
    return shapes[[c for _, c, _ in spec].index(ctx)]


def test_batch_autotune_and_bf16_error_vs_fp64(oracle):
    xr = load_xr()
    spec = _specimens(oracle)
    for _, ctx, _ in spec:
        ctx.set_option(xr.Option.STORAGE, 1)        # BF16 volumes and sinograms, stochastic rounding
        ctx.set_option(xr.Option.GRAPHS, 1)
    batch = xr.Batch([ctx for _, ctx, _ in spec])
    dbs = [torch.from_numpy(b).cuda().to(torch.bfloat16) for _, _, b in spec]
    dvs = [torch.full((13,) + (ctx.N,) * 3, 0.01, dtype=torch.bfloat16, device="cuda") for _, ctx, _ in spec]
    torch.cuda.synchronize()
    epochs, subsets = 3, 3
    batch.session_begin([d.data_ptr() for d in dbs], [d.data_ptr() for d in dvs], True, epochs, subsets)
    chosen, shapes = batch.autotune_shapes()
    assert all(v >= 0 for v in chosen)
    assert all(sh in (0, 1) for sh in shapes)   # three column axes: both launch shapes timed
    for _ in range(epochs):
        batch.epoch()
    batch.session_end()
    for (s, ctx, b), dv, vpc in zip(spec, dvs, chosen):
        v0 = np.full((13, s.N, s.N, s.N), 0.01, np.float64)
        ref64, _, _ = oracle.xtt_reconstruct(s, b.astype(np.float64), v0, epochs, subsets, dt=np.float64)
        err = rel_err(dv.float().cpu().numpy(), ref64)
        print(f"specimen N={s.N} V={s.V}: views/CTA {vpc}, axes one launch {ctx_shape(ctx, shapes, spec)}, "
              f"BF16 vs FP64 {err:.3e}")
        assert err <= 3e-2
    batch.close()
