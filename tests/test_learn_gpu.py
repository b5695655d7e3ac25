"""Tensor-core convolutions and the warm-start network on the GPU against the
CPU oracle (oracle/warmstart.py) on the same BF16 inputs.

Tolerances: fprop/dgrad outputs are stored in BF16 (8 significant bits), so
|gpu - oracle| <= 2^-7 |oracle| + 2^-7 * 1e-2 max|oracle| (one BF16 rounding
step either way of a value near a rounding boundary); wgrad and the loss are
FP32 sums of exact BF16 products: relative 1e-4.  Network gradients pass
through four BF16 roundings of activations and gradients; a value rounded
the other way changes its neighbours, so they are compared by relative L2
error <= 2e-2 and cosine >= 0.999.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import load_xr

import warmstart as ws

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev_bf16(a: np.ndarray):
    """float array -> torch int16 tensor holding BF16 bits, and the rounded values (float64)."""
    bits = ws.bf16_bits(a)
    return torch.from_numpy(bits.view(np.int16).copy()).cuda(), ws.bf16(a)


def _from_bf16(t) -> np.ndarray:
    u = t.cpu().numpy().view(np.uint16).astype(np.uint32) << 16
    return u.view(np.float32).astype(np.float64)


def _close_bf16(got, ref):
    m = np.abs(ref).max()
    err = np.abs(got - ref)
    ok = err <= 2.0 ** -7 * np.abs(ref) + 2.0 ** -7 * 1e-2 * m
    assert ok.mean() > 0.999, (err.max(), m)
    assert err.max() <= 2.0 ** -6 * m


SHAPES = [(9, 7, 13), (20, 36, 40)]   # (nz, ny, nx): 819 voxels (a partial tile); 28 800 (persistent loop)


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 16), (32, 32)])
@pytest.mark.parametrize("shape", SHAPES)
def test_conv_fprop_epilogues(cin, cout, shape):
    xr = load_xr()
    rng = np.random.default_rng(cin * 100 + cout + shape[2])
    x = rng.normal(size=shape + (cin,)).astype(np.float32)
    w = (rng.normal(size=(27, cout, cin)) * 0.1).astype(np.float32)
    b = rng.normal(size=cout).astype(np.float32)
    mask = rng.normal(size=shape + (cout,)).astype(np.float32)
    dx, xv = _dev_bf16(x)
    dw, wv = _dev_bf16(w)
    dm, mv = _dev_bf16(mask)
    db = torch.from_numpy(b).cuda()
    ref = ws.conv3d(xv, wv)
    for epi in (0, 1, 2):
        dy = torch.zeros(shape + (cout,), dtype=torch.int16, device="cuda")
        xr.conv3d_fprop(dx.data_ptr(), cin, dw.data_ptr(), db.data_ptr() if epi < 2 else 0,
                        dm.data_ptr() if epi == 2 else 0, dy.data_ptr(), cout, shape, epi)
        torch.cuda.synchronize()
        got = _from_bf16(dy)
        want = ref + b if epi < 2 else ref
        if epi == 1:
            want = np.maximum(want, 0.0)
        if epi == 2:
            want = want * (mv > 0)
        _close_bf16(got, want)


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 16), (32, 32)])
@pytest.mark.parametrize("shape", SHAPES)
def test_conv_wgrad(cin, cout, shape):
    xr = load_xr()
    rng = np.random.default_rng(7 + cin + cout + shape[0])
    x = rng.normal(size=shape + (cin,)).astype(np.float32)
    g = rng.normal(size=shape + (cout,)).astype(np.float32)
    dx, xv = _dev_bf16(x)
    dg, gv = _dev_bf16(g)
    dw = torch.zeros((27, cout, cin), dtype=torch.float32, device="cuda")
    xr.conv3d_wgrad(dx.data_ptr(), cin, dg.data_ptr(), cout, dw.data_ptr(), shape)
    torch.cuda.synchronize()
    ref = ws.conv3d_wgrad(xv, gv)
    got = dw.cpu().numpy().astype(np.float64)
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()


def test_dgrad_is_fprop_with_mirrored_transposed_weights():
    """dgrad through the fprop kernel: w'[26 - t][k][n] = w[t][n][k]."""
    xr = load_xr()
    rng = np.random.default_rng(11)
    shape = (10, 12, 14)
    g = rng.normal(size=shape + (32,)).astype(np.float32)
    w = (rng.normal(size=(27, 32, 16)) * 0.1).astype(np.float32)
    wt = np.ascontiguousarray(w[::-1].transpose(0, 2, 1))
    dg, gv = _dev_bf16(g)
    dwt, _ = _dev_bf16(wt)
    out = torch.zeros(shape + (16,), dtype=torch.int16, device="cuda")
    xr.conv3d_fprop(dg.data_ptr(), 32, dwt.data_ptr(), 0, 0, out.data_ptr(), 16, shape, 0)
    torch.cuda.synchronize()
    _close_bf16(_from_bf16(out), ws.conv3d_dgrad(gv, ws.bf16(w)))


def _net_case(seed=3, shape=(12, 14, 16), noise=0.1):
    rng = np.random.default_rng(seed)
    K = 13
    x = rng.uniform(0.0, 1.0, (K,) + shape).astype(np.float32)
    t = (0.8 * x + 0.05 + noise * rng.uniform(0.0, 1.0, x.shape)).astype(np.float32)
    return K, x, t


def test_net_loss_and_gradient_match_oracle():
    xr = load_xr()
    K, x, t = _net_case()
    net = xr.Net(K, 32, 4, seed=5)
    p = net.get_params()
    p[-K:] = 0.05                                   # non-zero last bias
    net.set_params(p)
    dx = torch.from_numpy(x).cuda()
    dt = torch.from_numpy(t).cuda()
    loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:], in_scale=2.0, want_grad=True)
    rl, rg, _ = ws.net_loss_grad(p.astype(np.float64), x, t, K, 32, 4, in_scale=2.0)
    assert abs(loss - rl) <= 1e-3 * rl
    rel = np.linalg.norm(g - rg) / np.linalg.norm(rg)
    cos = float(g @ rg / (np.linalg.norm(g) * np.linalg.norm(rg)))
    print(f"net gradient: rel L2 {rel:.3e}, cosine {cos:.6f}")
    assert rel <= 2e-2 and cos >= 0.999
    # per layer, the gradient of every weight block is non-trivial
    off = 0
    for cin, cout in ws.layer_shapes(K, 32, 4):
        n = 27 * cin * cout + cout
        blk, rblk = g[off:off + n], rg[off:off + n]
        assert np.linalg.norm(blk - rblk) <= 5e-2 * np.linalg.norm(rblk)
        off += n
    net.close()


def test_net_tensor_loss_matches_oracle():
    """The orientation term of the training loss: loss and gradient against
    the oracle with the XTT basis; weight 0 restores the plain MSE."""
    xr = load_xr()
    K, x, t = _net_case(seed=4)
    basis = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, -1, 0], [1, 0, 1], [1, 0, -1], [0, 1, 1],
                      [0, 1, -1], [1, 1, 1], [1, 1, -1], [1, -1, 1], [-1, 1, 1]], np.float64)
    basis /= np.linalg.norm(basis, axis=1, keepdims=True)
    net = xr.Net(K, 32, 4, seed=6)
    p = net.get_params()
    dx = torch.from_numpy(x).cuda()
    dt = torch.from_numpy(t).cuda()
    l_plain, _ = net.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:])
    net.set_tensor_loss(basis, 3.0)
    loss, g = net.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:], want_grad=True)
    rl, rg, _ = ws.net_loss_grad(p.astype(np.float64), x, t, K, 32, 4, tensor_basis=basis, tensor_weight=3.0)
    assert loss > 1.5 * l_plain
    assert abs(loss - rl) <= 1e-3 * rl
    rel = np.linalg.norm(g - rg) / np.linalg.norm(rg)
    cos = float(g @ rg / (np.linalg.norm(g) * np.linalg.norm(rg)))
    print(f"tensor-loss gradient: rel L2 {rel:.3e}, cosine {cos:.6f}")
    assert rel <= 2e-2 and cos >= 0.999
    net.set_tensor_loss(None, 0.0)
    l_off, _ = net.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:])
    assert abs(l_off - l_plain) <= 1e-9 * l_plain   # the loss sums per-block partials by atomics, in any order
    with pytest.raises(xr.XRError):
        net.set_tensor_loss(basis, -1.0)
    net.close()


@pytest.mark.parametrize("storage", [0, 1])
def test_net_infer_matches_oracle(storage):
    xr = load_xr()
    K, x, _ = _net_case(seed=9, shape=(10, 11, 17))
    net = xr.Net(K, 32, 4, seed=8)
    p = net.get_params()
    p[-K - 27 * 32 * K:-K] *= 10.0                  # a visible last layer
    net.set_params(p)
    dt = {0: torch.float32, 1: torch.bfloat16}[storage]
    dx = torch.from_numpy(x).cuda().to(dt)
    xin = dx.float().cpu().numpy()
    out = torch.empty_like(dx)
    net.infer(dx.data_ptr(), out.data_ptr(), x.shape[1:], storage=storage, in_scale=1.5, floor_value=0.0)
    torch.cuda.synchronize()
    got = out.float().cpu().numpy().astype(np.float64)
    ref = ws.net_forward(p.astype(np.float64), xin, K, 32, 4, in_scale=1.5, floor_value=0.0)
    tol = 2e-3 if storage == 0 else 1e-2
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    # in place: the output may overwrite the input
    net.infer(dx.data_ptr(), dx.data_ptr(), x.shape[1:], storage=storage, in_scale=1.5, floor_value=0.0)
    torch.cuda.synchronize()
    assert torch.equal(dx, out)
    net.close()


def test_net_training_reduces_loss_and_round_trips(tmp_path):
    xr = load_xr()
    K, x, t = _net_case(seed=21, shape=(16, 16, 16), noise=0.0)   # a learnable map
    net = xr.Net(K, 32, 4, seed=1)
    dx = torch.from_numpy(x).cuda()
    dt = torch.from_numpy(t).cuda()
    l0, _ = net.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:])
    for _ in range(100):
        net.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:])
        net.adam_step(2e-3)
    l1, _ = net.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:])
    print(f"training loss {l0:.4e} -> {l1:.4e}")
    assert l1 < 0.5 * l0
    path = str(tmp_path / "net.bin")
    net.save(path)
    other = xr.Net(K, 32, 4, seed=99)
    other.load(path)
    assert np.array_equal(other.get_params(), net.get_params())
    l2, _ = other.loss_grad(dx.data_ptr(), dt.data_ptr(), x.shape[1:])
    assert abs(l2 - l1) <= 1e-12 * l1     # FP64 loss sums in atomic order
    with pytest.raises(xr.XRError):
        xr.Net(K, 16, 4).load(path)
    net.close()
    other.close()
