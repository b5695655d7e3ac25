"""CPU oracle for the learned warm start (test infrastructure only: imported by
tests/, never by the product).

The reference has no learned component, so there is no reference source to
restate; this module restates the network of include/xr_learn.h in numpy:
3x3x3 convolutions with zero padding (tap = 9*(dz+1) + 3*(dy+1) + (dx+1)),
ReLU hidden layers, the residual output y = x + (conv_D + b_D) / s, the mean
squared error and its gradient by back-propagation.  With `bf16=True` it
rounds at the points where the tensor-core path stores BF16 (weights, packed
input, hidden activations, output gradients), accumulating in float64.

Pinning: with `bf16=False` the analytic gradient is checked against central
finite differences in float64 (tests/test_learn_oracle.py); the GPU kernels
are then checked against the BF16 emulation.
"""
from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(a: np.ndarray) -> np.ndarray:
    """BF16 bit patterns (uint16) of a float array, round to nearest even."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def taps():
    """(dz, dy, dx) of the 27 taps in kernel order."""
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def _shift(x: np.ndarray, dz: int, dy: int, dx: int) -> np.ndarray:
    """out[z, y, x] = x[z + dz, y + dy, x + dx], zero outside (x: [nz, ny, nx, c])."""
    nz, ny, nx = x.shape[:3]
    p = np.zeros((nz + 2, ny + 2, nx + 2) + x.shape[3:], x.dtype)
    p[1:-1, 1:-1, 1:-1] = x
    return p[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx]


def conv3d(x: np.ndarray, w: np.ndarray, b=None) -> np.ndarray:
    """y[v][n] = sum_t sum_k x[v + d(t)][k] w[t][n][k] (+ b[n]); x [nz,ny,nx,cin], w [27,cout,cin]."""
    y = np.zeros(x.shape[:3] + (w.shape[1],), np.float64)
    for t, (dz, dy, dx) in enumerate(taps()):
        y += _shift(x, dz, dy, dx) @ w[t].T
    if b is not None:
        y += b
    return y


def conv3d_dgrad(dy: np.ndarray, w: np.ndarray) -> np.ndarray:
    """dx[v][k] = sum_t sum_n dy[v - d(t)][n] w[t][n][k]."""
    dx = np.zeros(dy.shape[:3] + (w.shape[2],), np.float64)
    for t, (dz, ddy, ddx) in enumerate(taps()):
        dx += _shift(dy, -dz, -ddy, -ddx) @ w[t]
    return dx


def conv3d_wgrad(x: np.ndarray, dy: np.ndarray) -> np.ndarray:
    """dw[t][n][k] = sum_v dy[v][n] x[v + d(t)][k]."""
    cin, cout = x.shape[3], dy.shape[3]
    dw = np.zeros((27, cout, cin), np.float64)
    g = dy.reshape(-1, cout)
    for t, (dz, ddy, ddx) in enumerate(taps()):
        dw[t] = g.T @ _shift(x, dz, ddy, ddx).reshape(-1, cin)
    return dw


def layer_shapes(channels: int, width: int, depth: int):
    """(cin, cout) per layer."""
    return [((channels if l == 0 else width), (channels if l == depth - 1 else width)) for l in range(depth)]


def unflatten(p: np.ndarray, channels: int, width: int, depth: int):
    """Flat parameter vector -> [(W [27, cout, cin], b [cout])] in layer order."""
    out, off = [], 0
    for cin, cout in layer_shapes(channels, width, depth):
        W = p[off:off + 27 * cout * cin].reshape(27, cout, cin)
        off += 27 * cout * cin
        b = p[off:off + cout]
        off += cout
        out.append((np.asarray(W, np.float64), np.asarray(b, np.float64)))
    return out


def flatten(params) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in params])


def tensor_components(basis: np.ndarray) -> np.ndarray:
    """E[k] = (xx, yy, zz, xy, xz, yz) of S_k S_k^T, [K, 6]."""
    S = np.asarray(basis, np.float64).reshape(-1, 3)
    x, y, z = S[:, 0], S[:, 1], S[:, 2]
    return np.stack([x * x, y * y, z * z, x * y, x * z, y * z], axis=1)


def net_loss_grad(p: np.ndarray, x: np.ndarray, target: np.ndarray, channels: int, width: int, depth: int,
                  in_scale: float = 1.0, bf16_emulation: bool = True, tensor_basis=None, tensor_weight: float = 0.0):
    """Loss and flat gradient of the network on planar volumes x, target
    [K, nz, ny, nx].  Returns (loss, grad, pred).  With tensor_weight > 0 the
    loss adds tensor_weight * ||T(pred) - T(target)||_F^2 per voxel, T(mu) =
    sum_k mu_k S_k S_k^T (the tensor of calcEigenVector, pca.cu:12-55, on
    sqrt|mu|), over the same K * voxels."""
    R = bf16 if bf16_emulation else (lambda a: np.asarray(a, np.float64))
    params = unflatten(p, channels, width, depth)
    xs = np.moveaxis(np.asarray(x, np.float64), 0, -1)          # [nz, ny, nx, K]
    ts = np.moveaxis(np.asarray(target, np.float64), 0, -1)
    if bf16_emulation:
        h = R(np.asarray(xs * in_scale, np.float32))
    else:
        h = xs * in_scale
    acts = [h]
    for l, (W, b) in enumerate(params):
        z = conv3d(acts[-1], R(W), b)
        if l + 1 < depth:
            acts.append(R(np.maximum(z, 0.0)))
        else:
            out = z
    if bf16_emulation:
        pred = np.asarray(xs, np.float32).astype(np.float64) + out / in_scale
    else:
        pred = xs + out / in_scale
    n = pred.size
    diff = pred - ts
    loss = float((diff ** 2).sum() / n)
    gd = diff
    if tensor_weight > 0:
        E = tensor_components(tensor_basis)[:diff.shape[-1]]
        w = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])
        dT = diff @ E                                   # [..., 6]
        loss += float(tensor_weight * (w * dT ** 2).sum() / n)
        gd = diff + tensor_weight * (dT * w) @ E.T
    g = R(2.0 * gd / n / in_scale)
    grads = [None] * depth
    for l in range(depth - 1, -1, -1):
        W, b = params[l]
        dW = conv3d_wgrad(acts[l], g)
        db = g.reshape(-1, g.shape[-1]).sum(0)
        grads[l] = (dW, db)
        if l > 0:
            g = R(conv3d_dgrad(g, R(W)) * (acts[l] > 0))
    return loss, flatten(grads), np.moveaxis(pred, -1, 0)


def net_forward(p: np.ndarray, x: np.ndarray, channels: int, width: int, depth: int, in_scale: float = 1.0,
                floor_value: float = -np.inf, bf16_emulation: bool = True) -> np.ndarray:
    """Network output y = max(x + net(s x) / s, floor) on planar x [K, nz, ny, nx]."""
    zero = np.zeros_like(np.asarray(x, np.float64))
    _, _, pred = net_loss_grad(p, x, zero, channels, width, depth, in_scale, bf16_emulation)
    return np.maximum(pred, floor_value)
