"""The learned warm start end to end on the GPU, at a small size: the device
fiber phantom against the numpy generator, and what a network trained by
libxr's tensor-core kernels gains over the plain OS-EM iterate it starts
from (held-out phantom, same geometry)."""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

from conftest import PKG_DIR, load_xr
from scans import basis13, fiber_phantom

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ws():
    load_xr()
    if "xrd.warmstart" in sys.modules:
        return sys.modules["xrd.warmstart"]
    spec = importlib.util.spec_from_file_location("xrd.warmstart", os.path.join(PKG_DIR, "warmstart.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["xrd.warmstart"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_device_phantom_matches_numpy_generator():
    ws = _ws()
    N, seed = 40, 17
    d = torch.empty((13, N, N, N), dtype=torch.float32, device="cuda")
    ws.fiber_phantom_dev(d.data_ptr(), N, 12, seed, basis13())
    torch.cuda.synchronize()
    ref = fiber_phantom(N, 12, seed, basis13())
    got = d.cpu().numpy()
    same = np.isclose(got, ref, rtol=1e-6, atol=1e-7).all(axis=0).mean()
    assert same >= 0.999      # voxel centres within FP32 rounding of a fiber's surface may differ
    assert np.abs(got).max() > 0.5


def test_trained_network_improves_the_early_iterate():
    ws = _ws()
    xr = load_xr()
    scan = ws.Scan(32, V=60)
    xin, tgt = ws.make_pool(scan, range(100, 124), crops_per=2, crop=24, early_epochs=3, rng_seed=1)
    net = xr.Net(13, 32, 4, seed=3)
    net.set_stream(scan.stream.cuda_stream)
    trace = ws.train(net, xin, tgt, steps=600, lr=2e-3, lr_final=2e-4, log_every=100)
    print("training loss (single crops)", [round(l, 5) for _, l in trace])
    assert np.mean([l for _, l in trace[-3:]]) < trace[0][1]
    # held-out phantom: plain OS-EM iterate vs warm start, then both continued
    mu = scan.phantom(999)
    b = scan.project(mu)
    plain = torch.full_like(mu, 0.01)
    scan.osem(b, plain, 3, final_sqrt=False)
    warm = torch.full_like(mu, 0.01)
    ws.warm_start(scan, net, b, warm, early_epochs=3)
    err = lambda v: float(torch.linalg.vector_norm(v - mu) / torch.linalg.vector_norm(mu))
    e_plain, e_warm = err(plain), err(warm)
    r_plain, r_warm = scan.residual(plain, b), scan.residual(warm, b)
    scan.osem(b, plain, 3, final_sqrt=False)
    scan.osem(b, warm, 3, final_sqrt=False)
    r_plain6, r_warm6 = scan.residual(plain, b), scan.residual(warm, b)
    print(f"held-out, 3 epochs: volume error plain {e_plain:.4f} / warm start {e_warm:.4f}, data residual "
          f"{r_plain:.4e} / {r_warm:.4e}; after 3 more epochs {r_plain6:.4e} / {r_warm6:.4e}")
    assert e_warm < e_plain
    net.close()
