"""The reference's own CUDA kernels on the B200 (reconstruct/src/ir.cu built
for sm_100a by oracle/Makefile, driven like XTT::reconstruct with one launch
and synchronize per y slab and view, oracle/ref_gpu) against the oracle on
the same seeded inputs: a check that the build runs the reference's
arithmetic.  The oracle is bit-exact to the reference compiled for the host;
the reference compiled for the GPU is not: nvcc contracts its a*b+c into fused
multiply-adds and the device's cosf/sinf round differently, so its detector
coordinates differ in the last bits, and footprint-edge pixels, divided by
their small weight sums in correlationProjByLength, amplify that.  Bounds:
volume 1e-4 of the largest value, ratio images 1e-4 relative L2 and 1e-2 of
the largest value (the product, which rounds as the host build, meets 1e-5
on both: tests/test_gpu_parity.py, tests/test_parity_full_size.py)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import RefGPU, Scan
from scans import basis13, fiber_phantom, three_axes

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not RefGPU.available(), reason="oracle/_ref/libxrref_gpu.so not built")
@pytest.mark.parametrize("art", [False, True], ids=["mlem", "art"])
def test_reference_gpu_xtt_epoch_matches_oracle(oracle, art):
    rng = np.random.default_rng(91)
    s = Scan(sdd=1000.0, sod=500.0, det=2.0, N=20, Nd=30, V=12, rot=three_axes(), trans=rng.normal(0, 0.3, (3, 3)),
             offset=rng.normal(0, 0.2, (3, 3)), basis=basis13())
    truth = fiber_phantom(s.N, 4, 92, s.basis)
    b = oracle.forward_all(s, truth, 0, True)
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    ref, rproj, rl = oracle.xtt_reconstruct(s, b, v0, 2, 4, art=art, lam=1e-3)
    got, gproj, gl, ms = RefGPU().xtt_reconstruct(s, b, v0, 2, 4, art=art, lam=1e-3)
    err = float(np.abs(got.astype(np.float64) - ref).max() / np.abs(ref).max())
    d = gproj.astype(np.float64) - rproj
    perr = float(np.abs(d).max() / np.abs(rproj).max())
    pl2 = float(np.linalg.norm(d) / np.linalg.norm(rproj))
    print(f"reference CUDA kernels vs oracle ({'ART' if art else 'MLEM'}): volume {err:.2e}, ratio images "
          f"max {perr:.2e} / L2 {pl2:.2e}, {ms.mean():.1f} ms per epoch")
    assert err <= 1e-4
    assert pl2 <= 1e-4 and perr <= 1e-2
    assert np.allclose(gl, rl, rtol=1e-3)
