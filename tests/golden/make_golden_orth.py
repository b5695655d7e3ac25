"""Golden vectors of the reference's orientation-parametrised XTT kernels
(forwardOrth, backwardOrth, calcNormalVectorThreeDirec; reconstruct/src/ir.cu)
from its host build (oracle/_ref/libxrref.so, serial launch order).

    python tests/golden/make_golden_orth.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import RefHost, Scan, build  # noqa: E402
from scans import basis13, three_axes  # noqa: E402


def orth_scan() -> Scan:
    rng = np.random.default_rng(41)
    return Scan(sdd=1000.0, sod=500.0, det=2.0, N=12, Nd=20, V=10, rot=three_axes(),
                trans=rng.normal(0, 0.3, (3, 3)), offset=rng.normal(0, 0.2, (3, 3)), basis=basis13()[:3])


def main() -> None:
    build(ref=True)
    R = RefHost(parallel=False)
    s = orth_scan()
    R.setup(s)
    rng = np.random.default_rng(42)
    N, Nd, V = s.N, s.Nd, s.V
    out = {"geom": np.array([s.sdd, s.sod, s.det, N, Nd, V], np.float64), "rot": s.rot, "trans": s.trans,
           "offset": s.offset, "basis": s.basis}
    vol = rng.uniform(0.1, 1.0, (3, N, N, N)).astype(np.float32)
    coef = np.stack([rng.uniform(-3.1, 3.1, (N, N, N)), rng.uniform(0.05, 0.99, (N, N, N))]).astype(np.float32)
    ratio = rng.uniform(0.0, 2.0, (V, Nd, Nd)).astype(np.float32)
    out.update(vol=vol, coef=coef, ratio=ratio)
    for cond in range(3):
        n = 2 + 3 * cond
        p = np.zeros(V * Nd * Nd, np.float32)
        R.forward_orth(cond, n, vol.ravel().copy(), coef.ravel().copy(), p)
        out[f"fwd_c{cond}"] = p[n * Nd * Nd:(n + 1) * Nd * Nd].copy()
        tmp = np.zeros(3 * N * N, np.float32)
        fac = np.zeros(3 * N * N, np.float32)
        R.backward_orth(cond, 5, n, ratio.ravel().copy(), coef.ravel().copy(), tmp, fac)
        out[f"bwd_c{cond}_tmp"] = tmp
        out[f"bwd_c{cond}_fac"] = fac
    for rot in range(4):
        c = coef.ravel().copy()
        loss = np.zeros(N ** 3, np.float32)
        R.normal_three(vol.ravel().copy(), c, loss, rot)
        out[f"nrm_r{rot}_coef"] = c
        out[f"nrm_r{rot}_loss"] = loss
    path = os.path.join(HERE, "ref_orth_small.npz")
    np.savez_compressed(path, **out)
    print(path, len(out), "arrays")


if __name__ == "__main__":
    main()
