"""Golden vectors of the reference's fiber-model projectors (forwardProjFiber,
backwardProjFiber; reconstruct/src/fiber.cu) from its host build
(oracle/_ref/libxrref.so, serial launch order), for K = 3 and K = 4, and of
whole fiberModelReconstruct runs (reconstruct.cu:1242-1371, restated in
oracle/ref_shim/ref_driver.cpp over the reference's kernels): MLEM and ART,
CW and CCW, two epochs of three subsets (one case with V % batch != 0).

    python tests/golden/make_golden_fiber.py
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


def fiber_scan(K: int) -> Scan:
    rng = np.random.default_rng(90 + K)
    return Scan(sdd=1000.0, sod=500.0, det=2.0, N=12, Nd=20, V=10, rot=three_axes(),
                trans=rng.normal(0, 0.3, (3, 3)), offset=rng.normal(0, 0.2, (3, 3)), basis=basis13()[:K])


def main() -> None:
    build(ref=True)
    out = {}
    for K in (3, 4):
        R = RefHost(parallel=False)
        s = fiber_scan(K)
        R.setup(s)
        rng = np.random.default_rng(95 + K)
        N, Nd, V = s.N, s.Nd, s.V
        vol = rng.normal(0, 1, (K, N, N, N)).astype(np.float32)
        ratio = rng.uniform(0.0, 2.0, (V, Nd, Nd)).astype(np.float32)
        out[f"k{K}_geom"] = np.array([s.sdd, s.sod, s.det, N, Nd, V], np.float64)
        out.update({f"k{K}_rot": s.rot, f"k{K}_trans": s.trans, f"k{K}_offset": s.offset, f"k{K}_basis": s.basis,
                    f"k{K}_vol": vol, f"k{K}_ratio": ratio})
        # views n > 0 (Rotate::CW) and n < 0 (Rotate::CCW, image |n|)
        for cond in range(3):
            for sign, tag in ((1, ""), (-1, "_ccw")):
                n = sign * (2 + 3 * cond)
                m = abs(n)
                p = np.zeros(V * Nd * Nd, np.float32)
                R.fiber_forward(cond, n, vol.ravel().copy(), p)
                out[f"k{K}_fwd_c{cond}{tag}"] = p[m * Nd * Nd:(m + 1) * Nd * Nd].copy()
                tmp = np.zeros(K * N * N, np.float32)
                fac = np.zeros(K * N * N, np.float32)
                R.fiber_backward(cond, 4, n, ratio.ravel().copy(), vol.ravel().copy(), tmp, fac)
                out[f"k{K}_bwd_c{cond}{tag}_tmp"] = tmp
                out[f"k{K}_bwd_c{cond}{tag}_fac"] = fac
    # whole sessions: (K, art, ccw)
    rng = np.random.default_rng(120)
    # case 4: V % batch != 0, so the last subsets revisit views 0 and 1 (reconstruct.cu:1306)
    for i, (K, art, ccw, V) in enumerate([(3, False, 0, 6), (4, True, 1, 6), (4, False, 1, 6), (3, True, 0, 6),
                                          (4, False, 0, 7)]):
        R = RefHost(parallel=False)
        s = Scan(sdd=1000.0, sod=500.0, det=2.0, N=8, Nd=14, V=V, rot=three_axes(),
                 trans=rng.normal(0, 0.3, (3, 3)), offset=rng.normal(0, 0.2, (3, 3)),
                 basis=np.eye(4, 3, dtype=np.float32)[:K])
        R.setup(s)
        sino = rng.uniform(0.5, 1.5, (3, s.V, s.Nd, s.Nd)).astype(np.float32)
        v0 = np.full((K, s.N, s.N, s.N), 0.01, np.float32)
        vol, ratio, losses = R.fiber_reconstruct(sino, v0, 2, 3, ccw, art, 1e-2)
        out.update({f"s{i}_case": np.array([K, int(art), ccw], np.int32), f"s{i}_geom":
                    np.array([s.sdd, s.sod, s.det, s.N, s.Nd, s.V], np.float64), f"s{i}_rot": s.rot,
                    f"s{i}_trans": s.trans, f"s{i}_offset": s.offset, f"s{i}_basis": s.basis, f"s{i}_sino": sino,
                    f"s{i}_vol": vol, f"s{i}_ratio": ratio, f"s{i}_losses": losses})
    path = os.path.join(HERE, "ref_fiber_small.npz")
    np.savez_compressed(path, **out)
    print(path, len(out), "arrays")


if __name__ == "__main__":
    main()
