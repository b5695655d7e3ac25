"""Generate tests/golden/ref_fdk_small.npz from the reference itself.

Runs the reference's own FDK kernels (reconstruct/src/fdk.cu:13-170: calcWeight,
projConv, filteredBackProj / backwardonDevice) and orientation post-processing
(direction/src/pca.cu:67-106: calcAngleFromMD, directionNormalization),
compiled for the host from slices of those files by `make -C oracle ref`
(oracle/_ref/libxrref.so), with FDK::reconstruct's host loop restated in
oracle/ref_shim/ref_fdk_pca.cpp (reconstruct.cu:1651-1724).  Stores inputs and
outputs as .npz; the committed fixture then pins the oracle anywhere.

    python tests/golden/make_golden_fdk.py
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
from scans import ellipsoid_phantom, three_axes  # noqa: E402


def fdk_scan(seed: int, C: int, N: int = 14, Nd: int = 22, V: int = 12) -> Scan:
    rng = np.random.default_rng(seed)
    return Scan(sdd=1000.0, sod=500.0, det=2.0, N=N, Nd=Nd, V=V, rot=three_axes()[:C],
                trans=rng.normal(0, 0.3, (C, 3)), offset=rng.normal(0, 0.2, (C, 3)),
                basis=np.array([[0.0, 0.0, 1.0]], np.float32))


def main() -> None:
    build(ref=True)
    R = RefHost(parallel=False)
    out = {}
    # FDK of 2 axes (the reference back-projects axis 0's filtered block for
    # every axis, reconstruct.cu:1708), CW and CCW
    s = fdk_scan(61, 2)
    R.setup(s)
    out.update({"fdk_geom": np.array([s.sdd, s.sod, s.det, s.N, s.Nd, s.V], np.float64), "fdk_rot": s.rot,
                "fdk_trans": s.trans, "fdk_offset": s.offset})
    rng = np.random.default_rng(62)
    sino = rng.uniform(0.0, 2.0, (s.C, s.V, s.Nd, s.Nd)).astype(np.float32)
    sino[:, :, :, :3] += ellipsoid_phantom(s.Nd, 2, 63)[: s.V, :, :3]   # some structure along u
    out["fdk_sino"] = sino
    out["fdk_weight"] = R.fdk_weight()
    out["fdk_filter"] = R.fdk_filter()
    for ccw in (0, 1):
        vol, filt = R.fdk_reconstruct(sino, ccw)
        out[f"fdk_vol_{ccw}"] = vol
        out[f"fdk_filt_{ccw}"] = filt
    # orientation post-processing: main directions with lengths around the
    # 0.65 threshold, both signs of m_y, and exact zeros
    md = rng.normal(0.0, 0.6, (3, 6, 7, 8)).astype(np.float32)
    md[:, 0, 0, :4] = 0.0
    md[1, 1, :, :] = np.abs(md[1, 1, :, :])
    out["pca_md"] = md
    out["pca_angle"] = R.angle_from_md(md)
    out["pca_norm"] = R.direction_normalization(md)
    np.savez_compressed(os.path.join(HERE, "ref_fdk_small.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_fdk_small.npz"), sorted(out))


if __name__ == "__main__":
    main()
