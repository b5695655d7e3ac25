"""Golden vectors of the reference's main-direction (circle-estimate) kernels
(forwardOrthByMD, backwardOrthByMD, meanFiltFiberMD, calcMainDirection,
calcMDWithEst, updateEstimation) and of the coefficient-plane steps of its
orth drivers (meanFiltFiber, calcNormalVectorThreeDirecWithEst,
updateEstimationByCoef; reconstruct/src/ir.cu) from its host build
(oracle/_ref/libxrref.so, serial launch order).

    python tests/golden/make_golden_md.py
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


def md_scan() -> Scan:
    rng = np.random.default_rng(61)
    return Scan(sdd=1000.0, sod=500.0, det=2.0, N=12, Nd=20, V=10, rot=three_axes(),
                trans=rng.normal(0, 0.3, (3, 3)), offset=rng.normal(0, 0.2, (3, 3)), basis=basis13()[:3])


def md_inputs(s: Scan):
    rng = np.random.default_rng(62)
    N, Nd, V = s.N, s.Nd, s.V
    vol = rng.uniform(0.1, 1.0, (3, N, N, N)).astype(np.float32)
    md = rng.normal(0, 1, (3, N, N, N)).astype(np.float32)
    md[:, 3, 4, 5] = 0.0                      # zero main direction: identity rotation
    md[:2, 6, 6, 6] = 0.0                     # along z
    ratio = rng.uniform(0.0, 2.0, (V, Nd, Nd)).astype(np.float32)
    est = np.stack([rng.uniform(0.0, 2.0, (N, N, N)), rng.uniform(0.0, 3.5, (N, N, N))]).astype(np.float32)
    coef = np.stack([rng.uniform(-3.1, 3.1, (N, N, N)), rng.uniform(-0.99, 0.99, (N, N, N))]).astype(np.float32)
    return vol, md, ratio, est, coef


def main() -> None:
    build(ref=True)
    R = RefHost(parallel=False)
    s = md_scan()
    R.setup(s)
    N, Nd, V = s.N, s.Nd, s.V
    vol, md, ratio, est, coef = md_inputs(s)
    out = {"geom": np.array([s.sdd, s.sod, s.det, N, Nd, V], np.float64), "rot": s.rot, "trans": s.trans,
           "offset": s.offset, "basis": s.basis, "vol": vol, "md": md, "ratio": ratio, "est": est, "coef": coef}
    for cond in range(3):
        n = 1 + 3 * cond
        p = np.zeros(V * Nd * Nd, np.float32)
        fac = np.zeros(Nd * Nd, np.float32)
        R.forward_md(cond, n, vol.ravel().copy(), md.ravel().copy(), p, fac)
        out[f"fwd_c{cond}"] = p[n * Nd * Nd:(n + 1) * Nd * Nd].copy()
        out[f"fwd_c{cond}_fac"] = fac
        tmp = np.zeros(3 * N * N, np.float32)
        bf = np.zeros(3 * N * N, np.float32)
        R.backward_md(cond, 5, n, ratio.ravel().copy(), md.ravel().copy(), tmp, bf)
        out[f"bwd_c{cond}_tmp"] = tmp
        out[f"bwd_c{cond}_fac"] = bf
    filt = md.ravel().copy()
    for y in range(2, N - 2):
        R.md_filter(y, md.ravel().copy(), filt, 1.0)
    out["filter"] = filt
    for it in range(4):
        m = md.ravel().copy()
        R.main_direction(vol.ravel().copy(), m, it)
        out[f"main_it{it}"] = m
    m = md.ravel().copy()
    R.md_with_estimate(vol.ravel().copy(), m, est.ravel().copy())
    out["with_est"] = m
    e = est.ravel().copy()
    R.update_estimation(vol.ravel().copy(), md.ravel().copy(), e, 2)
    out["update_est"] = e
    c = coef.ravel().copy()
    loss = np.zeros(N ** 3, np.float32)
    R.normal_three_est(vol.ravel().copy(), c, loss, est.ravel().copy())
    out["nrm_est_coef"] = c
    out["nrm_est_loss"] = loss
    cf = coef.ravel().copy()
    for y in range(1, N - 1):
        R.coef_filter(y, coef.ravel().copy(), cf, vol.ravel().copy(), 1.0)
    out["coef_filter"] = cf
    e = est.ravel().copy()
    R.update_estimation_coef(vol.ravel().copy(), e, 3)
    out["update_est_coef"] = e
    path = os.path.join(HERE, "ref_md_small.npz")
    np.savez_compressed(path, **out)
    print(path, len(out), "arrays")


if __name__ == "__main__":
    main()
