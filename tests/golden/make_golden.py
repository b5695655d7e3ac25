"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own reconstruct/src/ir.cu, compiled for the host through
oracle/ref_shim (oracle/_ref/libxrref.so, built by `make -C oracle ref` from
the reference sources), serially so that every float sum has a fixed order,
and stores inputs and outputs as .npz.  Needs the reference sources; the
committed fixtures then pin the oracle anywhere.

    python tests/golden/make_golden.py
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


def small_scan(seed: int, C: int, K: int) -> Scan:
    rng = np.random.default_rng(seed)
    rot = three_axes()[:C]
    basis = basis13()[:K] if K > 1 else np.array([[0.0, 0.0, 1.0]], np.float32)
    return Scan(sdd=1000.0, sod=500.0, det=2.0, N=12, Nd=20, V=10, rot=rot,
                trans=rng.normal(0, 0.3, (C, 3)), offset=rng.normal(0, 0.2, (C, 3)), basis=basis)


def scan_dict(s: Scan, prefix: str) -> dict:
    return {f"{prefix}geom": np.array([s.sdd, s.sod, s.det, s.N, s.Nd, s.V], np.float64),
            f"{prefix}rot": s.rot, f"{prefix}trans": s.trans, f"{prefix}offset": s.offset,
            f"{prefix}basis": s.basis}


def main() -> None:
    build(ref=True)
    R = RefHost(parallel=False)
    out = {}

    # --- unit kernels: one view of each axis, plain and XTT (3 axes, K = 13)
    s = small_scan(11, 3, 13)
    R.setup(s)
    out.update(scan_dict(s, "unit_"))
    rng = np.random.default_rng(12)
    N, Nd, V = s.N, s.Nd, s.V
    vol = rng.uniform(0.1, 1.0, (s.K, N, N, N)).astype(np.float32)
    sino = rng.uniform(0.0, 3.0, (V, Nd, Nd)).astype(np.float32)
    out["unit_vol"] = vol
    out["unit_sino"] = sino
    for xtt in (0, 1):
        for cond in range(s.C):
            n = 3 + cond
            p = np.zeros(V * Nd * Nd, np.float32)
            f = np.zeros(Nd * Nd, np.float32)
            R.forward_view(cond, n, vol.ravel().copy(), p, f, xtt)
            out[f"fwd_x{xtt}_c{cond}_proj"] = p[n * Nd * Nd:(n + 1) * Nd * Nd].copy()
            out[f"fwd_x{xtt}_c{cond}_factor"] = f.copy()
            R.correlation(cond, n, p, f)
            out[f"cor_x{xtt}_c{cond}"] = p[n * Nd * Nd:(n + 1) * Nd * Nd].copy()
            for art in (0, 1):
                q = p.copy()
                loss = R.ratio(n, q, sino.ravel(), art)
                out[f"rat_x{xtt}_c{cond}_a{art}"] = q[n * Nd * Nd:(n + 1) * Nd * Nd].copy()
                out[f"rat_x{xtt}_c{cond}_a{art}_loss"] = np.array([loss], np.float32)
            q = p.copy()
            R.ratio(n, q, sino.ravel(), 0)
            t = np.zeros(N * N * s.K, np.float32)
            g = np.zeros(N * N * s.K, np.float32)
            R.backward_slab(cond, 5, n, q, t, g, xtt)
            out[f"bwd_x{xtt}_c{cond}_in"] = q[n * Nd * Nd:(n + 1) * Nd * Nd].copy()
            out[f"bwd_x{xtt}_c{cond}_tmp"] = t
            out[f"bwd_x{xtt}_c{cond}_factor"] = g
    out["fwdall_xtt"] = R.forward_all(vol, 0, True)

    # --- IR::reconstruct: one axis, V % batch != 0 (subset wrap-around)
    s1 = small_scan(21, 1, 1)
    R.setup(s1)
    out.update(scan_dict(s1, "ir_"))
    rng = np.random.default_rng(22)
    truth = rng.uniform(0.0, 1.0, (1, s1.N, s1.N, s1.N)).astype(np.float32)
    b = R.forward_all(truth[0], 0, False)
    out["ir_sino"] = b
    for art in (0, 1):
        v, l = R.ir_reconstruct(b, np.ones_like(truth), 3, 3, art=art, lam=1e-2)
        out[f"ir_a{art}_vol"] = v
        out[f"ir_a{art}_loss"] = l

    # --- XTT::reconstruct: 3 axes, K = 13
    s3 = small_scan(31, 3, 13)
    R.setup(s3)
    out.update(scan_dict(s3, "xtt_"))
    rng = np.random.default_rng(32)
    truth = rng.uniform(0.0, 0.5, (s3.K, s3.N, s3.N, s3.N)).astype(np.float32)
    b = R.forward_all(truth, 0, True)
    out["xtt_sino"] = b
    for art in (0, 1):
        v0 = np.full_like(truth, 0.01)
        v, p, l = R.xtt_reconstruct(b, v0, 2, 3, art=art, lam=1e-3)
        out[f"xtt_a{art}_vol"] = v
        out[f"xtt_a{art}_proj"] = p
        out[f"xtt_a{art}_loss"] = l

    path = os.path.join(HERE, "ref_ir_small.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
