"""The reference-signature C++ layer (include/xr_compat.hpp): a main.cu-style
driver compiles and links against it (CPU), and runs on the GPU, matching
the Python path and the oracle."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, ROOT, load_xr
from scans import basis13, fiber_phantom, three_axes

SRC = os.path.join(ROOT, "tests", "compat", "main_like.cpp")


def build_driver(tmp_path) -> str:
    load_xr().lib()
    exe = str(tmp_path / "main_like")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", PKG_DIR, "-l:libxr.so", f"-Wl,-rpath,{PKG_DIR}"], check=True)
    return exe


def test_compat_header_compiles_and_links(tmp_path):
    exe = build_driver(tmp_path)
    assert os.path.exists(exe)


def test_c99_caller_builds_and_runs(tmp_path):
    """The C ABI from plain C: tests/compat/c_caller.c compiles as pedantic
    C99 with warnings as errors, links against libxr.so and passes its
    device-free checks (context round trip, argument, state and
    configuration errors)."""
    load_xr().lib()
    exe = str(tmp_path / "c_caller")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "compat", "c_caller.c"), "-o", exe, "-L", PKG_DIR, "-l:libxr.so",
                    f"-Wl,-rpath,{PKG_DIR}"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, f"check {r.returncode} failed"
    assert "sm_100a" in r.stdout


def test_compat_signatures_match_the_reference():
    """tests/compat/signatures.cpp static_asserts the type of every compat
    entry point against the reference's declaration (reconstruct.cuh,
    pca.cuh, tvmin.h, quadfilt.h, params.h); it must compile."""
    src = os.path.join(ROOT, "tests", "compat", "signatures.cpp")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_compat_driver_runs(tmp_path, oracle):
    from oracle import Scan
    exe = build_driver(tmp_path)
    N, Nd, V = 12, 20, 9
    b13 = basis13()
    doc = {"recon_variable": {"blockSize": 32, "vector": 13, "condition": 3, "base": [float(x) for x in b13.ravel()]},
           "sim": {"proj_path": "p", "vol_path": "v", "direc_path": "d", "sod": 500.0, "sdd": 1000.0, "proj": V,
                   "num_det_u": Nd, "num_det_v": Nd, "det_size": 2.0, "num_voxel": N, "rot": 3,
                   "matrixRot": [float(x) for x in three_axes().ravel()], "vecTrans": [0.0] * 9,
                   "areaTrans": [0.0, 0.0, 0.0], "offset": [0.0] * 9, "sorting": False}}
    cfg = tmp_path / "settings.json"
    cfg.write_text(json.dumps(doc))
    s = Scan(sdd=1000.0, sod=500.0, det=2.0, N=N, Nd=Nd, V=V, rot=three_axes(), trans=np.zeros((3, 3)),
             offset=np.zeros((3, 3)), basis=b13)
    truth = fiber_phantom(N, 3, 4, b13)
    b = oracle.forward_all(s, truth, 0, True)
    b.tofile(str(tmp_path / "sino.raw"))
    r = subprocess.run([exe, str(cfg), "sim", str(tmp_path / "sino.raw"), str(tmp_path) + "/"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    mu = np.stack([np.fromfile(str(tmp_path / f"ct{k + 1}.raw"), np.float32) for k in range(13)])
    ref, _, _ = oracle.xtt_reconstruct(s, b, np.full((13, N, N, N), 0.01, np.float32), 2, 3, lam=1e-3)
    assert np.abs(mu.reshape(ref.shape) - ref).max() <= 1e-5 * np.abs(ref).max()
