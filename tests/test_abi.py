"""C-ABI boundary checks that need no GPU: libxr.so loads, exports every
function include/xr.h and include/xr_learn.h declare, parses settings files of the reference's
schema like init_params (params.cu:42-104), validates scans, and reports
XR_ERR_NODEV (instead of crashing) when no device is present."""
from __future__ import annotations

import ctypes
import json
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available, load_xr
from oracle import reference_root

HEADERS = [os.path.join(ROOT, "include", "xr.h"), os.path.join(ROOT, "include", "xr_learn.h")]
REF_SETTINGS = os.path.join(reference_root() or "-", "utility", "settings.json")


def declared_functions():
    text = "".join(open(h).read() for h in HEADERS)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xr_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ["xr_init_params", "xr_create", "xr_forward", "xr_forward_proj_only", "xr_ir_reconstruct",
                     "xr_xtt_reconstruct", "xr_fdk_reconstruct", "xr_orientation", "xr_residual",
                     "xr_dev_session_begin", "xr_dev_session_epoch", "xr_dev_session_end", "xr_last_error"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    xr = load_xr()
    L = xr.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert b"sm_100a" in L.xr_version()


def test_python_mirror_binds_every_symbol():
    xr = load_xr()
    assert set(declared_functions()) == set(xr._SIGS)


def _write_settings(tmp_path, presets):
    doc = {"recon_variable": {"blockSize": 32, "vector": 3, "condition": 2,
                              "base": [0.0, 0.0, 1.0, 0.6, 0.8, 0.0, 0.0, 0.6, 0.8]}}
    doc.update(presets)
    p = tmp_path / "settings.json"
    p.write_text(json.dumps(doc, indent=1))
    return str(p)


def _preset(sorting=None, index=None):
    d = {"proj_path": "../p/x", "vol_path": "../v/y", "direc_path": "../d/z", "sod": 500.0, "sdd": 1000.0,
         "proj": 12, "num_det_u": 20, "num_det_v": 20, "det_size": 2.0, "num_voxel": 16, "rot": 3,
         "matrixRot": [1, 0, 0, 0, 1, 0, 0, 0, 1,
                       0, 0, -1, 0, 1, 0, 1, 0, 0,
                       1, 0, 0, 0, 0, -1, 0, 1, 0],
         "vecTrans": [0.1, 0.2, 0.3, 1.0, 2.0, 3.0, -1.0, -2.0, -3.0],
         "areaTrans": [0.5, 0.25, 0.125],
         "offset": [0.01, 0, 0, 0.02, 0, 0, 0.03, 0, 0]}
    if sorting is not None:
        d["sorting"] = sorting
    if index is not None:
        d["index"] = index
    return d


def test_init_params_sorting_and_area_trans(tmp_path):
    xr = load_xr()
    path = _write_settings(tmp_path, {"a": _preset(True, [2, 0, 1]), "b": _preset(False), "c": _preset()})
    ctx = xr.Context.from_settings(path, "a")
    assert (ctx.N, ctx.Nd, ctx.V, ctx.C, ctx.K) == (16, 20, 12, 2, 3)
    pre = _preset()
    R = np.array(pre["matrixRot"], np.float32).reshape(3, 9)
    T = np.array(pre["vecTrans"], np.float32).reshape(3, 3) + np.array(pre["areaTrans"], np.float32)
    O = np.array(pre["offset"], np.float32).reshape(3, 3)
    assert np.array_equal(ctx.rot, R[[2, 0]])
    assert np.array_equal(ctx.trans, T[[2, 0]])
    assert np.array_equal(ctx.offset, O[[2, 0]])
    pp, vp, dp, li = ctx.paths()
    assert (pp, vp, dp, li) == ("../p/x", "../v/y", "../d/z", [3, 1])
    ctx.close()
    for tag in ("b", "c"):   # "c" has no "sorting" key: read as false
        ctx = xr.Context.from_settings(path, tag)
        assert np.array_equal(ctx.rot, R[:2]) and np.array_equal(ctx.trans, T[:2])
        assert ctx.paths()[3] == [1, 2]
        ctx.close()


@pytest.mark.skipif(not os.path.exists(REF_SETTINGS), reason="reference settings.json absent")
@pytest.mark.parametrize("tag", ["oilpan", "phaseCT", "cfrp_7d_13rot", "cfrp_7d_6rot", "simulation"])
def test_init_params_on_reference_settings(tag):
    """Every preset of the reference's own settings.json parses as
    init_params would, including `simulation`, which lacks "sorting" (the
    reference throws there, params.cu:69)."""
    xr = load_xr()
    doc = json.load(open(REF_SETTINGS))
    t, rv = doc[tag], doc["recon_variable"]
    C, K = rv["condition"], rv["vector"]
    if len(t["matrixRot"]) < 9 * C and not t.get("sorting", False):
        with pytest.raises(xr.XRError):
            xr.Context.from_settings(REF_SETTINGS, tag)
        return
    ctx = xr.Context.from_settings(REF_SETTINGS, tag)
    vt = np.array(t["vecTrans"], np.float32).reshape(-1, 3)
    vt[: t["rot"]] += np.array(t["areaTrans"], np.float32)
    idx = t["index"][:C] if t.get("sorting", False) else list(range(C))
    assert np.array_equal(ctx.rot, np.array(t["matrixRot"], np.float32).reshape(-1, 9)[idx])
    assert np.array_equal(ctx.trans, vt[idx])
    assert np.array_equal(ctx.offset, np.array(t["offset"], np.float32).reshape(-1, 3)[idx])
    assert np.array_equal(ctx.basis, np.array(rv["base"], np.float32).reshape(-1, 3)[:K])
    assert ctx.sod == np.float32(t["sod"]) and ctx.det == np.float32(t["det_size"])
    assert (ctx.N, ctx.Nd, ctx.V) == (t["num_voxel"], t["num_det_u"], t["proj"])
    ctx.close()


def test_init_params_errors(tmp_path):
    xr = load_xr()
    path = _write_settings(tmp_path, {"a": _preset()})
    with pytest.raises(xr.XRError) as e:
        xr.Context.from_settings(path, "missing_tag")
    assert e.value.status == 6
    with pytest.raises(xr.XRError) as e:
        xr.Context.from_settings(str(tmp_path / "nope.json"), "a")
    assert e.value.status == 5
    bad = tmp_path / "bad.json"
    bad.write_text('{"recon_variable": {"vector": 3,, }')
    with pytest.raises(xr.XRError) as e:
        xr.Context.from_settings(str(bad), "a")
    assert e.value.status == 6
    broken = _preset()
    del broken["sod"]
    path2 = _write_settings(tmp_path, {"a": broken})
    with pytest.raises(xr.XRError):
        xr.Context.from_settings(path2, "a")


def test_create_validates_scan():
    xr = load_xr()
    rot = np.eye(3, dtype=np.float32).ravel()
    ctx = xr.Context.create(1000, 500, 2, 16, 20, 12, rot)
    assert ctx.vs == 1.0 and ctx.K == 1
    ctx.close()
    for bad in [dict(N=0), dict(Nd=1), dict(V=0), dict(sdd=-1)]:
        kw = dict(sdd=1000, sod=500, det=2, N=16, Nd=20, V=12)
        kw.update(bad)
        with pytest.raises(xr.XRError):
            xr.Context.create(kw["sdd"], kw["sod"], kw["det"], kw["N"], kw["Nd"], kw["V"], rot)


def test_null_arguments_rejected():
    xr = load_xr()
    L = xr.lib()
    assert L.xr_create(None, 0, ctypes.byref(ctypes.c_void_p())) == 1
    assert L.xr_init_params(None, b"x", 0, ctypes.byref(ctypes.c_void_p())) == 1
    assert L.xr_dev_session_epoch(None, None) == 1
    rot = np.eye(3, dtype=np.float32).ravel()
    ctx = xr.Context.create(1000, 500, 2, 8, 12, 4, rot)
    assert L.xr_forward(ctx._h, None, None, 0, 0) == 1
    assert L.xr_dev_session_epoch(ctx._h, None) == 8          # XR_ERR_STATE: no session
    assert b"session" in L.xr_last_error(ctx._h)
    ctx.close()


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_device_calls_report_nodev_without_gpu():
    xr = load_xr()
    rot = np.eye(3, dtype=np.float32).ravel()
    ctx = xr.Context.create(1000, 500, 2, 8, 12, 4, rot)
    with pytest.raises(xr.XRError) as e:
        ctx.forward(np.ones((8, 8, 8), np.float32), xtt=False)
    assert e.value.status == 7
    ctx.close()


def test_raw_volume_io(tmp_path):
    xr = load_xr()
    v = xr.Volume(data=np.arange(24, dtype=np.float32).reshape(2, 3, 4))
    assert (v.x(), v.y(), v.z()) == (4, 3, 2)
    assert v(1, 2, 1) == np.float32(1 + 4 * 2 + 12 * 1)        # idx = x + X*y + X*Y*z
    name = str(tmp_path / xr.raw_name("vol", 1, 4, 3, 2))
    assert name.endswith("vol1_4x3x2.raw")
    v.save(name)
    w = xr.Volume()
    w.load(name, 4, 3, 2)
    assert np.array_equal(w.get(), v.get())
    with pytest.raises(IOError):
        w.load(name, 8, 8, 8)


def test_orientation_step_arguments_rejected():
    """The orientation-parametrised and main-direction entry points reject
    null buffers, out-of-range sign patterns and too few basis vectors with
    XR_ERR_ARG (1) / XR_ERR_CONFIG (6) before touching a device."""
    xr = load_xr()
    rot = np.eye(3, dtype=np.float32).ravel()
    basis = np.eye(3, dtype=np.float32)
    ctx = xr.Context.create(1000, 500, 2, 8, 12, 4, rot, basis=basis)
    calls = [lambda: ctx.md_filter(0, 0), lambda: ctx.md_main_direction(0, 0, 0),
             lambda: ctx.md_with_estimate(0, 0, 0), lambda: ctx.md_update_estimation(0, 0, 1),
             lambda: ctx.orth_filter(0, 0, 0), lambda: ctx.orth_update_estimation(0, 0, 1),
             lambda: ctx.orth_normal_update_est(0, 0, 0, 0), lambda: ctx.dev_forward_md(0, 0, 0),
             lambda: ctx.dev_session_begin_md(0, 0, 0, 1, 1), lambda: ctx.md_main_direction(8, 8, 4),
             lambda: ctx.md_filter(8, 8, 1.0, -1)]
    for call in calls:
        with pytest.raises(xr.XRError) as e:
            call()
        assert e.value.status == 1
    ctx.close()
    one = xr.Context.create(1000, 500, 2, 8, 12, 4, rot)            # K = 1
    for call in [lambda: one.md_main_direction(8, 8, 0), lambda: one.orth_update_estimation(8, 8, 0)]:
        with pytest.raises(xr.XRError) as e:
            call()
        assert e.value.status == 6
    one.close()


def test_fiber_arguments_rejected():
    """The fiber-model entry points reject null buffers and negative epoch
    counts with XR_ERR_ARG (1), and K outside {3, 4} or 16-bit volume storage
    with XR_ERR_CONFIG (6), before touching a device."""
    xr = load_xr()
    rot = np.eye(3, dtype=np.float32).ravel()
    ctx = xr.Context.create(1000, 500, 2, 8, 12, 4, rot, basis=np.eye(3, dtype=np.float32))
    for call in [lambda: ctx.dev_forward_fiber(0, 0), lambda: ctx.dev_session_begin_fiber(0, 0, 1, 1),
                 lambda: ctx.fiber_reconstruct(np.zeros((1, 4, 12, 12), np.float32), -1, 1)]:
        with pytest.raises(xr.XRError) as e:
            call()
        assert e.value.status == 1
    ctx.set_option(xr.Option.STORAGE, 1)
    with pytest.raises(xr.XRError) as e:
        ctx.dev_forward_fiber(8, 8)
    assert e.value.status == 6
    ctx.close()
    for K in (1, 13):
        bad = xr.Context.create(1000, 500, 2, 8, 12, 4, rot, basis=np.eye(3, dtype=np.float32)[np.arange(K) % 3])
        for call in [lambda: bad.dev_forward_fiber(8, 8), lambda: bad.dev_session_begin_fiber(8, 8, 1, 1),
                     lambda: bad.fiber_reconstruct(np.zeros((1, 4, 12, 12), np.float32), 1, 1)]:
            with pytest.raises(xr.XRError) as e:
                call()
            assert e.value.status == 6
        bad.close()


def test_axes_one_launch_option_values():
    """XR_OPT_AXES_ONE_LAUNCH takes 0 (a launch per column axis), 1 (one launch
    for all axes) and 2 (automatic, the default); anything else is XR_ERR_ARG."""
    xr = load_xr()
    ctx = xr.Context.create(1000, 500, 2, 8, 12, 4, np.eye(3, dtype=np.float32).ravel())
    for v in (0, 1, 2):
        ctx.set_option(xr.Option.AXES_ONE_LAUNCH, v)
    for v in (-1, 3):
        with pytest.raises(xr.XRError) as e:
            ctx.set_option(xr.Option.AXES_ONE_LAUNCH, v)
        assert e.value.status == 1
    ctx.close()


def test_ratio_texture_option_values():
    """XR_OPT_RATIO_TEXTURE takes 0 or 1 outside a session."""
    xr = load_xr()
    ctx = xr.Context.create(1000, 500, 2, 8, 12, 4, np.eye(3, dtype=np.float32).ravel())
    for v in (0, 1):
        ctx.set_option(xr.Option.RATIO_TEXTURE, v)
    ctx.close()
