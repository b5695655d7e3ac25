"""xray-directional-reconstruction_b200 — Python mirror of the reference's
reconstruction call surface over the C ABI of libxr.so (include/xr.h).

The reference (ixactly/Xray-directional-reconstruction) is C++; its surface is
(reconstruct/include/reconstruct.cuh:14-73, geometry.h, volume.h, params.h):

    init_params(tag)                        -> init_params(tag, json_path)
    Geometry(sdd, sod, detSize, voxel, detect, nProj)
    Volume<float>                           -> Volume (numpy-backed, x fastest)
    IR::reconstruct(sino, voxel, geom, epoch, batch, dir, method, lambda)
    XTT::reconstruct(sino, voxel, md, geom, epoch, batch, dir, method, lambda)
    FDK::reconstruct(sino, voxel, geom, dir)
    forwardProjOnly(sino, voxel, geom, dir)
    calcEigenVector / calcAngleFromMD / directionNormalization (direction/)

Every call runs the sm_100a kernels in libxr.so.  There is no CPU path: if the
library is missing the import fails; if no B200 is present the calls raise.
"""
from __future__ import annotations

import ctypes
import enum
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxr.so")

_F = ctypes.POINTER(ctypes.c_float)
_Fc = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)


class XRError(RuntimeError):
    """A libxr call returned a non-zero xr_status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"libxr status {status} ({STATUS_NAMES.get(status, '?')}): {msg}")
        self.status = status


STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_OOM", 3: "ERR_CUDA", 4: "ERR_TIMEOUT", 5: "ERR_IO",
                6: "ERR_CONFIG", 7: "ERR_NODEV", 8: "ERR_STATE"}


class Method(enum.IntEnum):
    """enum class Method, reconstruct.cuh:14-19."""
    XTT = 0
    MLEM = 1
    ART = 2
    FDK = 3


class Rotate(enum.IntEnum):
    """enum class Rotate, reconstruct.cuh:21-24."""
    CW = 0
    CCW = 1


class Filter(enum.IntEnum):
    REFERENCE = 0
    RAMLAK = 1


class Timing(enum.IntEnum):
    FORWARD = 0
    RATIO = 1
    BACK = 2
    SETUP = 3
    ORIENT = 4
    FDK = 5
    OTHER = 6


class Option(enum.IntEnum):
    TIMING = 1
    FDK_AXIS_BLOCKS = 2
    VIEWS_PER_CTA = 3
    STORAGE = 4
    GRAPHS = 5
    SINO_STORAGE = 6
    ROUNDING = 7
    XTT_SQRT = 8
    AXES_ONE_LAUNCH = 9
    RATIO_TEXTURE = 10


class Storage(enum.IntEnum):
    F32 = 0
    BF16 = 1
    F16 = 2


class _Scan(ctypes.Structure):
    _fields_ = [("sdd", ctypes.c_float), ("sod", ctypes.c_float), ("det_size", ctypes.c_float),
                ("num_voxel", ctypes.c_int), ("num_detect", ctypes.c_int), ("num_proj", ctypes.c_int),
                ("num_cond", ctypes.c_int), ("num_basis", ctypes.c_int),
                ("rot", _F), ("trans", _F), ("offset", _F), ("basis", _F)]


class _Timings(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * 7), ("launches", ctypes.c_long * 7)]


# Exported symbols of include/xr.h with their argument types.
_SIGS = {
    "xr_version": ([], ctypes.c_char_p),
    "xr_create": ([ctypes.POINTER(_Scan), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "xr_init_params": ([ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
                       ctypes.c_int),
    "xr_destroy": ([ctypes.c_void_p], None),
    "xr_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "xr_get_scan": ([ctypes.c_void_p, ctypes.POINTER(_Scan)], ctypes.c_int),
    "xr_get_paths": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_char_p),
                      ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "xr_set_stream": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_set_option": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "xr_get_timings": ([ctypes.c_void_p, ctypes.POINTER(_Timings)], ctypes.c_int),
    "xr_reset_timings": ([ctypes.c_void_p], ctypes.c_int),
    "xr_forward_proj_only": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "xr_forward": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "xr_ir_reconstruct": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                           ctypes.c_int, ctypes.c_int, ctypes.c_float, _F], ctypes.c_int),
    "xr_xtt_reconstruct": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, _F],
                           ctypes.c_int),
    "xr_fdk_reconstruct": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
                           ctypes.c_int),
    "xr_fiber_reconstruct": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_float, _F], ctypes.c_int),
    "xr_dev_forward_fiber": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "xr_dev_session_begin_fiber": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_float], ctypes.c_int),
    "xr_orientation": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_angle_from_md": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_direction_normalization": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_residual": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D, _D],
                    ctypes.c_int),
    "xr_dev_forward": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
                       ctypes.c_int),
    "xr_dev_residual": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D, _D],
                        ctypes.c_int),
    "xr_dev_orientation": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_dev_session_begin": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float], ctypes.c_int),
    "xr_dev_session_epoch": ([ctypes.c_void_p, _D], ctypes.c_int),
    "xr_dev_session_end": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_dev_session_proj": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "xr_dev_forward_proj_only_static": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p], ctypes.c_int),
    "xr_dev_forward_orth": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int],
                            ctypes.c_int),
    "xr_dev_session_begin_orth": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float], ctypes.c_int),
    "xr_orth_normal_update": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int],
                              ctypes.c_int),
    "xr_orth_normal_update_est": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p], ctypes.c_int),
    "xr_orth_filter": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                        ctypes.c_int], ctypes.c_int),
    "xr_orth_update_estimation": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "xr_dev_forward_md": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int],
                          ctypes.c_int),
    "xr_dev_session_begin_md": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float], ctypes.c_int),
    "xr_md_filter": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_int], ctypes.c_int),
    "xr_md_main_direction": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "xr_md_with_estimate": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_md_update_estimation": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "xr_dev_fill": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float], ctypes.c_int),
    "xr_tv_minimize": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                        ctypes.c_float, ctypes.c_int], ctypes.c_int),
    "xr_quad_form_filter": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                             ctypes.c_int, ctypes.c_float], ctypes.c_int),
    "xr_tv_minimize_host": ([ctypes.c_int, _F, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                             ctypes.c_float, ctypes.c_int], ctypes.c_int),
    "xr_quad_form_filter_host": ([ctypes.c_int, ctypes.POINTER(_F), ctypes.POINTER(_F), ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_float], ctypes.c_int),
    "xr_batch_create": ([ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
                        ctypes.c_int),
    "xr_batch_destroy": ([ctypes.c_void_p], None),
    "xr_batch_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "xr_batch_session_begin": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_float], ctypes.c_int),
    "xr_batch_epoch": ([ctypes.c_void_p, _D], ctypes.c_int),
    "xr_batch_session_end": ([ctypes.c_void_p], ctypes.c_int),
    "xr_batch_autotune": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "xr_batch_autotune_shapes": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
                                 ctypes.c_int),
    # include/xr_learn.h
    "xr_net_create": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                       ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "xr_net_destroy": ([ctypes.c_void_p], None),
    "xr_net_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "xr_net_set_stream": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "xr_net_num_params": ([ctypes.c_void_p], ctypes.c_size_t),
    "xr_net_get_params": ([ctypes.c_void_p, _F, ctypes.c_size_t], ctypes.c_int),
    "xr_net_set_params": ([ctypes.c_void_p, _F, ctypes.c_size_t], ctypes.c_int),
    "xr_net_save": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "xr_net_load": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "xr_net_infer": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                      ctypes.c_int, ctypes.c_float, ctypes.c_float], ctypes.c_int),
    "xr_net_loss_grad": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_float, _D, _F], ctypes.c_int),
    "xr_net_adam_step": ([ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float],
                         ctypes.c_int),
    "xr_net_set_tensor_loss": ([ctypes.c_void_p, _F, ctypes.c_float], ctypes.c_int),
    "xr_conv3d_fprop": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                         ctypes.c_int], ctypes.c_int),
    "xr_dev_fiber_phantom": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, _F, ctypes.c_void_p],
                             ctypes.c_int),
    "xr_conv3d_wgrad": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
}

_lib = None


def build(force: bool = False) -> str:
    """Compile libxr.so in place (nvcc, sm_100a)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_xr_build", os.path.join(HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


def lib() -> ctypes.CDLL:
    """The loaded libxr.so.  Raises if it has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libxr.so not built ({LIB_PATH}); run build() or "
                               "python xray-directional-reconstruction_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _f32(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


def _ptrs(arrs: Sequence[np.ndarray]):
    return (_F * len(arrs))(*[a.ctypes.data_as(_F) for a in arrs])


class Geometry:
    """Geometry(sdd, sod, detSize, voxel, detect, nProj), geometry.h:8-25;
    voxSize = sod*detSize/sdd in float32 (geometry.h:13)."""

    def __init__(self, sdd: float, sod: float, detSize: float, voxel: int, detect: int, nProj: int):
        self.sdd = float(np.float32(sdd))
        self.sod = float(np.float32(sod))
        self.detSize = float(np.float32(detSize))
        self.voxel = int(voxel)
        self.detect = int(detect)
        self.nProj = int(nProj)
        self.voxSize = float(np.float32(np.float32(sod) * np.float32(detSize)) / np.float32(sdd))


class Volume:
    """Volume<float> (volume.h:18-165): a host 3-D float array, x fastest
    (idx = x + X*y + X*Y*z).  Backed by a numpy array of shape (z, y, x)."""

    def __init__(self, x: int = 0, y: int = 0, z: int = 0, data: Optional[np.ndarray] = None):
        if data is not None:
            self.data = _f32(data)
            if self.data.ndim != 3:
                raise ValueError("Volume data must be 3-D (z, y, x)")
        else:
            self.data = np.zeros((z, y, x), np.float32)

    def x(self) -> int: return self.data.shape[2]
    def y(self) -> int: return self.data.shape[1]
    def z(self) -> int: return self.data.shape[0]
    def get(self) -> np.ndarray: return self.data

    def __call__(self, x, y, z):
        return self.data[z, y, x]

    def load(self, filename: str, x: int, y: int, z: int) -> None:
        """volume.h:105-120: raw float32, x fastest.  Raises on a missing or
        short file (the reference prints and continues with garbage)."""
        raw = np.fromfile(filename, dtype=np.float32)
        if raw.size < x * y * z:
            raise IOError(f"{filename}: {raw.size} floats, need {x * y * z}")
        self.data = raw[: x * y * z].reshape(z, y, x).copy()

    def save(self, filename: str) -> None:
        """volume.h:122-132."""
        self.data.tofile(filename)

    def forEach(self, f) -> None:
        """volume.h:139-148 (vectorised: f must accept numpy arrays)."""
        self.data = _f32(f(self.data))

    def mean(self) -> float:
        return float(self.data.astype(np.float64).mean())


def raw_name(prefix: str, index: int, x: int, y: int, z: int) -> str:
    """The reference's raw file naming <prefix><i>_<X>x<Y>x<Z>.raw (main.cu:31-32,86-97)."""
    return f"{prefix}{index}_{x}x{y}x{z}.raw"


class Context:
    """An xr_ctx: scan geometry, per-axis rotation/offsets and the scattering
    basis (the reference's globals), plus the device workspace."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle
        s = _Scan()
        self._check(lib().xr_get_scan(self._h, ctypes.byref(s)))
        self.sdd, self.sod, self.det = s.sdd, s.sod, s.det_size
        self.N, self.Nd, self.V, self.C, self.K = s.num_voxel, s.num_detect, s.num_proj, s.num_cond, s.num_basis
        self.rot = np.ctypeslib.as_array(s.rot, (self.C * 9,)).copy().reshape(self.C, 9)
        self.trans = np.ctypeslib.as_array(s.trans, (self.C * 3,)).copy().reshape(self.C, 3)
        self.offset = np.ctypeslib.as_array(s.offset, (self.C * 3,)).copy().reshape(self.C, 3)
        self.basis = np.ctypeslib.as_array(s.basis, (self.K * 3,)).copy().reshape(self.K, 3)

    # ---- construction
    @classmethod
    def create(cls, sdd, sod, det, N, Nd, V, rot, trans=None, offset=None, basis=None, device: int = 0):
        rot = _f32(rot).reshape(-1, 9)
        C = rot.shape[0]
        trans = _f32(np.zeros((C, 3)) if trans is None else trans).reshape(C, 3)
        offset = _f32(np.zeros((C, 3)) if offset is None else offset).reshape(C, 3)
        basis = _f32(np.array([[0, 0, 1.0]]) if basis is None else basis).reshape(-1, 3)
        s = _Scan(float(sdd), float(sod), float(det), int(N), int(Nd), int(V), C, basis.shape[0],
                  rot.ctypes.data_as(_F), trans.ctypes.data_as(_F), offset.ctypes.data_as(_F),
                  basis.ctypes.data_as(_F))
        h = ctypes.c_void_p()
        st = lib().xr_create(ctypes.byref(s), int(device), ctypes.byref(h))
        if st:
            raise XRError(st, "xr_create rejected the scan")
        return cls(h)

    @classmethod
    def from_settings(cls, json_path: str, tag: str, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().xr_init_params(json_path.encode(), tag.encode(), int(device), ctypes.byref(h))
        if st:
            raise XRError(st, f"init_params({tag!r}) from {json_path}")
        return cls(h)

    def close(self):
        if getattr(self, "_h", None):
            lib().xr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st:
            msg = lib().xr_last_error(self._h)
            raise XRError(st, msg.decode() if msg else "")

    # ---- introspection
    @property
    def vs(self) -> float:
        return float(np.float32(np.float32(self.sod) * np.float32(self.det)) / np.float32(self.sdd))

    def paths(self):
        pp, vp, dp = ctypes.c_char_p(), ctypes.c_char_p(), ctypes.c_char_p()
        li = (ctypes.c_int * self.C)()
        self._check(lib().xr_get_paths(self._h, ctypes.byref(pp), ctypes.byref(vp), ctypes.byref(dp), li))
        return pp.value.decode(), vp.value.decode(), dp.value.decode(), list(li)

    def set_option(self, key: int, value: int):
        self._check(lib().xr_set_option(self._h, int(key), int(value)))

    def set_stream(self, stream_ptr: int):
        self._check(lib().xr_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def timings(self):
        t = _Timings()
        self._check(lib().xr_get_timings(self._h, ctypes.byref(t)))
        return {Timing(k).name.lower(): (t.ms[k], t.launches[k]) for k in range(7)}

    def reset_timings(self):
        self._check(lib().xr_reset_timings(self._h))

    # ---- host-buffer calls (numpy); volumes (.., N, N, N) z-major, sinograms (C, V, Nd, Nd)
    def _vols(self, vol, n):
        v = _f32(vol).reshape(n, self.N, self.N, self.N)
        return [v[i] for i in range(n)]

    def forward(self, vol, xtt: bool, rotate: int = Rotate.CW) -> np.ndarray:
        vols = self._vols(vol, self.K if xtt else 1)
        out = np.zeros((self.C, self.V, self.Nd, self.Nd), np.float32)
        self._check(lib().xr_forward(self._h, _ptrs(vols), _ptrs([out[c] for c in range(self.C)]), int(rotate),
                                     int(bool(xtt))))
        return out

    def forward_proj_only(self, vol, rotate: int = Rotate.CW) -> np.ndarray:
        vols = self._vols(vol, 1)
        out = np.zeros((self.C, self.V, self.Nd, self.Nd), np.float32)
        self._check(lib().xr_forward_proj_only(self._h, _ptrs(vols), _ptrs([out[c] for c in range(self.C)]),
                                               int(rotate)))
        return out

    def ir_reconstruct(self, sino, vol, epoch, batch, rotate=Rotate.CW, method=Method.MLEM, lam=1e-2):
        """Returns (volumes (C, N, N, N), losses (C, epoch))."""
        sino = _f32(sino).reshape(self.C, self.V, self.Nd, self.Nd).copy()
        vols = _f32(vol).reshape(self.C, self.N, self.N, self.N).copy()
        losses = np.zeros(self.C * max(epoch, 1), np.float32)
        self._check(lib().xr_ir_reconstruct(self._h, _ptrs([sino[c] for c in range(self.C)]),
                                            _ptrs([vols[c] for c in range(self.C)]), int(epoch), int(batch),
                                            int(rotate), int(method), float(lam), losses.ctypes.data_as(_F)))
        return vols, losses[: self.C * epoch].reshape(self.C, epoch)

    def xtt_reconstruct(self, sino, vol, epoch, batch, rotate=Rotate.CW, method=Method.MLEM, lam=1e-2,
                        orientation: bool = True):
        """Returns (mu (K, N, N, N) after sqrt, last ratio images (C, V, Nd, Nd),
        md (3, N, N, N) or None, evalue (3, N, N, N) or None, losses (epoch,))."""
        sino = _f32(sino).reshape(self.C, self.V, self.Nd, self.Nd).copy()
        vols = _f32(vol).reshape(self.K, self.N, self.N, self.N).copy()
        md = np.zeros((3, self.N, self.N, self.N), np.float32) if orientation else None
        ev = np.zeros((3, self.N, self.N, self.N), np.float32) if orientation else None
        losses = np.zeros(max(epoch, 1), np.float32)
        self._check(lib().xr_xtt_reconstruct(
            self._h, _ptrs([sino[c] for c in range(self.C)]), _ptrs([vols[k] for k in range(self.K)]),
            _ptrs([md[i] for i in range(3)]) if orientation else None,
            _ptrs([ev[i] for i in range(3)]) if orientation else None,
            int(epoch), int(batch), int(rotate), int(method), float(lam), losses.ctypes.data_as(_F)))
        return vols, sino, md, ev, losses[:epoch]

    def fiber_reconstruct(self, sino, epoch, batch, rotate=Rotate.CW, method=Method.MLEM, lam=1e-2):
        """XTT::fiberModelReconstruct (reconstruct.cu:1242-1371): every channel
        starts at 0.01.  Returns (volume (K, N, N, N), last ratio images
        (C, V, Nd, Nd), losses (epoch,))."""
        sino = _f32(sino).reshape(self.C, self.V, self.Nd, self.Nd).copy()
        vols = np.zeros((self.K, self.N, self.N, self.N), np.float32)
        losses = np.zeros(max(epoch, 1), np.float32)
        self._check(lib().xr_fiber_reconstruct(self._h, _ptrs([sino[c] for c in range(self.C)]),
                                               _ptrs([vols[k] for k in range(self.K)]), int(epoch), int(batch),
                                               int(rotate), int(method), float(lam), losses.ctypes.data_as(_F)))
        return vols, sino, losses[:epoch]

    def fdk_reconstruct(self, sino, rotate=Rotate.CW, filt=Filter.REFERENCE):
        """Returns (volumes (C, N, N, N), filtered sinograms (C, V, Nd, Nd))."""
        sino = _f32(sino).reshape(self.C, self.V, self.Nd, self.Nd).copy()
        vols = np.zeros((self.C, self.N, self.N, self.N), np.float32)
        self._check(lib().xr_fdk_reconstruct(self._h, _ptrs([sino[c] for c in range(self.C)]),
                                             _ptrs([vols[c] for c in range(self.C)]), int(rotate), int(filt)))
        return vols, sino

    def orientation(self, mu):
        mus = self._vols(mu, self.K)
        md = np.zeros((3, self.N, self.N, self.N), np.float32)
        ev = np.zeros((3, self.N, self.N, self.N), np.float32)
        self._check(lib().xr_orientation(self._h, _ptrs(mus), _ptrs([md[i] for i in range(3)]),
                                         _ptrs([ev[i] for i in range(3)])))
        return md, ev

    def angle_from_md(self, md):
        mds = self._vols(md, 3)
        ang = np.zeros((2, self.N, self.N, self.N), np.float32)
        self._check(lib().xr_angle_from_md(self._h, _ptrs(mds), _ptrs([ang[0], ang[1]])))
        return ang

    def direction_normalization(self, md):
        m = _f32(md).reshape(3, self.N, self.N, self.N).copy()
        self._check(lib().xr_direction_normalization(self._h, _ptrs([m[i] for i in range(3)])))
        return m

    def residual(self, vol, sino, xtt: bool, rotate=Rotate.CW):
        vols = self._vols(vol, self.K if xtt else 1)
        s = _f32(sino).reshape(self.C, self.V, self.Nd, self.Nd)
        r, l1 = ctypes.c_double(), ctypes.c_double()
        self._check(lib().xr_residual(self._h, _ptrs(vols), _ptrs([s[c] for c in range(self.C)]), int(rotate),
                                      int(bool(xtt)), ctypes.byref(r), ctypes.byref(l1)))
        return r.value, l1.value

    # ---- device-buffer calls (raw device pointers, e.g. torch tensor.data_ptr())
    def dev_forward(self, d_vol: int, d_sino: int, xtt: bool, rotate=Rotate.CW):
        self._check(lib().xr_dev_forward(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_sino), int(rotate),
                                         int(bool(xtt))))

    def dev_orientation(self, d_mu: int, d_md: int, d_ev: int = 0):
        """calcEigenVector (pca.cu:12-55) of every voxel: d_mu K planes of the
        storage type, d_md three FP32 planes, d_ev three FP32 planes or 0."""
        self._check(lib().xr_dev_orientation(self._h, ctypes.c_void_p(d_mu), ctypes.c_void_p(d_md),
                                             ctypes.c_void_p(d_ev or None)))

    def dev_residual(self, d_vol: int, d_sino: int, xtt: bool, rotate=Rotate.CW):
        r, l1 = ctypes.c_double(), ctypes.c_double()
        self._check(lib().xr_dev_residual(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_sino), int(rotate),
                                          int(bool(xtt)), ctypes.byref(r), ctypes.byref(l1)))
        return r.value, l1.value

    def dev_session_begin(self, d_sino: int, d_vol: int, xtt: bool, epochs: int, batch: int, rotate=Rotate.CW,
                          method=Method.MLEM, lam=1e-2):
        self._check(lib().xr_dev_session_begin(self._h, ctypes.c_void_p(d_sino), ctypes.c_void_p(d_vol),
                                               int(bool(xtt)), int(epochs), int(batch), int(rotate), int(method),
                                               float(lam)))

    def dev_forward_orth(self, d_vol: int, d_coef: int, d_sino: int, rotate=Rotate.CW):
        """forwardOrth over every axis and view (ir.cu:294-364), device buffers."""
        self._check(lib().xr_dev_forward_orth(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_coef),
                                              ctypes.c_void_p(d_sino), int(rotate)))

    def dev_session_begin_orth(self, d_sino: int, d_vol: int, d_coef: int, epochs: int, batch: int,
                               rotate=Rotate.CW, method=Method.MLEM, lam=1e-2):
        """Orientation-parametrised XTT session (forwardOrth / backwardOrth)."""
        self._check(lib().xr_dev_session_begin_orth(self._h, ctypes.c_void_p(d_sino), ctypes.c_void_p(d_vol),
                                                    ctypes.c_void_p(d_coef), int(epochs), int(batch), int(rotate),
                                                    int(method), float(lam)))

    def orth_normal_update(self, d_vol: int, d_coef: int, d_loss: int, rot: int = 0):
        """calcNormalVectorThreeDirec (ir.cu:856-974) on device buffers."""
        self._check(lib().xr_orth_normal_update(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_coef),
                                                ctypes.c_void_p(d_loss), int(rot)))

    def orth_normal_update_est(self, d_vol: int, d_coef: int, d_loss: int, d_est: int):
        """calcNormalVectorThreeDirecWithEst (ir.cu:976-1071) on device buffers."""
        self._check(lib().xr_orth_normal_update_est(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_coef),
                                                    ctypes.c_void_p(d_loss), ctypes.c_void_p(d_est)))

    def orth_filter(self, d_coef: int, d_tmp: int, d_vol: int, weight: float = 1.0, passes: int = 1):
        """meanFiltFiber (ir.cu:1231-1302), `passes` times, on device planes."""
        self._check(lib().xr_orth_filter(self._h, ctypes.c_void_p(d_coef), ctypes.c_void_p(d_tmp),
                                         ctypes.c_void_p(d_vol), float(weight), int(passes)))

    def orth_update_estimation(self, d_vol: int, d_est: int, iteration: int):
        """updateEstimationByCoef (ir.cu:1073-1120)."""
        self._check(lib().xr_orth_update_estimation(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_est),
                                                    int(iteration)))

    def dev_forward_fiber(self, d_vol: int, d_sino: int, rotate=Rotate.CW):
        """forwardProjFiber (fiber.cu:13-153) over every axis and view, device buffers."""
        self._check(lib().xr_dev_forward_fiber(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_sino),
                                               int(rotate)))

    def dev_session_begin_fiber(self, d_sino: int, d_vol: int, epochs: int, batch: int, rotate=Rotate.CW,
                                method=Method.MLEM, lam=1e-2):
        """fiberModelReconstruct's epochs as a session (channel 0 updated)."""
        self._check(lib().xr_dev_session_begin_fiber(self._h, ctypes.c_void_p(d_sino), ctypes.c_void_p(d_vol),
                                                     int(epochs), int(batch), int(rotate), int(method), float(lam)))

    def dev_forward_md(self, d_vol: int, d_md: int, d_sino: int, rotate=Rotate.CW):
        """forwardOrthByMD + chord normalisation over every axis and view (ir.cu:154-231)."""
        self._check(lib().xr_dev_forward_md(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_md),
                                            ctypes.c_void_p(d_sino), int(rotate)))

    def dev_session_begin_md(self, d_sino: int, d_vol: int, d_md: int, epochs: int, batch: int,
                             rotate=Rotate.CW, method=Method.MLEM, lam=1e-2):
        """Main-direction XTT session (circleEstReconstruct's inner epochs)."""
        self._check(lib().xr_dev_session_begin_md(self._h, ctypes.c_void_p(d_sino), ctypes.c_void_p(d_vol),
                                                  ctypes.c_void_p(d_md), int(epochs), int(batch), int(rotate),
                                                  int(method), float(lam)))

    def md_filter(self, d_md: int, d_tmp: int, weight: float = 1.0, passes: int = 1):
        """meanFiltFiberMD (ir.cu:1304-1363), `passes` times, on device planes."""
        self._check(lib().xr_md_filter(self._h, ctypes.c_void_p(d_md), ctypes.c_void_p(d_tmp), float(weight),
                                       int(passes)))

    def md_main_direction(self, d_vol: int, d_md: int, iteration: int = 0):
        """calcMainDirection (ir.cu:624-710)."""
        self._check(lib().xr_md_main_direction(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_md),
                                               int(iteration)))

    def md_with_estimate(self, d_vol: int, d_md: int, d_est: int):
        """calcMDWithEst (ir.cu:712-789)."""
        self._check(lib().xr_md_with_estimate(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_md),
                                              ctypes.c_void_p(d_est)))

    def md_update_estimation(self, d_vol: int, d_est: int, iteration: int):
        """updateEstimation (ir.cu:791-844)."""
        self._check(lib().xr_md_update_estimation(self._h, ctypes.c_void_p(d_vol), ctypes.c_void_p(d_est),
                                                  int(iteration)))

    def dev_fill(self, d: int, n: int, value: float):
        """fillVolume (ir.cu:846-854): n device floats <- value."""
        self._check(lib().xr_dev_fill(self._h, ctypes.c_void_p(d), ctypes.c_size_t(n), float(value)))

    def dev_session_epoch(self, want_loss: bool = False):
        if not want_loss:
            self._check(lib().xr_dev_session_epoch(self._h, None))
            return None
        buf = (ctypes.c_double * 32)()
        self._check(lib().xr_dev_session_epoch(self._h, buf))
        return list(buf)

    def dev_session_end(self, d_md: int = 0, d_ev: int = 0):
        self._check(lib().xr_dev_session_end(self._h, ctypes.c_void_p(d_md or None), ctypes.c_void_p(d_ev or None)))

    def dev_session_proj(self) -> int:
        p = ctypes.c_void_p()
        self._check(lib().xr_dev_session_proj(self._h, ctypes.byref(p)))
        return p.value


# ---------------------------------------------------------------------------
# The reference's free-function surface, driven by a module-level context (the
# reference keeps these as globals filled by init_params, params.cu:14-40).

_ctx: Optional[Context] = None


def init_params(tag: str, json_path: str, device: int = 0) -> Context:
    """init_params(tag), params.cu:42-104 (the path is an argument here)."""
    global _ctx
    if _ctx is not None:
        _ctx.close()
    _ctx = Context.from_settings(json_path, tag, device)
    return _ctx


def _need_ctx() -> Context:
    if _ctx is None:
        raise RuntimeError("call init_params(tag, json_path) first")
    return _ctx


def _check_geom(ctx: Context, geom: Geometry):
    if (geom.voxel, geom.detect, geom.nProj) != (ctx.N, ctx.Nd, ctx.V):
        raise ValueError("Geometry does not match the settings loaded by init_params")


class IR:
    @staticmethod
    def reconstruct(sinogram: Sequence[Volume], voxel: Sequence[Volume], geom: Geometry, epoch: int, batch: int,
                    dir: Rotate, method: Method, lambda_: float = 1e-2) -> np.ndarray:
        """IR::reconstruct (reconstruct.cu:23-156): voxel[cond] updated in place.
        Returns the loss sums (C, epoch)."""
        ctx = _need_ctx()
        _check_geom(ctx, geom)
        sino = np.stack([s.get() for s in sinogram[: ctx.C]])
        vol = np.stack([v.get() for v in voxel[: ctx.C]])
        out, losses = ctx.ir_reconstruct(sino, vol, epoch, batch, dir, method, lambda_)
        for c in range(ctx.C):
            voxel[c].data = out[c]
        return losses


class XTT:
    @staticmethod
    def reconstruct(sinogram: Sequence[Volume], voxel: Sequence[Volume], md: Optional[Sequence[Volume]],
                    geom: Geometry, epoch: int, batch: int, dir: Rotate, method: Method,
                    lambda_: float = 1e-2) -> np.ndarray:
        """XTT::reconstruct (reconstruct.cu:799-954): voxel[k] <- sqrt|mu_k|,
        md[0..2] <- fiber direction, sinogram[c] <- last ratio images."""
        ctx = _need_ctx()
        _check_geom(ctx, geom)
        sino = np.stack([s.get() for s in sinogram[: ctx.C]])
        vol = np.stack([v.get() for v in voxel[: ctx.K]])
        mu, ratio, m, _, losses = ctx.xtt_reconstruct(sino, vol, epoch, batch, dir, method, lambda_,
                                                      orientation=md is not None)
        for k in range(ctx.K):
            voxel[k].data = mu[k]
        for c in range(ctx.C):
            sinogram[c].data = ratio[c]
        if md is not None:
            for i in range(3):
                md[i].data = m[i]
        return losses


class FDK:
    @staticmethod
    def reconstruct(sinogram: Sequence[Volume], voxel: Sequence[Volume], geom: Geometry, dir: Rotate,
                    filt: Filter = Filter.REFERENCE) -> None:
        """FDK::reconstruct (reconstruct.cu:1651-1724)."""
        ctx = _need_ctx()
        _check_geom(ctx, geom)
        sino = np.stack([s.get() for s in sinogram[: ctx.C]])
        vols, filtered = ctx.fdk_reconstruct(sino, dir, filt)
        for c in range(ctx.C):
            voxel[c].data = vols[c]
            sinogram[c].data = filtered[c]


def forwardProjOnly(sinogram: Sequence[Volume], voxel: Sequence[Volume], geom: Geometry, dir: Rotate) -> None:
    """forwardProjOnly (reconstruct.cu:1890-1949)."""
    ctx = _need_ctx()
    _check_geom(ctx, geom)
    out = ctx.forward_proj_only(voxel[0].get(), dir)
    for c in range(ctx.C):
        sinogram[c].data = out[c]


def calcEigenVectorAll(ct: Sequence[Volume], md: Sequence[Volume], evalue: Sequence[Volume]) -> None:
    """calcEigenVector (direction/src/pca.cu:12-55) for every voxel at once."""
    ctx = _need_ctx()
    m, e = ctx.orientation(np.stack([v.get() for v in ct[: ctx.K]]))
    for i in range(3):
        md[i].data = m[i]
        evalue[i].data = e[i]


def calcAngleFromMD(md: Sequence[Volume], angle: Sequence[Volume]) -> None:
    """calcAngleFromMD (direction/src/pca.cu:67-83)."""
    ctx = _need_ctx()
    a = ctx.angle_from_md(np.stack([v.get() for v in md[:3]]))
    angle[0].data, angle[1].data = a[0], a[1]


def directionNormalization(md: Sequence[Volume]) -> None:
    """directionNormalization (direction/src/pca.cu:85-106)."""
    ctx = _need_ctx()
    m = ctx.direction_normalization(np.stack([v.get() for v in md[:3]]))
    for i in range(3):
        md[i].data = m[i]


def totalVariationMinimized(vol: Volume, rho: float, lam: float, iters: int, device: int = 0) -> None:
    """totalVariationMinimized (solver/src/tvmin.cpp:6-98), in place, on the GPU."""
    a = _f32(vol.get()).copy()
    Z, Y, X = a.shape
    st = lib().xr_tv_minimize_host(int(device), a.ctypes.data_as(_F), X, Y, Z, float(rho), float(lam), int(iters))
    if st:
        raise XRError(st, "xr_tv_minimize_host")
    vol.data = a


def quadlicFormFilterCPU(voxel: Sequence[Volume], coefficient: Sequence[Volume], lam: float,
                         device: int = 0) -> None:
    """quadlicFormFilterCPU (reconstruct/src/quadfilt.cpp:11-134), in place, on the GPU."""
    v = [_f32(x.get()).copy() for x in voxel[:3]]
    c = [_f32(x.get()).copy() for x in coefficient[:2]]
    Z, Y, X = v[0].shape
    st = lib().xr_quad_form_filter_host(int(device), _ptrs(v), _ptrs(c), X, Y, Z, float(lam))
    if st:
        raise XRError(st, "xr_quad_form_filter_host")
    for i in range(3):
        voxel[i].data = v[i]
    for i in range(2):
        coefficient[i].data = c[i]


def version() -> str:
    return lib().xr_version().decode()


class Batch:
    """Several specimens' OS-EM sessions run together (xr_batch_*): one epoch
    of every specimen per call, their kernels overlapping on the GPU, the
    whole multi-specimen epoch replayed as one CUDA graph when the first
    context has Option.GRAPHS set.  Holds references to the contexts."""

    def __init__(self, contexts: Sequence["Context"]):
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[c._h for c in self.contexts])
        h = ctypes.c_void_p()
        st = lib().xr_batch_create(arr, len(self.contexts), ctypes.byref(h))
        if st:
            raise XRError(st, "xr_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().xr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st:
            msg = lib().xr_batch_last_error(self._h)
            raise XRError(st, msg.decode() if msg else "")

    def session_begin(self, d_sinos, d_vols, xtt: bool, epochs: int, subsets: int, rotate: int = 0,
                      method: int = 1, lam: float = 1e-2):
        n = len(self.contexts)
        s = (ctypes.c_void_p * n)(*[int(p) for p in d_sinos])
        v = (ctypes.c_void_p * n)(*[int(p) for p in d_vols])
        self._check(lib().xr_batch_session_begin(self._h, s, v, int(xtt), int(epochs), int(subsets), int(rotate),
                                                 int(method), float(lam)))

    def epoch(self) -> np.ndarray:
        loss = np.zeros(len(self.contexts), np.float64)
        self._check(lib().xr_batch_epoch(self._h, loss.ctypes.data_as(_D)))
        return loss

    def session_end(self):
        self._check(lib().xr_batch_session_end(self._h))

    def autotune(self) -> list:
        out = (ctypes.c_int * len(self.contexts))()
        self._check(lib().xr_batch_autotune(self._h, out))
        return list(out)

    def autotune_shapes(self):
        """(views per CTA, axes in one launch 0 / 1) chosen per specimen."""
        vpc = (ctypes.c_int * len(self.contexts))()
        shape = (ctypes.c_int * len(self.contexts))()
        self._check(lib().xr_batch_autotune_shapes(self._h, vpc, shape))
        return list(vpc), list(shape)


# ---------------------------------------------------------------------------
# Learned warm start (include/xr_learn.h; no counterpart in the reference)
# ---------------------------------------------------------------------------

class Net:
    """The warm-start network: depth 3x3x3 convolutions of `width` channels
    on K-channel volumes, y = x + net(s*x)/s, trained and run on the tensor
    cores by libxr.  Device buffers are passed as raw pointers (e.g.
    torch.Tensor.data_ptr())."""

    def __init__(self, channels: int = 13, width: int = 32, depth: int = 4, seed: int = 0, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().xr_net_create(int(device), int(channels), int(width), int(depth), int(seed), ctypes.byref(h))
        if st:
            raise XRError(st, "xr_net_create")
        self._h = h
        self.channels, self.width, self.depth = channels, width, depth

    def close(self):
        if getattr(self, "_h", None):
            lib().xr_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st:
            msg = lib().xr_net_last_error(self._h)
            raise XRError(st, msg.decode() if msg else "")

    def set_stream(self, stream_handle: int):
        self._check(lib().xr_net_set_stream(self._h, ctypes.c_void_p(stream_handle)))

    @property
    def num_params(self) -> int:
        return int(lib().xr_net_num_params(self._h))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.num_params, np.float32)
        self._check(lib().xr_net_get_params(self._h, p.ctypes.data_as(_F), p.size))
        return p

    def set_params(self, p) -> None:
        p = _f32(p).ravel()
        self._check(lib().xr_net_set_params(self._h, p.ctypes.data_as(_F), p.size))

    def save(self, path: str) -> None:
        self._check(lib().xr_net_save(self._h, path.encode()))

    def load(self, path: str) -> None:
        self._check(lib().xr_net_load(self._h, path.encode()))

    def infer(self, d_in: int, d_out: int, shape, storage: int = 0, in_scale: float = 1.0,
              floor_value: float = 0.0) -> None:
        """d_out = max(net(d_in), floor_value); shape = (nz, ny, nx) of each
        of the K planes; storage 0 FP32, 1 BF16, 2 FP16."""
        nz, ny, nx = shape
        self._check(lib().xr_net_infer(self._h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), int(storage), nx, ny,
                                       nz, float(in_scale), float(floor_value)))

    def loss_grad(self, d_in: int, d_target: int, shape, in_scale: float = 1.0, want_grad: bool = False):
        """(loss, gradient or None) of the FP32 device volumes; the gradient
        stays on the device for adam_step."""
        nz, ny, nx = shape
        loss = ctypes.c_double()
        g = np.empty(self.num_params, np.float32) if want_grad else None
        self._check(lib().xr_net_loss_grad(self._h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_target), nx, ny, nz,
                                           float(in_scale), ctypes.byref(loss),
                                           g.ctypes.data_as(_F) if g is not None else None))
        return loss.value, g

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self._check(lib().xr_net_adam_step(self._h, float(lr), float(beta1), float(beta2), float(eps)))

    def set_tensor_loss(self, basis, weight: float) -> None:
        """Adds weight * ||T(pred) - T(target)||_F^2 per voxel to the training
        loss, T(mu) = sum_k mu_k S_k S_k^T (the tensor of the main direction);
        basis: K x 3 scattering vectors; weight 0 turns it off."""
        b = _f32(np.zeros((0, 3)) if basis is None else basis).reshape(-1, 3)
        if basis is not None and b.shape[0] < self.channels:
            raise ValueError("the tensor loss needs one basis vector per channel")
        self._check(lib().xr_net_set_tensor_loss(self._h, b.ctypes.data_as(_F) if b.size else None, float(weight)))


def conv3d_fprop(x: int, cin: int, w: int, bias: int, mask: int, y: int, cout: int, shape, epilogue: int,
                 stream: int = 0) -> None:
    """Layer-level tensor-core convolution (device pointers, BF16 channels-last)."""
    nz, ny, nx = shape
    st = lib().xr_conv3d_fprop(ctypes.c_void_p(stream), ctypes.c_void_p(x), cin, ctypes.c_void_p(w),
                               ctypes.c_void_p(bias or None), ctypes.c_void_p(mask or None), ctypes.c_void_p(y),
                               cout, nx, ny, nz, epilogue)
    if st:
        raise XRError(st, "xr_conv3d_fprop")


def conv3d_wgrad(x: int, cin: int, dy: int, cout: int, dw: int, shape, stream: int = 0) -> None:
    """Layer-level weight gradient, accumulated into the FP32 dw[27][cout][cin]."""
    nz, ny, nx = shape
    st = lib().xr_conv3d_wgrad(ctypes.c_void_p(stream), ctypes.c_void_p(x), cin, ctypes.c_void_p(dy), cout,
                               ctypes.c_void_p(dw), nx, ny, nz)
    if st:
        raise XRError(st, "xr_conv3d_wgrad")
