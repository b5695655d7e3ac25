"""ctypes front-end of the checkers — TEST INFRASTRUCTURE ONLY.

`Oracle` wraps oracle/liboracle.so, the project's CPU restatement of the
reference's reconstruction path (FP32 in the reference's operation order, and
FP64).  `RefHost` wraps oracle/_ref/libxrref.so, the reference's own
reconstruct/src/ir.cu compiled for the host through oracle/ref_shim.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only to check or to time the reference; the product never
does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def reference_root() -> str:
    """The reference checkout oracle/Makefile builds from (XR_REFERENCE, else
    the recipe's default); it may be absent (e.g. where only the prebuilt
    checkers travel)."""
    if os.environ.get("XR_REFERENCE"):
        return os.environ["XR_REFERENCE"]
    r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


def build(ref: bool = False) -> None:
    """Build liboracle.so (and, with ref=True, the reference host build)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


@dataclass
class Scan:
    """A scan description: the reference's Geometry plus its per-axis globals
    (elemR, elemT, INIT_OFFSET) and the scattering basis (params.cu:14-40)."""
    sdd: float
    sod: float
    det: float
    N: int
    Nd: int
    V: int
    rot: np.ndarray            # (C, 9)
    trans: np.ndarray          # (C, 3)
    offset: np.ndarray         # (C, 3)
    basis: np.ndarray          # (K, 3)
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.rot = np.ascontiguousarray(np.asarray(self.rot, np.float32).reshape(-1, 9))
        self.trans = np.ascontiguousarray(np.asarray(self.trans, np.float32).reshape(-1, 3))
        self.offset = np.ascontiguousarray(np.asarray(self.offset, np.float32).reshape(-1, 3))
        self.basis = np.ascontiguousarray(np.asarray(self.basis, np.float32).reshape(-1, 3))

    @property
    def C(self) -> int:
        return self.rot.shape[0]

    @property
    def K(self) -> int:
        return self.basis.shape[0]

    @property
    def vs(self) -> float:
        return float(np.float32(np.float32(self.sod) * np.float32(self.det)) / np.float32(self.sdd))


class _OrScan(ctypes.Structure):
    _fields_ = [("sdd", ctypes.c_float), ("sod", ctypes.c_float), ("det", ctypes.c_float),
                ("N", ctypes.c_int), ("Nd", ctypes.c_int), ("V", ctypes.c_int),
                ("C", ctypes.c_int), ("K", ctypes.c_int),
                ("rot", _F), ("trans", _F), ("offset", _F), ("basis", _F)]


def _p(a: np.ndarray, dt=np.float32):
    assert a.dtype == dt and a.flags.c_contiguous
    return a.ctypes.data_as(_F if dt == np.float32 else _D)


def _ptr_array(arrs, dt):
    t = _F if dt == np.float32 else _D
    return (t * len(arrs))(*[a.ctypes.data_as(t) for a in arrs])


class Oracle:
    """The project's CPU restatement (liboracle.so)."""

    def __init__(self):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)

    def _scan(self, s: Scan) -> _OrScan:
        return _OrScan(s.sdd, s.sod, s.det, s.N, s.Nd, s.V, s.C, s.K,
                       _p(s.rot), _p(s.trans), _p(s.offset), _p(s.basis))

    def _fn(self, name, dt):
        return getattr(self.lib, ("or32_" if dt == np.float32 else "or64_") + name)

    def forward_view(self, s, cond, n, vol, proj, factor, xtt, dt=np.float32):
        self._fn("forward_view", dt)(ctypes.byref(self._scan(s)), cond, n, _p(vol, dt), _p(proj, dt),
                                     _p(factor, dt), int(xtt))

    def forward_orth_view(self, s, cond, n, vol, coef, proj, dt=np.float32):
        """forwardOrth (ir.cu:294-364) of one view into proj (axis block, all views)."""
        self._fn("forward_orth_view", dt)(ctypes.byref(self._scan(s)), cond, n, _p(vol, dt), _p(coef, dt),
                                          _p(proj, dt))

    def backward_orth_slab(self, s, cond, y, n, proj, coef, tmp, factor, dt=np.float32):
        """backwardOrth (ir.cu:366-423) of slab y, view n."""
        self._fn("backward_orth_slab", dt)(ctypes.byref(self._scan(s)), cond, y, n, _p(proj, dt), _p(coef, dt),
                                           _p(tmp, dt), _p(factor, dt))

    def normal_three(self, s, vol, coef, loss, rot, dt=np.float32):
        """calcNormalVectorThreeDirec (ir.cu:856-974): coef and loss updated in place."""
        self._fn("normal_three", dt)(ctypes.byref(self._scan(s)), _p(vol, dt), _p(coef, dt), _p(loss, dt), int(rot))

    def forward_md_view(self, s, cond, n, vol, md, proj, factor, dt=np.float32):
        """forwardOrthByMD (ir.cu:154-231) of one view; factor accumulates the weights."""
        self._fn("forward_md_view", dt)(ctypes.byref(self._scan(s)), cond, n, _p(vol, dt), _p(md, dt),
                                        _p(proj, dt), _p(factor, dt))

    def backward_md_slab(self, s, cond, y, n, proj, md, tmp, factor, dt=np.float32):
        """backwardOrthByMD (ir.cu:233-292) of slab y, view n."""
        self._fn("backward_md_slab", dt)(ctypes.byref(self._scan(s)), cond, y, n, _p(proj, dt), _p(md, dt),
                                         _p(tmp, dt), _p(factor, dt))

    def md_filter_slab(self, s, y, md, out, coef, dt=np.float32):
        """meanFiltFiberMD (ir.cu:1304-1363) of slab y into out."""
        c = ctypes.c_float(coef) if dt == np.float32 else ctypes.c_double(coef)
        self._fn("md_filter_slab", dt)(ctypes.byref(self._scan(s)), int(y), _p(md, dt), _p(out, dt), c)

    def main_direction(self, s, vol, md, iteration, dt=np.float32):
        """calcMainDirection (ir.cu:624-710): md updated in place."""
        self._fn("main_direction", dt)(ctypes.byref(self._scan(s)), _p(vol, dt), _p(md, dt), int(iteration))

    def md_with_estimate(self, s, vol, md, est, dt=np.float32):
        """calcMDWithEst (ir.cu:712-789): md updated in place."""
        self._fn("md_with_estimate", dt)(ctypes.byref(self._scan(s)), _p(vol, dt), _p(md, dt), _p(est, dt))

    def update_estimation(self, s, vol, est, iteration, dt=np.float32):
        """updateEstimation (ir.cu:791-844): est (2 planes) updated in place."""
        self._fn("update_estimation", dt)(ctypes.byref(self._scan(s)), _p(vol, dt), _p(est, dt), int(iteration))

    def normal_three_est(self, s, vol, coef, loss, est, dt=np.float32):
        """calcNormalVectorThreeDirecWithEst (ir.cu:976-1071): coef and loss updated in place."""
        self._fn("normal_three_est", dt)(ctypes.byref(self._scan(s)), _p(vol, dt), _p(coef, dt), _p(loss, dt),
                                         _p(est, dt))

    def coef_filter_slab(self, s, y, coef, vol, out, w, dt=np.float32):
        """meanFiltFiber (ir.cu:1231-1302) of slab y into out."""
        c = ctypes.c_float(w) if dt == np.float32 else ctypes.c_double(w)
        self._fn("coef_filter_slab", dt)(ctypes.byref(self._scan(s)), int(y), _p(coef, dt), _p(vol, dt),
                                         _p(out, dt), c)

    def update_estimation_coef(self, s, vol, est, iteration, dt=np.float32):
        """updateEstimationByCoef (ir.cu:1073-1120): est updated in place."""
        self._fn("update_estimation_coef", dt)(ctypes.byref(self._scan(s)), _p(vol, dt), _p(est, dt),
                                               int(iteration))

    def fiber_forward_view(self, s, cond, n, vol, proj, dt=np.float32):
        """forwardProjFiber (fiber.cu:13-153) of one view into proj (axis block, all views)."""
        self._fn("fiber_forward_view", dt)(ctypes.byref(self._scan(s)), cond, n, _p(vol, dt), _p(proj, dt))

    def fiber_backward_slab(self, s, cond, y, n, proj, vol, tmp, factor, dt=np.float32):
        """backwardProjFiber (fiber.cu:155-226) of slab y, view n."""
        self._fn("fiber_backward_slab", dt)(ctypes.byref(self._scan(s)), cond, y, n, _p(proj, dt), _p(vol, dt),
                                            _p(tmp, dt), _p(factor, dt))

    def fiber_reconstruct(self, s, sino, vol, epoch, batch, rotate_ccw=0, art=False, lam=1e-2):
        """XTT::fiberModelReconstruct (reconstruct.cu:1242-1371) from the volume
        given (the reference starts every channel at 0.01, :1245-1247), FP32,
        with the oracle's kernels: per subset forwardProjFiber + projRatio /
        projSubtract over every axis (:1302-1326), then per slab
        backwardProjFiber over every axis and view and voxelProduct / voxelPlus
        (ir.cu:1637-1693) of channel 0 alone (:1328-1347).  Subset order: a
        default std::mt19937_64 shuffles the persistent order every epoch
        (:1296-1298).  sino: (C, V, Nd, Nd); vol: (K, N, N, N).  Returns
        (volume, last ratio images (C, V, Nd, Nd), per-epoch sums of |b - p|)."""
        N, Nd, V, K, C = s.N, s.Nd, s.V, s.K, s.C
        rot = -1 if rotate_ccw else 1
        sub_size = (V + batch - 1) // batch
        alpha = np.float32(lam) / np.float32(sub_size)
        vol = np.ascontiguousarray(vol, np.float32).reshape(K, -1).copy()
        sino = np.ascontiguousarray(sino, np.float32).reshape(C, -1)
        orders = self.subset_orders(batch, epoch, True)
        proj = np.zeros((C, V * Nd * Nd), np.float32)
        losses = np.zeros(epoch, np.float64)
        v0 = vol[0].reshape(N, N, N)                       # [z][y][x], a view of vol
        for e in range(epoch):
            proj[:] = 0
            for sub in orders[e]:
                views = [rot * ((int(sub) + batch * j) % V) for j in range(sub_size)]
                for c in range(C):
                    for n in views:
                        self.fiber_forward_view(s, c, n, vol.ravel(), proj[c])
                        losses[e] += self.ratio(s, n, proj[c], sino[c], art)
                for y in range(N):
                    tmp = np.zeros(K * N * N, np.float32)
                    fac = np.zeros(K * N * N, np.float32)
                    for c in range(C):
                        for n in views:
                            self.fiber_backward_slab(s, c, y, n, proj[c], vol.ravel(), tmp, fac)
                    t0, f0 = tmp[:N * N].reshape(N, N), fac[:N * N].reshape(N, N)   # [z][x]
                    if art:
                        v0[:, y, :] = v0[:, y, :] + alpha * t0
                    else:
                        with np.errstate(divide="ignore", invalid="ignore"):
                            upd = (v0[:, y, :] * t0) / f0
                        v0[:, y, :] = np.where(f0 == 0, np.float32(0), upd)
        return vol.reshape(K, N, N, N), proj.reshape(C, V, Nd, Nd), losses

    def correlation(self, s, cond, n, proj, factor, dt=np.float32):
        self._fn("correlation", dt)(ctypes.byref(self._scan(s)), cond, n, _p(proj, dt), _p(factor, dt))

    def ratio(self, s, n, proj, sino, art, dt=np.float32):
        acc = np.zeros(1, dt)
        self._fn("ratio", dt)(ctypes.byref(self._scan(s)), n, _p(proj, dt), _p(sino, dt), int(art), _p(acc, dt))
        return float(acc[0])

    def backward_slab(self, s, cond, y, n, proj, tmp, factor, xtt, dt=np.float32):
        self._fn("backward_slab", dt)(ctypes.byref(self._scan(s)), cond, y, n, _p(proj, dt), _p(tmp, dt),
                                      _p(factor, dt), int(xtt))

    def forward_all(self, s, vol, rotate_ccw=0, xtt=False, dt=np.float32):
        vol = np.ascontiguousarray(vol, dt)
        proj = np.zeros(s.C * s.V * s.Nd * s.Nd, dt)
        self._fn("forward_all", dt)(ctypes.byref(self._scan(s)), _p(vol, dt), _p(proj, dt), int(rotate_ccw),
                                    int(xtt))
        return proj.reshape(s.C, s.V, s.Nd, s.Nd)

    def subset_orders(self, batch, rows, fresh_engine_each_row):
        out = np.zeros(rows * batch, np.int32)
        self.lib.or_subset_orders(batch, rows, int(fresh_engine_each_row), out.ctypes.data_as(_I))
        return out.reshape(rows, batch)

    def ir_reconstruct(self, s, sino, vol, epoch, batch, rotate_ccw=0, art=False, lam=1e-2, dt=np.float32):
        """sino: (C, V, Nd, Nd); vol: (C, N, N, N) initial volumes (copied).
        Returns (volumes, losses[C, epoch])."""
        sino = [np.ascontiguousarray(x, dt).ravel() for x in sino]
        vols = [np.ascontiguousarray(x, dt).ravel().copy() for x in vol]
        orders = self.subset_orders(batch, s.C * epoch, False)
        losses = np.zeros(s.C * epoch, dt)
        self._fn("ir_reconstruct", dt)(ctypes.byref(self._scan(s)), _ptr_array(sino, dt), _ptr_array(vols, dt),
                                       epoch, batch, int(rotate_ccw), int(art),
                                       (ctypes.c_float if dt == np.float32 else ctypes.c_double)(lam),
                                       _p(losses, dt), orders.ctypes.data_as(_I))
        return np.stack(vols).reshape(s.C, s.N, s.N, s.N), losses.reshape(s.C, epoch)

    def xtt_reconstruct(self, s, sino, vol, epoch, batch, rotate_ccw=0, art=False, lam=1e-2, dt=np.float32):
        """sino: (C, V, Nd, Nd); vol: (K, N, N, N).  Returns (vol after sqrt,
        last ratio images (C, V, Nd, Nd), losses[epoch])."""
        sino = np.ascontiguousarray(sino, dt).ravel()
        vol = np.ascontiguousarray(vol, dt).ravel().copy()
        proj = np.zeros_like(sino)
        orders = self.subset_orders(batch, epoch, True)
        losses = np.zeros(epoch, dt)
        self._fn("xtt_reconstruct", dt)(ctypes.byref(self._scan(s)), _p(sino, dt), _p(vol, dt), _p(proj, dt),
                                        epoch, batch, int(rotate_ccw), int(art),
                                        (ctypes.c_float if dt == np.float32 else ctypes.c_double)(lam),
                                        _p(losses, dt), orders.ctypes.data_as(_I))
        return (vol.reshape(s.K, s.N, s.N, s.N), proj.reshape(s.C, s.V, s.Nd, s.Nd), losses)

    def fdk_reconstruct(self, s, sino, rotate_ccw=0, ramlak=False, block0=True, dt=np.float32):
        sino = np.ascontiguousarray(sino, dt).ravel()
        vol = np.zeros(s.C * s.N ** 3, dt)
        filt = np.zeros_like(sino)
        self._fn("fdk_reconstruct", dt)(ctypes.byref(self._scan(s)), _p(sino, dt), _p(vol, dt), _p(filt, dt),
                                        int(rotate_ccw), int(ramlak), int(block0))
        return vol.reshape(s.C, s.N, s.N, s.N), filt.reshape(s.C, s.V, s.Nd, s.Nd)

    def fdk_filter(self, s, ramlak=False, dt=np.float32):
        f = np.zeros(s.Nd, dt)
        self._fn("fdk_filter", dt)(ctypes.byref(self._scan(s)), int(ramlak), _p(f, dt))
        return f

    def fdk_weight(self, s, dt=np.float32):
        w = np.zeros(s.Nd * s.Nd, dt)
        self._fn("fdk_weight", dt)(ctypes.byref(self._scan(s)), _p(w, dt))
        return w.reshape(s.Nd, s.Nd)

    def orientation(self, basis, mu):
        """mu: (K, ...) float32.  Returns md (3, ...), evalue (3, ...)."""
        K = mu.shape[0]
        shp = mu.shape[1:]
        mu = np.ascontiguousarray(mu, np.float32).reshape(K, -1)
        nv = mu.shape[1]
        md = np.zeros((3, nv), np.float32)
        ev = np.zeros((3, nv), np.float32)
        b = np.ascontiguousarray(np.asarray(basis, np.float32).ravel())
        self.lib.or_orientation(ctypes.c_long(nv), K, _p(b), _p(mu), _p(md), _p(ev))
        return md.reshape((3,) + shp), ev.reshape((3,) + shp)

    def angle_from_md(self, md):
        """calcAngleFromMD (pca.cu:67-83): md (3, ...) -> angle (2, ...)."""
        shp = md.shape[1:]
        md = np.ascontiguousarray(md, np.float32).reshape(3, -1)
        out = np.zeros((2, md.shape[1]), np.float32)
        self.lib.or_angle_from_md(ctypes.c_long(md.shape[1]), _p(md), _p(out))
        return out.reshape((2,) + shp)

    def direction_normalization(self, md):
        """directionNormalization (pca.cu:85-106) of a copy of md (3, ...)."""
        shp = md.shape[1:]
        out = np.ascontiguousarray(md, np.float32).reshape(3, -1).copy()
        self.lib.or_direction_normalization(ctypes.c_long(out.shape[1]), _p(out))
        return out.reshape((3,) + shp)

    def jacobi3(self, A):
        A = np.ascontiguousarray(A, np.float64).ravel()
        w = np.zeros(3)
        V = np.zeros(9)
        self.lib.or_jacobi3(_p(A, np.float64), _p(w, np.float64), _p(V, np.float64))
        return w, V.reshape(3, 3)


class RefHost:
    """The reference's own ir.cu kernels compiled for the host (libxrref.so)."""

    def __init__(self, parallel: bool = False):
        path = os.path.join(HERE, "_ref", "libxrref.so")
        if not os.path.exists(path):
            build(ref=True)
        self.lib = ctypes.CDLL(path)
        self.lib.xr_ref_ratio.restype = ctypes.c_float
        self.lib.xr_ref_vox_size.restype = ctypes.c_float
        self.lib.xr_ref_set_parallel(1 if parallel else 0)

    @staticmethod
    def available() -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", "libxrref.so"))

    def setup(self, s: Scan):
        self.s = s
        self.lib.xr_ref_setup(ctypes.c_float(s.sdd), ctypes.c_float(s.sod), ctypes.c_float(s.det), s.N, s.Nd,
                              s.V, s.C, s.K, _p(s.rot), _p(s.trans), _p(s.offset), _p(s.basis))

    def set_parallel(self, on: bool):
        self.lib.xr_ref_set_parallel(1 if on else 0)

    def forward_view(self, cond, n, vol, proj, factor, xtt):
        self.lib.xr_ref_forward_view(cond, n, _p(vol), _p(proj), _p(factor), int(xtt))

    def correlation(self, cond, n, proj, factor):
        self.lib.xr_ref_correlation(cond, n, _p(proj), _p(factor))

    def forward_orth(self, cond, n, vol, coef, proj):
        self.lib.xr_ref_forward_orth(cond, n, _p(vol), _p(coef), _p(proj))

    def backward_orth(self, cond, y, n, proj, coef, tmp, factor):
        self.lib.xr_ref_backward_orth(cond, y, n, _p(proj), _p(coef), _p(tmp), _p(factor))

    def normal_three(self, vol, coef, loss, rot):
        self.lib.xr_ref_normal_three(_p(vol), _p(coef), _p(loss), int(rot))

    def forward_md(self, cond, n, vol, md, proj, factor):
        self.lib.xr_ref_forward_md(cond, n, _p(vol), _p(md), _p(proj), _p(factor))

    def backward_md(self, cond, y, n, proj, md, tmp, factor):
        self.lib.xr_ref_backward_md(cond, y, n, _p(proj), _p(md), _p(tmp), _p(factor))

    def normal_three_est(self, vol, coef, loss, est):
        self.lib.xr_ref_normal_three_est(_p(vol), _p(coef), _p(loss), _p(est))

    def coef_filter(self, y, coef, out, vol, w):
        self.lib.xr_ref_coef_filter(int(y), _p(coef), _p(out), _p(vol), ctypes.c_float(w))

    def update_estimation_coef(self, vol, est, iteration):
        loss = np.zeros(self.s.N ** 3, np.float32)
        self.lib.xr_ref_update_estimation_coef(_p(vol), _p(loss), _p(est), int(iteration))

    def fiber_forward(self, cond, n, vol, proj):
        self.lib.xr_ref_fiber_forward(cond, n, _p(vol), _p(proj))

    def fiber_backward(self, cond, y, n, proj, vol, tmp, factor):
        self.lib.xr_ref_fiber_backward(cond, y, n, _p(proj), _p(vol), _p(tmp), _p(factor))

    def md_filter(self, y, md, out, coef):
        self.lib.xr_ref_md_filter(int(y), _p(md), _p(out), ctypes.c_float(coef))

    def main_direction(self, vol, md, iteration):
        loss = np.zeros(self.s.N ** 3, np.float32)
        self.lib.xr_ref_main_direction(_p(vol), _p(md), _p(loss), int(iteration))

    def md_with_estimate(self, vol, md, est):
        self.lib.xr_ref_md_with_estimate(_p(vol), _p(md), _p(est))

    def update_estimation(self, vol, md, est, iteration):
        loss = np.zeros(self.s.N ** 3, np.float32)
        self.lib.xr_ref_update_estimation(_p(vol), _p(md), _p(loss), _p(est), int(iteration))

    def ratio(self, n, proj, sino, art):
        return float(self.lib.xr_ref_ratio(n, _p(proj), _p(sino), int(art)))

    def fdk_weight(self):
        """calcWeight (fdk.cu:13-26): (Nd, Nd)."""
        w = np.zeros(self.s.Nd * self.s.Nd, np.float32)
        self.lib.xr_ref_fdk_weight(_p(w))
        return w.reshape(self.s.Nd, self.s.Nd)

    def fdk_filter(self):
        """The filter table of FDK::reconstruct (reconstruct.cu:1692-1698)."""
        f = np.zeros(self.s.Nd, np.float32)
        self.lib.xr_ref_fdk_filter(_p(f))
        return f

    def fdk_reconstruct(self, sino, rotate_ccw=0):
        """FDK::reconstruct (reconstruct.cu:1651-1724) with the reference's
        fdk.cu kernels: returns (volumes (C, N, N, N), filtered sinograms)."""
        s = self.s
        sino = np.ascontiguousarray(sino, np.float32).ravel()
        vol = np.zeros(s.C * s.N ** 3, np.float32)
        filt = np.zeros_like(sino)
        self.lib.xr_ref_fdk_reconstruct(_p(sino), _p(vol), _p(filt), int(rotate_ccw))
        return vol.reshape(s.C, s.N, s.N, s.N), filt.reshape(s.C, s.V, s.Nd, s.Nd)

    def angle_from_md(self, md):
        """calcAngleFromMD (pca.cu:67-83) on md (3, nz, ny, nx)."""
        nz, ny, nx = md.shape[1:]
        md = np.ascontiguousarray(md, np.float32)
        out = np.zeros((2, nz, ny, nx), np.float32)
        self.lib.xr_ref_angle_from_md(_p(md), _p(out), nx, ny, nz)
        return out

    def direction_normalization(self, md):
        """directionNormalization (pca.cu:85-106) of a copy of md (3, nz, ny, nx)."""
        nz, ny, nx = md.shape[1:]
        out = np.ascontiguousarray(md, np.float32).copy()
        self.lib.xr_ref_direction_normalization(_p(out), nx, ny, nz)
        return out

    def backward_slab(self, cond, y, n, proj, tmp, factor, xtt):
        self.lib.xr_ref_backward_slab(cond, y, n, _p(proj), _p(tmp), _p(factor), int(xtt))

    def forward_all(self, vol, rotate_ccw=0, xtt=False):
        s = self.s
        vol = np.ascontiguousarray(vol, np.float32).ravel().copy()
        proj = np.zeros(s.C * s.V * s.Nd * s.Nd, np.float32)
        self.lib.xr_ref_forward_all(_p(vol), _p(proj), int(rotate_ccw), int(xtt))
        return proj.reshape(s.C, s.V, s.Nd, s.Nd)

    def ir_reconstruct(self, sino, vol, epoch, batch, rotate_ccw=0, art=False, lam=1e-2):
        s = self.s
        sino = [np.ascontiguousarray(x, np.float32).ravel().copy() for x in sino]
        vols = [np.ascontiguousarray(x, np.float32).ravel().copy() for x in vol]
        losses = np.zeros(epoch, np.float32)
        self.lib.xr_ref_ir_reconstruct(_ptr_array(sino, np.float32), _ptr_array(vols, np.float32), epoch, batch,
                                       int(rotate_ccw), int(art), ctypes.c_float(lam), _p(losses))
        return np.stack(vols).reshape(s.C, s.N, s.N, s.N), losses

    def xtt_reconstruct(self, sino, vol, epoch, batch, rotate_ccw=0, art=False, lam=1e-2):
        s = self.s
        sino = [np.ascontiguousarray(x, np.float32).ravel().copy() for x in sino]
        vols = [np.ascontiguousarray(x, np.float32).ravel().copy() for x in vol]
        losses = np.zeros(epoch, np.float32)
        self.lib.xr_ref_xtt_reconstruct(_ptr_array(sino, np.float32), _ptr_array(vols, np.float32), epoch, batch,
                                        int(rotate_ccw), int(art), ctypes.c_float(lam), _p(losses))
        return (np.stack(vols).reshape(s.K, s.N, s.N, s.N), np.stack(sino).reshape(s.C, s.V, s.Nd, s.Nd),
                losses)

    def fiber_reconstruct(self, sino, vol, epoch, batch, rotate_ccw=0, art=False, lam=1e-2):
        """fiberModelReconstruct's epochs from the volume given; returns
        (volume (K, N, N, N), last ratio images (C, V, Nd, Nd), float losses)."""
        s = self.s
        sino = [np.ascontiguousarray(x, np.float32).ravel().copy() for x in sino]
        vols = [np.ascontiguousarray(x, np.float32).ravel().copy() for x in vol]
        losses = np.zeros(epoch, np.float32)
        self.lib.xr_ref_fiber_reconstruct(_ptr_array(sino, np.float32), _ptr_array(vols, np.float32), epoch, batch,
                                          int(rotate_ccw), int(art), ctypes.c_float(lam), _p(losses))
        return (np.stack(vols).reshape(s.K, s.N, s.N, s.N), np.stack(sino).reshape(s.C, s.V, s.Nd, s.Nd),
                losses)


class RefGPU:
    """The reference's own CUDA kernels (reconstruct/src/ir.cu built for the
    B200 into oracle/_ref/libxrref_gpu.so) driven like XTT::reconstruct, one
    launch and synchronize per y slab and view (oracle/ref_gpu)."""

    def __init__(self):
        path = os.path.join(HERE, "_ref", "libxrref_gpu.so")
        if not os.path.exists(path):
            build(ref=True)
        self.lib = ctypes.CDLL(path)
        self.lib.xr_refgpu_xtt_reconstruct.restype = ctypes.c_int

    @staticmethod
    def available() -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", "libxrref_gpu.so"))

    def xtt_reconstruct(self, s: Scan, sino, vol, epoch, batch, rotate_ccw=0, art=False, lam=1e-2,
                        want_ratio=True):
        """Returns (vol after voxelSqrt (K, N, N, N), last ratio images or None,
        losses (epoch,), milliseconds per epoch (epoch,))."""
        sino = np.ascontiguousarray(sino, np.float32).ravel()
        v = np.ascontiguousarray(vol, np.float32).ravel().copy()
        ratio = np.zeros_like(sino) if want_ratio else None
        losses = np.zeros(max(epoch, 1), np.float32)
        ms = np.zeros(max(epoch, 1), np.float64)
        st = self.lib.xr_refgpu_xtt_reconstruct(
            ctypes.c_float(s.sdd), ctypes.c_float(s.sod), ctypes.c_float(s.det), s.N, s.Nd, s.V, s.C, s.K,
            _p(s.rot), _p(s.trans), _p(s.offset), _p(s.basis), _p(sino), _p(v),
            _p(ratio) if want_ratio else None, int(epoch), int(batch), int(rotate_ccw), int(art),
            ctypes.c_float(lam), _p(losses), ms.ctypes.data_as(_D))
        if st:
            raise RuntimeError(f"reference GPU run failed: CUDA error {st}")
        return (v.reshape(s.K, s.N, s.N, s.N), ratio.reshape(s.C, s.V, s.Nd, s.Nd) if want_ratio else None,
                losses[:epoch], ms[:epoch])
