#!/usr/bin/env python
"""Benchmark: XTT reconstruction throughput on B200.

Workload (the XTT 256^3 x 13 configuration): 256^3 voxels x K = 13 scattering
channels, 3 sample-rotation axes x 180 views over 360 degrees, 384 x 384
detector, SOD 500 / SDD 1000 / 1 mm voxels, 12 seeded straight fiber
cylinders; OS-EM (the reference's XTT::reconstruct, method MLEM, 5 subsets as
main.cu:60) from mu = 0.01.  One step = one OS-EM epoch: forward + ratio +
back-projection/update of every view of every axis.

metric  effective projector bandwidth: every epoch applies the forward and
        the back projector once to each of the C*V views, each charged
        bytes_view = K*N^3*4 + Nd^2*4 (the volume streamed once plus one
        detector image), so value = 2*C*V*bytes_view / epoch time.
e2e     the same metric through the public host-buffer call
        (xr_xtt_reconstruct, one epoch, pinned host buffers, including the
        H2D of sinograms + initial volume and the D2H of volume, ratio
        images and orientation).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "xray-directional-reconstruction_b200")

W = dict(N=256, Nd=384, V=180, C=3, K=13, batch=5, sdd=1000.0, sod=500.0, det=2.0, n_fibers=12, seed=5)
# --size profile: the same kernels on a smaller case for ncu captures (volume
# 192^3 x 13 = 368 MB, still larger than L2), with the full workload's 36 views
# per subset and axis, so per-launch instruction counts scale by voxel-views.
W_PROFILE = dict(W, N=192, Nd=288, V=180)
WORKLOAD = ("XTT 256^3 x K13, 3 axes x 180 views, 384^2 detector, OS-EM 5 subsets, FP32 "
            "(12 seeded fiber cylinders, SOD 500 / SDD 1000 mm, 1 mm voxels)")
METRIC = "XTT 256^3x13 projector GB/s (effective, forward+back per OS-EM epoch)"


def load_pkg():
    if "xrd" in sys.modules:
        return sys.modules["xrd"]
    spec = importlib.util.spec_from_file_location("xrd", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["xrd"] = mod
    spec.loader.exec_module(mod)
    return mod


def three_axes():
    return np.array([[1, 0, 0, 0, 1, 0, 0, 0, 1], [0, 0, -1, 0, 1, 0, 1, 0, 0], [1, 0, 0, 0, 0, -1, 0, 1, 0]],
                    np.float32)


def basis13():
    d = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1), (0, 1, 1), (0, 1, -1),
         (1, 1, 1), (1, 1, -1), (1, -1, 1), (-1, 1, 1)]
    return np.array([np.asarray(v, np.float64) / np.linalg.norm(v) for v in d], np.float32)


def fiber_phantom(N, n_fib, seed, basis):
    """Fibers of radius U[2,5] voxels with unit direction f uniform on the
    sphere; channel k = |S_k x f|^2 inside, 0 outside.  (K, N, N, N) float32."""
    rng = np.random.default_rng(seed)
    c = (np.arange(N, dtype=np.float32) - (N - 1) / 2.0)
    vol = np.zeros((basis.shape[0], N, N, N), np.float32)
    for _ in range(n_fib):
        f = rng.normal(size=3)
        f /= np.linalg.norm(f)
        p0 = rng.uniform(-0.3 * N, 0.3 * N, 3)
        r = rng.uniform(2.0, 5.0)
        eta = np.sum(np.cross(basis.astype(np.float64), f[None, :]) ** 2, axis=1).astype(np.float32)
        for z in range(N):
            dz = c[z] - p0[2]
            dy = (c - p0[1])[:, None]
            dx = (c - p0[0])[None, :]
            t = dx * f[0] + dy * f[1] + dz * f[2]
            d2 = dx * dx + dy * dy + dz * dz - t * t
            inside = d2 <= r * r
            if inside.any():
                for k in range(basis.shape[0]):
                    vol[k, z][inside] = eta[k]
    return vol


def bytes_view(K, N, Nd, s=4):
    return K * N ** 3 * s + Nd * Nd * s


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def conv_roofline(local: int, N: int = 256, reps: int = 3):
    """Tensor-core roofline of the warm-start network's inference on an
    N^3 x 13 BF16 volume (in place): algorithmic FLOPs = 2 * nvox * 27 *
    sum_l cin_l * cout_l (unpadded channels) over the CUDA-event time of one
    inference (the network's conv launches plus the input packing)."""
    import struct
    import torch
    ws = load_warmstart()
    if not os.path.exists(ws.WEIGHTS):
        return None
    with open(ws.WEIGHTS, "rb") as f:
        channels, width, depth = struct.unpack("<3i", f.read(20)[8:20])
    net = ws.load_net(ws.WEIGHTS, local)
    stream = torch.cuda.current_stream()
    net.set_stream(stream.cuda_stream)
    vol = torch.full((channels, N, N, N), 0.5, dtype=torch.bfloat16, device="cuda")
    net.infer(vol.data_ptr(), vol.data_ptr(), (N, N, N), storage=1, floor_value=-1e30)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        net.infer(vol.data_ptr(), vol.data_ptr(), (N, N, N), storage=1, floor_value=-1e30)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    macs = 27 * sum(ci * co for ci, co in
                    [((channels if l == 0 else width), (channels if l == depth - 1 else width)) for l in range(depth)])
    flops = 2.0 * N ** 3 * macs
    peak, kind = measured_tensor_peak()
    net.close()
    return {"bound": "tensor", "kernel": "k_conv_ws (tcgen05, BF16 x BF16 -> FP32)", "achieved": flops / ms / 1e9,
            "peak": peak, "unit": "TFLOP/s", "frac": flops / ms / 1e9 / peak, "peak_kind": kind,
            "infer_ms": ms, "flops_per_inference": flops, "workload": f"{N}^3 x {channels}, depth {depth}, width {width}"}


PROFILE_JSON = os.path.join(ROOT, "profiles", "xtt_projectors_ncu.json")


def profile_figures():
    """Per-kernel figures of one ncu capture of the projector kernels on the
    profile case (profiles/xtt_projectors_ncu.json: warp instructions and DRAM
    bytes per launch, the voxel-views and sizes of that launch, the command)."""
    if not os.path.exists(PROFILE_JSON):
        return None
    return json.load(open(PROFILE_JSON))


def issue_roofline(kernel: str, launch_s: float, vox_views: float, n_vox: float, det_px_views: float,
                   sm_mhz: float, hbm_peak: float):
    """Roofline of a projector kernel against the resource that binds it: warp
    instruction issue (4 schedulers per SM, one warp instruction per cycle
    each).  achieved = warp instructions per launch / launch time, where the
    instructions per launch are the captured count per voxel-view times this
    launch's voxel-views; peak = 148 SMs x 4 x the SM clock sampled during
    the timed region.  traffic = the captured DRAM read and write bytes, each
    scaled to this launch by the unit the capture names for it (voxels for
    volume-side traffic, pixel-views for detector images), and
    hbm_frac_actual = traffic / launch time / measured HBM copy bandwidth."""
    figs = profile_figures()
    if not figs or kernel not in figs.get("kernels", {}):
        return None
    k = figs["kernels"][kernel]
    inst = k["warp_inst_per_launch"] / k["voxel_views_per_launch"] * vox_views
    unit = {"voxels": (n_vox, k["voxels_per_launch"]), "pixel_views": (det_px_views, k["pixel_views_per_launch"])}
    traffic = sum(k[f"dram_{d}_bytes_per_launch"] * unit[k[f"scale_{d}"]][0] / unit[k[f"scale_{d}"]][1]
                  for d in ("read", "write"))
    peak = 148 * 4 * sm_mhz * 1e6
    return {"bound": "issue", "kernel": kernel, "achieved": inst / launch_s / 1e9, "peak": peak / 1e9,
            "unit": "G warp-instructions/s", "frac": inst / launch_s / peak, "traffic": traffic,
            "hbm_frac_actual": traffic / launch_s / (hbm_peak * 1e9), "warp_inst_per_voxel_view":
            k["warp_inst_per_launch"] / k["voxel_views_per_launch"], "sm_mhz": sm_mhz,
            "source": os.path.relpath(PROFILE_JSON, ROOT) + " (" + figs.get("case", "") + ")"}


def l1_roofline(kernel: str, launch_s: float, vox_views: float, sm_mhz: float):
    """Roofline of a projector kernel against the L1 data pipe (one LSU
    wavefront per cycle per SM: the shared-memory atomics of the forward
    splat's tiles, the gathers of the back-projection).  achieved = captured
    wavefronts per voxel-view x this launch's voxel-views / launch time; peak =
    148 SMs x the SM clock sampled during the timed region."""
    figs = profile_figures()
    if not figs or kernel not in figs.get("kernels", {}):
        return None
    k = figs["kernels"][kernel]
    if "l1_wavefronts_per_launch" not in k:
        return None
    per_vv = k["l1_wavefronts_per_launch"] / k["voxel_views_per_launch"]
    peak = 148 * sm_mhz * 1e6
    ach = per_vv * vox_views / launch_s
    return {"bound": "l1", "kernel": kernel, "achieved": ach / 1e9, "peak": peak / 1e9, "unit": "G wavefronts/s",
            "frac": ach / peak, "wavefronts_per_voxel_view": per_vv, "sm_mhz": sm_mhz,
            "source": os.path.relpath(PROFILE_JSON, ROOT) + " (" + figs.get("case", "") + ")"}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap,utilization.gpu",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return out
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7 and parts[0].replace(".", "").isdigit():
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        loaded = [r for r in rows if r[6].isdigit() and int(r[6]) > 0] or rows
        out["sm_mhz"] = statistics.median(float(r[0]) for r in loaded)
        out["sm_max_mhz"] = max(float(r[1]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        out["reasons"] = [n for i, n in enumerate(names) if any(r[2 + i].lower() == "active" for r in loaded)]
        out["samples"] = len(loaded)
        return out


def bench_config(args, world: int):
    """The workload named in both arms' JSON lines (the same dict)."""
    N, Nd, V, C, K = W["N"], W["Nd"], W["V"], W["C"], W["K"]
    vol_mb, sino_mb = K * N ** 3 * 4 / 2 ** 20, C * V * Nd * Nd * 4 / 2 ** 20
    return {"workload": WORKLOAD if args.size == "full" else
            f"XTT {N}^3 x K{K}, {C} axes x {V} views, {Nd}^2 detector, OS-EM {W['batch']} subsets, FP32 "
            "(profile case: the kernels of the full workload at a size ncu captures)",
            "N": N, "K": K, "axes": C, "views": V, "detector": Nd, "subsets": W["batch"],
            "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 (volume {vol_mb:.0f} MiB, sinograms {sino_mb:.0f} MiB)"}


def cpu_reference_sample(mu_host: np.ndarray, b_host, n_views: int, warm: int = 0, first: int = 0):
    """Time the reference's own projector kernels (reconstruct/src/ir.cu built
    for the host, OpenMP over detector/voxel rows) on n_views (axis, view)
    pairs of the workload, starting at pair `first` of a fixed sequence that
    visits the three axes in turn: per pair forward + correlation + ratio
    against the measured image, then the back-projection of every y slab.
    mu_host is the current iterate; b_host(cond, n) returns the measured image
    of a pair (flat float32).  Returns (seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefHost, Scan
    s = Scan(sdd=W["sdd"], sod=W["sod"], det=W["det"], N=W["N"], Nd=W["Nd"], V=W["V"], rot=three_axes(),
             trans=np.zeros((3, 3)), offset=np.zeros((3, 3)), basis=basis13())
    R = RefHost(parallel=True)
    R.setup(s)
    N, Nd, K = s.N, s.Nd, s.K
    vol = np.ascontiguousarray(mu_host.reshape(-1))
    proj = np.zeros(s.V * Nd * Nd, np.float32)
    fac = np.zeros(Nd * Nd, np.float32)
    tmp = np.zeros(N * N * K, np.float32)
    bfac = np.zeros(N * N * K, np.float32)
    t_total = 0.0
    for i in range(warm + n_views):
        cond, n = reference_pair(first + i)
        sino = np.zeros(s.V * Nd * Nd, np.float32)
        sino[n * Nd * Nd:(n + 1) * Nd * Nd] = b_host(cond, n)
        t0 = time.perf_counter()
        R.forward_view(cond, n, vol, proj, fac, 1)
        R.correlation(cond, n, proj, fac)
        R.ratio(n, proj, sino, 0)
        for y in range(N):
            tmp[:] = 0
            bfac[:] = 0
            R.backward_slab(cond, y, n, proj, tmp, bfac, 1)
        dt = time.perf_counter() - t0
        if i >= warm:
            t_total += dt
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return t_total, threads


def reference_pair(i: int):
    """(axis, view) of the i-th pair of the CPU samples: the axes in turn, the
    views of each axis in a stride-37 order over the scan."""
    return i % W["C"], (37 * (i // W["C"])) % W["V"]


def reference_measured(mu_true: np.ndarray):
    """The measured images b = A mu_true of the sampled pairs, made with the
    reference's own host forward operator (forwardProjXTT +
    correlationProjByLength) of the phantom the GPU arm reconstructs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefHost, Scan
    s = Scan(sdd=W["sdd"], sod=W["sod"], det=W["det"], N=W["N"], Nd=W["Nd"], V=W["V"], rot=three_axes(),
             trans=np.zeros((3, 3)), offset=np.zeros((3, 3)), basis=basis13())
    R = RefHost(parallel=True)
    R.setup(s)
    Nd = s.Nd
    vol = np.ascontiguousarray(mu_true.reshape(-1))
    cache = {}

    def get(cond, n):
        if (cond, n) not in cache:
            proj = np.zeros(s.V * Nd * Nd, np.float32)
            fac = np.zeros(Nd * Nd, np.float32)
            R.forward_view(cond, n, vol, proj, fac, 1)
            R.correlation(cond, n, proj, fac)
            cache[(cond, n)] = proj[n * Nd * Nd:(n + 1) * Nd * Nd].copy()
        return cache[(cond, n)]
    return get


def run_reference(args, rank):
    """--impl reference: the reference's CPU implementation of the path on
    the host cores (oracle/_ref, its own ir.cu), same metric and config: the
    phantom the GPU arm reconstructs, its measured images made by the
    reference's own forward operator, the OS-EM start mu = 0.01; each step a
    sample of 3 (axis, view) pairs (one per axis) of the epoch's 540."""
    if rank != 0:
        return
    bv = bytes_view(W["K"], W["N"], W["Nd"])
    mu_true = fiber_phantom(W["N"], W["n_fibers"], W["seed"], basis13())
    b = reference_measured(mu_true)
    mu = np.full_like(mu_true, 0.01)
    per_step_views = 3
    times = []
    threads = 1
    for i in range(args.warmup + args.steps):
        t, threads = cpu_reference_sample(mu, b, per_step_views, 0, first=i * per_step_views)
        if i >= args.warmup:
            times.append(t)
    t_step = float(np.mean(times))
    value = 2 * per_step_views * bv / t_step / 1e9
    sample = (f"{per_step_views} of {W['C'] * W['V']} (axis, view) pairs per step (one per axis), forward + "
              "correlation + ratio + back-projection of all K channels; reference ir.cu kernels compiled for the "
              "host, OpenMP; same phantom and OS-EM start as the GPU arm, measured images by the reference's own "
              "forward operator")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(args, 1),
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def load_replicas():
    spec = importlib.util.spec_from_file_location("xr_replicas", os.path.join(PKG, "replicas.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_warmstart():
    if "xrd.warmstart" in sys.modules:
        return sys.modules["xrd.warmstart"]
    load_pkg()
    spec = importlib.util.spec_from_file_location("xrd.warmstart", os.path.join(PKG, "warmstart.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["xrd.warmstart"] = mod
    spec.loader.exec_module(mod)
    return mod


def orientation_of(scan, mu):
    """Per-voxel main direction (calcEigenVector, pca.cu:12-55, libxr's FP64
    kernel) of sqrt|mu|, the voxelSqrt that XTT::reconstruct applies before it
    (reconstruct.cu:919-942): (3, N, N, N) FP32 on the device."""
    import torch
    xr = load_pkg()
    root = mu.float().abs().sqrt().contiguous()
    md = torch.empty((3,) + tuple(mu.shape[1:]), dtype=torch.float32, device=mu.device)
    scan.ctx.set_option(xr.Option.STORAGE, 0)
    scan.ctx.dev_orientation(root.data_ptr(), md.data_ptr(), 0)
    torch.cuda.synchronize()
    return md


def angle_stats(md_a, md_b, mask):
    """Angle between the main directions md_a and md_b (unsigned axes) over
    the voxels of `mask`: mean / median / 90th percentile in degrees."""
    import torch
    a, b = md_a[:, mask].double(), md_b[:, mask].double()
    na, nb = a.norm(dim=0), b.norm(dim=0)
    ok = (na > 0) & (nb > 0)
    c = ((a * b).sum(0).abs()[ok] / (na[ok] * nb[ok])).clamp(max=1.0)
    ang = torch.rad2deg(torch.acos(c))
    if ang.numel() == 0:
        return {"voxels": 0}
    return {"voxels": int(ang.numel()), "mean_deg": float(ang.mean()), "median_deg": float(ang.median()),
            "p90_deg": float(ang.kthvalue(max(1, int(math.ceil(0.9 * ang.numel()))))[0])}


def run_ttr(args, local):
    """Time to a relative data residual ||A mu - b|| / ||b|| <= --target (FP64
    norms) on the XTT 256^3 x 13 workload, arms on the same data b = A mu_true
    (device fiber phantom, seed held out from the training seeds):
      plain_f32:    FP32 OS-EM (5 subsets) from mu = 0.01 (main.cu:38-43);
      learned_bf16: BF16 volumes (FP32 data): 5 OS-EM epochs from mu = 0.01,
                    the warm-start network in place, then OS-EM to the target;
      plain_bf16:   BF16 volumes without the network (isolates the storage).
    Device time (CUDA events): session set-up, epochs and inference, after an
    untimed warm-up epoch of every arm (kernels loaded, the geometry-only
    per-subset sensitivity on the context), so no arm pays those one-time
    costs.  The residual is checked every --check-every epochs and after
    every epoch once it is within 5 % of the target, outside the timed
    work."""
    import torch
    ws = load_warmstart()
    xr = load_pkg()
    weights = args.weights or ws.WEIGHTS
    torch.cuda.set_device(local)
    scan = ws.Scan(W["N"], W["V"], device=local, n_fibers=W["n_fibers"])
    mu_true = scan.phantom(W["seed"])
    b = scan.project(mu_true)
    torch.cuda.synchronize()
    K, N = scan.K, scan.N
    arms = {}
    # orientation of the true volume, over the fiber voxels (not timed)
    fiber_mask = mu_true.sum(0) > 0
    md_arm = {}
    try:
        md_true, ori_err = orientation_of(scan, mu_true), None
    except Exception as ex:      # an analysis failure is reported, it does not cost the timings
        md_true, ori_err = None, f"{type(ex).__name__}: {ex}"

    def run_arm(name, storage, learned):
        dt = {0: torch.float32, 1: torch.bfloat16}[storage]
        vol = torch.full((K, N, N, N), 0.01, dtype=dt, device="cuda")
        ms0, e0, r0 = 0.0, 0, None
        if learned:
            if not os.path.exists(weights):
                arms[name] = {"unavailable": "no trained weights at " + os.path.relpath(weights, ROOT)}
                return
            net = ws.load_net(weights, local)
            net.set_stream(scan.stream.cuda_stream)
            ms0 = ws.warm_start(scan, net, b, vol, args.early, W["batch"], storage, 0)
            e0 = args.early
            r0 = scan.residual(vol, b, storage, 0)
            net.close()
        e, ms, trace = scan.osem(b, vol, 0, W["batch"], storage, 0, residual_every=args.check_every,
                                 target=args.target, max_epochs=args.max_epochs, final_sqrt=False)
        reached = bool(trace) and trace[-1][2] <= args.target
        err = float(torch.linalg.vector_norm(vol.float() - mu_true) / torch.linalg.vector_norm(mu_true))
        ori = {"error": ori_err}
        if md_true is not None:
            try:
                md_arm[name] = orientation_of(scan, vol)
                ori = angle_stats(md_arm[name], md_true, fiber_mask)
            except Exception as ex:
                ori = {"error": f"{type(ex).__name__}: {ex}"}
        arms[name] = {"storage": {0: "f32", 1: "bf16"}[storage], "sinogram": "f32", "learned": learned,
                      "reached": reached, "epochs": e0 + e, "seconds": (ms0 + ms) / 1e3 if reached else None,
                      "seconds_run": (ms0 + ms) / 1e3, "residual_final": trace[-1][2] if trace else r0,
                      "residual_after_warm_start": r0, "volume_rel_error_final": err,
                      "orientation_error_vs_truth": ori,
                      "history": [{"epoch": e0 + ep, "ms": ms0 + t, "rel_l2": r} for ep, t, r in trace]}
        del vol

    # Untimed warm-up, one epoch per arm (and one inference for a learned
    # arm): CUDA loads each kernel at its first launch, and the first session
    # of a context computes the per-subset sensitivity (geometry only, then
    # kept on the context).  Without it both one-time costs land in whichever
    # arm runs first with those kernels.
    for name in args.arms.split(","):
        storage = 0 if name.endswith("f32") else 1
        wv = torch.full((K, N, N, N), 0.01, dtype={0: torch.float32, 1: torch.bfloat16}[storage], device="cuda")
        if name.startswith("learned") and os.path.exists(weights):
            net = ws.load_net(weights, local)
            net.set_stream(scan.stream.cuda_stream)
            ws.warm_start(scan, net, b, wv, 1, W["batch"], storage, 0)
            net.close()
        scan.osem(b, wv, 1, W["batch"], storage, 0, final_sqrt=False)
        scan.residual(wv, b, storage, 0)
        del wv
    torch.cuda.synchronize()

    for name in args.arms.split(","):
        run_arm(name, 0 if name.endswith("f32") else 1, name.startswith("learned"))
    line = {"mode": "time_to_residual", "metric": "XTT 256^3x13 time-to-%g residual (learned+BF16 vs plain FP32)"
            % args.target, "unit": "s", "higher_is_better": False, "workload": WORKLOAD, "target": args.target,
            "check_every": args.check_every, "max_epochs": args.max_epochs, "arms": arms}
    p, l = arms.get("plain_f32", {}), arms.get("learned_bf16", {})
    line["speedup_learned_bf16_vs_plain_f32"] = (p["seconds"] / l["seconds"]) if p.get("seconds") and \
        l.get("seconds") else None
    cross = None
    if "learned_bf16" in md_arm and "plain_f32" in md_arm:
        try:
            cross = angle_stats(md_arm["learned_bf16"], md_arm["plain_f32"], fiber_mask)
        except Exception as ex:
            cross = {"error": f"{type(ex).__name__}: {ex}"}
    line["orientation_learned_bf16_vs_plain_f32"] = cross
    line["network"] = os.path.relpath(weights, ROOT)
    # gate: the learned arm's median orientation error within 0.25 degrees of plain FP32's
    po = arms.get("plain_f32", {}).get("orientation_error_vs_truth", {})
    lo = arms.get("learned_bf16", {}).get("orientation_error_vs_truth", {})
    if "median_deg" in po and "median_deg" in lo:
        line["orientation_gate"] = {"learned_median_deg": lo["median_deg"], "plain_median_deg": po["median_deg"],
                                    "allowed_excess_deg": 0.25,
                                    "pass": bool(lo["median_deg"] <= po["median_deg"] + 0.25)}
    # plain FP32 after as many epochs as the learned arm ran (not timed): the
    # direction at equal epochs, beside the gate's comparison at equal residual
    le = arms.get("learned_bf16", {}).get("epochs")
    if md_true is not None and le and arms.get("learned_bf16", {}).get("reached"):
        try:
            vol = torch.full((K, N, N, N), 0.01, dtype=torch.float32, device="cuda")
            scan.osem(b, vol, int(le), W["batch"], 0, 0, final_sqrt=False)
            eq = angle_stats(orientation_of(scan, vol), md_true, fiber_mask)
            eq["epochs"] = int(le)
            eq["residual"] = scan.residual(vol, b, 0, 0)
            line["orientation_plain_f32_at_learned_epochs"] = eq
            del vol
        except Exception as ex:
            line["orientation_plain_f32_at_learned_epochs"] = {"error": f"{type(ex).__name__}: {ex}"}
    line["orientation_note"] = ("angle between per-voxel main directions (calcEigenVector of sqrt|mu|) over the "
                                "fiber voxels of the phantom; the truth is the orientation of the true volume")
    del md_arm, md_true
    scan.ctx.close()
    return line


def run_c4(args, local):
    """Uneven batch: 8 XTT specimens with N drawn from {96, 128, 160, 192}
    (seed 4), 3 axes x U{90..180} views, 256^2 detector, K = 13; BF16
    volumes and sinograms with stochastic rounding, FP32 arithmetic, FP64
    residual norms.  One batched epoch (all specimens forked onto their
    streams, replayed as one CUDA graph, views per CTA and the forward's launch
    shape autotuned) against the
    same epochs run specimen after specimen; per specimen the BF16 result's
    error against an FP32 run of the same epochs."""
    import torch
    ws = load_warmstart()
    xr = load_pkg()
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    rng = np.random.default_rng(4)
    sizes = [int(v) for v in rng.choice([96, 128, 160, 192], 8)]
    views = [int(v) for v in rng.integers(90, 181, 8)]
    basis = basis13()
    specs = []
    for i, (N, V) in enumerate(zip(sizes, views)):
        ctx = xr.Context.create(1000.0, 500.0, 2.0, N, 256, V, three_axes(), None, None, basis, device=local)
        ctx.set_stream(stream.cuda_stream)   # batch forks onto each context's own stream below
        mu = torch.empty((13, N, N, N), dtype=torch.float32, device="cuda")
        ws.fiber_phantom_dev(mu.data_ptr(), N, 12, 400 + i, basis, stream.cuda_stream)
        b = torch.empty((3, V, 256, 256), dtype=torch.float32, device="cuda")
        ctx.dev_forward(mu.data_ptr(), b.data_ptr(), True)
        specs.append({"N": N, "V": V, "ctx": ctx, "b32": b, "b16": b.to(torch.bfloat16)})
    torch.cuda.synchronize()
    E = args.steps

    def fresh(storage):
        dt = torch.bfloat16 if storage else torch.float32
        return [torch.full((13, sp["N"], sp["N"], sp["N"]), 0.01, dtype=dt, device="cuda") for sp in specs]

    def set_opts(storage, graphs):
        for sp in specs:
            sp["ctx"].set_option(xr.Option.STORAGE, storage)
            sp["ctx"].set_option(xr.Option.GRAPHS, graphs)
            sp["ctx"].set_option(xr.Option.XTT_SQRT, 0)

    # FP32 reference results (specimen after specimen)
    set_opts(0, 0)
    ref = fresh(0)
    for sp, v in zip(specs, ref):
        sp["ctx"].dev_session_begin(sp["b32"].data_ptr(), v.data_ptr(), True, E + 1, 5)
        for _ in range(E + 1):
            sp["ctx"].dev_session_epoch()
        sp["ctx"].dev_session_end(0, 0)
    # sequential BF16: each specimen's own session and graphs
    set_opts(1, 1)
    seq = fresh(1)
    seq_ms = 0.0
    for sp, v in zip(specs, seq):
        c = sp["ctx"]
        c.dev_session_begin(sp["b16"].data_ptr(), v.data_ptr(), True, E + 1, 5)
        c.dev_session_epoch()                                  # warm-up (graph capture)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(E):
            c.dev_session_epoch()
        e1.record(stream)
        torch.cuda.synchronize()
        seq_ms += e0.elapsed_time(e1)
        c.dev_session_end(0, 0)
    # batched BF16: every specimen's epoch in one graph
    for sp in specs:
        sp["ctx"].set_stream(0)                                # each context back on its own stream
    bat = fresh(1)
    batch = xr.Batch([sp["ctx"] for sp in specs])
    batch.session_begin([sp["b16"].data_ptr() for sp in specs], [v.data_ptr() for v in bat], True, E + 1, 5)
    chosen, shapes = batch.autotune_shapes()
    batch.epoch()                                              # warm-up (graph capture)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(E):
        batch.epoch()
    bat_ms = (time.perf_counter() - t0) * 1e3                  # each epoch call ends with a synchronize
    batch.session_end()                                        # XTT_SQRT 0: the iterates stay
    batch.close()
    per = []
    for sp, v, r, vpc, shape in zip(specs, bat, ref, chosen, shapes):
        c = sp["ctx"]
        c.set_option(xr.Option.SINO_STORAGE, 0)                # residual against the FP32 data
        res, _ = c.dev_residual(v.data_ptr(), sp["b32"].data_ptr(), True)
        err = float((v.float() - r).abs().max() / r.abs().max())
        per.append({"N": sp["N"], "views": sp["V"], "views_per_cta": vpc, "axes_one_launch": shape,
                    "residual_rel_l2": res,
                    "bf16_vs_fp32_max_rel": err})
    vox_views = sum(3 * sp["V"] * sp["N"] ** 3 for sp in specs)
    line = {"mode": "uneven_batch", "specimens": per, "epochs_timed": E, "storage": "bf16 volumes and sinograms, "
            "stochastic rounding", "sequential_ms_per_epoch": seq_ms / E, "batched_ms_per_epoch": bat_ms / E,
            "speedup_batched": seq_ms / bat_ms, "gvoxel_views_per_s_batched": 2 * vox_views / (bat_ms / E / 1e3) / 1e9,
            "note": "batched time by host clock around synchronized epoch calls; sequential by CUDA events; each "
                    "specimen's BF16 result against an FP32 run of the same epochs on the GPU (the FP64 oracle "
                    "comparison of batched BF16 sessions is in the GPU tests, at sizes the oracle finishes)"}
    for sp in specs:
        sp["ctx"].close()
    torch.cuda.synchronize()
    torch.cuda.set_stream(torch.cuda.default_stream())
    return line


def run_c3(args, local):
    """XTT plain vs batched at 128^3 x 13 (12 seeded fiber cylinders, 3
    sample-rotation axes x 120 views, 192^2 detector, OS-EM 5 subsets, FP32):
    the same epochs with the forward splat as one launch per column axis
    (XR_OPT_AXES_ONE_LAUNCH 0; the back-projection always covers all axes and
    K channels in one launch) and as one launch over all axes (1); device
    time by CUDA events after warm-up epochs, the forward / back split from
    the library's per-class timers, the two forward operators compared."""
    import torch
    xr = load_pkg()
    N, Nd, V, K, C = 128, 192, 120, 13, 3
    basis = basis13()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = xr.Context.create(W["sdd"], W["sod"], W["det"], N, Nd, V, three_axes(), None, None, basis, device=local)
    ctx.set_stream(stream.cuda_stream)
    mu = torch.from_numpy(fiber_phantom(N, 12, 3, basis)).cuda()
    b = torch.empty((C, V, Nd, Nd), dtype=torch.float32, device="cuda")
    ctx.dev_forward(mu.data_ptr(), b.data_ptr(), True)
    arms = {}
    fwd = {}
    for name, opt in (("launch_per_column_axis", 0), ("one_launch", 1)):
        ctx.set_option(xr.Option.AXES_ONE_LAUNCH, opt)
        p = torch.empty_like(b)
        ctx.dev_forward(mu.data_ptr(), p.data_ptr(), True)
        fwd[name] = p
        v = torch.full((K, N, N, N), 0.01, dtype=torch.float32, device="cuda")
        ctx.dev_session_begin(b.data_ptr(), v.data_ptr(), True, args.warmup + 2 * args.steps, 5)
        for _ in range(args.warmup):
            ctx.dev_session_epoch()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            ctx.dev_session_epoch()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.set_option(xr.Option.TIMING, 1)
        ctx.reset_timings()
        for _ in range(args.steps):
            ctx.dev_session_epoch()
        torch.cuda.synchronize()
        tim = ctx.timings()
        ctx.set_option(xr.Option.TIMING, 0)
        ctx.dev_session_end(0, 0)
        arms[name] = {"epoch_ms": e0.elapsed_time(e1) / args.steps,
                      "forward_ms": tim["forward"][0] / args.steps, "back_ms": tim["back"][0] / args.steps,
                      "ratio_ms": tim["ratio"][0] / args.steps,
                      "forward_launches_per_epoch": 5 * (3 if opt == 0 else 1)}
    ctx.set_option(xr.Option.AXES_ONE_LAUNCH, 2)
    a, o = fwd["launch_per_column_axis"].double(), fwd["one_launch"].double()
    bv = bytes_view(K, N, Nd)
    line = {"mode": "xtt_plain_vs_batched", "workload": f"XTT {N}^3 x K{K}, {C} axes x {V} views, {Nd}^2 detector, "
            "OS-EM 5 subsets, FP32 (12 seeded fiber cylinders)", "arms": arms,
            "speedup_one_launch": arms["launch_per_column_axis"]["epoch_ms"] / arms["one_launch"]["epoch_ms"],
            "effective_gbs_one_launch": 2 * C * V * bv / (arms["one_launch"]["epoch_ms"] * 1e-3) / 1e9,
            "forward_max_rel_diff_between_arms": float((a - o).abs().max() / a.abs().max()),
            "default": "one launch for all axes below 2048 bricks per axis (N < 192), one per column axis above",
            "steps": args.steps, "warmup": args.warmup}
    ctx.close()
    torch.cuda.synchronize()
    torch.cuda.set_stream(torch.cuda.default_stream())
    return line


C2 = dict(N=256, Nd=384, V=360, n_ell=20, seed=2, photons=1e5, mu_per_mm=0.002, epochs=50, batch=5, lam=0.005)


def ellipsoids_dev(N, n_ell, seed):
    """Additive random ellipsoids on the device (the generator of
    tests/scans.ellipsoid_phantom: centres and semi-axes uniform within 0.8 of
    the half field of view, random orientation, values U[0.1, 1.0]); z-major."""
    import torch
    rng = np.random.default_rng(seed)
    c = torch.arange(N, device="cuda", dtype=torch.float32) - (N - 1) / 2.0
    vol = torch.zeros((N, N, N), device="cuda")
    half = 0.8 * N / 2.0
    for _ in range(n_ell):
        ctr = rng.uniform(-half, half, 3) * 0.5
        ax = rng.uniform(0.1, 1.0, 3) * half * 0.5
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, cc, d = q
        R = np.array([[a * a + b * b - cc * cc - d * d, 2 * (b * cc - a * d), 2 * (b * d + a * cc)],
                      [2 * (b * cc + a * d), a * a - b * b + cc * cc - d * d, 2 * (cc * d - a * b)],
                      [2 * (b * d - a * cc), 2 * (cc * d + a * b), a * a - b * b - cc * cc + d * d]])
        val = rng.uniform(0.1, 1.0)
        Rt = torch.tensor(R / ax[None, :], device="cuda", dtype=torch.float32)   # columns scaled by 1/axes
        for z in range(N):
            zz = c[z] - ctr[2]
            yy = (c - ctr[1])[:, None]
            xx = (c - ctr[0])[None, :]
            u = [xx * Rt[0, i] + yy * Rt[1, i] + zz * Rt[2, i] for i in range(3)]
            inside = (u[0] ** 2 + u[1] ** 2 + u[2] ** 2) <= 1.0
            vol[z] += inside.float() * val
    return vol


def run_c2(args, local):
    """Plain cone-beam FDK + OS-ART (the reference's FDK::reconstruct then
    IR::reconstruct with Method::ART, reconstruct.cu:1651-1724, :23-156):
    256^3 volume of 20 seeded ellipsoids, 360 views over 360 degrees, 384^2
    detector, SOD 500 / SDD 1000 mm, 1 mm voxels.  Noisy data: the phantom's
    values are attenuation in units of 0.002 / mm (value 1 = 0.2 / cm), counts
    I ~ Poisson(1e5 exp(-b)) per ray, b = -ln(max(I, 1) / 1e5).  FDK with the
    Ram-Lak filter; its volume, moved from the FDK frame (source at -sod,
    centred grid) to the iterative one (+1 voxel on each axis) and scaled by
    the least-squares factor <A f, b> / <A f, A f>, starts 50 OS-ART epochs (5
    subsets, lambda 0.005: the step the ray length of 256 voxels allows).
    Device times by CUDA events (the library's per-class timers)."""
    import torch
    xr = load_pkg()
    P = C2
    N, Nd, V = P["N"], P["Nd"], P["V"]
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = xr.Context.create(W["sdd"], W["sod"], W["det"], N, Nd, V, np.eye(3, dtype=np.float32).reshape(1, 9),
                            device=local)
    ctx.set_stream(stream.cuda_stream)
    mu = ellipsoids_dev(N, P["n_ell"], P["seed"]).contiguous()
    b = torch.empty((1, V, Nd, Nd), dtype=torch.float32, device="cuda")
    ctx.dev_forward(mu.data_ptr(), b.data_ptr(), False)
    g = torch.Generator(device="cuda").manual_seed(P["seed"])
    counts = torch.poisson(P["photons"] * torch.exp(-b * P["mu_per_mm"]), generator=g)
    bn = (-torch.log(counts.clamp_min(1.0) / P["photons"]) / P["mu_per_mm"]).contiguous()
    torch.cuda.synchronize()
    noise_rel = float(torch.linalg.vector_norm(bn - b) / torch.linalg.vector_norm(b))
    # FDK on host buffers (the reference's call surface), device time by its timer
    ctx.set_option(xr.Option.TIMING, 1)
    ctx.reset_timings()
    t0 = time.perf_counter()
    f_vol, _ = ctx.fdk_reconstruct(bn.cpu().numpy(), xr.Rotate.CW, xr.Filter.RAMLAK)
    fdk_wall = time.perf_counter() - t0
    fdk_ms = ctx.timings()["fdk"][0]
    f = torch.from_numpy(f_vol[0]).cuda().roll(shifts=(1, 1, 1), dims=(0, 1, 2)).contiguous()
    af = torch.empty_like(b)
    ctx.dev_forward(f.data_ptr(), af.data_ptr(), False)
    torch.cuda.synchronize()
    scale = float((af.double() * bn.double()).sum() / (af.double() * af.double()).sum())
    vol = (f * scale).contiguous()
    r_fdk, _ = ctx.dev_residual(vol.data_ptr(), bn.data_ptr(), False)
    err_fdk = float(torch.linalg.vector_norm(vol - mu) / torch.linalg.vector_norm(mu))
    ctx.reset_timings()
    ctx.dev_session_begin(bn.data_ptr(), vol.data_ptr(), False, P["epochs"], P["batch"], method=xr.Method.ART,
                          lam=P["lam"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(P["epochs"]):
        ctx.dev_session_epoch()
    e1.record(stream)
    torch.cuda.synchronize()
    art_ms = e0.elapsed_time(e1)
    tim = ctx.timings()
    ctx.dev_session_end(0, 0)
    ctx.set_option(xr.Option.TIMING, 0)
    r_art, _ = ctx.dev_residual(vol.data_ptr(), bn.data_ptr(), False)
    r_clean, _ = ctx.dev_residual(vol.data_ptr(), b.data_ptr(), False)
    err_art = float(torch.linalg.vector_norm(vol - mu) / torch.linalg.vector_norm(mu))
    bv = bytes_view(1, N, Nd)
    fwd_ms, back_ms = tim["forward"][0] / P["epochs"], tim["back"][0] / P["epochs"]
    line = {"workload": f"plain cone-beam {N}^3, {V} views over 360 deg, {Nd}^2 detector, {P['n_ell']} ellipsoids, "
            f"Poisson {P['photons']:.0e} photons; FDK (Ram-Lak) + {P['epochs']} OS-ART epochs ({P['batch']} subsets, "
            f"lambda {P['lam']})", "noise_rel_l2": noise_rel,
            "fdk_ms": fdk_ms, "fdk_host_call_s": fdk_wall, "fdk_scale_to_iterative_units": scale,
            "residual_rel_l2_noisy_after_fdk": r_fdk, "residual_rel_l2_noisy_after_art": r_art,
            "residual_rel_l2_clean_after_art": r_clean, "volume_rel_error_after_fdk": err_fdk,
            "volume_rel_error_after_art": err_art, "art_ms_per_epoch": art_ms / P["epochs"],
            "forward_ms_per_epoch": fwd_ms, "back_ms_per_epoch": back_ms,
            "forward_effective_gbs": V * bv / (fwd_ms * 1e-3) / 1e9,
            "back_effective_gbs": V * bv / (back_ms * 1e-3) / 1e9,
            "forward_compulsory_hbm_frac": (5 * N ** 3 * 4 + V * Nd * Nd * 4) / (fwd_ms * 1e-3) / 1e9 /
            measured_peaks()[0],
            "back_compulsory_hbm_frac": (5 * 2 * N ** 3 * 4 + V * Nd * Nd * 4) / (back_ms * 1e-3) / 1e9 /
            measured_peaks()[0],
            "note": "effective GB/s charge bytes_view = N^3*4 + Nd^2*4 per view; compulsory = per subset launch the "
                    "volume read (and written by the back) once plus its views' images"}
    ctx.close()
    del mu, b, bn, counts, vol, f, af
    torch.cuda.empty_cache()
    return line


def run_reference_gpu(d_b, local, epochs: int = 1):
    """The reference's own CUDA kernels on this GPU (reconstruct/src/ir.cu
    built for sm_100a, oracle/_ref/libxrref_gpu.so), driven like its
    XTT::reconstruct: one launch and one device synchronize per y slab and
    view (reconstruct.cu:857-911), on the same workload and data as the
    timed epochs (b = A mu_true, mu = 0.01).  Times of whole epochs by CUDA
    events inside the driver."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefGPU, Scan
    if not RefGPU.available():
        return {"unavailable": "oracle/_ref/libxrref_gpu.so not built (make -C oracle ref with the reference sources)"}
    s = Scan(sdd=W["sdd"], sod=W["sod"], det=W["det"], N=W["N"], Nd=W["Nd"], V=W["V"], rot=three_axes(),
             trans=np.zeros((3, 3)), offset=np.zeros((3, 3)), basis=basis13())
    b = d_b.cpu().numpy()
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    _, _, losses, ms = RefGPU().xtt_reconstruct(s, b, v0, epochs, W["batch"], want_ratio=False)
    return {"ms_per_epoch": float(np.mean(ms)), "epochs": epochs, "loss_first_epoch": float(losses[0]),
            "launches_per_epoch": int(2 * s.C * s.V * s.N + s.C * s.V * 2 + W["batch"] * s.N * (1 + s.K)),
            "note": "the reference's ir.cu kernels compiled for this B200 and its per-slab launch + "
                    "cudaDeviceSynchronize structure; FP32, same workload and data as the timed epochs"}


def run_fiber(args, local):
    """Fiber model (fiber.cu, fiberModelReconstruct): forwardProjFiber over
    every (axis, view) pair, and OS-EM epochs (5 subsets) of forward, ratio and
    back-projection with the update of channel 0, on a 128^3 x 4 volume of
    signed fiber vectors plus an isotropic term, 3 axes x 120 views, 192^2
    detector.  Device time by CUDA events on the library's stream, after
    --warmup untimed repetitions."""
    import torch
    xr = load_pkg()
    N, Nd, V, K, C = 128, 192, 120, 4, 3
    rng = np.random.default_rng(11)
    vol_h = rng.uniform(-1.0, 1.0, (K, N, N, N)).astype(np.float32)
    vol_h[3] = np.abs(vol_h[3]) * 0.5
    ctx = xr.Context.create(W["sdd"], W["sod"], W["det"], N, Nd, V, three_axes(), None, None,
                            np.eye(4, 3, dtype=np.float32), device=local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    vol = torch.from_numpy(vol_h).cuda()
    sino = torch.empty((C, V, Nd, Nd), dtype=torch.float32, device="cuda")
    ctx.dev_forward_fiber(vol.data_ptr(), sino.data_ptr())
    out = torch.empty_like(sino)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        ctx.dev_forward_fiber(vol.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        ctx.dev_forward_fiber(vol.data_ptr(), out.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / args.steps
    rec = torch.full_like(vol, 0.01)
    ctx.dev_session_begin_fiber(sino.data_ptr(), rec.data_ptr(), args.warmup + args.steps, 5)
    for _ in range(args.warmup):
        ctx.dev_session_epoch()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        ctx.dev_session_epoch()
    e1.record(stream)
    torch.cuda.synchronize()
    ep_ms = e0.elapsed_time(e1) / args.steps
    ctx.dev_session_end(0, 0)
    bv = bytes_view(K, N, Nd)
    line = {"mode": "fiber_model", "workload": f"fiber model {N}^3 x K{K}, {C} axes x {V} views, {Nd}^2 detector, "
            "OS-EM 5 subsets, FP32", "forward_ms": fwd_ms, "epoch_ms": ep_ms,
            "forward_effective_gbs": C * V * bv / (fwd_ms * 1e-3) / 1e9,
            "epoch_effective_gbs": 2 * C * V * bv / (ep_ms * 1e-3) / 1e9, "steps": args.steps, "warmup": args.warmup}
    ctx.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--size", default="full", choices=["full", "profile"])
    ap.add_argument("--ttr", action="store_true",
                    help="time-to-residual: OS-EM from mu = 0.01 until ||A mu - b|| / ||b|| <= --target")
    ap.add_argument("--target", type=float, default=1e-3)
    ap.add_argument("--max-epochs", type=int, default=1000)
    ap.add_argument("--check-every", type=int, default=10)
    ap.add_argument("--early", type=int, default=5, help="--ttr: OS-EM epochs before the warm-start network")
    ap.add_argument("--arms", default="plain_f32,learned_bf16", help="--ttr arms (also plain_bf16, learned_f32)")
    ap.add_argument("--weights", default="", help="--ttr: warm-start network file (default: the package's)")
    ap.add_argument("--no-ttr", action="store_true", help="skip the time-to-residual comparison of the default run")
    ap.add_argument("--c4", action="store_true", help="uneven batch of 8 specimens (BF16), batched vs sequential")
    ap.add_argument("--c2", action="store_true", help="plain cone-beam FDK + 50 OS-ART epochs at 256^3, 360 views")
    ap.add_argument("--c3", action="store_true", help="XTT 128^3 x 13: forward per column axis vs one launch")
    ap.add_argument("--no-configs", action="store_true", help="skip the FDK+ART and uneven-batch lines of the default run")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the epoch of the reference's CUDA kernels")
    ap.add_argument("--fiber", action="store_true", help="fiber-model forward and epoch timing (128^3 x 4)")
    ap.add_argument("--conv", type=int, default=0, metavar="N",
                    help="only the warm-start network's tensor-core roofline on an N^3 x 13 volume")
    args = ap.parse_args()
    if args.size == "profile":
        W.update(W_PROFILE)
        args.no_e2e = True
        args.no_cpu_baseline = True
    if args.warmup < 3:
        args.warmup = 3

    rp = load_replicas()
    rank, world, local = rp.rank_env()

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch

    torch.cuda.set_device(local)
    if args.conv:
        if rank == 0:
            torch.cuda.set_stream(torch.cuda.Stream())
            print(json.dumps(conv_roofline(local, args.conv)), flush=True)
        return
    if args.ttr or args.c4 or args.fiber or args.c2 or args.c3:
        if rank == 0:          # one GPU: these comparisons run on rank 0 only
            if args.ttr:
                print(json.dumps(run_ttr(args, local)), flush=True)
            elif args.c3:
                print(json.dumps(run_c3(args, local)), flush=True)
            elif args.fiber:
                print(json.dumps(run_fiber(args, local)), flush=True)
            elif args.c2:
                print(json.dumps(run_c2(args, local)), flush=True)
            else:
                print(json.dumps(run_c4(args, local)), flush=True)
        return
    if world > 1:
        rp.init("nccl")

    xr = load_pkg()
    s_basis = basis13()
    ctx = xr.Context.create(W["sdd"], W["sod"], W["det"], W["N"], W["Nd"], W["V"], three_axes(), None, None,
                            s_basis, device=local)
    # one non-default stream shared by torch and the library, so the CUDA
    # events below bracket the library's kernels
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    N, Nd, V, C, K = W["N"], W["Nd"], W["V"], W["C"], W["K"]
    mu_true = fiber_phantom(N, W["n_fibers"], rp.specimen_seed(W["seed"], rank), s_basis)   # one specimen per replica
    d_true = torch.from_numpy(mu_true).cuda()
    d_b = torch.empty((C, V, Nd, Nd), dtype=torch.float32, device="cuda")
    ctx.dev_forward(d_true.data_ptr(), d_b.data_ptr(), True)           # b = A mu_true
    d_vol = torch.full((K, N, N, N), 0.01, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    ctx.dev_session_begin(d_b.data_ptr(), d_vol.data_ptr(), True, args.warmup + args.steps, W["batch"])
    for _ in range(args.warmup):
        ctx.dev_session_epoch()
    torch.cuda.synchronize()
    ctx.set_option(xr.Option.TIMING, 1)
    ctx.reset_timings()

    sampler = ClockSampler(local)
    if world > 1:
        rp.barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        ctx.dev_session_epoch()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    t_ms = ev0.elapsed_time(ev1) / args.steps
    tim = ctx.timings()
    ctx.set_option(xr.Option.TIMING, 0)
    rel, _ = ctx.dev_residual(d_vol.data_ptr(), d_b.data_ptr(), True)   # ||A mu - b|| / ||b|| after the epochs
    ctx.dev_session_end(0, 0)

    def epoch_ms(storage, graphs, steps, split=None):
        """Mean epoch time of a fresh session (same inputs) with the given
        storage type and graph replay; warm-up epochs untimed.  split: a dict
        that receives the per-class device times per epoch, averaged over the
        timed epochs, which then run with the per-class timing events on, as
        the FP32 epochs of the headline do (direct epochs only: timing events
        are not recorded inside graphs)."""
        ctx.set_option(xr.Option.STORAGE, storage)
        ctx.set_option(xr.Option.GRAPHS, graphs)
        dt = {0: torch.float32, 1: torch.bfloat16, 2: torch.float16}[storage]
        db = d_b.to(dt)
        dv = torch.full((K, N, N, N), 0.01, dtype=dt, device="cuda")
        torch.cuda.synchronize()
        ctx.dev_session_begin(db.data_ptr(), dv.data_ptr(), True, args.warmup + steps, W["batch"])
        for _ in range(args.warmup):
            ctx.dev_session_epoch()
        torch.cuda.synchronize()
        if split is not None:
            ctx.set_option(xr.Option.TIMING, 1)
            ctx.reset_timings()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(steps):
            ctx.dev_session_epoch()
        a1.record(stream)
        torch.cuda.synchronize()
        ms = a0.elapsed_time(a1) / steps
        if split is not None:
            split.update({k: v[0] / steps for k, v in ctx.timings().items() if v[1]})
            ctx.set_option(xr.Option.TIMING, 0)
        ctx.dev_session_end(0, 0)
        ctx.set_option(xr.Option.GRAPHS, 0)
        ctx.set_option(xr.Option.STORAGE, 0)
        del db, dv
        return ms

    bf16_split = {}
    variants = {"f32_graphs": epoch_ms(0, 1, args.steps), "bf16": epoch_ms(1, 0, args.steps, bf16_split),
                "bf16_graphs": epoch_ms(1, 1, args.steps), "bf16_kernel_ms": bf16_split}

    bv = bytes_view(K, N, Nd)
    per_gpu_bytes = 2 * C * V * bv
    value = world * per_gpu_bytes / (t_ms / 1e3) / 1e9

    # roofline of the dominant kernel (forward or back), per launch.  The
    # forward of a subset is one k_fwd_col launch per column axis g (the three
    # axes here have g = z, x, y: 3 launches of V/batch views); the fused back
    # projection + update is one k_back_col launch over all axes' views.
    subset = (V + W["batch"] - 1) // W["batch"]
    rot = three_axes().reshape(C, 3, 3)
    n_groups = len({int(np.argmax(np.abs(r[:, 2]))) for r in rot})
    if ((N + 15) // 16) ** 2 * ((N + 7) // 8) < 2048:   # XR_OPT_AXES_ONE_LAUNCH's default: one launch for all axes
        n_groups = 1
    fwd_ms, fwd_n = tim["forward"]
    back_ms, back_n = tim["back"]
    if fwd_ms >= back_ms:
        dom, dom_ms, dom_n, units = "k_fwd_col<1,g,float>", fwd_ms, fwd_n * n_groups, C * subset // n_groups
    else:
        dom, dom_ms, dom_n, units = "k_back_col<3,float>", back_ms, back_n, C * subset
    peak, peak_kind = measured_peaks()
    avg_launch_s = dom_ms / max(dom_n, 1) / 1e3
    # compulsory DRAM bytes of one launch: the forward reads the volume once and
    # writes its views' detector images; the back reads the volume, the
    # per-subset sensitivity and the ratio images and writes the volume
    if dom.startswith("k_fwd"):
        # channels whose grating weight (S_k . G)^2 is zero for an axis are not read
        grat = rot[:, :, 2]                                  # G = elemR e_z per axis
        active = float(np.mean([(np.abs(s_basis @ gv) > 1e-6).sum() for gv in grat]))
        compulsory = active * N ** 3 * 4 + units * Nd * Nd * 4
    else:
        compulsory = 3 * K * N ** 3 * 4 + units * Nd * Nd * 4
    hbm = {"bound": "hbm", "kernel": dom, "achieved": compulsory / avg_launch_s / 1e9, "peak": peak, "unit": "GB/s",
           "frac": compulsory / avg_launch_s / 1e9 / peak, "peak_kind": peak_kind, "bytes_per_launch": compulsory,
           "note": "compulsory bytes of one launch (each operand moved once) over its CUDA-event time"}
    effective = {"kernel": dom, "gbs": units * bv / avg_launch_s / 1e9, "bytes_per_unit": bv, "units_per_launch": units,
                 "note": "bytes_view = K*N^3*4 + Nd^2*4 charged per view: one volume read serves every view of the "
                         "launch, so this exceeds the HBM peak and is not a roofline fraction"}
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    roofline = issue_roofline(dom, avg_launch_s, float(N) ** 3 * units, float(N) ** 3, float(Nd * Nd) * units,
                              sm_mhz, peak)
    if roofline is None:           # no captured instruction counts: the HBM view alone
        roofline = dict(hbm, traffic=None)
    roofline_l1 = l1_roofline(dom, avg_launch_s, float(N) ** 3 * units, sm_mhz)
    roofline.update({"avg_launch_ms": avg_launch_s * 1e3, "units_per_launch": units, "peak_kind": "sampled SM clock"
                     if roofline["bound"] == "issue" else peak_kind})
    # kernels in the timed region: per subset n_groups forward launches, one
    # ratio launch, one back launch
    launches = int(fwd_n * n_groups + tim["ratio"][1] + back_n)

    # e2e through the public host-buffer API (pinned host memory), every rank
    e2e = None
    e2e_ms = None
    if not args.no_e2e:
        h_b = d_b.cpu().pin_memory()
        h_v0 = torch.full((K, N, N, N), 0.01, dtype=torch.float32).pin_memory()
        h_vol = torch.empty((K, N, N, N), dtype=torch.float32).pin_memory()
        h_sino = torch.empty((C, V, Nd, Nd), dtype=torch.float32).pin_memory()
        h_md = torch.empty((3, N, N, N), dtype=torch.float32).pin_memory()
        FP = ctypes.POINTER(ctypes.c_float)

        def ptrs(t, n):
            base = t.data_ptr()
            step = t[0].numel() * 4
            return (FP * n)(*[ctypes.cast(base + i * step, FP) for i in range(n)])

        L = xr.lib()
        times = []
        for i in range(3 + args.steps):
            h_vol.copy_(h_v0)
            h_sino.copy_(h_b)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            # the reference's XTT::reconstruct returns the volume, the last ratio
            # images and the main directions (as the compat layer's call): no eigenvalues
            st = L.xr_xtt_reconstruct(ctx._h, ptrs(h_sino, C), ptrs(h_vol, K), ptrs(h_md, 3),
                                      None, 1, W["batch"], 0, 1, ctypes.c_float(1e-2), None)
            e1.record(stream)
            torch.cuda.synchronize()
            if st:
                raise RuntimeError(L.xr_last_error(ctx._h).decode())
            if i >= 3:
                times.append(e0.elapsed_time(e1))
        e2e_ms = float(np.mean(times))

    if world > 1:
        t_max, e_max = rp.max_over_ranks([t_ms, e2e_ms or 0.0], device="cuda")
        t_ms, e2e_ms = t_max, (e_max if e2e_ms else None)
        value = rp.whole_job_rate(per_gpu_bytes, world, t_ms) / 1e9
        if rank != 0:
            ctx.close()
            rp.finish()
            return
    if e2e_ms:
        h2d = C * V * Nd * Nd * 4 + K * N ** 3 * 4
        d2h = K * N ** 3 * 4 + C * V * Nd * Nd * 4 + 3 * N ** 3 * 4
        e2e = {"value": world * per_gpu_bytes / (e2e_ms / 1e3) / 1e9, "unit": "GB/s",
               "ms_per_step": e2e_ms, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "call": "xr_xtt_reconstruct(epoch=1) with pinned host buffers, incl. sqrt + main directions "
                       "(the outputs of the reference's XTT::reconstruct)"}

    cpu = None
    if not args.no_cpu_baseline and world == 1:
        n_views = 3
        hb = d_b.cpu().numpy()
        t, threads = cpu_reference_sample(np.full_like(mu_true, 0.01), lambda cond, n: hb[cond, n].ravel(),
                                          n_views, 0)
        cpu = {"value": 2 * n_views * bv / t / 1e9, "unit": "GB/s", "cores": threads, "kind": "reference",
               "sample": f"{n_views} of {C * V} (axis, view) pairs (one per axis), forward + correlation + ratio + "
                         "back-projection of all K channels, reference ir.cu kernels compiled for the host, OpenMP; "
                         "the GPU arm's measured images and OS-EM start"}

    ref_gpu = None
    if world == 1 and args.size == "full" and not args.no_ref_gpu:
        try:
            ref_gpu = run_reference_gpu(d_b, local)
            if "ms_per_epoch" in ref_gpu:
                ref_gpu["libxr_ms_per_epoch"] = t_ms
                ref_gpu["libxr_speedup"] = ref_gpu["ms_per_epoch"] / t_ms
        except Exception as ex:      # the reference's run is reported, it does not cost the line
            ref_gpu = {"error": f"{type(ex).__name__}: {ex}"}
    ttr = None
    if world == 1 and not args.no_ttr and args.size == "full":
        ctx.close()
        del d_true, d_b, d_vol
        torch.cuda.empty_cache()
        t = run_ttr(args, local)
        ttr = {"target_rel_residual": t["target"], "speedup_learned_bf16_vs_plain_f32":
               t["speedup_learned_bf16_vs_plain_f32"], "note": "device time to the target, residual checked every "
               f"{t['check_every']} epochs and after every epoch within 5 % of the target, outside the timed work; "
               "same data b = A mu_true (held-out phantom)",
               "orientation_learned_bf16_vs_plain_f32": t["orientation_learned_bf16_vs_plain_f32"],
               "orientation_note": t["orientation_note"], "orientation_gate": t.get("orientation_gate"),
               "orientation_plain_f32_at_learned_epochs": t.get("orientation_plain_f32_at_learned_epochs"),
               "network": t.get("network")}
        for k, a in t["arms"].items():
            ttr[k] = {x: a.get(x) for x in ("seconds", "epochs", "reached", "residual_final", "storage",
                                            "orientation_error_vs_truth", "unavailable") if x in a}
    conv = None
    if world == 1 and args.size == "full":
        conv = conv_roofline(local)
    c2 = c3 = c4 = None
    if world == 1 and args.size == "full" and not args.no_configs:
        c2 = run_c2(args, local)
        c3 = run_c3(args, local)
        c4 = run_c4(args, local)
    line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(args, world), "residual_rel_l2_after": rel,
            "e2e": e2e, "roofline": roofline, "roofline_l1": roofline_l1, "roofline_hbm": hbm,
            "effective_projector": effective,
            "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in tim.items() if v[1]},
            "variants_ms_per_step": variants, "time_to_residual": ttr, "roofline_conv": conv,
            "fdk_art_256": c2, "xtt_plain_vs_batched_128": c3, "uneven_batch_bf16": c4, "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        rp.finish()


if __name__ == "__main__":
    main()
