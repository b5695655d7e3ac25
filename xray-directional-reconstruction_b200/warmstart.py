"""Learned warm start for XTT OS-EM: training-data synthesis, training on the
tensor cores, and the warm-started reconstruction (include/xr_learn.h).

The reference has no learned component; this module drives libxr's own
kernels only (projector, OS-EM sessions, tensor-core convolutions, Adam).
torch provides device memory and streams.

Pairs: a seeded fiber phantom mu_true (12 cylinders, radius U[2,5] voxels,
direction uniform on the sphere, eta_k = |S_k x f|^2 inside), its noiseless
XTT projections b = A mu_true, and the output of the reference-style
XTT::reconstruct after `early_epochs` OS-EM epochs from a constant start
(the voxelSqrt of the iterate).  The training target is, by choice:
  converged  the method's own converged reconstruction: plain FP32 OS-EM
             from the same constant start run until the relative data
             residual reaches `target_residual` (the iterate, no voxelSqrt).
             The 13 channels are not all determined by 3 axes x V views, so
             plain OS-EM converges to one particular solution of A mu = b;
             this is the one a warm start should lead it to.
  truth      mu_true itself (the phantom; a solution of A mu = b, though not
             the one the iteration reaches from a constant start).
The network learns early iterate -> target on random cubic crops.

    python xray-directional-reconstruction_b200/warmstart.py train --target converged --depths 4 --out W.bin
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "warmstart_k13.bin")


def _pkg():
    if "xrd" in sys.modules:
        return sys.modules["xrd"]
    spec = importlib.util.spec_from_file_location("xrd", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["xrd"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_net(path: str = WEIGHTS, device: int = 0):
    """A network of the shape recorded in a weights file (xr_net_save
    format: magic, int32 channels, width, depth, FP32 parameters)."""
    import struct
    with open(path, "rb") as f:
        head = f.read(20)
    if len(head) < 20 or head[:6] != b"XRNET1":
        raise ValueError(f"not a network file: {path}")
    channels, width, depth = struct.unpack("<3i", head[8:20])
    net = _pkg().Net(channels, width, depth, device=device)
    net.load(path)
    return net


def cubic13() -> np.ndarray:
    """13 unit scattering directions, one per antipodal pair of the cubic
    symmetry directions: 3 axes, 6 face diagonals, 4 body diagonals."""
    d = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1),
         (0, 1, 1), (0, 1, -1), (1, 1, 1), (1, 1, -1), (1, -1, 1), (-1, 1, 1)]
    return np.array([np.asarray(v, np.float64) / np.linalg.norm(v) for v in d], np.float32)


def three_axes() -> np.ndarray:
    """Sample-rotation axes of the three-axis scans: identity and the two
    90-degree tilts (rotation axis along x, along y)."""
    return np.array([[1, 0, 0, 0, 1, 0, 0, 0, 1],
                     [0, 0, -1, 0, 1, 0, 1, 0, 0],
                     [1, 0, 0, 0, 0, -1, 0, 1, 0]], np.float32)


def fiber_params(N: int, n_fib: int, seed: int) -> np.ndarray:
    """(n_fib, 7) rows (f, p0, r) drawn in the order of the numpy phantom
    generator: f ~ normalised N(0, I), p0 ~ U[-0.3N, 0.3N]^3, r ~ U[2, 5]."""
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(n_fib):
        f = rng.normal(size=3)
        f /= np.linalg.norm(f)
        p0 = rng.uniform(-0.3 * N, 0.3 * N, 3)
        r = rng.uniform(2.0, 5.0)
        rows.append(np.concatenate([f, p0, [r]]))
    return np.array(rows, np.float32).reshape(n_fib, 7)


def fiber_phantom_dev(out_ptr: int, N: int, n_fib: int, seed: int, basis: np.ndarray, stream: int = 0) -> None:
    """Fiber phantom (K, N, N, N) FP32 written on the device by libxr."""
    import ctypes
    xr = _pkg()
    b = np.ascontiguousarray(basis, np.float32)
    fib = fiber_params(N, n_fib, seed)
    F = ctypes.POINTER(ctypes.c_float)
    st = xr.lib().xr_dev_fiber_phantom(ctypes.c_void_p(stream), N, b.shape[0], b.ctypes.data_as(F), n_fib,
                                       fib.ctypes.data_as(F), ctypes.c_void_p(out_ptr))
    if st:
        raise xr.XRError(st, "xr_dev_fiber_phantom")


class Scan:
    """The three-axis XTT scan of the warm-start workloads (SOD 500 / SDD 1000,
    2 mm pixels: 1 mm voxels), scaled to N: N_d = 1.5 N."""

    def __init__(self, N: int, V: int = 180, device: int = 0, n_fibers: int = 12):
        import torch
        self.xr = _pkg()
        self.N, self.V, self.Nd, self.C = N, V, (3 * N) // 2, 3
        self.basis = cubic13()
        self.K = self.basis.shape[0]
        self.n_fibers = n_fibers
        self.ctx = self.xr.Context.create(1000.0, 500.0, 2.0, N, self.Nd, V, three_axes(), None, None, self.basis,
                                          device=device)
        # one non-default stream for torch's copies and libxr's kernels (CUDA
        # graph capture needs a non-default stream)
        self.stream = torch.cuda.Stream()
        torch.cuda.set_stream(self.stream)
        self.ctx.set_stream(self.stream.cuda_stream)

    def phantom(self, seed: int):
        import torch
        t = torch.empty((self.K, self.N, self.N, self.N), dtype=torch.float32, device="cuda")
        fiber_phantom_dev(t.data_ptr(), self.N, self.n_fibers, seed, self.basis, self.stream.cuda_stream)
        return t

    def project(self, mu):
        import torch
        b = torch.empty((self.C, self.V, self.Nd, self.Nd), dtype=torch.float32, device="cuda")
        self.ctx.dev_forward(mu.data_ptr(), b.data_ptr(), True)
        return b

    def osem(self, b, vol, epochs: int, batch: int = 5, storage: int = 0, sino_storage: int = -1,
             residual_every: int = 0, target: float = 0.0, max_epochs: int = 0, graphs: bool = False,
             final_sqrt: bool = True, fine_within: float = 0.05):
        """OS-EM (XTT MLEM) epochs on the device volume `vol` in place (b and
        vol of the given storage types).  With residual_every > 0, runs until
        the relative data residual <= target or max_epochs, checking it every
        residual_every epochs and after every epoch once it is within
        fine_within (relative) of the target, so the epoch that reaches the
        target is found exactly.  final_sqrt: end like the reference's
        XTT::reconstruct (voxelSqrt of the result), else leave the iterate.
        Returns (epochs run, device milliseconds of session set-up + epochs,
        residual trace [(epoch, ms, residual)]); residual checks are not
        timed."""
        import torch
        xr = self.xr
        self.ctx.set_option(xr.Option.XTT_SQRT, 1 if final_sqrt else 0)
        self.ctx.set_option(xr.Option.STORAGE, storage)
        self.ctx.set_option(xr.Option.SINO_STORAGE, sino_storage)
        self.ctx.set_option(xr.Option.GRAPHS, 1 if graphs else 0)
        total = max_epochs if residual_every else epochs
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        self.ctx.dev_session_begin(b.data_ptr(), vol.data_ptr(), True, total, batch)
        ms, trace, e = 0.0, [], 0
        first = True
        step = residual_every
        while e < total:
            n = min(step, total - e) if residual_every else total
            if not first:
                e0.record(self.stream)
            first = False
            for _ in range(n):
                self.ctx.dev_session_epoch()
            e1.record(self.stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            e += n
            if residual_every:
                r, _ = self.ctx.dev_residual(vol.data_ptr(), b.data_ptr(), True)
                trace.append((e, ms, r))
                if r <= target:
                    break
                if r <= target * (1.0 + fine_within):
                    step = 1
        self.ctx.dev_session_end(0, 0)
        self.ctx.set_option(xr.Option.STORAGE, 0)
        self.ctx.set_option(xr.Option.SINO_STORAGE, -1)
        self.ctx.set_option(xr.Option.GRAPHS, 0)
        self.ctx.set_option(xr.Option.XTT_SQRT, 1)
        return e, ms, trace

    def residual(self, vol, b, storage: int = 0, sino_storage: int = -1) -> float:
        xr = self.xr
        self.ctx.set_option(xr.Option.STORAGE, storage)
        self.ctx.set_option(xr.Option.SINO_STORAGE, sino_storage)
        r, _ = self.ctx.dev_residual(vol.data_ptr(), b.data_ptr(), True)
        self.ctx.set_option(xr.Option.STORAGE, 0)
        self.ctx.set_option(xr.Option.SINO_STORAGE, -1)
        return r


def make_pool(scan: Scan, seeds, crops_per: int, crop: int, early_epochs: int = 5, batch: int = 5,
              mu0: float = 0.01, rng_seed: int = 0, storage: int = 0, target: str = "truth",
              target_residual: float = 1e-3, max_epochs: int = 2000, check_every: int = 10, log=None):
    """Random crops of (early iterate, target) pairs, stacked on the device:
    two (P, K, crop, crop, crop) FP32 tensors.  The early iterate runs with
    volumes of the given storage type (FP32 data); target "truth" is mu_true,
    "converged" plain FP32 OS-EM from mu0 to `target_residual`."""
    import torch
    if target not in ("truth", "converged"):
        raise ValueError("target must be 'truth' or 'converged'")
    rng = np.random.default_rng(rng_seed)
    xs, ts = [], []
    N = scan.N
    dt = {0: torch.float32, 1: torch.bfloat16, 2: torch.float16}[storage]
    for s in seeds:
        mu = scan.phantom(int(s))
        b = scan.project(mu)
        vol = torch.full(mu.shape, mu0, dtype=dt, device="cuda")
        scan.osem(b, vol, early_epochs, batch, storage=storage, sino_storage=0)
        if target == "converged":
            ref = torch.full(mu.shape, mu0, dtype=torch.float32, device="cuda")
            e, ms, trace = scan.osem(b, ref, 0, batch, residual_every=check_every, target=target_residual,
                                     max_epochs=max_epochs, final_sqrt=False)
            if log is not None:
                log.append({"seed": int(s), "epochs": e, "ms": ms, "residual": trace[-1][2] if trace else None})
            del mu
            mu = ref
        for _ in range(crops_per):
            o = rng.integers(0, N - crop + 1, 3)
            sl = (slice(None), slice(o[0], o[0] + crop), slice(o[1], o[1] + crop), slice(o[2], o[2] + crop))
            xs.append(vol[sl].float().contiguous())
            ts.append(mu[sl].contiguous())
        del mu, b, vol
    return torch.stack(xs), torch.stack(ts)


def train(net, xin, tgt, steps: int, lr: float = 2e-3, lr_final: float = 1e-4, seed: int = 0, log_every: int = 100):
    """Adam on random pool entries, learning rate decayed geometrically from
    lr to lr_final; returns the loss trace [(step, loss)]."""
    rng = np.random.default_rng(seed)
    P = xin.shape[0]
    shape = tuple(xin.shape[2:])
    trace = []
    for it in range(steps):
        i = int(rng.integers(0, P))
        loss, _ = net.loss_grad(xin[i].data_ptr(), tgt[i].data_ptr(), shape)
        a = lr * (lr_final / lr) ** (it / max(steps - 1, 1))
        net.adam_step(a)
        if it % log_every == 0 or it == steps - 1:
            trace.append((it, loss))
    return trace


def warm_start(scan: Scan, net, b, vol, early_epochs: int = 5, batch: int = 5, storage: int = 0,
               sino_storage: int = -1):
    """The warm-started reconstruction's first part: `early_epochs` OS-EM
    epochs ending like the reference's XTT::reconstruct (its output is the
    voxelSqrt of the iterate), then the network in place on the device
    volume, clamped at 0: it maps that output to an estimate of the
    converged iterate mu, from which OS-EM continues (final_sqrt=False until
    the end).  Returns the milliseconds spent (set-up, epochs, inference;
    CUDA events)."""
    import torch
    _, ms, _ = scan.osem(b, vol, early_epochs, batch, storage, sino_storage)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(scan.stream)
    net.infer(vol.data_ptr(), vol.data_ptr(), (scan.N, scan.N, scan.N), storage=storage, floor_value=0.0)
    e1.record(scan.stream)
    torch.cuda.synchronize()
    return ms + e0.elapsed_time(e1)


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser(description="train the warm-start network on synthetic fiber phantoms")
    ap.add_argument("cmd", choices=["train"])
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--phantoms", type=int, default=200)
    ap.add_argument("--seed0", type=int, default=1000)
    ap.add_argument("--crops", type=int, default=4)
    ap.add_argument("--crop", type=int, default=64)
    ap.add_argument("--early", type=int, default=5)
    ap.add_argument("--depths", default="4", help="comma-separated network depths, each trained on the same pool")
    ap.add_argument("--tensor-loss", default="0",
                    help="comma-separated weights of the loss's direction-tensor term (0: plain MSE), each trained "
                         "on the same pool")
    ap.add_argument("--target", default="converged", choices=["converged", "truth"])
    ap.add_argument("--target-residual", type=float, default=1e-3)
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--lr", type=float, default=1.5e-3)
    ap.add_argument("--storage", type=int, default=1, help="volume storage of the early iterates (1 = BF16)")
    ap.add_argument("--log", default="")
    args = ap.parse_args(argv)
    xr = _pkg()
    torch.cuda.set_device(0)
    scan = Scan(args.N)
    t0 = time.time()
    tlog = []
    xin, tgt = make_pool(scan, range(args.seed0, args.seed0 + args.phantoms), args.crops, args.crop, args.early,
                         storage=args.storage, target=args.target, target_residual=args.target_residual, log=tlog)
    t1 = time.time()
    depths = [int(d) for d in args.depths.split(",")]
    tweights = [float(w) for w in args.tensor_loss.split(",")]
    recs = []
    for depth in depths:
        for tw in tweights:
            t2 = time.time()
            net = xr.Net(scan.K, 32, depth, seed=0)
            net.set_stream(scan.stream.cuda_stream)
            net.set_tensor_loss(scan.basis, tw)
            trace = train(net, xin, tgt, args.steps, args.lr)
            torch.cuda.synchronize()
            t3 = time.time()
            out = args.out
            if len(depths) > 1:
                out = out.replace(".bin", f"_d{depth}.bin")
            if len(tweights) > 1:
                out = out.replace(".bin", f"_t{tw:g}.bin")
            os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
            net.save(out)
            net.close()
            recs.append({"out": os.path.basename(out), "depth": depth, "tensor_loss": tw, "train_s": t3 - t2,
                         "loss_trace": trace})
    rec = {"pairs": int(xin.shape[0]), "phantoms": args.phantoms, "seeds": [args.seed0, args.seed0 + args.phantoms - 1],
           "N": args.N, "crop": args.crop, "crops_per_phantom": args.crops, "early_epochs": args.early,
           "target": args.target, "target_residual": args.target_residual, "steps": args.steps, "lr": args.lr,
           "storage": args.storage, "pool_s": t1 - t0, "targets": tlog, "networks": recs}
    print(json.dumps(rec))
    if args.log:
        with open(args.log, "w") as f:
            json.dump(rec, f, indent=1)


if __name__ == "__main__":
    main()
