"""Replica-parallel bookkeeping on CPU with the gloo backend, world size 2:
distinct specimens per rank, MAX of per-rank device times, whole-job rate,
and a short process-group timeout when a rank never joins."""
from __future__ import annotations

import importlib.util
import os
import socket

import pytest

from conftest import PKG_DIR

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _replicas():
    spec = importlib.util.spec_from_file_location("xr_replicas", os.path.join(PKG_DIR, "replicas.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    rp = _replicas()
    r, w, local = rp.rank_env()
    rp.init("gloo", timeout_s=30)
    seed = rp.specimen_seed(5, r)
    t_ms = 100.0 + 50.0 * r          # rank 1 is the slow one
    e2e_ms = 300.0 - 10.0 * r
    mx = rp.max_over_ranks([t_ms, e2e_ms])
    rate = rp.whole_job_rate(1.0e9, w, mx[0])
    out.put((r, w, local, seed, mx, rate))
    rp.finish()


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 for x in res)
    assert res[0][3] != res[1][3]                        # different specimens
    for x in res:
        assert x[4] == [150.0, 300.0]                    # slowest rank's device time, on every rank
        assert abs(x[5] - 2 * 1.0e9 / 0.150) < 1e-3 * x[5]


def _lonely(port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="2", LOCAL_RANK="0")
    rp = _replicas()
    try:
        rp.init("gloo", timeout_s=3)
        rp.max_over_ranks([1.0])
        out.put("no error")
    except Exception as e:  # rendezvous or collective timeout
        out.put(type(e).__name__)


def test_missing_rank_times_out_on_host():
    """A rank that never joins: the other's rendezvous ends with an error
    within the short timeout (failure made on the host, no GPU involved)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely, args=(_free_port(), q))
    p.start()
    msg = q.get(timeout=120)
    p.join(timeout=60)
    assert msg != "no error"
