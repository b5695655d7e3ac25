"""Pin the oracle: its FP32 restatement must reproduce, bit for bit, the
golden vectors produced by the reference's own reconstruct/src/ir.cu compiled
for the host (tests/golden/make_golden.py).  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import RefHost, Scan


def _scan(g, p) -> Scan:
    sdd, sod, det, N, Nd, V = g[p + "geom"]
    return Scan(sdd=float(sdd), sod=float(sod), det=float(det), N=int(N), Nd=int(Nd), V=int(V),
                rot=g[p + "rot"], trans=g[p + "trans"], offset=g[p + "offset"], basis=g[p + "basis"])


@pytest.mark.parametrize("xtt", [0, 1])
@pytest.mark.parametrize("cond", [0, 1, 2])
def test_unit_kernels_bit_exact(oracle, golden, xtt, cond):
    s = _scan(golden, "unit_")
    N, Nd, V = s.N, s.Nd, s.V
    vol = golden["unit_vol"].ravel().copy()
    sino = golden["unit_sino"].ravel().copy()
    n = 3 + cond
    sl = slice(n * Nd * Nd, (n + 1) * Nd * Nd)
    p = np.zeros(V * Nd * Nd, np.float32)
    f = np.zeros(Nd * Nd, np.float32)
    oracle.forward_view(s, cond, n, vol, p, f, xtt)                 # a1-a4
    assert np.array_equal(p[sl], golden[f"fwd_x{xtt}_c{cond}_proj"])
    assert np.array_equal(f, golden[f"fwd_x{xtt}_c{cond}_factor"])
    oracle.correlation(s, cond, n, p, f)                            # a5
    assert np.array_equal(p[sl], golden[f"cor_x{xtt}_c{cond}"])
    for art in (0, 1):                                              # a6
        q = p.copy()
        loss = oracle.ratio(s, n, q, sino, art)
        assert np.array_equal(q[sl], golden[f"rat_x{xtt}_c{cond}_a{art}"])
        assert np.float32(loss) == golden[f"rat_x{xtt}_c{cond}_a{art}_loss"][0]
    q = np.zeros(V * Nd * Nd, np.float32)
    q[sl] = golden[f"bwd_x{xtt}_c{cond}_in"]
    t = np.zeros(N * N * s.K, np.float32)
    g = np.zeros(N * N * s.K, np.float32)
    oracle.backward_slab(s, cond, 5, n, q, t, g, xtt)               # a7-a8
    assert np.array_equal(t, golden[f"bwd_x{xtt}_c{cond}_tmp"])
    assert np.array_equal(g, golden[f"bwd_x{xtt}_c{cond}_factor"])


def test_forward_all_xtt_bit_exact(oracle, golden):
    s = _scan(golden, "unit_")
    got = oracle.forward_all(s, golden["unit_vol"], 0, True)
    assert np.array_equal(got, golden["fwdall_xtt"])


@pytest.mark.parametrize("art", [0, 1])
def test_ir_reconstruct_bit_exact(oracle, golden, art):
    """IR::reconstruct (a9, a11): 3 epochs, batch 3 over 10 views (so the
    subset wrap-around revisits views), MLEM and ART."""
    s = _scan(golden, "ir_")
    vol, loss = oracle.ir_reconstruct(s, golden["ir_sino"], np.ones((1, s.N, s.N, s.N), np.float32),
                                      3, 3, art=bool(art), lam=1e-2)
    assert np.array_equal(vol, golden[f"ir_a{art}_vol"])
    assert np.array_equal(loss[-1], golden[f"ir_a{art}_loss"])


@pytest.mark.parametrize("art", [0, 1])
def test_xtt_reconstruct_bit_exact(oracle, golden, art):
    """XTT::reconstruct (a4, a8-a11): 3 axes, K = 13, sqrt at the end."""
    s = _scan(golden, "xtt_")
    v0 = np.full((s.K, s.N, s.N, s.N), 0.01, np.float32)
    vol, proj, loss = oracle.xtt_reconstruct(s, golden["xtt_sino"], v0, 2, 3, art=bool(art), lam=1e-3)
    assert np.array_equal(vol, golden[f"xtt_a{art}_vol"])
    assert np.array_equal(proj, golden[f"xtt_a{art}_proj"])
    assert np.array_equal(loss, golden[f"xtt_a{art}_loss"])


def test_fp64_oracle_close_to_fp32(oracle, golden):
    """The FP64 instantiation computes the same operator (sanity of the
    template): relative difference at FP32 rounding level."""
    s = _scan(golden, "unit_")
    a = oracle.forward_all(s, golden["unit_vol"], 0, True)
    b = oracle.forward_all(s, golden["unit_vol"].astype(np.float64), 0, True, dt=np.float64)
    assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()


def test_subset_orders_match_reference_engine(oracle):
    """The reference shuffles with a default-seeded std::mt19937_64
    (reconstruct.cu:75,858): the order for batch 5 is fixed by libstdc++."""
    o = oracle.subset_orders(5, 3, True)
    assert all(sorted(r) == list(range(5)) for r in o)
    # XTT re-seeds every epoch and shuffles the persistent order: row e+1 is
    # the same permutation applied once more to row e.
    assert list(o[1]) == [o[0][o[0][i]] for i in range(5)]
    o2 = oracle.subset_orders(5, 3, True)
    assert np.array_equal(o, o2)


def test_jacobi_known_answer(oracle):
    """FP64 Jacobi eigensolver (orientation step) on known matrices."""
    w, V = oracle.jacobi3(np.diag([3.0, 1.0, 2.0]))
    assert np.allclose(w, [1, 2, 3])
    assert np.allclose(np.abs(V[:, 0]), [0, 1, 0])
    rng = np.random.default_rng(0)
    for _ in range(20):
        A = rng.normal(size=(3, 3))
        A = A + A.T
        w, V = oracle.jacobi3(A)
        wr = np.linalg.eigvalsh(A)
        assert np.allclose(w, wr, atol=1e-12)
        assert np.allclose(A @ V, V * w, atol=1e-10)


def test_orientation_against_lapack(oracle):
    """calcEigenVector (direction/src/pca.cu:12-55) against LAPACK's eigh of
    the same tensor: smallest-eigenvalue direction, z-sign rule, mean-mu
    scaling and normalised eigenvalues.  A fiber voxel (coefficients
    |S_k x f|) points close to f."""
    from scans import basis13
    b = basis13().astype(np.float64)
    rng = np.random.default_rng(5)
    f = np.array([0.3, -0.5, 0.81])
    f /= np.linalg.norm(f)
    fiber = np.sqrt(np.sum(np.cross(b, f) ** 2, 1))
    mu = np.concatenate([fiber[:, None], rng.uniform(0, 1, (13, 50))], 1).astype(np.float32)
    md, ev = oracle.orientation(b.astype(np.float32), mu)
    for i in range(mu.shape[1]):
        m = mu[:, i].astype(np.float64)
        T = (b * m[:, None] ** 2).T @ b / 13.0
        w, V = np.linalg.eigh(T)
        v = V[:, 0] * (1.0 if V[2, 0] >= 0 else -1.0)
        assert np.allclose(md[:, i], m.mean() * v, atol=1e-5)
        assert np.allclose(ev[:, i], w / w.sum(), atol=1e-5)
    v0 = md[:, 0] / np.linalg.norm(md[:, 0])
    assert abs(v0 @ f) > 0.95


@pytest.mark.skipif(not RefHost.available(), reason="reference host build absent")
def test_reference_build_loads():
    r = RefHost()
    assert r.lib.xr_ref_vox_size is not None
