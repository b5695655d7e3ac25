"""CPU oracle for the regularisers (test infrastructure only: imported by
tests/, never by the product).

Restates, with numpy / scipy.sparse in float64:
* totalVariationMinimized (solver/src/tvmin.cpp:6-98): F built row by row as
  the reference's triplet loop builds it (forward differences at voxels with
  x < X-1, y < Y-1, z < Z-1; rows (3 v + c)), y = u = 1, and per ADMM
  iteration the exact solution of (I + rho F^T F) x = F^T (rho y - u) + x0
  (a sparse direct solve, standing in for the reference's BiCGSTAB run to
  machine precision), then the soft threshold and the dual update.
* quadlicFormFilterCPU (reconstruct/src/quadfilt.cpp:11-134): the per-voxel
  Rodrigues rotation from (phi, cos theta), Q = R^T diag(m, m, 0) R with
  m = mu0 + mu1 + mu2 and mu = (v1, v2, v0), TV on the 6 elements (rho 3,
  20 iterations), and the eigen-decomposition (numpy eigh, ascending).

Parity unpinned: the reference runs these on the host with Eigen, a
third-party library absent here (find_package(Eigen3 3.3), version not
pinned), so no reference output could be produced; the restatement is
checked by its own identities (tests/test_regularisers_oracle.py).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def tv_operator(X: int, Y: int, Z: int) -> sp.csr_matrix:
    """F (3N x N), rows 3 * co(x, y, z) + c, as tvmin.cpp:23-41."""
    N = X * Y * Z
    rows, cols, vals = [], [], []
    co = lambda x, y, z: x + X * y + X * Y * z
    for x in range(X - 1):
        for y in range(Y - 1):
            for z in range(Z - 1):
                v = co(x, y, z)
                for c, w in enumerate((co(x + 1, y, z), co(x, y + 1, z), co(x, y, z + 1))):
                    rows += [3 * v + c, 3 * v + c]
                    cols += [w, v]
                    vals += [1.0, -1.0]
    return sp.csr_matrix((vals, (rows, cols)), shape=(3 * N, N))


def tv_minimize(vol: np.ndarray, rho: float, lam: float, iters: int) -> np.ndarray:
    """vol: (Z, Y, X) array; returns the ADMM result of the same shape."""
    Z, Y, X = vol.shape
    N = X * Y * Z
    F = tv_operator(X, Y, Z)
    x0 = np.asarray(vol, np.float64).ravel()
    yy = np.ones(3 * N)
    uu = np.ones(3 * N)
    lhs = (sp.identity(N, format="csc") + rho * (F.T @ F)).tocsc()
    solve = spla.factorized(lhs)
    xx = x0.copy()
    for _ in range(iters):
        rhs = F.T @ (rho * yy - uu) + x0
        xx = solve(rhs)
        fx = F @ xx
        z = fx + uu / rho
        yy = np.where(z > 0, np.maximum(z - lam / rho, 0.0), np.minimum(z + lam / rho, 0.0))
        uu = uu + rho * (fx - yy)
    return xx.reshape(Z, Y, X)


def quad_tensor(vox: np.ndarray, coef: np.ndarray) -> np.ndarray:
    """vox (3, ...), coef (2, ...) -> the 6 elements (Q00, Q11, Q22, Q01, Q02, Q12)."""
    vox = np.asarray(vox, np.float64)
    phi, c = np.asarray(coef[0], np.float64), np.asarray(coef[1], np.float64)
    m = vox[1] + vox[2] + vox[0]
    x, y, z = np.cos(phi), np.sin(phi), np.zeros_like(phi)
    s = np.sqrt(1.0 - c * c)
    nrm = np.sqrt(x * x + y * y + z * z)
    nx, ny, nz = x / nrm, y / nrm, z / nrm
    oc = 1.0 - c
    R = np.array([[oc * nx * nx + c, oc * nx * ny - nz * s, oc * nx * nz + ny * s],
                  [oc * nx * ny + nz * s, oc * ny * ny + c, oc * ny * nz - nx * s],
                  [oc * nx * nz - ny * s, oc * ny * nz + nx * s, oc * nz * nz + c]])
    qe = lambda a, b: m * (R[0, a] * R[0, b] + R[1, a] * R[1, b])
    return np.stack([qe(0, 0), qe(1, 1), qe(2, 2), qe(0, 1), qe(0, 2), qe(1, 2)])


def quad_decompose(q: np.ndarray):
    """Filtered elements -> (vox (3, ...), coef (2, ...)) as quadfilt.cpp:97-132."""
    shape = q.shape[1:]
    Q = np.zeros(shape + (3, 3))
    Q[..., 0, 0], Q[..., 1, 1], Q[..., 2, 2] = q[0], q[1], q[2]
    Q[..., 0, 1] = Q[..., 1, 0] = q[3]
    Q[..., 0, 2] = Q[..., 2, 0] = q[4]
    Q[..., 1, 2] = Q[..., 2, 1] = q[5]
    w, V = np.linalg.eigh(Q)
    n = V[..., :, 0]
    n = n / np.linalg.norm(n, axis=-1, keepdims=True)
    n = np.where(n[..., 2:3] >= 0, n, -n)
    coef = np.stack([np.arctan2(-n[..., 0], n[..., 1]), n[..., 2]])
    vox = np.stack([w[..., 1], w[..., 2], w[..., 0]])
    return vox, coef


def quad_form_filter(vox: np.ndarray, coef: np.ndarray, lam: float):
    """vox (3, Z, Y, X), coef (2, Z, Y, X) -> filtered (vox, coef)."""
    q = quad_tensor(vox, coef)
    q = np.stack([tv_minimize(q[e], 3.0, lam, 20) for e in range(6)])
    return quad_decompose(q)
