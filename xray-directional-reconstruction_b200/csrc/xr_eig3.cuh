/*
 * Symmetric 3x3 eigen-decomposition in FP64 by cyclic Jacobi rotations
 * (Golub & Van Loan, Matrix Computations, section 8.5): A (row-major, full)
 * is overwritten, w receives the diagonal (eigenvalues, unordered), V the
 * eigenvectors as columns.  Stops when the off-diagonal mass falls below
 * 1e-34 of the diagonal's (or 50 sweeps).
 */
#ifndef XR_EIG3_CUH
#define XR_EIG3_CUH

namespace xr {

__device__ inline void jacobi3(double A[9], double w[3], double V[9]) {
#pragma unroll
    for (int i = 0; i < 9; i++) V[i] = (i % 4 == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 50; sweep++) {
        const double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
        const double dia = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
        if (off <= 1e-300 || off <= 1e-34 * dia) break;
#pragma unroll
        for (int pq = 0; pq < 3; pq++) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            const double apq = A[3 * p + q];
            if (apq == 0.0) continue;
            const double theta = (A[3 * q + q] - A[3 * p + p]) / (2.0 * apq);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double akp = A[3 * k + p], akq = A[3 * k + q];
                A[3 * k + p] = c * akp - s * akq;
                A[3 * k + q] = s * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double apk = A[3 * p + k], aqk = A[3 * q + k];
                A[3 * p + k] = c * apk - s * aqk;
                A[3 * q + k] = s * apk + c * aqk;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double vkp = V[3 * k + p], vkq = V[3 * k + q];
                V[3 * k + p] = c * vkp - s * vkq;
                V[3 * k + q] = s * vkp + c * vkq;
            }
        }
    }
    w[0] = A[0];
    w[1] = A[4];
    w[2] = A[8];
}

/* Ascending order of w (stable), as an index permutation. */
__device__ inline void order3(const double w[3], int idx[3]) {
    idx[0] = 0; idx[1] = 1; idx[2] = 2;
    for (int a = 0; a < 3; a++)
        for (int b = a + 1; b < 3; b++)
            if (w[idx[b]] < w[idx[a]]) { const int t = idx[a]; idx[a] = idx[b]; idx[b] = t; }
}

}  // namespace xr

#endif
