/*
 * The oracle — TEST INFRASTRUCTURE ONLY.  A CPU restatement of the
 * reference's reconstruction hot path (see xr_oracle_impl.h for what each
 * function follows).  Built by oracle/Makefile into oracle/liboracle.so.
 * Nothing in the product links or calls this library; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and only
 * to check results.
 *
 * Exports or32_* (FP32, the reference's operation order) and or64_* (FP64),
 * plus or_orientation (FP64 Jacobi restatement of direction/src/pca.cu:12-55)
 * and or_angle_from_md / or_direction_normalization (pca.cu:67-106).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "xr_oracle.h"

#define OR_CAT2(a, b) a##b
#define OR_CAT(a, b) OR_CAT2(a, b)

/* The reference's atan2(float, float) in host code resolves to the double
 * function (its <cmath> float overloads are not brought in for atan2), so
 * the FP32 restatement rounds the double result. */
static float or_atan2f(float y, float x) { return (float)atan2((double)y, (double)x); }

/* ---- FP32 instantiation ---- */
#define real float
#define OR_PFX or32_
#define OR_IS_FLOAT 1
#define RCOS cosf
#define RSIN sinf
#define RSQRT sqrtf
#define RFLOOR floorf
#define RFABS fabsf
#define RATAN2 or_atan2f
#include "xr_oracle_impl.h"
#undef real
#undef OR_PFX
#undef OR_IS_FLOAT
#undef RCOS
#undef RSIN
#undef RSQRT
#undef RFLOOR
#undef RFABS
#undef RATAN2

/* ---- FP64 instantiation ---- */
#define real double
#define OR_PFX or64_
#define OR_IS_FLOAT 0
#define RCOS cos
#define RSIN sin
#define RSQRT sqrt
#define RFLOOR floor
#define RFABS fabs
#define RATAN2 atan2
#include "xr_oracle_impl.h"

/* Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix (FP64),
 * eigenvalues ascending with their unit eigenvectors in the columns of V.
 * Restates what pca.cu:33-36 asks of Eigen::SelfAdjointEigenSolver (Eigen
 * itself is third-party and absent; the Jacobi method is Golub & Van Loan,
 * Matrix Computations, section 8.5). */
void or_jacobi3(const double *Ain, double *w, double *V) {
    double A[9];
    memcpy(A, Ain, sizeof(A));
    for (int i = 0; i < 9; i++) V[i] = (i % 4 == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 50; sweep++) {
        const double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
        const double dia = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
        if (off <= 1e-300 || off <= 1e-34 * dia) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                const double apq = A[3 * p + q];
                if (apq == 0.0) continue;
                const double theta = (A[3 * q + q] - A[3 * p + p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) { /* A <- J^T A J */
                    const double akp = A[3 * k + p], akq = A[3 * k + q];
                    A[3 * k + p] = c * akp - s * akq;
                    A[3 * k + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {
                    const double apk = A[3 * p + k], aqk = A[3 * q + k];
                    A[3 * p + k] = c * apk - s * aqk;
                    A[3 * q + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    const double vkp = V[3 * k + p], vkq = V[3 * k + q];
                    V[3 * k + p] = c * vkp - s * vkq;
                    V[3 * k + q] = s * vkp + c * vkq;
                }
            }
    }
    int idx[3] = {0, 1, 2};
    double d[3] = {A[0], A[4], A[8]};
    for (int i = 0; i < 3; i++) /* stable ascending sort */
        for (int j = i + 1; j < 3; j++)
            if (d[idx[j]] < d[idx[i]]) { int tt = idx[i]; idx[i] = idx[j]; idx[j] = tt; }
    double Vs[9];
    for (int c = 0; c < 3; c++) {
        w[c] = d[idx[c]];
        for (int r = 0; r < 3; r++) Vs[3 * r + c] = V[3 * r + idx[c]];
    }
    memcpy(V, Vs, sizeof(Vs));
}

/* calcEigenVector (direction/src/pca.cu:12-55) for every voxel, in FP64:
 * T = (1/K) sum_k (mu_k S_k)(mu_k S_k)^T; v = unit eigenvector of the smallest
 * eigenvalue; md = sign(v_z >= 0 ? 1 : -1) * mean(mu) * v; evalue_i =
 * lambda_i / sum(lambda).  mu: K channels of nvox; md, ev: 3 channels. */
void or_orientation(long nvox, int K, const float *basis, const float *mu, float *md, float *ev) {
    for (long i = 0; i < nvox; i++) {
        double T[9] = {0}, mean = 0;
        for (int k = 0; k < K; k++) {
            const double m = mu[(long)k * nvox + i];
            const double sc[3] = {m * basis[3 * k], m * basis[3 * k + 1], m * basis[3 * k + 2]};
            mean += m;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) T[3 * a + b] += sc[a] * sc[b];
        }
        mean /= K;
        for (int a = 0; a < 9; a++) T[a] /= K;
        double w[3], V[9];
        or_jacobi3(T, w, V);
        double v0[3] = {V[0], V[3], V[6]};
        const double nv = sqrt(v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2]);
        for (int a = 0; a < 3; a++) v0[a] /= nv;
        const double sg = v0[2] >= 0 ? 1.0 : -1.0;
        const double tr = w[0] + w[1] + w[2];
        for (int a = 0; a < 3; a++) {
            md[(long)a * nvox + i] = (float)(sg * mean * v0[a]);
            ev[(long)a * nvox + i] = (float)(w[a] / tr);
        }
    }
}

/* calcAngleFromMD, direction/src/pca.cu:67-83, elementwise over nvox voxels
 * of three planes: the reference's std::atan2 and std::sqrt of floats are
 * their float overloads (atan2f, sqrtf).  angle: phi plane, theta plane. */
void or_angle_from_md(long nvox, const float *md, float *angle) {
    for (long i = 0; i < nvox; i++) {
        const float m0 = md[i], m1 = md[nvox + i], m2 = md[2 * nvox + i];
        if (m1 < 0.f) {
            angle[i] = atan2f(-m1, -m0);
            angle[nvox + i] = atan2f(sqrtf(m1 * m1 + m0 * m0), -m2);
        } else {
            angle[i] = atan2f(m1, m0);
            angle[nvox + i] = atan2f(sqrtf(m1 * m1 + m0 * m0), m2);
        }
    }
}

/* directionNormalization, direction/src/pca.cu:85-106, in place: unit
 * vectors where the length exceeds 0.65, zero vectors elsewhere. */
void or_direction_normalization(long nvox, float *md) {
    for (long i = 0; i < nvox; i++) {
        const float x = md[i], y = md[nvox + i], z = md[2 * nvox + i];
        const float norm = sqrtf(x * x + y * y + z * z);
        if (norm > 0.65f) {
            md[i] = x / norm;
            md[nvox + i] = y / norm;
            md[2 * nvox + i] = z / norm;
        } else {
            md[i] = 0.f;
            md[nvox + i] = 0.f;
            md[2 * nvox + i] = 0.f;
        }
    }
}
