/*
 * CPU restatement of the reference's reconstruction hot path — TEST
 * INFRASTRUCTURE ONLY (the oracle).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it, and only as the checker.
 *
 * This file is included twice by xr_oracle.c: once with real = float (the
 * reference's FP32 arithmetic, operation by operation, so that per-voxel
 * detector coordinates and weights are bit-identical to the reference compiled
 * for the host) and once with real = double (the FP64 oracle used to state the
 * error of every GPU result).
 *
 * Pinned against: oracle/_ref/libxrref.so, the reference's own
 * reconstruct/src/ir.cu compiled through oracle/ref_shim, via the golden
 * vectors in tests/golden (tests/golden/make_golden.py).  The FDK part is
 * pinned the same way against the reference's fdk.cu kernels (lines 1-170,
 * built for the host from a slice: the file's later Hilbert variant holds a
 * kernel launch) by tests/golden/make_golden_fdk.py.  The orientation step
 * needs Eigen, which is absent: a restatement without a reference-run pin.
 *
 * Layouts follow the reference: volumes x-fastest (idx = x + N*y + N*N*z,
 * volume.h:65-71), K channels of N^3 back to back (ir.cu:1788-1790);
 * projections u-fastest, then v, then view (ir.cu:1518), C blocks of V views.
 */

#define RV(name) OR_CAT(OR_PFX, name)

typedef struct {
    real R[9];      /* Rotate = elemR[cond] * Rz(theta)          ir.cu:1865-1872 */
    real off[3];    /* Rotate * INIT_OFFSET[cond]                ir.cu:1873       */
    real t[3];      /* elemT[cond]                               ir.cu:1870       */
    real src[3];    /* Rotate * (0, sod, 0)                      ir.cu:1874,1879  */
    real eu[3];     /* Rotate * (1, 0, 0)                        ir.cu:1875,1896  */
    real ev[3];     /* Rotate * (0, 0, 1)                        ir.cu:1876,1897  */
    real ss;        /* src . src                                 ir.cu:1893       */
} RV(frame);

/* Matrix3X::operator*(Matrix3X) (vec.h:171-181): w = 0; w += a*b over k. */
static void RV(mat3mul)(const real *a, const real *b, real *w) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            real s = (real)0;
            for (int k = 0; k < 3; k++) s += a[3 * i + k] * b[3 * k + j];
            w[3 * i + j] = s;
        }
}

/* Matrix3X::operator*(Vector3X) (vec.h:193-201). */
static void RV(mat3vec)(const real *a, const real *v, real *w) {
    for (int i = 0; i < 3; i++) {
        real s = (real)0;
        for (int j = 0; j < 3; j++) s += a[3 * i + j] * v[j];
        w[i] = s;
    }
}

/* Vector3X::operator*(Vector3X) (vec.h:66-68). */
static real RV(dot3)(const real *a, const real *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* The per-(axis, view) part of rayCasting, ir.cu:1860-1879 (also the head of
 * correlationProjByLength ir.cu:1541-1553 and FDK's backwardonDevice
 * fdk.cu:111-130, which differs only in the source sign). */
void RV(view_frame)(const or_scan *s, int cond, int n, int fdk_frame, RV(frame) * f) {
    const real theta = (real)2.0 * (real)M_PI * (real)n / (real)s->V;
    const real c = RCOS(theta), sn = RSIN(theta);
    const real Rz[9] = {c, -sn, (real)0, sn, c, (real)0, (real)0, (real)0, (real)1};
    real cR[9], off0[3];
    for (int i = 0; i < 9; i++) cR[i] = (real)s->rot[9 * cond + i];
    for (int i = 0; i < 3; i++) {
        off0[i] = (real)s->offset[3 * cond + i];
        f->t[i] = (real)s->trans[3 * cond + i];
    }
    RV(mat3mul)(cR, Rz, f->R);
    RV(mat3vec)(f->R, off0, f->off);
    const real o2s[3] = {(real)0, fdk_frame ? -(real)s->sod : (real)s->sod, (real)0};
    const real bu[3] = {(real)1, (real)0, (real)0}, bv[3] = {(real)0, (real)0, (real)1};
    RV(mat3vec)(f->R, o2s, f->src);
    RV(mat3vec)(f->R, bu, f->eu);
    RV(mat3vec)(f->R, bv, f->ev);
    f->ss = RV(dot3)(f->src, f->src);
}

static real RV(vox_size)(const or_scan *s) { return (real)s->sod * (real)s->det / (real)s->sdd; } /* geometry.h:13 */

/* rayCasting, ir.cu:1852-1902 (per voxel).  fdk_frame selects FDK's centred
 * voxel grid (fdk.cu:132-135).  Returns u, v, the unit ray B and, through o,
 * origin2voxel (FDK's magnification weight needs its y). */
void RV(raycast)(const or_scan *s, const RV(frame) * f, int fdk_frame, int x, int y, int z, real *u,
                 real *v, real *B, real *o) {
    const real vs = RV(vox_size)(s);
    const real N = (real)s->N;
    const int xyz[3] = {x, y, z};
    real org[3], d[3], p[3];
    for (int i = 0; i < 3; i++) {
        if (fdk_frame)
            org[i] = ((real)2.0 * (real)xyz[i] - N + (real)1.0) * (real)0.5 * vs - f->off[i] - f->t[i];
        else
            org[i] = ((real)2.0 * (real)xyz[i] - N - (real)1.0) * (real)0.5 * vs - f->off[i] - f->t[i];
    }
    for (int i = 0; i < 3; i++) d[i] = org[i] - f->src[i];
    const real coeff = -(f->ss) / RV(dot3)(f->src, d);
    for (int i = 0; i < 3; i++) p[i] = f->src[i] + coeff * d[i];
    const real mag = (real)s->sdd / (real)s->sod;
    *u = RV(dot3)(p, f->eu) * mag / (real)s->det + (real)0.5 * (real)s->Nd;
    *v = RV(dot3)(p, f->ev) * mag / (real)s->det + (real)0.5 * (real)s->Nd;
    if (B) { /* Vector3X::normalize(1e-8), vec.h:93-105 */
        const real val = RSQRT(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int i = 0; i < 3; i++) B[i] = (val > (real)1e-8f) ? d[i] / val : (real)0;
    }
    if (o)
        for (int i = 0; i < 3; i++) o[i] = org[i];
}

/* Detector window and bilinear taps, e.g. ir.cu:1501-1509. Returns 0 outside. */
static int RV(taps)(const or_scan *s, real u, real v, long *iu, long *iv, real c[4]) {
    const real lim = (real)s->Nd - (real)0.55f;
    if (!((real)0.55f < u && u < lim && (real)0.55f < v && v < lim)) return 0;
    const real ut = u - (real)0.5, vt = v - (real)0.5;
    *iu = (long)RFLOOR(ut);
    *iv = (long)RFLOOR(vt);
    const real fu = ut - (real)*iu, fv = vt - (real)*iv;
    c[0] = ((real)1 - fu) * fv;          /* (iu,   iv+1) */
    c[1] = fu * fv;                      /* (iu+1, iv+1) */
    c[2] = fu * ((real)1 - fv);          /* (iu+1, iv)   */
    c[3] = ((real)1 - fu) * ((real)1 - fv); /* (iu, iv)  */
    return 1;
}

/* (|B x S_k| * |S_k . G|)^2, ir.cu:1785-1786. */
static real RV(xtt_weight)(const real *B, const real *S, const real *G) {
    const real cx = B[1] * S[2] - B[2] * S[1];
    const real cy = B[2] * S[0] - B[0] * S[2];
    const real cz = B[0] * S[1] - B[1] * S[0];
    const real vkm = RSQRT(cx * cx + cy * cy + cz * cz) * RFABS(RV(dot3)(S, G));
    return vkm * vkm;
}

/* rodriguesRotation, ir.cu:597-623: rotation about (x, y, z) normalised by
 * the angle with the given cosine / sine (identity below |n| < 1e-8), as
 * (1 - cos) n n^T + [cos, -nz sin, ny sin; nz sin, cos, -nx sin; -ny sin, nx sin, cos]. */
static void RV(rodrigues)(real x, real y, real z, real c, real sn, real *R) {
    if (RSQRT(x * x + y * y + z * z) < (real)1e-8f) {
        for (int i = 0; i < 9; i++) R[i] = (i % 4 == 0) ? (real)1 : (real)0;
        return;
    }
    const real nx = x / RSQRT(x * x + y * y + z * z);
    const real ny = y / RSQRT(x * x + y * y + z * z);
    const real nz = z / RSQRT(x * x + y * y + z * z);
    const real r1[9] = {nx * nx, nx * ny, nx * nz, nx * ny, ny * ny, ny * nz, nx * nz, ny * nz, nz * nz};
    const real r2[9] = {c, -nz * sn, ny * sn, nz * sn, c, -nx * sn, -ny * sn, nx * sn, c};
    for (int i = 0; i < 9; i++) R[i] = ((real)1 - c) * r1[i] + r2[i];
}

/* The per-voxel rotation of the orientation-parametrised projectors
 * (ir.cu:319-331, :390-395): coef planes (phi, cos theta) ->
 * rodrigues(cos phi, sin phi, 0, cos theta, sqrt(1 - cos^2 theta)). */
static void RV(orth_rotation)(const real *coef, long N3, long idx, real *R) {
    const real phi = coef[idx], ct = coef[N3 + idx];
    RV(rodrigues)(RCOS(phi), RSIN(phi), (real)0, ct, RSQRT((real)1 - ct * ct), R);
}

/* forwardProj/forwardonDevice (ir.cu:1480-1531, xtt == 0) or
 * forwardProjXTT/forwardXTTonDevice (ir.cu:133-141,1753-1804, xtt != 0) for
 * one view over every y slab, in the reference's launch order (y, then z, then
 * x).  proj is the axis block base (all views); factor is the per-view weight
 * image, accumulated (the caller zeroes it, reconstruct.cu:88/:866). */
void RV(forward_view)(const or_scan *s, int cond, int n, const real *vol, real *proj, real *factor,
                      int xtt) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd;
    const long nn = n < 0 ? -n : n;
    const real vs = RV(vox_size)(s);
    const real ratio = (vs * vs) / ((real)s->det * ((real)s->sod / (real)s->sdd) * (real)s->det *
                                    ((real)s->sod / (real)s->sdd));
    real G[3];
    { const real bz[3] = {(real)0, (real)0, (real)1}; RV(mat3vec)(f.R, bz, G); }
    for (long y = 0; y < N; y++)
        for (long z = 0; z < N; z++)
            for (long x = 0; x < N; x++) {
                real u, v, B[3], c[4];
                long iu, iv;
                RV(raycast)(s, &f, 0, (int)x, (int)y, (int)z, &u, &v, xtt ? B : 0, 0);
                if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
                const long idx = x + N * y + N * N * z;
                real val[4];
                if (!xtt) {
                    for (int i = 0; i < 4; i++) val[i] = c[i] * ratio * vol[idx];
                } else {
                    real pr = (real)0;
                    for (int k = 0; k < s->K; k++) {
                        real S[3] = {(real)s->basis[3 * k], (real)s->basis[3 * k + 1], (real)s->basis[3 * k + 2]};
                        const real w = RV(xtt_weight)(B, S, G);
                        pr += w * vs * ratio * vol[idx + (long)k * N * N * N];
                    }
                    for (int i = 0; i < 4; i++) val[i] = c[i] * pr;
                }
                const long base = Nd * Nd * nn;
                proj[iu + Nd * (iv + 1) + base] += val[0];
                proj[(iu + 1) + Nd * (iv + 1) + base] += val[1];
                proj[(iu + 1) + Nd * iv + base] += val[2];
                proj[iu + Nd * iv + base] += val[3];
                factor[iu + Nd * (iv + 1)] += c[0];
                factor[(iu + 1) + Nd * (iv + 1)] += c[1];
                factor[(iu + 1) + Nd * iv] += c[2];
                factor[iu + Nd * iv] += c[3];
            }
}

/* forwardOrth, ir.cu:294-364: the XTT forward of one view with every voxel's
 * basis rotated by its coefficient planes (S <- R S), no weight image. */
void RV(forward_orth_view)(const or_scan *s, int cond, int n, const real *vol, const real *coef, real *proj) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd, N3 = N * N * N;
    const long nn = n < 0 ? -n : n;
    const real vs = RV(vox_size)(s);
    const real ratio = (vs * vs) / ((real)s->det * ((real)s->sod / (real)s->sdd) * (real)s->det *
                                    ((real)s->sod / (real)s->sdd));
    real G[3];
    { const real bz[3] = {(real)0, (real)0, (real)1}; RV(mat3vec)(f.R, bz, G); }
    for (long y = 0; y < N; y++)
        for (long z = 0; z < N; z++)
            for (long x = 0; x < N; x++) {
                real u, v, B[3], c[4], R[9];
                long iu, iv;
                RV(raycast)(s, &f, 0, (int)x, (int)y, (int)z, &u, &v, B, 0);
                if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
                const long idx = x + N * y + N * N * z;
                RV(orth_rotation)(coef, N3, idx, R);
                real pr = (real)0;
                for (int k = 0; k < s->K; k++) {
                    const real S0[3] = {(real)s->basis[3 * k], (real)s->basis[3 * k + 1], (real)s->basis[3 * k + 2]};
                    real S[3];
                    RV(mat3vec)(R, S0, S);
                    const real w = RV(xtt_weight)(B, S, G);
                    pr += w * vs * ratio * vol[idx + (long)k * N3];
                }
                const long base = Nd * Nd * nn;
                proj[iu + Nd * (iv + 1) + base] += c[0] * pr;
                proj[(iu + 1) + Nd * (iv + 1) + base] += c[1] * pr;
                proj[(iu + 1) + Nd * iv + base] += c[2] * pr;
                proj[iu + Nd * iv + base] += c[3] * pr;
            }
}

/* correlationProjByLength, ir.cu:1533-1603: the chord length L of the ray
 * through the (shifted) volume box, and proj *= L / (factor + 1e-5).  Only the
 * first two face hits are stored (the reference's coord[6] overflows past two,
 * ir.cu:1576-1595).  The reference indexes the view with the signed n
 * (ir.cu:1601); this restatement uses |n| (identical for clockwise scans). */
void RV(correlation)(const or_scan *s, int cond, int n, real *proj, const real *factor) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd;
    const long nn = n < 0 ? -n : n;
    const real vs = RV(vox_size)(s);
    const real src[3] = {(real)0, (real)s->sod, (real)0};
    real o2s[3];
    RV(mat3vec)(f.R, src, o2s);
    real plane[6];
    for (int a = 0; a < 3; a++) {
        plane[2 * a] = -((real)(N + 1) / (real)2.0) * vs - f.off[a] - f.t[a];
        plane[2 * a + 1] = ((real)(N + 1) / (real)2.0) * vs - f.off[a] - f.t[a];
    }
    for (long v = 0; v < Nd; v++)
        for (long u = 0; u < Nd; u++) {
            const real pix[3] = {((real)u - ((real)Nd - (real)1.0) * (real)0.5) * (real)s->det,
                                 -((real)s->sdd - (real)s->sod),
                                 ((real)v - ((real)Nd - (real)1.0) * (real)0.5) * (real)s->det};
            real o2p[3], s2p[3];
            RV(mat3vec)(f.R, pix, o2p);
            for (int i = 0; i < 3; i++) s2p[i] = o2s[i] - o2p[i];
            int cnt = 0;
            real coord[6] = {0, 0, 0, 0, 0, 0};
            for (int p = 0; p < 3; p++)
                for (int sg = 0; sg < 2; sg++) {
                    const real tt = (plane[2 * p + sg] - o2s[p]) / s2p[p];
                    real pl[3];
                    for (int i = 0; i < 3; i++) pl[i] = tt * s2p[i] + o2s[i];
                    const int p1 = (p + 1) % 3, p2 = (p + 2) % 3;
                    if (plane[2 * p1] < pl[p1] && pl[p1] < plane[2 * p1 + 1] && plane[2 * p2] < pl[p2] &&
                        pl[p2] < plane[2 * p2 + 1]) {
                        if (cnt < 2)
                            for (int i = 0; i < 3; i++) coord[i + 3 * cnt] = pl[i];
                        cnt++;
                    }
                }
            const real L = RSQRT((coord[0] - coord[3]) * (coord[0] - coord[3]) +
                                 (coord[1] - coord[4]) * (coord[1] - coord[4]) +
                                 (coord[2] - coord[5]) * (coord[2] - coord[5]));
            const long idx = u + Nd * v + Nd * Nd * nn;
            proj[idx] *= L / (factor[u + Nd * v] + (real)1e-5f);
        }
}

/* projRatio (ir.cu:1616-1635, art == 0) / projSubtract (ir.cu:1656-1666).
 * Adds every |b - p| to *loss in the reference's serial order (one running
 * sum over all views, as the reference's single loss1 accumulator). */
void RV(ratio)(const or_scan *s, int n, real *proj, const real *sino, int art, real *loss) {
    const long Nd = s->Nd;
    const long nn = n < 0 ? -n : n;
    for (long v = 0; v < Nd; v++)
        for (long u = 0; u < Nd; u++) {
            const long idx = u + Nd * v + Nd * Nd * nn;
            *loss += RFABS(sino[idx] - proj[idx]);
            if (art) {
                proj[idx] = sino[idx] - proj[idx];
            } else {
                if (proj[idx] != (real)0) proj[idx] = sino[idx] / proj[idx];
                if (proj[idx] > (real)2.0) proj[idx] = (real)2.0;
            }
        }
}

/* backwardProj/backwardonDevice (ir.cu:1605-1614,1720-1751, xtt == 0) or
 * backwardProjXTT/backwardXTTonDevice (ir.cu:143-152,1807-1850) for one y slab
 * and one view; tmp/factor are the slab accumulators (K planes of N*N). */
void RV(backward_slab)(const or_scan *s, int cond, int y, int n, const real *proj, real *tmp,
                       real *factor, int xtt) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd;
    const long nn = n < 0 ? -n : n;
    real G[3];
    { const real bz[3] = {(real)0, (real)0, (real)1}; RV(mat3vec)(f.R, bz, G); }
    for (long z = 0; z < N; z++)
        for (long x = 0; x < N; x++) {
            real u, v, B[3], c[4];
            long iu, iv;
            RV(raycast)(s, &f, 0, (int)x, y, (int)z, &u, &v, xtt ? B : 0, 0);
            if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
            const long base = Nd * Nd * nn;
            const real p0 = proj[iu + Nd * (iv + 1) + base], p1 = proj[(iu + 1) + Nd * (iv + 1) + base];
            const real p2 = proj[(iu + 1) + Nd * iv + base], p3 = proj[iu + Nd * iv + base];
            const long idx = x + N * z;
            if (!xtt) {
                const real nb = c[0] * p0 + c[1] * p1 + c[2] * p2 + c[3] * p3;
                factor[idx] += (real)1.0;
                tmp[idx] += nb;
            } else {
                for (int k = 0; k < s->K; k++) {
                    real S[3] = {(real)s->basis[3 * k], (real)s->basis[3 * k + 1], (real)s->basis[3 * k + 2]};
                    const real w = RV(xtt_weight)(B, S, G);
                    const real bf = w * c[0] * p0 + w * c[1] * p1 + w * c[2] * p2 + w * c[3] * p3;
                    factor[idx + (long)k * N * N] += w;
                    tmp[idx + (long)k * N * N] += bf;
                }
            }
        }
}

/* backwardOrth, ir.cu:366-423: backward_slab's XTT form with the rotated basis. */
void RV(backward_orth_slab)(const or_scan *s, int cond, int y, int n, const real *proj, const real *coef,
                            real *tmp, real *factor) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd, N3 = N * N * N;
    const long nn = n < 0 ? -n : n;
    real G[3];
    { const real bz[3] = {(real)0, (real)0, (real)1}; RV(mat3vec)(f.R, bz, G); }
    for (long z = 0; z < N; z++)
        for (long x = 0; x < N; x++) {
            real u, v, B[3], c[4], R[9];
            long iu, iv;
            RV(raycast)(s, &f, 0, (int)x, y, (int)z, &u, &v, B, 0);
            if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
            RV(orth_rotation)(coef, N3, x + N * y + N * N * z, R);
            const long base = Nd * Nd * nn;
            const real p0 = proj[iu + Nd * (iv + 1) + base], p1 = proj[(iu + 1) + Nd * (iv + 1) + base];
            const real p2 = proj[(iu + 1) + Nd * iv + base], p3 = proj[iu + Nd * iv + base];
            const long idx = x + N * z;
            for (int k = 0; k < s->K; k++) {
                const real S0[3] = {(real)s->basis[3 * k], (real)s->basis[3 * k + 1], (real)s->basis[3 * k + 2]};
                real S[3];
                RV(mat3vec)(R, S0, S);
                const real w = RV(xtt_weight)(B, S, G);
                const real bf = w * c[0] * p0 + w * c[1] * p1 + w * c[2] * p2 + w * c[3] * p3;
                factor[idx + (long)k * N * N] += w;
                tmp[idx + (long)k * N * N] += bf;
            }
        }
}

/* Vector3X::normalize (vec.h:94-106): divide by the norm above 1e-8, else zero. */
static void RV(normalize3)(real *v) {
    const real l = RSQRT(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > (real)1e-8f) {
        v[0] /= l; v[1] /= l; v[2] /= l;
    } else {
        v[0] = v[1] = v[2] = (real)0;
    }
}

/* calcNormalVectorThreeDirec, ir.cu:856-974: from the three orthogonal
 * coefficients mu (planes 0..2) and the sign pattern rot, the plane normal
 * (mu0 S0 - mu1' S1) x (mu0 S0 - mu2' S2), rotated by the voxel's current R,
 * z >= 0, gives the new (phi, cos theta); loss = |(R e_z) x norm|. */
static void RV(normal_three_voxel)(const or_scan *s, const real *vol, real *coef, real *loss, long N3, long i,
                                   int rot);

void RV(normal_three)(const or_scan *s, const real *vol, real *coef, real *loss, int rot) {
    const long N3 = (long)s->N * s->N * s->N;
    for (long i = 0; i < N3; i++) RV(normal_three_voxel)(s, vol, coef, loss, N3, i, rot);
}

/* calcNormalVectorThreeDirecWithEst, ir.cu:976-1071: the sign pattern of each
 * voxel from its estimate plane 1 (< 0.5, < 1.5, < 2.5, else). */
void RV(normal_three_est)(const or_scan *s, const real *vol, real *coef, real *loss, const real *est) {
    const long N3 = (long)s->N * s->N * s->N;
    for (long i = 0; i < N3; i++) {
        const real r = est[N3 + i];
        RV(normal_three_voxel)(s, vol, coef, loss, N3, i, r < (real)0.5f ? 0 : (r < (real)1.50f ? 1 : (r < (real)2.50f ? 2 : 3)));
    }
}

static void RV(normal_three_voxel)(const or_scan *s, const real *vol, real *coef, real *loss, long N3, long i,
                                   int rot) {
    {
        real R[9];
        RV(orth_rotation)(coef, N3, i, R);
        const real mu0 = vol[i], m1 = vol[N3 + i], m2 = vol[2 * N3 + i];
        real mu1 = m1, mu2 = m2;
        if (rot == 1) { mu1 = -m1; mu2 = m2; }
        else if (rot == 2) { mu1 = -m1; mu2 = -m2; }
        else if (rot == 3) { mu1 = m1; mu2 = -m2; }
        const float *b = s->basis;
        real v1[3], v2[3], nrm[3];
        for (int j = 0; j < 3; j++) {
            v1[j] = mu0 * (real)b[j] - mu1 * (real)b[3 + j];
            v2[j] = mu0 * (real)b[j] - mu2 * (real)b[6 + j];
        }
        nrm[0] = v1[1] * v2[2] - v1[2] * v2[1];
        nrm[1] = v1[2] * v2[0] - v1[0] * v2[2];
        nrm[2] = v1[0] * v2[1] - v1[1] * v2[0];
        RV(normalize3)(nrm);
        real rn[3];
        RV(mat3vec)(R, nrm, rn);
        /* norm + 0 * base */
        for (int j = 0; j < 3; j++) rn[j] = rn[j] + (real)0 * (j == 2 ? (real)1 : (real)0);
        if (rn[2] < (real)0) { rn[0] = -rn[0]; rn[1] = -rn[1]; rn[2] = -rn[2]; }
        RV(normalize3)(rn);
        real be[3];
        { const real bz[3] = {(real)0, (real)0, (real)1}; RV(mat3vec)(R, bz, be); }
        const real dx = be[1] * rn[2] - be[2] * rn[1], dy = be[2] * rn[0] - be[0] * rn[2],
                   dz = be[0] * rn[1] - be[1] * rn[0];
        /* rotAxis = base x norm */
        const real ax = (real)0 * rn[2] - (real)1 * rn[1], ay = (real)1 * rn[0] - (real)0 * rn[2];
        loss[i] = RSQRT(dx * dx + dy * dy + dz * dz);
        coef[i] = RATAN2(ay, ax);
        coef[N3 + i] = (real)0 * rn[0] + (real)0 * rn[1] + (real)1 * rn[2];
    }
}

/* The per-voxel rotation by main direction (forwardOrthByMD ir.cu:183-189,
 * backwardOrthByMD :262-268, calcMainDirection :693-700): md planes
 * (m0, m1, m2) -> rodrigues(-m1, m0, 0, m2 / |m|, sqrt(m0^2 + m1^2) / |m|). */
static void RV(md_rotation)(const real *md, long N3, long idx, real *R) {
    const real m0 = md[idx], m1 = md[N3 + idx], m2 = md[2 * N3 + idx];
    RV(rodrigues)(-m1, m0, (real)0, m2 / RSQRT(m0 * m0 + m1 * m1 + m2 * m2),
                  RSQRT(m0 * m0 + m1 * m1) / RSQRT(m0 * m0 + m1 * m1 + m2 * m2), R);
}

/* forwardOrthByMD, ir.cu:154-231: one view over every y slab with each
 * voxel's basis rotated by its main direction, accumulating the weight image
 * like forwardProjXTT; unlike the other forwards it applies no vs * ratio
 * factor (ir.cu:180-181 computes the ratio and never uses it). */
void RV(forward_md_view)(const or_scan *s, int cond, int n, const real *vol, const real *md, real *proj,
                         real *factor) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd, N3 = N * N * N;
    const long nn = n < 0 ? -n : n;
    real G[3];
    { const real bz[3] = {(real)0, (real)0, (real)1}; RV(mat3vec)(f.R, bz, G); }
    for (long y = 0; y < N; y++)
        for (long z = 0; z < N; z++)
            for (long x = 0; x < N; x++) {
                real u, v, B[3], c[4], R[9];
                long iu, iv;
                RV(raycast)(s, &f, 0, (int)x, (int)y, (int)z, &u, &v, B, 0);
                if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
                const long idx = x + N * y + N * N * z;
                RV(md_rotation)(md, N3, idx, R);
                real pr = (real)0;
                for (int k = 0; k < s->K; k++) {
                    const real S0[3] = {(real)s->basis[3 * k], (real)s->basis[3 * k + 1], (real)s->basis[3 * k + 2]};
                    real S[3];
                    RV(mat3vec)(R, S0, S);
                    pr += RV(xtt_weight)(B, S, G) * vol[idx + (long)k * N3];
                }
                const long base = Nd * Nd * nn;
                proj[iu + Nd * (iv + 1) + base] += c[0] * pr;
                proj[(iu + 1) + Nd * (iv + 1) + base] += c[1] * pr;
                proj[(iu + 1) + Nd * iv + base] += c[2] * pr;
                proj[iu + Nd * iv + base] += c[3] * pr;
                factor[iu + Nd * (iv + 1)] += c[0];
                factor[(iu + 1) + Nd * (iv + 1)] += c[1];
                factor[(iu + 1) + Nd * iv] += c[2];
                factor[iu + Nd * iv] += c[3];
            }
}

/* backwardOrthByMD, ir.cu:233-292: backward_orth_slab with the rotation by
 * main direction. */
void RV(backward_md_slab)(const or_scan *s, int cond, int y, int n, const real *proj, const real *md, real *tmp,
                          real *factor) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd, N3 = N * N * N;
    const long nn = n < 0 ? -n : n;
    real G[3];
    { const real bz[3] = {(real)0, (real)0, (real)1}; RV(mat3vec)(f.R, bz, G); }
    for (long z = 0; z < N; z++)
        for (long x = 0; x < N; x++) {
            real u, v, B[3], c[4], R[9];
            long iu, iv;
            RV(raycast)(s, &f, 0, (int)x, y, (int)z, &u, &v, B, 0);
            if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
            RV(md_rotation)(md, N3, x + N * y + N * N * z, R);
            const long base = Nd * Nd * nn;
            const real p0 = proj[iu + Nd * (iv + 1) + base], p1 = proj[(iu + 1) + Nd * (iv + 1) + base];
            const real p2 = proj[(iu + 1) + Nd * iv + base], p3 = proj[iu + Nd * iv + base];
            const long idx = x + N * z;
            for (int k = 0; k < s->K; k++) {
                const real S0[3] = {(real)s->basis[3 * k], (real)s->basis[3 * k + 1], (real)s->basis[3 * k + 2]};
                real S[3];
                RV(mat3vec)(R, S0, S);
                const real w = RV(xtt_weight)(B, S, G);
                const real bf = w * c[0] * p0 + w * c[1] * p1 + w * c[2] * p2 + w * c[3] * p3;
                factor[idx + (long)k * N * N] += w;
                tmp[idx + (long)k * N * N] += bf;
            }
        }
}

/* meanFiltFiberMD, ir.cu:1304-1363, on slab y (2 <= y < N-2, as the driver
 * reconstruct.cu:1458-1461 calls it) for 2 <= x, z < N-2: the 27 neighbours
 * signed by their agreement with the centre (dot > 0 added, < 0 subtracted,
 * weight coef), normalised (zero -> e_z), scaled to the centre's length. */
void RV(md_filter_slab)(const or_scan *s, int y, const real *md, real *out, real coef) {
    const long N = s->N, N3 = N * N * N;
    for (long z = 2; z < N - 2; z++)
        for (long x = 2; x < N - 2; x++) {
            const long c = x + N * y + N * N * z;
            const real c0 = md[c], c1 = md[N3 + c], c2 = md[2 * N3 + c];
            real nv[3] = {(real)0, (real)0, (real)0};
            const real len = RSQRT(c0 * c0 + c1 * c1 + c2 * c2);
            for (int i = -1; i < 2; i++)
                for (int j = -1; j < 2; j++)
                    for (int k = -1; k < 2; k++) {
                        const long o = (x - i) + N * (y - j) + N * N * (z - k);
                        const real o0 = md[o], o1 = md[N3 + o], o2 = md[2 * N3 + o];
                        const real d = c0 * o0 + c1 * o1 + c2 * o2;
                        if (d > (real)0) {
                            nv[0] = nv[0] + coef * o0; nv[1] = nv[1] + coef * o1; nv[2] = nv[2] + coef * o2;
                        } else if (d < -(real)0) {
                            nv[0] = nv[0] - coef * o0; nv[1] = nv[1] - coef * o1; nv[2] = nv[2] - coef * o2;
                        }
                    }
            RV(normalize3)(nv);
            if (RSQRT(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]) < (real)1e-8f) {
                nv[0] = (real)0; nv[1] = (real)0; nv[2] = (real)1;
            }
            out[c] = len * nv[0];
            out[N3 + c] = len * nv[1];
            out[2 * N3 + c] = len * nv[2];
        }
}

/* The main direction shared by calcMainDirection (ir.cu:624-710) and
 * calcMDWithEst (:712-789) for voxel i: from mu (planes 0..2) the in-plane
 * magnitudes (fx, fy, fz) after removing the (+-1, +-1, +-1) component,
 * signed by `sgn` (0: none, 1: -fx, 2: -fx -fy, 3: -fy), times half the sum
 * of mu, rotated by the voxel's previous md and turned to z >= 0. */
static void RV(main_direction_voxel)(const real *vol, real *md, long N3, long i, int sgn) {
    const real mu0 = vol[i], mu1 = vol[N3 + i], mu2 = vol[2 * N3 + i];
    real n0 = (real)0, n1 = (real)0, n2 = (real)0;
    if (mu2 + mu1 - mu0 < (real)0) { n0 = -(real)1; n1 = (real)1; n2 = (real)1; }
    else if (mu0 + mu2 - mu1 < (real)0) { n0 = (real)1; n1 = -(real)1; n2 = (real)1; }
    else if (mu1 + mu0 - mu2 < (real)0) { n0 = (real)1; n1 = (real)1; n2 = -(real)1; }
    const real co = (mu0 * n0 + mu1 * n1 + mu2 * n2) / (real)3.f;
    const real v0 = mu0 - co * n0, v1 = mu1 - co * n1, v2 = mu2 - co * n2;
    real fx = RSQRT((real)0.5f * RFABS(v2 + v1 - v0)), fy = RSQRT((real)0.5f * RFABS(v0 + v2 - v1));
    const real fz = RSQRT((real)0.5f * RFABS(v1 + v0 - v2));
    if (sgn == 1) fx = -fx;
    else if (sgn == 2) { fx = -fx; fy = -fy; }
    else if (sgn == 3) fy = -fy;
    const real mean = (mu0 + mu1 + mu2) / (real)2.0f;
    const real m[3] = {mean * fx, mean * fy, mean * fz};
    real R[9], r[3];
    RV(md_rotation)(md, N3, i, R);
    RV(mat3vec)(R, m, r);
    if (r[2] < (real)0) { r[0] = -r[0]; r[1] = -r[1]; r[2] = -r[2]; }
    md[i] = r[0];
    md[N3 + i] = r[1];
    md[2 * N3 + i] = r[2];
}

/* calcMainDirection, ir.cu:624-710, every voxel (sign pattern = iter). */
void RV(main_direction)(const or_scan *s, const real *vol, real *md, int iter) {
    const long N3 = (long)s->N * s->N * s->N;
    for (long i = 0; i < N3; i++) RV(main_direction_voxel)(vol, md, N3, i, iter);
}

/* calcMDWithEst, ir.cu:712-789: the sign pattern of each voxel from its
 * estimate plane 1 (< 0.5, < 1.5, < 2.5, else). */
void RV(md_with_estimate)(const or_scan *s, const real *vol, real *md, const real *est) {
    const long N3 = (long)s->N * s->N * s->N;
    for (long i = 0; i < N3; i++) {
        const real rot = est[N3 + i];
        const int sgn = rot < (real)0.5f ? 0 : (rot < (real)1.50f ? 1 : (rot < (real)2.50f ? 2 : 3));
        RV(main_direction_voxel)(vol, md, N3, i, sgn);
    }
}

/* updateEstimation, ir.cu:791-844: loss = mu2^2 + (1 - lo/hi)^2 of the first
 * two channels; where it beats estimate plane 0, planes 0/1 <- (loss, iter). */
void RV(update_estimation)(const or_scan *s, const real *vol, real *est, int iter) {
    const long N3 = (long)s->N * s->N * s->N;
    for (long i = 0; i < N3; i++) {
        const real mu0 = vol[i], mu1 = vol[N3 + i], mu2 = vol[2 * N3 + i];
        real lo, hi;
        if (mu0 < mu1) { lo = mu0; hi = mu1; } else { lo = mu1; hi = mu0; }
        const real loss = mu2 * mu2 + ((real)1.0f - lo / hi) * ((real)1.0f - lo / hi);
        if (loss < est[i]) {
            est[i] = loss;
            est[N3 + i] = (real)iter;
        }
    }
}

/* meanFiltFiber, ir.cu:1231-1302, on slab y (1 <= y < N-1, as the driver
 * reconstruct.cu:534-537 calls it) for 1 <= x, z < N-1: each neighbour's
 * direction from its (phi, cos theta) planes as mu (sin t cos(phi - pi/2),
 * sin t sin(phi - pi/2), cos t), mu the sum of its three coefficients; pairs
 * (i, 26 - i) within 60 degrees of the centre (|dot| > 0.5) added signed to
 * it, normalised, z >= 0, back to (phi, cos theta).  -pi/2 + phi is
 * evaluated in double (M_PI) and rounded to float. */
void RV(coef_filter_slab)(const or_scan *s, int y, const real *coef, const real *vol, real *out, real w) {
    const long N = s->N, N3 = N * N * N;
    for (long z = 1; z < N - 1; z++)
        for (long x = 1; x < N - 1; x++) {
            real nv[27][3];
            int cnt = 0;
            for (int i = -1; i < 2; i++)
                for (int j = -1; j < 2; j++)
                    for (int k = -1; k < 2; k++) {
                        const long o = (x - i) + N * (y - j) + N * N * (z - k);
                        const real ct = coef[N3 + o];
                        const real st = RSQRT((real)1.f - ct * ct);
                        const real phi = (real)(-M_PI / 2.0f + (double)coef[o]);
                        const real mu = vol[o] + vol[N3 + o] + vol[2 * N3 + o];
                        nv[cnt][0] = mu * (st * RCOS(phi));
                        nv[cnt][1] = mu * (st * RSIN(phi));
                        nv[cnt][2] = mu * ct;
                        cnt++;
                    }
            real c[3] = {nv[13][0], nv[13][1], nv[13][2]};
            for (int i = 0; i < 13; i++) {
                const real *a = nv[i], *b = nv[26 - i];
                const real da = a[0] * nv[13][0] + a[1] * nv[13][1] + a[2] * nv[13][2];
                if (da > (real)0.5f) { c[0] = c[0] + w * a[0]; c[1] = c[1] + w * a[1]; c[2] = c[2] + w * a[2]; }
                else if (da < -(real)0.5f) { c[0] = c[0] - w * a[0]; c[1] = c[1] - w * a[1]; c[2] = c[2] - w * a[2]; }
                const real db = b[0] * nv[13][0] + b[1] * nv[13][1] + b[2] * nv[13][2];
                if (db > (real)0.5f) { c[0] = c[0] + w * b[0]; c[1] = c[1] + w * b[1]; c[2] = c[2] + w * b[2]; }
                else if (db < -(real)0.5f) { c[0] = c[0] - w * b[0]; c[1] = c[1] - w * b[1]; c[2] = c[2] - w * b[2]; }
            }
            RV(normalize3)(c);
            if (c[2] < (real)0) { c[0] = -c[0]; c[1] = -c[1]; c[2] = -c[2]; }
            /* rotAxis = e_z x c, cos = e_z . c */
            const real ax = (real)0 * c[2] - (real)1 * c[1], ay = (real)1 * c[0] - (real)0 * c[2];
            const long ci = x + N * y + N * N * z;
            out[ci] = RATAN2(ay, ax);
            out[N3 + ci] = (real)0 * c[0] + (real)0 * c[1] + (real)1 * c[2];
        }
}

/* updateEstimationByCoef, ir.cu:1073-1120: the plane normal of the three
 * coefficients (no signs), z >= 0; where its cosine to e_z exceeds estimate
 * plane 0, planes 0/1 <- (cosine, iter). */
void RV(update_estimation_coef)(const or_scan *s, const real *vol, real *est, int iter) {
    const long N3 = (long)s->N * s->N * s->N;
    const float *b = s->basis;
    for (long i = 0; i < N3; i++) {
        const real mu0 = vol[i], mu1 = vol[N3 + i], mu2 = vol[2 * N3 + i];
        real v1[3], v2[3], n[3];
        for (int j = 0; j < 3; j++) {
            v1[j] = mu0 * (real)b[j] - mu1 * (real)b[3 + j];
            v2[j] = mu0 * (real)b[j] - mu2 * (real)b[6 + j];
        }
        n[0] = v1[1] * v2[2] - v1[2] * v2[1];
        n[1] = v1[2] * v2[0] - v1[0] * v2[2];
        n[2] = v1[0] * v2[1] - v1[1] * v2[0];
        RV(normalize3)(n);
        if (n[2] < (real)0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
        RV(normalize3)(n);
        const real c = (real)0 * n[0] + (real)0 * n[1] + (real)1 * n[2];
        if (c > est[i]) {
            est[i] = c;
            est[N3 + i] = (real)iter;
        }
    }
}

/* rayCastingFiber, fiber.cu:228-278: rayCasting's source and rotation, but
 * voxel centres at (2i - N + 1)/2 and the detector v axis along -R e_z. */
static void RV(raycast_fiber)(const or_scan *s, const RV(frame) * f, int x, int y, int z, real *u, real *v,
                              real *B) {
    const real vs = RV(vox_size)(s);
    const real N = (real)s->N;
    const int xyz[3] = {x, y, z};
    real org[3], d[3], p[3];
    for (int i = 0; i < 3; i++)
        org[i] = ((real)2.0 * (real)xyz[i] - N + (real)1.0) * (real)0.5 * vs - f->off[i] - f->t[i];
    for (int i = 0; i < 3; i++) d[i] = org[i] + (-f->src[i]);
    const real coeff = -(f->ss) / RV(dot3)(f->src, d);
    for (int i = 0; i < 3; i++) p[i] = f->src[i] + coeff * d[i];
    const real mag = (real)s->sdd / (real)s->sod;
    const real evn[3] = {-f->ev[0], -f->ev[1], -f->ev[2]};
    *u = RV(dot3)(p, f->eu) * mag / (real)s->det + (real)0.5 * (real)s->Nd;
    *v = RV(dot3)(p, evn) * mag / (real)s->det + (real)0.5 * (real)s->Nd;
    const real val = RSQRT(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int i = 0; i < 3; i++) B[i] = (val > (real)1e-8f) ? d[i] / val : (real)0;
}

/* The fiber model's signed projection of voxel idx: ps = (B x G).(f0, f1, f2)
 * + f3 (fiber.cu:52-65, channels beyond the fourth are not read); the weight
 * used is |ps|, its sign s. */
static real RV(fiber_signed)(const or_scan *s, const real *B, const real *G, const real *vol, long idx, long N3,
                             real *bxg) {
    bxg[0] = B[1] * G[2] - B[2] * G[1];
    bxg[1] = B[2] * G[0] - B[0] * G[2];
    bxg[2] = B[0] * G[1] - B[1] * G[0];
    real ps = (real)0;
    const int K = s->K < 4 ? s->K : 4;
    for (int i = 0; i < K; i++) ps += (i >= 3 ? (real)1.0f : bxg[i]) * vol[idx + (long)i * N3];
    return ps;
}

/* forwardProjFiber / forwardFiberModel, fiber.cu:13-78 and 80-153: one view
 * over every y slab, proj[tap] += c * vs * ratio * |ps|; no weight image. */
void RV(fiber_forward_view)(const or_scan *s, int cond, int n, const real *vol, real *proj) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd, N3 = N * N * N;
    const long nn = n < 0 ? -n : n;
    const real vs = RV(vox_size)(s);
    const real ratio = (vs * vs) / ((real)s->det * ((real)s->sod / (real)s->sdd) * (real)s->det *
                                    ((real)s->sod / (real)s->sdd));
    for (long y = 0; y < N; y++)
        for (long z = 0; z < N; z++)
            for (long x = 0; x < N; x++) {
                real u, v, B[3], c[4], bxg[3];
                long iu, iv;
                RV(raycast_fiber)(s, &f, (int)x, (int)y, (int)z, &u, &v, B);
                if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
                const long idx = x + N * y + N * N * z;
                const real ps = RV(fiber_signed)(s, B, f.ev, vol, idx, N3, bxg);
                const real pr = ps * (ps >= (real)0 ? (real)1.0f : -(real)1.0f);
                const long base = Nd * Nd * nn;
                proj[iu + Nd * (iv + 1) + base] += c[0] * vs * ratio * pr;
                proj[(iu + 1) + Nd * (iv + 1) + base] += c[1] * vs * ratio * pr;
                proj[(iu + 1) + Nd * iv + base] += c[2] * vs * ratio * pr;
                proj[iu + Nd * iv + base] += c[3] * vs * ratio * pr;
            }
}

/* backwardProjFiber / backwardFiberModel, fiber.cu:155-226, slab y, view n:
 * channel i gets w_i = |(B x G)_i s| (i < 3) or 1, tmp_i += w_i sum c r,
 * factor_i += w_i (K planes of N*N). */
void RV(fiber_backward_slab)(const or_scan *s, int cond, int y, int n, const real *proj, const real *vol, real *tmp,
                             real *factor) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 0, &f);
    const long N = s->N, Nd = s->Nd, N3 = N * N * N;
    const long nn = n < 0 ? -n : n;
    const int K = s->K < 4 ? s->K : 4;
    for (long z = 0; z < N; z++)
        for (long x = 0; x < N; x++) {
            real u, v, B[3], c[4], bxg[3];
            long iu, iv;
            RV(raycast_fiber)(s, &f, (int)x, y, (int)z, &u, &v, B);
            if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
            const real ps = RV(fiber_signed)(s, B, f.ev, vol, x + N * y + N * N * z, N3, bxg);
            const real sg = ps >= (real)0 ? (real)1.0f : -(real)1.0f;
            const long base = Nd * Nd * nn;
            const real p0 = proj[iu + Nd * (iv + 1) + base], p1 = proj[(iu + 1) + Nd * (iv + 1) + base];
            const real p2 = proj[(iu + 1) + Nd * iv + base], p3 = proj[iu + Nd * iv + base];
            for (int i = 0; i < K; i++) {
                const real w = (i >= 3) ? (real)1.0f : RFABS(bxg[i] * sg);
                const real bf = w * c[0] * p0 + w * c[1] * p1 + w * c[2] * p2 + w * c[3] * p3;
                const long idx = x + N * z + (long)i * N * N;
                factor[idx] += w;
                tmp[idx] += bf;
            }
        }
}

/* voxelProduct (ir.cu:1637-1654, MLEM) or voxelPlus (ir.cu:1682-1693, ART)
 * on slab y of one channel. */
void RV(voxel_update)(const or_scan *s, int y, real *vol, const real *tmp, const real *factor, int art,
                      real alpha) {
    const long N = s->N;
    for (long z = 0; z < N; z++)
        for (long x = 0; x < N; x++) {
            const long iv = x + N * y + N * N * z, ip = x + N * z;
            if (art)
                vol[iv] = vol[iv] + alpha * tmp[ip];
            else
                vol[iv] = (factor[ip] == (real)0) ? (real)0 : vol[iv] * tmp[ip] / factor[ip];
        }
}

/* voxelSqrt, ir.cu:1707-1717, over all K channels. */
void RV(voxel_sqrt)(const or_scan *s, real *vol) {
    const long n = (long)s->N * s->N * s->N * s->K;
    for (long i = 0; i < n; i++) vol[i] = vol[i] < (real)0 ? RSQRT(-vol[i]) : RSQRT(vol[i]);
}

/* The normalised forward operator A of the reconstruction loops: forward +
 * correlation for every axis and view (what the loops compare with b).  The
 * (axis, view) pairs run in parallel (OpenMP): each writes only its own view
 * image with a private weight image, so the result is the serial one bit for
 * bit. */
void RV(forward_all)(const or_scan *s, const real *vol, real *proj, int rotate_ccw, int xtt) {
    const long Nd = s->Nd, V = s->V;
    const long lenD = Nd * Nd * V;
    const int rotation = rotate_ccw ? -1 : 1;
    memset(proj, 0, sizeof(real) * lenD * s->C);
#pragma omp parallel
    {
        real *factor = (real *)malloc(sizeof(real) * Nd * Nd);
#pragma omp for schedule(dynamic, 1)
        for (long i = 0; i < (long)s->C * V; i++) {
            const int cond = (int)(i / V);
            const int n = rotation * (int)(i % V);
            memset(factor, 0, sizeof(real) * Nd * Nd);
            RV(forward_view)(s, cond, n, vol, proj + lenD * cond, factor, xtt);
            RV(correlation)(s, cond, n, proj + lenD * cond, factor);
        }
        free(factor);
    }
}

/* The forward + correlation of one subset's views of every axis, in parallel:
 * within a subset the views (sub + batch*j) % V are distinct (a wrapped index
 * is congruent to sub - V modulo batch, never to sub), so every (axis, view)
 * pair writes its own image; the serial loops' order of float sums inside each
 * image is kept. */
static void RV(forward_subset)(const or_scan *s, const real *vol, real *proj, int n_cond, int sub, int batch,
                               int subsetSize, int rotation, int xtt) {
    const long Nd = s->Nd, V = s->V;
    const long lenD = Nd * Nd * V;
#pragma omp parallel
    {
        real *pf = (real *)malloc(sizeof(real) * Nd * Nd);
#pragma omp for schedule(dynamic, 1)
        for (long i = 0; i < (long)n_cond * subsetSize; i++) {
            const int cond = (int)(i / subsetSize), j = (int)(i % subsetSize);
            const int n = rotation * (int)((sub + batch * j) % V);
            memset(pf, 0, sizeof(real) * Nd * Nd);
            RV(forward_view)(s, cond, n, vol, proj + lenD * cond, pf, xtt);
            RV(correlation)(s, cond, n, proj + lenD * cond, pf);
        }
        free(pf);
    }
}

/* IR::reconstruct, reconstruct.cu:23-156.  orders holds C*epoch rows of the
 * subset order (the reference shuffles one std::mt19937_64 stream, :75,81);
 * losses receives C*epoch raw loss sums. */
void RV(ir_reconstruct)(const or_scan *s, real **sino, real **vol, int epoch, int batch, int rotate_ccw,
                        int art, real lambda, real *losses, const int *orders) {
    const long N = s->N, Nd = s->Nd, V = s->V;
    const long lenD = Nd * Nd * V;
    const int rotation = rotate_ccw ? -1 : 1;
    const int subsetSize = (int)((V + batch - 1) / batch);
    real *proj = (real *)malloc(sizeof(real) * lenD);
    for (int cond = 0; cond < s->C; cond++) {
        /* one axis at a time (the reference's outer loop, :64): a scan of
         * this axis alone, so the subset helper sees one axis block */
        or_scan one = *s;
        one.C = 1;
        one.rot = s->rot + 9 * cond;
        one.trans = s->trans + 3 * cond;
        one.offset = s->offset + 3 * cond;
        for (int ep = 0; ep < epoch; ep++) {
            const int *order = orders + ((long)cond * epoch + ep) * batch;
            real loss = (real)0;
            memset(proj, 0, sizeof(real) * lenD);
            for (int b = 0; b < batch; b++) {
                const int sub = order[b];
                /* forward + correlation in parallel, then the ratios in the
                 * serial order of the single loss accumulator */
                RV(forward_subset)(&one, vol[cond], proj, 1, sub, batch, subsetSize, rotation, 0);
                for (int j = 0; j < subsetSize; j++) {
                    const int n = rotation * (int)((sub + batch * j) % V);
                    RV(ratio)(s, n, proj, sino[cond], art, &loss);
                }
#pragma omp parallel
                {
                    real *tmp = (real *)malloc(sizeof(real) * N * N);
                    real *fac = (real *)malloc(sizeof(real) * N * N);
#pragma omp for schedule(dynamic, 1)
                    for (int y = 0; y < N; y++) {
                        memset(tmp, 0, sizeof(real) * N * N);
                        memset(fac, 0, sizeof(real) * N * N);
                        for (int j = 0; j < subsetSize; j++) {
                            const int n = rotation * (int)((sub + batch * j) % V);
                            RV(backward_slab)(&one, 0, y, n, proj, tmp, fac, 0);
                        }
                        RV(voxel_update)(s, y, vol[cond], tmp, fac, art, lambda / (real)subsetSize);
                    }
                    free(tmp);
                    free(fac);
                }
            }
            if (losses) losses[(long)cond * epoch + ep] = loss;
        }
    }
    free(proj);
}

/* XTT::reconstruct, reconstruct.cu:799-927 (without the orientation step;
 * see orientation below).  vol is ONE buffer of K*N^3 (the device layout,
 * reconstruct.cu:819,828-829); proj (C*lenD) receives the last ratio images
 * (the reference copies them over the sinograms, :924-925).  orders holds
 * epoch rows (a fresh engine shuffles a persistent order each epoch, :858-859). */
void RV(xtt_reconstruct)(const or_scan *s, const real *sino, real *vol, real *proj, int epoch, int batch,
                         int rotate_ccw, int art, real lambda, real *losses, const int *orders) {
    const long N = s->N, Nd = s->Nd, V = s->V, K = s->K;
    const long lenD = Nd * Nd * V, lenV = N * N * N, lenP = N * N;
    const int rotation = rotate_ccw ? -1 : 1;
    const int subsetSize = (int)((V + batch - 1) / batch);
    for (int ep = 0; ep < epoch; ep++) {
        const int *order = orders + (long)ep * batch;
        real loss = (real)0;
        memset(proj, 0, sizeof(real) * lenD * s->C);
        for (int b = 0; b < batch; b++) {
            const int sub = order[b];
            /* forward + correlation of the subset in parallel, then the
             * ratios in the serial order of the single loss accumulator */
            RV(forward_subset)(s, vol, proj, s->C, sub, batch, subsetSize, rotation, 1);
            for (int cond = 0; cond < s->C; cond++)
                for (int j = 0; j < subsetSize; j++) {
                    const int n = rotation * (int)((sub + batch * j) % V);
                    RV(ratio)(s, n, proj + lenD * cond, sino + lenD * cond, art, &loss);
                }
            /* slabs in parallel: each reads the ratio images and updates its
             * own y slab of every channel */
#pragma omp parallel
            {
                real *tmp = (real *)malloc(sizeof(real) * lenP * K);
                real *fac = (real *)malloc(sizeof(real) * lenP * K);
#pragma omp for schedule(dynamic, 1)
                for (int y = 0; y < N; y++) {
                    memset(tmp, 0, sizeof(real) * lenP * K);
                    memset(fac, 0, sizeof(real) * lenP * K);
                    for (int cond = 0; cond < s->C; cond++)
                        for (int j = 0; j < subsetSize; j++) {
                            const int n = rotation * (int)((sub + batch * j) % V);
                            RV(backward_slab)(s, cond, y, n, proj + lenD * cond, tmp, fac, 1);
                        }
                    for (long k = 0; k < K; k++)
                        RV(voxel_update)(s, y, vol + lenV * k, tmp + lenP * k, fac + lenP * k, art,
                                         lambda / (real)subsetSize);
                }
                free(tmp);
                free(fac);
            }
        }
        if (losses) losses[ep] = loss;
    }
    RV(voxel_sqrt)(s, vol);
}

/* ---------------------------------------------------------------- FDK ---- */

/* calcWeight, fdk.cu:13-26. */
void RV(fdk_weight)(const or_scan *s, real *w) {
    const long Nd = s->Nd;
    for (long v = 0; v < Nd; v++)
        for (long u = 0; u < Nd; u++) {
            const real ur = ((real)u + (real)0.5 - (real)Nd / (real)2.0) * (real)s->det;
            const real vr = ((real)v + (real)0.5 - (real)Nd / (real)2.0) * (real)s->det;
            w[u + Nd * v] = (real)s->sdd / RSQRT((real)s->sdd * (real)s->sdd + ur * ur + vr * vr);
        }
}

/* The filter table built on the host, reconstruct.cu:1694-1698 (ramlak=0), or
 * a Ram-Lak (band-limited ramp) table in the same scaling (the sample spacing d
 * and the 1/2 of a full 360-degree scan folded in): h[0] = 1/(8d),
 * h[odd k] = -1/(2 pi^2 k^2 d), h[even k > 0] = 0 (ramlak=1; the reference has
 * no Ram-Lak). */
void RV(fdk_filter)(const or_scan *s, int ramlak, real *filt) {
    const real d = (real)s->det * ((real)s->sod / (real)s->sdd);
    for (long k = 0; k < s->Nd; k++) {
        if (!ramlak) {
#if OR_IS_FLOAT
            filt[k] = 1.0f / (float)(M_PI * M_PI * d * (1.0f - 4.0f * (float)(k * k)));
#else
            filt[k] = 1.0 / (M_PI * M_PI * d * (1.0 - 4.0 * (double)(k * k)));
#endif
        } else {
            if (k == 0) filt[k] = (real)1 / ((real)8 * d);
            else if (k % 2) filt[k] = -(real)1 / ((real)2 * (real)(M_PI * M_PI) * (real)(k * k) * d);
            else filt[k] = (real)0;
        }
    }
}

/* projConv, fdk.cu:28-43, for view |n|: dst += sum_j filt[|u-j|] src[j] w[j]
 * along each detector row (dst starts at zero: the reference never clears it,
 * reconstruct.cu:1669, which is taken as zero). */
void RV(fdk_conv)(const or_scan *s, int n, const real *src, const real *filt, const real *w, real *dst) {
    const long Nd = s->Nd;
    const long nn = n < 0 ? -n : n;
    for (long v = 0; v < Nd; v++)
        for (long u = 0; u < Nd; u++) {
            const long idx = u + Nd * v + Nd * Nd * nn;
            real acc = dst[idx];
            for (long j = 0; j < Nd; j++) {
                const real fk = (u > j) ? filt[u - j] : filt[j - u];
                acc += fk * src[Nd * v + j + Nd * Nd * nn] * w[Nd * v + j];
            }
            dst[idx] = acc;
        }
}

/* filteredBackProj/backwardonDevice (FDK), fdk.cu:51-170: for one signed view
 * n, vol[x,y,z] += (sod/(sod+o_y))^2 * (2 pi / V) * bilinear(proj). */
void RV(fdk_backproject_view)(const or_scan *s, int cond, int n, const real *proj, real *vol) {
    RV(frame) f;
    RV(view_frame)(s, cond, n, 1, &f);
    const long N = s->N, Nd = s->Nd;
    const long nn = n < 0 ? -n : n;
    const real Cw = (real)2.0 * (real)M_PI / (real)s->V;
    for (long y = 0; y < N; y++)
        for (long z = 0; z < N; z++)
            for (long x = 0; x < N; x++) {
                real u, v, c[4], o[3];
                long iu, iv;
                RV(raycast)(s, &f, 1, (int)x, (int)y, (int)z, &u, &v, 0, o);
                if (!RV(taps)(s, u, v, &iu, &iv, c)) continue;
                const real U = (real)s->sod / ((real)s->sod + o[1]);
                const long base = Nd * Nd * nn;
                const real nb = c[0] * proj[iu + Nd * (iv + 1) + base] + c[1] * proj[(iu + 1) + Nd * (iv + 1) + base] +
                                c[2] * proj[(iu + 1) + Nd * iv + base] + c[3] * proj[iu + Nd * iv + base];
                vol[x + N * y + N * N * z] += U * U * Cw * nb;
            }
}

/* FDK::reconstruct, reconstruct.cu:1651-1724.  sino: C blocks; vol: C
 * channels of N^3 (the reference writes channel `cond`, fdk.cu:163); filt_out
 * (C blocks, may be NULL) receives the filtered projections (the reference
 * copies them over the sinograms, :1713-1714).  block0 != 0 reproduces the
 * reference's back-projection of axis 0's filtered block for every axis
 * (:1708 passes devSinoFilt without the axis offset). */
void RV(fdk_reconstruct)(const or_scan *s, const real *sino, real *vol, real *filt_out, int rotate_ccw,
                         int ramlak, int block0) {
    const long N = s->N, Nd = s->Nd, V = s->V;
    const long lenD = Nd * Nd * V, lenV = N * N * N;
    const int rotation = rotate_ccw ? -1 : 1;
    real *w = (real *)malloc(sizeof(real) * Nd * Nd);
    real *filt = (real *)malloc(sizeof(real) * Nd);
    real *sf = (real *)calloc((size_t)(lenD * s->C), sizeof(real));
    RV(fdk_weight)(s, w);
    RV(fdk_filter)(s, ramlak, filt);
    memset(vol, 0, sizeof(real) * lenV * s->C);
    for (int cond = 0; cond < s->C; cond++)
        for (long n = 0; n < V; n++) {
            RV(fdk_conv)(s, (int)n, sino + lenD * cond, filt, w, sf + lenD * cond);
            RV(fdk_backproject_view)(s, cond, rotation * (int)n, sf + (block0 ? 0 : lenD * cond), vol + lenV * cond);
        }
    if (filt_out) memcpy(filt_out, sf, sizeof(real) * lenD * s->C);
    free(w); free(filt); free(sf);
}

/* Data residual in FP64 over all axes, views and pixels:
 * out[0] = ||p - b||_2 / ||b||_2, out[1] = sum |b - p| (the reference's loss). */
void RV(residual)(long n, const real *p, const real *b, double *out) {
    double num = 0, den = 0, l1 = 0;
    for (long i = 0; i < n; i++) {
        const double d = (double)p[i] - (double)b[i];
        num += d * d;
        den += (double)b[i] * (double)b[i];
        l1 += fabs(d);
    }
    out[0] = den > 0 ? sqrt(num / den) : 0.0;
    out[1] = l1;
}

#undef RV
