/* The oracle's scan description — TEST INFRASTRUCTURE ONLY.  The fields are
 * the reference's globals and Geometry (params.cu:14-40, geometry.h:8-25). */
#ifndef XR_ORACLE_H
#define XR_ORACLE_H
typedef struct {
    float sdd, sod, det;   /* Geometry(sdd, sod, detSize, ...)              */
    int N, Nd, V, C, K;    /* voxels/side, detector px/side, views, axes, basis vectors */
    const float *rot;      /* 9*C elemR (row-major)                          */
    const float *trans;    /* 3*C elemT (areaTrans already added, params.cu:74-78) */
    const float *offset;   /* 3*C INIT_OFFSET                                 */
    const float *basis;    /* 3*K basisVector                                 */
} or_scan;
#endif
