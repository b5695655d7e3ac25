/*
 * xr.h — C ABI of the B200 (sm_100a) reconstruction library libxr.so.
 *
 * Drop-in boundary for the reference's reconstruction hot path
 * (ixactly/Xray-directional-reconstruction): every entry point below names the
 * reference interface it replaces.  Plain pointers and sizes only; the caller
 * owns every buffer and the library keeps no host pointer after a call.
 *
 * Layouts are the reference's:
 *   volume     N*N*N floats, x fastest: idx = x + N*y + N*N*z   (volume.h:65-71)
 *   sinogram   V views of Nd*Nd, u fastest, then v, then view   (ir.cu:1518)
 * Host-buffer entry points take one pointer per axis / per basis channel, as
 * the reference's Volume<float> arrays (reconstruct.cuh:27-45).  Device-buffer
 * entry points (xr_dev_*) take contiguous device memory: K channels of N^3
 * back to back and C axis blocks of V*Nd*Nd back to back
 * (reconstruct.cu:816-829).
 *
 * Every call returns an xr_status; xr_last_error() gives the message.  A
 * context is not thread-safe: use one context per host thread.  Work runs on
 * the context's stream (xr_set_stream), host-buffer calls synchronize it
 * before returning.
 */
#ifndef XR_H
#define XR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum xr_status {
    XR_OK = 0,
    XR_ERR_ARG = 1,      /* bad argument (null pointer, size, enum)         */
    XR_ERR_OOM = 2,      /* device allocation failed                         */
    XR_ERR_CUDA = 3,     /* CUDA runtime / launch error                      */
    XR_ERR_TIMEOUT = 4,  /* a bounded device wait gave up                    */
    XR_ERR_IO = 5,       /* file could not be read / written                 */
    XR_ERR_CONFIG = 6,   /* settings file malformed or key missing           */
    XR_ERR_NODEV = 7,    /* no CUDA device, or not an sm_100 device          */
    XR_ERR_STATE = 8     /* call out of order (e.g. epoch before begin)      */
} xr_status;

/* enum class Method, reconstruct.cuh:14-19 */
typedef enum xr_method { XR_METHOD_XTT = 0, XR_METHOD_MLEM = 1, XR_METHOD_ART = 2, XR_METHOD_FDK = 3 } xr_method;
/* enum class Rotate, reconstruct.cuh:21-24 (CW: view n at +2*pi*n/V) */
typedef enum xr_rotate { XR_ROTATE_CW = 0, XR_ROTATE_CCW = 1 } xr_rotate;
/* FDK filter tables: the reference's (reconstruct.cu:1692-1698) or Ram-Lak */
typedef enum xr_filter { XR_FILTER_REFERENCE = 0, XR_FILTER_RAMLAK = 1 } xr_filter;

/* Scan description: Geometry (geometry.h:8-25) plus the globals init_params
 * fills (params.cu:14-40).  voxSize is derived, sod*det_size/sdd
 * (geometry.h:13).  Arrays are read at xr_create and copied. */
typedef struct xr_scan {
    float sdd;          /* source-detector distance  (SRC_DETECT_DISTANCE)       */
    float sod;          /* source-object distance    (SRC_OBJ_DISTANCE)          */
    float det_size;     /* detector pixel pitch      (DETECTOR_SIZE)             */
    int num_voxel;      /* N, voxels per side        (NUM_VOXEL)                 */
    int num_detect;     /* Nd, pixels per side       (NUM_DETECT_U == _V)        */
    int num_proj;       /* V, views per axis over 360 degrees (NUM_PROJ)         */
    int num_cond;       /* C, sample rotation axes   (NUM_PROJ_COND)             */
    int num_basis;      /* K, scattering vectors     (NUM_BASIS_VECTOR)          */
    const float *rot;   /* 9*C  elemR, row-major per axis                        */
    const float *trans; /* 3*C  elemT (areaTrans already added, params.cu:74-78) */
    const float *offset;/* 3*C  INIT_OFFSET                                      */
    const float *basis; /* 3*K  basisVector                                      */
} xr_scan;

typedef struct xr_ctx xr_ctx;

/* Per-kernel-class device time, accumulated while XR_OPT_TIMING is on
 * (CUDA events on the context stream).  Classes: */
enum {
    XR_T_FORWARD = 0,   /* forward splat (plain / XTT)                  */
    XR_T_RATIO = 1,     /* normalisation + ratio/subtract + loss        */
    XR_T_BACK = 2,      /* back-projection fused with the voxel update  */
    XR_T_SETUP = 3,     /* normaliser precompute (weights + chord)      */
    XR_T_ORIENT = 4,    /* sqrt + per-voxel eigen                       */
    XR_T_FDK = 5,       /* FDK weight/convolution/back-projection       */
    XR_T_OTHER = 6,     /* residual, memsets, copies                    */
    XR_T_COUNT = 7
};
typedef struct xr_timings {
    double ms[XR_T_COUNT];
    long launches[XR_T_COUNT];
} xr_timings;

/* Options (xr_set_option) */
enum {
    XR_OPT_TIMING = 1,        /* 1: record per-class device times                 */
    XR_OPT_FDK_AXIS_BLOCKS = 2,/* 1: FDK back-projects each axis's own filtered
                                  block; 0 (default): axis 0's block for every
                                  axis, as the reference (reconstruct.cu:1708)   */
    XR_OPT_VIEWS_PER_CTA = 3,  /* forward splat: views per CTA (0 = automatic)    */
    XR_OPT_STORAGE = 4,        /* storage of volumes and measured sinograms in HBM:
                                  0 FP32 (default), 1 BF16, 2 FP16; arithmetic
                                  and accumulation stay FP32 (FP64 for losses and
                                  residual norms).  Device-buffer calls then take
                                  volumes / sinograms of that type; host-buffer
                                  calls keep float arrays and convert on the GPU */
    XR_OPT_GRAPHS = 5,         /* 1: each session epoch runs as a CUDA graph, one
                                  captured per distinct subset order and replayed
                                  (ignored while XR_OPT_TIMING is on)            */
    XR_OPT_SINO_STORAGE = 6,   /* storage of measured sinograms alone: -1 (default)
                                  the XR_OPT_STORAGE type, else 0 / 1 / 2 as there
                                  (e.g. BF16 volumes with FP16 or FP32 data)      */
    XR_OPT_ROUNDING = 7,       /* 16-bit volume updates: 1 (default) stochastic
                                  rounding, 0 round to nearest even.  Nearest
                                  rounding drops every update below half a unit
                                  in the last place, so late OS-EM epochs stall */
    XR_OPT_XTT_SQRT = 8,       /* 1 (default): an XTT session ends with the
                                  reference's voxelSqrt (reconstruct.cu:919-922);
                                  0: it leaves the iterate itself, so a later
                                  session can continue it                         */
    XR_OPT_AXES_ONE_LAUNCH = 9,/* XTT forward splat of the rotation axes whose
                                  grating is a grid axis: 1 all of them in one
                                  launch (each CTA's axis picks its column axis);
                                  0 one launch per column axis; 2 (default) one
                                  launch when a single axis has fewer than 2048
                                  bricks of 16 x 16 x 8 voxels (N < 192), where
                                  the per-axis launches would have to split the
                                  views of a subset over CTAs to fill the GPU   */
    XR_OPT_RATIO_TEXTURE = 10  /* 1 (default): sessions keep the subset's ratio
                                  images in a 2D-layered CUDA array as well (XTT
                                  sessions whose axes are all column-aligned; IR
                                  sessions for each column-aligned axis), and
                                  the back-projection gathers each voxel's 4
                                  taps with one texture instruction; likewise
                                  FDK's filtered projections for its column-form
                                  back-projection; 0: they load the 4 taps from
                                  the linear images                              */
};

/* ---- context ----------------------------------------------------------- */

/* Replaces Geometry(sdd, sod, detSize, voxel, detect, nProj) + the globals of
 * init_params (geometry.h:10-14, params.cu:42-104).  device: CUDA ordinal. */
xr_status xr_create(const xr_scan *scan, int device, xr_ctx **out);

/* init_params(tag), params.cu:42-104: reads `tag` from a settings.json of the
 * reference's schema (utility/settings.json), including the sorting/index
 * axis permutation (:80-95) and areaTrans (:74-78).  The path is an argument
 * (the reference hard-codes it, :43); a preset without "sorting" reads as
 * sorting=false. */
xr_status xr_init_params(const char *json_path, const char *tag, int device, xr_ctx **out);

void xr_destroy(xr_ctx *ctx);
const char *xr_last_error(const xr_ctx *ctx);
/* Scan as stored (pointers valid while ctx lives). */
xr_status xr_get_scan(const xr_ctx *ctx, xr_scan *out);
/* PROJ_PATH, VOLUME_PATH, DIRECTION_PATH and LOAD_INDEX (params.cu:46-95);
 * load_index receives C ints (1-based file indices). */
xr_status xr_get_paths(const xr_ctx *ctx, const char **proj_path, const char **vol_path,
                       const char **direc_path, int *load_index);
/* Use `stream` (a cudaStream_t) for all device work; NULL = the context's own. */
xr_status xr_set_stream(xr_ctx *ctx, void *stream);
xr_status xr_set_option(xr_ctx *ctx, int key, int value);
xr_status xr_get_timings(const xr_ctx *ctx, xr_timings *out);
xr_status xr_reset_timings(xr_ctx *ctx);

/* ---- host-buffer entry points (the reference's call surface) ------------ */

/* forwardProjOnly, reconstruct.cu:1890-1949: the raw voxel-driven splat of
 * channel 0 (forwardProj, ir.cu:1480-1531) for every axis and view, without
 * the chord-length normalisation.  voxel[1], sino[C]. */
xr_status xr_forward_proj_only(xr_ctx *ctx, const float *const *voxel, float *const *sino, xr_rotate dir);

/* The normalised forward operator of the reconstruction loops (forward splat +
 * correlationProjByLength, ir.cu:1480-1603 / :1753-1804): what the loops
 * compare with the measured sinogram.  xtt=0: channel 0, plain weights;
 * xtt=1: K channels, dark-field weights.  voxel[1 or K], sino[C]. */
xr_status xr_forward(xr_ctx *ctx, const float *const *voxel, float *const *sino, xr_rotate dir, int xtt);

/* IR::reconstruct, reconstruct.cu:23-156 (reconstruct.cuh:27-28): OS-EM
 * (XR_METHOD_MLEM) or OS-ART (XR_METHOD_ART, step lambda/subsetSize) of each
 * axis independently into voxel[cond].  sino[C], voxel[C] (in: initial
 * volume, out: result).  losses: NULL or C*epoch raw sums of |b - Ax| per
 * epoch (the reference keeps the last axis's, :131). */
xr_status xr_ir_reconstruct(xr_ctx *ctx, float *const *sino, float *const *voxel, int epoch, int batch,
                            xr_rotate dir, xr_method method, float lambda, float *losses);

/* XTT::reconstruct, reconstruct.cu:799-954 (reconstruct.cuh:42-45): joint
 * OS-EM / OS-ART of the K scattering channels over all axes, then
 * mu_k = sqrt|mu_k| and, when md != NULL, the per-voxel orientation
 * (calcEigenVector, direction/src/pca.cu:12-55) into md[3] (and evalue[3]
 * when evalue != NULL).  sino[C] is overwritten with the last ratio images,
 * as the reference does (:924-925).  losses: NULL or epoch raw sums. */
xr_status xr_xtt_reconstruct(xr_ctx *ctx, float *const *sino, float *const *voxel, float *const *md,
                             float *const *evalue, int epoch, int batch, xr_rotate dir, xr_method method,
                             float lambda, float *losses);

/* FDK::reconstruct, reconstruct.cu:1651-1724: cosine weight (fdk.cu:13-26),
 * row convolution (fdk.cu:28-43) and weighted back-projection
 * (fdk.cu:51-170) of each axis into voxel[cond] (zeroed first).  sino[C] is
 * overwritten with the filtered projections (:1713-1714). */
xr_status xr_fdk_reconstruct(xr_ctx *ctx, float *const *sino, float *const *voxel, xr_rotate dir,
                             xr_filter filter);

/* calcEigenVector over every voxel (pca.cu:12-55, called at
 * reconstruct.cu:935-942), in FP64 on the GPU.  mu[K] in, md[3] out,
 * evalue[3] out (may be NULL). */
xr_status xr_orientation(xr_ctx *ctx, const float *const *mu, float *const *md, float *const *evalue);

/* calcAngleFromMD (pca.cu:67-83): angle[0] = phi, angle[1] = theta. */
xr_status xr_angle_from_md(xr_ctx *ctx, const float *const *md, float *const *angle);
/* directionNormalization (pca.cu:85-106): unit vectors where |md| > 0.65, else 0. */
xr_status xr_direction_normalization(xr_ctx *ctx, float *const *md);

/* Data residual (no reference counterpart; the reference logs only the L1
 * sum, reconstruct.cu:951-953): rel_l2 = ||A x - b||_2 / ||b||_2 and
 * l1 = sum |A x - b| over all axes, views and pixels, in FP64. */
xr_status xr_residual(xr_ctx *ctx, const float *const *voxel, const float *const *sino, xr_rotate dir,
                      int xtt, double *rel_l2, double *l1);

/* ---- device-buffer entry points (no host copies) ------------------------ */
/* Volumes (d_vol, d_mu) hold elements of the storage type (XR_OPT_STORAGE),
 * measured sinograms (d_sino of the residual and of sessions) of the
 * sinogram storage type (XR_OPT_SINO_STORAGE); forward projections,
 * orientations and eigenvalues are FP32. */

xr_status xr_dev_forward(xr_ctx *ctx, const void *d_vol, float *d_sino, xr_rotate dir, int xtt);
xr_status xr_dev_residual(xr_ctx *ctx, const void *d_vol, const void *d_sino, xr_rotate dir, int xtt,
                          double *rel_l2, double *l1);
xr_status xr_dev_orientation(xr_ctx *ctx, const void *d_mu, float *d_md, float *d_evalue);

/* An XTT / IR reconstruction session on device buffers, split so a caller
 * (or a CUDA graph) can drive epochs one at a time:
 *   begin: geometry tables, normaliser and subset lists (iteration-invariant);
 *          `epochs` is the planned epoch count (IR draws every axis's subset
 *          orders from one engine, axis-major, reconstruct.cu:75-81, so the
 *          order of (axis, epoch) depends on it; XTT ignores it);
 *   epoch: one OS-EM/OS-ART epoch over all subsets; *loss = raw |b - Ax| sum
 *          (may be NULL; reading it synchronizes the stream);
 *   end:   XTT only — mu_k = sqrt|mu_k| and, when d_md != NULL, orientation.
 * d_sino: C*V*Nd^2; d_vol: K*N^3 (XTT) or C*N^3 (IR).  Both stay owned by
 * the caller and must outlive the session. */
xr_status xr_dev_session_begin(xr_ctx *ctx, const void *d_sino, void *d_vol, int xtt, int epochs,
                               int batch, xr_rotate dir, xr_method method, float lambda);
xr_status xr_dev_session_epoch(xr_ctx *ctx, double *loss);
xr_status xr_dev_session_end(xr_ctx *ctx, float *d_md, float *d_evalue);
/* The session's current ratio images (C*V*Nd^2 floats, device pointer). */
xr_status xr_dev_session_proj(xr_ctx *ctx, const float **d_proj);

/* ---- orientation-parametrised XTT (ir.cu:294-423, :856-974) ------------- */
/* The XTT operators with every voxel's scattering basis rotated by its own
 * Rodrigues rotation rodriguesRotation(cos phi, sin phi, 0, cos theta,
 * sin theta) (ir.cu:597-623); d_coef holds the phi plane then the cos theta
 * plane (2 * N^3 floats, FP32).  The forward is the reference's forwardOrth
 * (ir.cu:294-364): no chord-length normalisation. */
xr_status xr_dev_forward_orth(xr_ctx *ctx, const void *d_vol, const float *d_coef, float *d_sino, xr_rotate dir);
/* An XTT session (xr_dev_session_epoch / _end as usual) whose forward,
 * ratio and back-projection are forwardOrth -> projRatio -> backwardOrth with
 * voxelProduct / voxelPlus, the loop of orthTwiceReconstruct's inner epochs
 * (reconstruct.cu:1067-1127); the planes stay fixed during the session.  The
 * subset order is the XTT session's (a default std::mt19937_64 each epoch),
 * where the reference seeds its engine from std::random_device. */
xr_status xr_dev_session_begin_orth(xr_ctx *ctx, const void *d_sino, void *d_vol, const float *d_coef, int epochs,
                                    int batch, xr_rotate dir, xr_method method, float lambda);
/* calcNormalVectorThreeDirec (ir.cu:856-974) on every voxel: d_vol holds the
 * three coefficients (FP32, K >= 3, basis vectors 0..2), d_coef is updated in
 * place, d_loss (N^3) receives |(R e_z) x n|; rot in 0..3 picks the signs. */
xr_status xr_orth_normal_update(xr_ctx *ctx, const float *d_vol, float *d_coef, float *d_loss, int rot);

/* calcNormalVectorThreeDirecWithEst (ir.cu:976-1071): as xr_orth_normal_update
 * with each voxel's sign pattern from plane 1 of d_est (2 N^3 floats). */
xr_status xr_orth_normal_update_est(xr_ctx *ctx, const float *d_vol, float *d_coef, float *d_loss,
                                    const float *d_est);
/* meanFiltFiber (ir.cu:1231-1302), `passes` times: each voxel with
 * 1 <= x, y, z < N-1 gets the direction of its neighbours (weight `weight`,
 * from their (phi, cos theta) planes in d_coef scaled by the sum of their
 * three coefficients in d_vol) that lie within 60 degrees of its own, signed
 * and summed; d_tmp (2 N^3 floats) is scratch; the outer one-voxel border
 * keeps its values (the reference copies its uninitialised scratch there,
 * reconstruct.cu:538). */
xr_status xr_orth_filter(xr_ctx *ctx, float *d_coef, float *d_tmp, const float *d_vol, float weight, int passes);
/* updateEstimationByCoef (ir.cu:1073-1120): where the cosine between e_z and
 * the plane normal of the three coefficients exceeds d_est plane 0, planes
 * 0 / 1 <- (that cosine, iter). */
xr_status xr_orth_update_estimation(xr_ctx *ctx, const float *d_vol, float *d_est, int iter);

/* ---- main-direction XTT (circleEstReconstruct, reconstruct.cu:1373-1649) -- */
/* The XTT operators with every voxel's basis rotated by its main direction
 * m (d_md: three planes m_x, m_y, m_z of N^3 floats, FP32): about (-m_y, m_x, 0)
 * by the angle of cosine m_z / |m| (identity where m_x = m_y = 0).  The
 * forward is forwardOrthByMD (ir.cu:154-231) followed by the chord-length
 * normalisation (correlationProjByLength, reconstruct.cu:1505-1506); like the
 * reference it carries no vs * ratio factor. */
xr_status xr_dev_forward_md(xr_ctx *ctx, const void *d_vol, const float *d_md, float *d_sino, xr_rotate dir);
/* An XTT session (xr_dev_session_epoch / _end as usual) of circleEstReconstruct's
 * inner epochs (reconstruct.cu:1486-1543): forwardOrthByMD -> normalisation ->
 * projRatio / projSubtract, backwardOrthByMD -> voxelProduct / voxelPlus; the
 * main direction stays fixed during the session.  Subset order as
 * xr_dev_session_begin_orth. */
xr_status xr_dev_session_begin_md(xr_ctx *ctx, const void *d_sino, void *d_vol, const float *d_md, int epochs,
                                  int batch, xr_rotate dir, xr_method method, float lambda);
/* meanFiltFiberMD (ir.cu:1304-1363), `passes` times: each voxel with
 * 2 <= x, y, z < N-2 becomes the sum of its 27 neighbours signed by their
 * agreement with it (weight `weight`), normalised (zero -> e_z) and scaled
 * to its own length; d_tmp (3 N^3 floats) is scratch.  The outer two-voxel
 * border keeps its values (the reference copies its uninitialised scratch
 * there, reconstruct.cu:1462). */
xr_status xr_md_filter(xr_ctx *ctx, float *d_md, float *d_tmp, float weight, int passes);
/* calcMainDirection (ir.cu:624-710): d_md <- main direction of the three
 * coefficients d_vol (FP32, K >= 3) with sign pattern iter (0..3), turned by
 * the previous d_md. */
xr_status xr_md_main_direction(xr_ctx *ctx, const float *d_vol, float *d_md, int iter);
/* calcMDWithEst (ir.cu:712-789): as xr_md_main_direction with each voxel's
 * sign pattern from plane 1 of d_est (2 N^3 floats: loss, pattern). */
xr_status xr_md_with_estimate(xr_ctx *ctx, const float *d_vol, float *d_md, const float *d_est);
/* updateEstimation (ir.cu:791-844): where mu_2^2 + (1 - lo/hi)^2 of the
 * coefficients is below d_est plane 0, planes 0 / 1 <- (that loss, iter). */
xr_status xr_md_update_estimation(xr_ctx *ctx, const float *d_vol, float *d_est, int iter);
/* ---- fiber model (reconstruct/src/fiber.cu; XTT::fiberModelReconstruct,
 *      reconstruct.cuh:54-55, reconstruct.cu:1242-1371) ------------------ */
/* Every voxel holds a fiber vector F = (mu_0, mu_1, mu_2) and, with K = 4, an
 * isotropic term mu_3; a ray of unit direction B through the grating of
 * direction G sees ps = (B x G) . F + mu_3 (fiber.cu:52-65).  The ray casting
 * is rayCastingFiber's (fiber.cu:228-278): voxel centres at (2i - N + 1)/2
 * and the detector v axis along -G.  These calls need K = 3 or 4 (the
 * reference indexes exactly four planes, fiber.cu:19-24) and FP32 volumes.
 *
 * forwardProjFiber (fiber.cu:13-153) of every axis and view: d_sino
 * (C*V*Nd^2, cleared first) receives c * vs * ratio * |ps| per bilinear tap;
 * no chord-length normalisation, no weight image. */
xr_status xr_dev_forward_fiber(xr_ctx *ctx, const float *d_vol, float *d_sino, xr_rotate dir);
/* A session (xr_dev_session_epoch / _end as usual) of fiberModelReconstruct's
 * epochs (reconstruct.cu:1286-1352): per subset forwardProjFiber ->
 * projRatio / projSubtract over every axis, then backwardProjFiber
 * (fiber.cu:155-226) over every axis and view with voxelProduct / voxelPlus of
 * channel 0 alone (the reference updates the first N^3 of devVoxel,
 * :1341-1345); the subset order is the XTT session's (a default
 * std::mt19937_64 each epoch, :1296-1297).  The session end applies no
 * voxelSqrt and no orientation (d_md and d_evalue are ignored). */
xr_status xr_dev_session_begin_fiber(xr_ctx *ctx, const void *d_sino, float *d_vol, int epochs, int batch,
                                     xr_rotate dir, xr_method method, float lambda);
/* fiberModelReconstruct on host buffers: voxel[K] is set to 0.01 first
 * (:1245-1247) and receives the result; sino[C] is overwritten with the last
 * ratio images (:1355-1356; zeros when epoch = 0).  losses: NULL or epoch raw
 * sums of |b - Ax|. */
xr_status xr_fiber_reconstruct(xr_ctx *ctx, float *const *sino, float *const *voxel, int epoch, int batch,
                               xr_rotate dir, xr_method method, float lambda, float *losses);

/* fillVolume (ir.cu:846-854): n device floats <- value. */
xr_status xr_dev_fill(xr_ctx *ctx, float *d, size_t n, float value);

/* ---- regularisers (solver/, reconstruct/src/quadfilt.cpp) --------------- */
/* totalVariationMinimized(vol, rho, lambda, iter), solver/src/tvmin.cpp:6-98:
 * anisotropic TV denoising by ADMM of a device volume (nx*ny*nz floats, x
 * fastest), in place.  The linear step (I + rho F^T F) x = F^T(rho y - u) + x0
 * is solved by conjugate gradients on the GPU to a relative residual of 1e-6
 * (FP64 inner products) where the reference runs Eigen's BiCGSTAB to machine
 * precision; F, the initial y = u = 1 and the updates are the reference's. */
xr_status xr_tv_minimize(void *stream, float *d_vol, int nx, int ny, int nz, float rho, float lambda, int iter);
/* quadlicFormFilterCPU(voxel[3], coefficient, lambda), quadfilt.cpp:11-134:
 * d_voxel 3 planes (the orthogonal coefficients), d_coef 2 planes (phi, cos
 * theta), both updated in place; each of the 6 tensor elements is TV-filtered
 * with rho 3 and 20 iterations. */
xr_status xr_quad_form_filter(void *stream, float *d_voxel, float *d_coef, int nx, int ny, int nz, float lambda);
/* Host-buffer forms of the two (copy in, run on `device`, copy out). */
xr_status xr_tv_minimize_host(int device, float *vol, int nx, int ny, int nz, float rho, float lambda, int iter);
xr_status xr_quad_form_filter_host(int device, float *const *voxel, float *const *coef, int nx, int ny, int nz,
                                   float lambda);

/* ---- several specimens at once (no reference counterpart) -------------- */
/* A batch runs the OS-EM sessions of several independent specimens (each its
 * own context: geometry, size, storage options) together: one epoch of every
 * specimen is enqueued on the specimens' streams, forked from and joined to
 * the batch's stream, so their kernels overlap on the GPU; with
 * XR_OPT_GRAPHS set on the first context the whole multi-specimen epoch is
 * captured once per distinct combination of subset orders and replayed as
 * one CUDA graph.  The reference reconstructs one specimen per run
 * (reconstruct.cu:799-954); each specimen's result equals its own session's. */
typedef struct xr_batch xr_batch;

/* Contexts on one device; the batch holds (does not own) them. */
xr_status xr_batch_create(xr_ctx *const *ctxs, int n, xr_batch **out);
void xr_batch_destroy(xr_batch *batch);
const char *xr_batch_last_error(const xr_batch *batch);
/* xr_dev_session_begin on every specimen (same epochs / subsets / method). */
xr_status xr_batch_session_begin(xr_batch *batch, const void *const *d_sinos, void *const *d_vols, int xtt, int epochs,
                                 int subsets, xr_rotate dir, xr_method method, float lambda);
/* One epoch of every specimen; losses[i] (may be NULL) = specimen i's epoch loss
 * (XTT: its single loss; IR: its axis 0 loss). */
xr_status xr_batch_epoch(xr_batch *batch, double *losses);
xr_status xr_batch_session_end(xr_batch *batch);
/* Autotuner: for each specimen, times its XTT forward splat over one subset
 * for each candidate views-per-CTA chunk and keeps the fastest
 * (XR_OPT_VIEWS_PER_CTA of that context); chosen[i] receives it (may be NULL). */
xr_status xr_batch_autotune(xr_batch *batch, int *chosen);
/* The same over views-per-CTA chunk x launch shape: when a specimen's axes
 * are all grid-aligned with more than one column axis, each chunk is timed
 * both as one launch per column axis and as one launch for all axes, and the
 * fastest pair is kept (XR_OPT_VIEWS_PER_CTA and XR_OPT_AXES_ONE_LAUNCH 0 / 1
 * of that context); views_per_cta[i], axes_one_launch[i] receive them (either
 * may be NULL). */
xr_status xr_batch_autotune_shapes(xr_batch *batch, int *views_per_cta, int *axes_one_launch);

/* The raw forward splat of xr_forward_proj_only on device buffers, for
 * callers that cannot allocate device memory: code whose device memory is
 * all owned by another allocator (a framework's caching pool) or whose
 * steady-state loop must not allocate.  No counterpart in the reference.
 * Allocates nothing: its only scratch (the per-view geometry table, the
 * view list and a flag word) is a fixed array inside libxr of
 * num_cond * num_proj <= 4096 (axis, view) pairs, held by every GPU that
 * loads the library until exit; larger scans get XR_ERR_ARG.  d_vol: N^3
 * floats (channel 0); d_sino: C*V*Nd^2 floats, cleared then accumulated.
 * Work is enqueued on `stream` (a cudaStream_t, NULL = legacy default)
 * without synchronizing; the caller's current device is restored on
 * return.  Like the other entry points it returns XR_ERR_NODEV on a device
 * that is not sm_100.  All calls share the scratch and it keeps the last
 * call's contents, so calls that overlap on the GPU race; serialise them.
 * The first call on a device resolves the scratch address
 * (cudaGetSymbolAddress), and the first call on a context no other entry
 * point has set up runs the detector-pitch division check (a kernel and a
 * synchronize).  Every call copies the geometry table from host stack
 * memory, so none may be captured into a CUDA graph: a call on a capturing
 * stream returns XR_ERR_ARG and enqueues nothing. */
xr_status xr_dev_forward_proj_only_static(xr_ctx *ctx, const float *d_vol, float *d_sino, xr_rotate dir,
                                          void *stream);

/* Library version string. */
const char *xr_version(void);

#ifdef __cplusplus
}
#endif
#endif /* XR_H */
