/*
 * Internal types of libxr: the context, the per-view geometry table and the
 * kernel launchers shared by the host code (xr_host.cpp) and the device code
 * (xr_kernels.cu, xr_fdk.cu, xr_orient.cu).
 */
#ifndef XR_INTERNAL_H
#define XR_INTERNAL_H

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/xr.h"

namespace xr {

constexpr int kMaxCond = 32;
constexpr int kMaxBasis = 32;
constexpr int kLossSlots = 64;   /* [0, 32): per-axis epoch losses; [40, 43): residual sums */
/* Flag or-ed into the storage argument of the update launchers: 16-bit
 * volumes are written with stochastic rounding. */
constexpr int kStoreStochastic = 0x10;

/* Per-(axis, view) constants of the reference's rayCasting (ir.cu:1860-1879),
 * computed once on the host with the reference's float operations.  The
 * kernels then repeat only the per-voxel part, op for op. */
struct ViewFrame {
    float src[3];  /* Rotate * (0, +-sod, 0)                        */
    float ss;      /* src . src                                     */
    float eu[3];   /* Rotate * (1,0,0): detector u axis (column 0)  */
    float e1x;     /* column 1 of Rotate (x)                        */
    float ev[3];   /* Rotate * (0,0,1): detector v axis == grating  */
    float e1y;     /* column 1 of Rotate (y)                        */
    float off[3];  /* Rotate * INIT_OFFSET[cond]                    */
    float e1z;     /* column 1 of Rotate (z)                        */
    float t[3];    /* elemT[cond]                                   */
    int view;      /* |n|: the view's index in the sinogram         */
};
static_assert(sizeof(ViewFrame) == 80, "ViewFrame layout");

/* Scalars every kernel needs (copied by value into kernel parameters). */
struct GeomConst {
    int N, Nd, V, C, K;
    float vs;      /* voxSize = sod*det/sdd (geometry.h:13)          */
    float mag;     /* sdd / sod                                      */
    float det;     /* detector pitch                                 */
    float half;    /* 0.5f * Nd                                      */
    float lim;     /* (float)Nd - 0.55f: detector window             */
    float ratio;   /* vs^2 / (det*(sod/sdd)*det*(sod/sdd)) (ir.cu:1513) */
    float sod, sdd;
    float rdet;    /* RN(1/det)                                      */
    int exact_rdet;/* 1: a/det as a Markstein-corrected product, checked
                      bit for bit against IEEE division on this device */
};

/* XTT basis constants: S_k, |S_k|^2 and g_kc = |S_k . G_c|^2 where
 * G_c = elemR[c] * e_z is the grating axis of axis c (the same for every view
 * of an axis: Rz(theta) leaves e_z fixed). */
struct BasisConst {
    float S[3 * kMaxBasis];
    float S2[kMaxBasis];
    float g[kMaxCond * kMaxBasis];  /* g[c*K + k] */
    float G[3 * kMaxCond];          /* per axis: grating direction elemR_c e_z */
};

struct Timing {
    bool on = false;
    double ms[XR_T_COUNT] = {};
    long launches[XR_T_COUNT] = {};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[XR_T_COUNT];
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
};

/* A device allocation owned by the context. */
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct Session {
    bool active = false;
    bool xtt = true;
    int epochs = 0, epoch_done = 0, batch = 1, subset_size = 1;
    int rotation = 1;
    bool art = false;
    float lambda = 0.f;
    const void *d_sino = nullptr;     /* storage type */
    void *d_vol = nullptr;            /* storage type */
    int storage = 0;                  /* volume                      */
    int sino_storage = 0;             /* measured sinogram           */
    int update_storage = 0;           /* volume, | kStoreStochastic  */
    const float *coef = nullptr;      /* orientation-parametrised XTT: rotation planes */
    int coef_kind = 0;                /* 0: (phi, cos theta); 1: main direction (3 planes) */
    bool fiber = false;               /* fiber model: fiber projectors, channel 0 updated   */
    cudaEvent_t sino_ready = nullptr; /* set: the first ratio launch waits for it (sinogram upload) */
    cudaEvent_t sino_rest = nullptr;  /* set: the second ratio launch waits for it (rest of the sinogram) */
    int vol_slabs = 0;                /* > 0: the first forward runs by z-slabs, each after its upload event */
    bool rtex = false;                /* XTT column session: ratio images through the layered texture */
    /* Host-call tail: when tail_slabs > 0, the last subset of the next epoch
     * back-projects by z-slabs and each slab is then voxelSqrt'ed, its
     * orientation computed into tail_md / tail_ev (may be null) and its
     * volume and orientation planes downloaded to vol_dst / md_dst / ev_dst
     * on the copy stream while the next slab runs; tail_done records it. */
    int tail_slabs = 0;
    float *const *vol_dst = nullptr;
    float *const *md_dst = nullptr;
    float *const *ev_dst = nullptr;
    float *tail_md = nullptr, *tail_ev = nullptr;
    bool tail_done = false;
    const cudaEvent_t *slab_ev = nullptr;
    float *const *ratio_dst = nullptr; /* set: each view's final ratio image to these host planes */
    std::vector<int> order;            /* persistent subset order (XTT)     */
    std::vector<int> ir_orders;        /* C*epochs rows (IR)                */
    std::map<std::vector<int>, cudaGraphExec_t> graphs;  /* per subset order */
};

}  // namespace xr

struct xr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaStream_t copy_stream = nullptr;  /* host-buffer calls: transfers beside the compute stream */
    cudaEvent_t copy_ev[3] = {nullptr, nullptr, nullptr};
    std::string err;

    float sdd = 0, sod = 0, det = 0;
    int N = 0, Nd = 0, V = 0, C = 0, K = 0;
    std::vector<float> rot, trans, offset, basis;
    std::string proj_path, vol_path, direc_path;
    std::vector<int> load_index;

    int fdk_axis_blocks = 0;
    std::vector<int> fdk_axis_g;       /* per axis: column axis of the FDK frames, -1 general */
    std::vector<float> fdk_magsig;     /* per axis: ev[g] * mag of the FDK frames */
    int views_per_cta = 0;
    int storage = 0;
    int sino_storage = -1;            /* -1: same as storage */
    bool stochastic = true;           /* 16-bit updates: stochastic rounding */
    bool xtt_sqrt = true;             /* XTT session end applies voxelSqrt   */
    bool use_graphs = false;
    int axes_one_launch = 2;          /* XTT forward: column-aligned axes in one launch (XR_OPT_AXES_ONE_LAUNCH) */

    xr::GeomConst gc{};
    xr::BasisConst bc{};
    xr::Timing timing;

    /* device workspace */
    int frames_rotation = 0;           /* rotation the frame table holds (0: none) */
    xr::DevBuf frames;                 /* C*V ViewFrame, n = rotation * view        */
    xr::DevBuf norm;                   /* C*V*Nd*Nd: L / (sum c + 1e-5)            */
    bool norm_valid = false;
    xr::DevBuf proj;                   /* C*V*Nd*Nd: forward / ratio images         */
    xr::DevBuf subsets;                /* batch*subset_size view indices            */
    xr::DevBuf loss;                   /* doubles: loss accumulators                */
    xr::DevBuf fiber_flag;             /* int: a fiber session's ratio images held inf/NaN */
    /* XTT column sessions: the subset's ratio images as a 2D-layered array
     * (layer = axis * subset size + list position), written by the ratio
     * kernel through rsurf and gathered by the back kernel through rtex */
    cudaArray_t rarr = nullptr;
    cudaTextureObject_t rtex = 0;
    cudaSurfaceObject_t rsurf = 0;
    int rlayers = 0, rnd = 0;
    /* FDK: the filtered projections as a 2D-layered array (layer = axis * V + view) */
    cudaArray_t farr = nullptr;
    cudaTextureObject_t ftex = 0;
    cudaSurfaceObject_t fsurf = 0;
    int flayers = 0, fnd = 0;
    bool ratio_texture = true;        /* XR_OPT_RATIO_TEXTURE */
    xr::DevBuf scratch_vol, scratch_sino, scratch_md, stage;
    xr::DevBuf basis_dev;              /* BasisConst                                */
    xr::DevBuf fdk_frames;             /* C*V ViewFrame with the FDK source         */
    int fdk_rotation = 0;
    xr::DevBuf fdk_filt, fdk_weight, fdk_sf;
    bool dev_ready = false;
    double *h_loss = nullptr;          /* pinned, kLossSlots doubles                */
    static constexpr int kSlabs = 8;   /* host-call volume upload and final download in z-slabs */
    cudaEvent_t slab_ev[kSlabs] = {};
    cudaEvent_t tail_ev[kSlabs] = {};  /* final download: a slab's orientation is done */
    int sens_batch = 0, sens_rotation = 0; /* the sensitivity buffer holds these subsets (0: nothing) */
    int static_rdet = -1;              /* xr_dev_forward_proj_only_static: its own
                                          result of the division check (-1: not run) */

    /* column-aligned axes (grating direction = +-grid axis for every view) */
    int col_rotation = 0;              /* rotation the column info was built for   */
    std::vector<int> axis_g;           /* per axis: column axis 0/1/2, -1 general   */
    bool all_aligned = false;
    xr::DevBuf colinfo;                /* int axis_g[C], float magsig[C], int conds[C] */
    xr::DevBuf sens;                   /* XTT: batch x K x N^3 per-subset sensitivity  */

    xr::Session sess;
};

namespace xr {

/* ---- host helpers (xr_host.cpp) ---- */
xr_status fail(xr_ctx *c, xr_status st, const std::string &msg);
xr_status cuda_check(xr_ctx *c, cudaError_t e, const char *what);
xr_status ensure(xr_ctx *c, DevBuf &b, size_t bytes, const char *what);
void timing_begin(xr_ctx *c, int cls, cudaEvent_t *ev);
void timing_end(xr_ctx *c, int cls, cudaEvent_t ev);

/* ---- kernel launchers (xr_kernels.cu) ---- */
/* coef (the forward / back launchers): non-null selects the orientation-
 * parametrised XTT, every voxel's basis rotated: coef_kind 0 by its
 * (phi, cos theta) planes (forwardOrth / backwardOrth, ir.cu:294-423), 1 by
 * its main-direction planes (forwardOrthByMD / backwardOrthByMD, ir.cu:
 * 154-292; that forward carries no vs * ratio factor). */
/* Forward splat of one set of views (all listed views of every listed axis).
 * mode 0: plain, value = ratio * vol[0]; mode 1: XTT K channels; mode 2:
 * weights only (value 1, the reference's devProjFactor).  out: C blocks of
 * V*Nd*Nd, accumulated with float atomics. */
cudaError_t launch_forward(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                           const int *view_list, int n_views, int cond0, int n_cond, const void *vol,
                           float *out, int mode, int views_per_cta, int storage, cudaStream_t s,
                           const float *coef = nullptr, int coef_kind = 0);
/* Chord-length normaliser: norm = L / (norm + 1e-5) in place, every view. */
cudaError_t launch_chord(const GeomConst &g, const ViewFrame *frames, float *norm, int n_cond, cudaStream_t s);
/* Normalise (skipped when norm is null) + ratio (MLEM) or subtract (ART) on
 * listed views of every axis, FP64 loss sum added to *loss.  surf (non-zero):
 * the ratio images also go to layer (axis * n_views + list position) of that
 * 2D-layered surface. */
cudaError_t launch_ratio(const GeomConst &g, const int *view_list, int n_views, int n_cond, float *proj,
                         const float *norm, const void *sino, int art, double *loss, int storage, cudaStream_t s,
                         cudaSurfaceObject_t surf = 0);
/* Normalise only (proj *= norm) on every view: the forward operator A. */
cudaError_t launch_normalize(const GeomConst &g, int n_cond, float *proj, const float *norm, cudaStream_t s);
/* Back-projection of the listed views fused with the MLEM / ART update. */
cudaError_t launch_back_update(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                               const int *view_list, int n_views, int cond0, int n_cond, const float *proj,
                               void *vol, int xtt, int art, float alpha, int storage, cudaStream_t s,
                               const float *coef = nullptr, int coef_kind = 0);
/* FP64 sums: out[0] += sum (p-b)^2, out[1] += sum b^2, out[2] += sum |p-b|. */
cudaError_t launch_residual(long n, const float *p, const void *b, double *out, int storage, cudaStream_t s);
/* mu = sqrt|mu| over n values. */
cudaError_t launch_sqrt_abs(long n, void *mu, int storage, cudaStream_t s);
/* n values from one storage type to another (0 FP32, 1 BF16, 2 FP16). */
cudaError_t launch_convert(long n, const void *src, int src_storage, void *dst, int dst_storage, cudaStream_t s);

/* ---- xr_column.cu: kernels for axes whose grating direction is a grid axis ---- */
cudaError_t check_exact_rdet(float det, float rdet, unsigned *d_flag, unsigned *h_result, cudaStream_t s);
/* zlo, zhi: only the bricks whose first voxel's z lies in [zlo, zhi) (z-slab
 * launches over a volume that arrives slab by slab; slab bounds multiples of 16).
 * G < 0 (modes 1-3): the listed axes may have different column axes, given
 * per axis by d_axis_g; one launch covers them all. */
cudaError_t launch_forward_col(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                               const int *view_list, int n_views, const int *d_conds, int n_cond, int G,
                               const float *d_magsig, const void *vol, float *out, int mode, int views_per_cta,
                               int storage, cudaStream_t s, const float *coef = nullptr, int coef_kind = 0,
                               int zlo = 0, int zhi = 1 << 30, const int *d_axis_g = nullptr);
/* mode 0: plain (one axis, update in place); 1: XTT (fac_in = sensitivity);
 * 2: sensitivity of the listed views into fac_out.  zb0, zb1: only the
 * bricks of 8 z-planes numbered [zb0, zb1) (zb1 = -1: to the last). */
cudaError_t launch_back_col(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                            const int *view_list, int n_views, const int *d_conds, int n_cond, const int *d_axis_g,
                            const float *d_magsig, const float *proj, void *vol, const float *fac_in, float *fac_out,
                            int mode, int art, float alpha, int storage, cudaStream_t s,
                            const float *coef = nullptr, int coef_kind = 0, cudaTextureObject_t rtex = 0,
                            int zb0 = 0, int zb1 = -1);

/* ---- xr_orient.cu ---- */
/* calcNormalVectorThreeDirec (ir.cu:856-974) on every voxel: vol holds the
 * three coefficients (FP32), coef (phi, cos theta) is updated, loss |(R e_z) x n|;
 * with est, the sign pattern of each voxel from est plane 1
 * (calcNormalVectorThreeDirecWithEst, ir.cu:976-1071). */
/* Main-direction kernels of circleEstReconstruct (ir.cu:624-844, 1304-1363),
 * FP32 planes of N^3: meanFiltFiberMD over 2 <= x, y, z < N-2 into out;
 * calcMainDirection (est null, sign pattern iter) or calcMDWithEst (est
 * planes (loss, pattern)); updateEstimation. */
cudaError_t launch_md_filter(int N, const float *md, float *out, float coef, cudaStream_t s);
cudaError_t launch_main_direction(int N, const float *vol, float *md, const float *est, int iter, cudaStream_t s);
cudaError_t launch_update_estimation(int N, const float *vol, float *est, int iter, cudaStream_t s);
cudaError_t launch_fill(long n, float *p, float value, cudaStream_t s);
cudaError_t launch_normal_three(long nvox, const BasisConst *d_basis, const float *vol, float *coef, float *loss,
                                int rot, cudaStream_t s, const float *est = nullptr);
/* meanFiltFiber (ir.cu:1231-1302) over 1 <= x, y, z < N-1 into out;
 * updateEstimationByCoef (ir.cu:1073-1120). */
cudaError_t launch_coef_filter(int N, const float *coef, const float *vol, float *out, float w, cudaStream_t s);
cudaError_t launch_update_estimation_coef(long nvox, const BasisConst *d_basis, const float *vol, float *est, int iter,
                                          cudaStream_t s);
cudaError_t launch_orientation(long nvox, int K, const BasisConst *d_basis, const void *mu, float *md,
                               float *ev, int storage, cudaStream_t s);
/* The same for voxels [i0, i1) of volumes with channel stride nvox. */
cudaError_t launch_orientation_range(long nvox, long i0, long i1, int K, const BasisConst *d_basis, const void *mu,
                                     float *md, float *ev, int storage, cudaStream_t s);
cudaError_t launch_angle_from_md(long nvox, const float *md, float *angle, cudaStream_t s);
cudaError_t launch_direction_normalization(long nvox, float *md, cudaStream_t s);

/* ---- xr_fiber.cu: the fiber model (reconstruct/src/fiber.cu) ---- */
/* forwardProjFiber of the listed views of the axes d_conds[0..n_cond) into out (C blocks of
 * V*Nd*Nd, accumulated): c * vs * ratio * |(B x G).(mu_0, mu_1, mu_2) + mu_3|
 * per tap, rayCastingFiber's frame; vol holds min(K, 4) FP32 planes of N^3. */
cudaError_t launch_fiber_forward(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                                 const int *d_conds, int n_cond, const float *vol, float *out, cudaStream_t s);
/* the same for n_cond axes of column axis G (d_magsig: sign(ev[G]) * mag) */
cudaError_t launch_fiber_forward_col(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                                     const int *d_conds, int n_cond, int G, const float *d_magsig, const float *vol,
                                     float *out, cudaStream_t s);
/* backwardProjFiber of the listed views of n_cond axes fused with the update
 * of channel 0 (voxelProduct, or voxelPlus with step alpha when art).
 * d_axis_g / d_magsig: per axis the column axis (-1: general) and
 * sign(ev[g]) * mag; *d_nonfinite (a device int the caller clears once per
 * session) is set when a ratio image read holds an infinity or a NaN; rtex
 * (non-zero): the ratio images as a 2D-layered array (layer = axis * n_views
 * + list position), gathered by the column axes. */
cudaError_t launch_fiber_back(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                              int n_cond, const int *d_axis_g, const float *d_magsig, const float *proj, float *vol,
                              int art, float alpha, int *d_nonfinite, cudaStream_t s, cudaTextureObject_t rtex = 0);

/* ---- xr_fdk.cu ---- */
/* h_axis_g / h_magsig (host arrays, may be null): per axis the column axis of
 * its FDK frames (-1: general) and ev[g] * mag.  fsurf / ftex (non-zero): a
 * 2D-layered array of C * V layers the filtered projections also go to, and
 * the column back-projection gathers its taps from. */
cudaError_t launch_fdk(const GeomConst &g, const ViewFrame *fdk_frames, int n_cond, const float *sino,
                       float *sino_filt, float *vol, const float *filt, float *weight, int axis_blocks,
                       cudaStream_t s, const int *h_axis_g = nullptr, const float *h_magsig = nullptr,
                       cudaSurfaceObject_t fsurf = 0, cudaTextureObject_t ftex = 0);

}  // namespace xr

#endif
