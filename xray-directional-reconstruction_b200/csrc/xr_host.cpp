/*
 * Host side of libxr: context, settings reader, per-view geometry tables,
 * the OS-EM / OS-ART / FDK schedulers and the C ABI of include/xr.h.
 *
 * Compiled with g++ -ffp-contract=off and no -march flags: the per-view
 * tables are computed with the same float operations, in the same order and
 * the same rounding as the reference's rayCasting (ir.cu:1860-1879), so the
 * kernels see bit-identical rotation, source and offset vectors.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "xr_internal.h"
#include "xr_json.h"

namespace xr {
inline size_t storage_bytes(int storage) { return storage == 0 ? 4 : 2; }
}

namespace xr {

constexpr int kMaxBasisXTT = 16; /* XTT back-projection keeps 2 accumulators per channel in registers */

xr_status fail(xr_ctx *c, xr_status st, const std::string &msg) {
    if (c) c->err = msg;
    return st;
}

xr_status cuda_check(xr_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return XR_OK;
    const xr_status st = (e == cudaErrorMemoryAllocation) ? XR_ERR_OOM : XR_ERR_CUDA;
    return fail(c, st, std::string(what) + ": " + cudaGetErrorString(e));
}

xr_status ensure(xr_ctx *c, DevBuf &b, size_t bytes, const char *what) {
    if (b.bytes >= bytes && b.p) return XR_OK;
    if (b.p) {
        cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
    }
    if (bytes == 0) return XR_OK;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, XR_ERR_OOM, std::string("cudaMalloc(") + what + ", " + std::to_string(bytes) +
                                       " bytes): " + cudaGetErrorString(e));
    }
    b.bytes = bytes;
    return XR_OK;
}

static void release(DevBuf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

void timing_begin(xr_ctx *c, int cls, cudaEvent_t *ev) {
    *ev = nullptr;
    if (!c->timing.on) return;
    (void)cls;
    std::pair<cudaEvent_t, cudaEvent_t> pr{nullptr, nullptr};
    if (!c->timing.pool.empty()) {
        pr = c->timing.pool.back();
        c->timing.pool.pop_back();
    } else {
        cudaEventCreate(&pr.first);
        cudaEventCreate(&pr.second);
    }
    cudaEventRecord(pr.first, c->stream);
    *ev = pr.first;
    c->timing.pending[cls].push_back(pr);
}

void timing_end(xr_ctx *c, int cls, cudaEvent_t ev) {
    if (!c->timing.on || !ev) return;
    auto &v = c->timing.pending[cls];
    if (!v.empty() && v.back().first == ev) {
        cudaEventRecord(v.back().second, c->stream);
        c->timing.launches[cls]++;
    }
}

static void timing_collect(xr_ctx *c) {
    for (int k = 0; k < XR_T_COUNT; k++) {
        for (auto &pr : c->timing.pending[k]) {
            cudaEventSynchronize(pr.second);
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) c->timing.ms[k] += ms;
            c->timing.pool.push_back(pr);
        }
        c->timing.pending[k].clear();
    }
    cudaGetLastError();
}

/* RAII helper: time one launch of class `cls` on the context stream. */
struct Timed {
    xr_ctx *c;
    int cls;
    cudaEvent_t ev;
    Timed(xr_ctx *c_, int cls_) : c(c_), cls(cls_) { timing_begin(c, cls, &ev); }
    ~Timed() { timing_end(c, cls, ev); }
};

/* ---------------------------------------------------------------- geometry */

/* Matrix3X::operator*(Matrix3X), vec.h:171-181. */
static void mat3mul(const float *a, const float *b, float *w) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            float s = 0.0f;
            for (int k = 0; k < 3; k++) s += a[3 * i + k] * b[3 * k + j];
            w[3 * i + j] = s;
        }
}

/* Matrix3X::operator*(Vector3X), vec.h:193-201. */
static void mat3vec(const float *a, const float *v, float *w) {
    for (int i = 0; i < 3; i++) {
        float s = 0.0f;
        for (int j = 0; j < 3; j++) s += a[3 * i + j] * v[j];
        w[i] = s;
    }
}

/* Per-(axis, signed view n) part of rayCasting (ir.cu:1860-1879); fdk selects
 * the FDK source position (0, -sod, 0) (fdk.cu:125). */
static ViewFrame make_frame(const xr_ctx *c, int cond, int n, bool fdk) {
    ViewFrame f;
    std::memset(&f, 0, sizeof(f));
    const float theta = 2.0f * (float)M_PI * (float)n / (float)c->V;
    const float cs = cosf(theta), sn = sinf(theta);
    const float Rz[9] = {cs, -sn, 0.0f, sn, cs, 0.0f, 0.0f, 0.0f, 1.0f};
    float R[9];
    mat3mul(&c->rot[9 * cond], Rz, R);
    mat3vec(R, &c->offset[3 * cond], f.off);
    const float o2s[3] = {0.0f, fdk ? -c->sod : c->sod, 0.0f};
    const float bu[3] = {1.0f, 0.0f, 0.0f}, bv[3] = {0.0f, 0.0f, 1.0f};
    mat3vec(R, o2s, f.src);
    mat3vec(R, bu, f.eu);
    mat3vec(R, bv, f.ev);
    f.e1x = R[1];
    f.e1y = R[4];
    f.e1z = R[7];
    f.ss = f.src[0] * f.src[0] + f.src[1] * f.src[1] + f.src[2] * f.src[2];
    for (int i = 0; i < 3; i++) f.t[i] = c->trans[3 * cond + i];
    f.view = n < 0 ? -n : n;
    return f;
}

ViewFrame host_view_frame(const xr_ctx *c, int cond, int n, bool fdk) { return make_frame(c, cond, n, fdk); }

static void fill_consts(xr_ctx *c) {
    GeomConst &g = c->gc;
    g.N = c->N;
    g.Nd = c->Nd;
    g.V = c->V;
    g.C = c->C;
    g.K = c->K;
    g.vs = c->sod * c->det / c->sdd;                 /* geometry.h:13 */
    g.mag = c->sdd / c->sod;                         /* ir.cu:1896    */
    g.det = c->det;
    g.half = 0.5f * (float)c->Nd;
    g.lim = (float)c->Nd - 0.55f;                    /* ir.cu:1501    */
    g.ratio = (g.vs * g.vs) / (c->det * (c->sod / c->sdd) * c->det * (c->sod / c->sdd)); /* ir.cu:1513 */
    g.sod = c->sod;
    g.sdd = c->sdd;
    g.rdet = 1.0f / c->det;
    g.exact_rdet = 0;                                /* set by ensure_device after the check */
    BasisConst &b = c->bc;
    std::memset(&b, 0, sizeof(b));
    for (int k = 0; k < c->K; k++) {
        const float s0 = c->basis[3 * k], s1 = c->basis[3 * k + 1], s2 = c->basis[3 * k + 2];
        b.S[3 * k] = s0;
        b.S[3 * k + 1] = s1;
        b.S[3 * k + 2] = s2;
        b.S2[k] = s0 * s0 + s1 * s1 + s2 * s2;
    }
    for (int cond = 0; cond < c->C; cond++) {
        /* G = Rotate * e_z = elemR[cond] * e_z for every view (Rz fixes e_z);
         * |S . G| as ir.cu:1786, squared. */
        const ViewFrame f = make_frame(c, cond, 0, false);
        for (int j = 0; j < 3; j++) b.G[3 * cond + j] = f.ev[j];
        for (int k = 0; k < c->K; k++) {
            const float h = std::fabs(b.S[3 * k] * f.ev[0] + b.S[3 * k + 1] * f.ev[1] + b.S[3 * k + 2] * f.ev[2]);
            b.g[cond * c->K + k] = h * h;
        }
    }
}

/* Select the device, create the stream and upload the basis constants. */
static xr_status ensure_device(xr_ctx *c) {
    if (c->dev_ready) return cuda_check(c, cudaSetDevice(c->device), "cudaSetDevice");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= c->device) {
        cudaGetLastError();
        return fail(c, XR_ERR_NODEV, "no CUDA device available (libxr needs a B200, sm_100a)");
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess)
        return fail(c, XR_ERR_NODEV, "cudaGetDeviceProperties failed");
    if (prop.major != 10)
        return fail(c, XR_ERR_NODEV, std::string("libxr is built for sm_100a; device is ") + prop.name + " sm_" +
                                         std::to_string(prop.major) + std::to_string(prop.minor));
    xr_status st = cuda_check(c, cudaSetDevice(c->device), "cudaSetDevice");
    if (st) return st;
    if (!c->own_stream) {
        st = cuda_check(c, cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        if (st) return st;
    }
    if (!c->stream) c->stream = c->own_stream;
    if ((st = ensure(c, c->basis_dev, sizeof(BasisConst), "basis"))) return st;
    st = cuda_check(c, cudaMemcpy(c->basis_dev.p, &c->bc, sizeof(BasisConst), cudaMemcpyHostToDevice),
                    "upload basis");
    if (st) return st;
    if (!c->h_loss) {
        st = cuda_check(c, cudaMallocHost(&c->h_loss, kLossSlots * sizeof(double)), "cudaMallocHost");
        if (st) return st;
    }
    if ((st = ensure(c, c->loss, kLossSlots * sizeof(double), "loss"))) return st;
    /* a/det as a corrected product only where it equals IEEE division bit for bit */
    unsigned *h_bad = reinterpret_cast<unsigned *>(c->h_loss);
    st = cuda_check(c, check_exact_rdet(c->det, c->gc.rdet, (unsigned *)c->loss.p, h_bad, c->stream),
                    "division check");
    if (st) return st;
    c->gc.exact_rdet = (*h_bad == 0) ? 1 : 0;
    c->dev_ready = true;
    return XR_OK;
}

static const BasisConst *dbasis(xr_ctx *c) { return (const BasisConst *)c->basis_dev.p; }

/* Device layout of the column information (xr_ctx::colinfo). */
struct ColInfo {
    int axis_g[kMaxCond];        /* column axis of each axis, -1: general    */
    float magsig[kMaxCond];      /* sign(ev[g]) * sdd/sod                    */
    int all[kMaxCond];           /* 0, 1, ..., C-1                           */
    int group[3][kMaxCond];      /* axes whose column axis is 0, 1, 2        */
};

/* An axis is column-aligned when, for every view, the detector v axis is
 * exactly +-e_g and the source and u axis have exactly zero g component:
 * then u is the same along every voxel column parallel to g. */
static int aligned_axis(const std::vector<ViewFrame> &h, int cond, int V, float *sign) {
    const ViewFrame &f0 = h[(size_t)cond * V];
    int g = -1;
    for (int i = 0; i < 3; i++)
        if (f0.ev[i] == 1.0f || f0.ev[i] == -1.0f) g = i;
    if (g < 0) return -1;
    *sign = f0.ev[g];
    for (int v = 0; v < V; v++) {
        const ViewFrame &f = h[(size_t)cond * V + v];
        for (int i = 0; i < 3; i++) {
            if (i == g) {
                if (f.ev[i] != *sign) return -1;
            } else if (f.ev[i] != 0.0f) {
                return -1;
            }
        }
        if (f.src[g] != 0.0f || f.eu[g] != 0.0f) return -1;
        /* the column kernels compute o_g = (p_g - off_g) - t_g once per voxel
         * for all views: off_g (= +-INIT_OFFSET_z, exact) and t_g must not vary */
        if (f.off[g] != f0.off[g] || f.t[g] != f0.t[g]) return -1;
    }
    return g;
}

/* storage type of measured sinograms */
static int sino_st(const xr_ctx *c) { return c->sino_storage < 0 ? c->storage : c->sino_storage; }

static const ColInfo *dcol(xr_ctx *c) { return (const ColInfo *)c->colinfo.p; }

/* Forward splat of the listed views of the listed axes: column kernels for
 * column-aligned axes (grouped by column axis), the general kernel else.
 * vol is the channel base (plain: the axis's own volume when one axis). */
static cudaError_t forward_dispatch(xr_ctx *c, const int *vl, int n_views, const std::vector<int> &conds,
                                    const void *vol, float *out, int mode, int storage,
                                    const float *coef = nullptr, int coef_kind = 0, int zlo = 0, int zhi = 1 << 30) {
    const ViewFrame *fr = (const ViewFrame *)c->frames.p;
    const ColInfo *ci = dcol(c);
    std::vector<int> grp[3];
    for (int cond : conds) {
        const int g = c->axis_g[cond];
        if (g < 0) {
            cudaError_t e = launch_forward(c->gc, dbasis(c), fr, vl, n_views, cond, 1, vol, out, mode,
                                           c->views_per_cta, storage, c->stream, coef, coef_kind);
            if (e != cudaSuccess) return e;
        } else {
            grp[g].push_back(cond);
        }
    }
    const long bricks = (long)((c->N + 15) / 16) * ((c->N + 15) / 16) * ((c->N + 7) / 8);
    const bool one = c->axes_one_launch == 1 || (c->axes_one_launch == 2 && bricks < 2048);
    if (one && (int)conds.size() == c->C && c->all_aligned &&
        (!grp[0].empty() + !grp[1].empty() + !grp[2].empty()) > 1 && mode != 0) {
        /* every axis, several column axes: one launch (per-CTA column axis) */
        return launch_forward_col(c->gc, dbasis(c), fr, vl, n_views, ci->all, c->C, -1, ci->magsig, vol, out, mode,
                                  c->views_per_cta, storage, c->stream, coef, coef_kind, zlo, zhi, ci->axis_g);
    }
    for (int g = 0; g < 3; g++) {
        if (grp[g].empty()) continue;
        /* the device group list holds every axis of column axis g in order;
         * a single axis uses its entry of the identity list instead */
        const int *dl = (grp[g].size() == 1) ? &ci->all[grp[g][0]] : ci->group[g];
        if (grp[g].size() != 1) {
            int n_in_group = 0;
            for (int cond = 0; cond < c->C; cond++) n_in_group += (c->axis_g[cond] == g);
            if ((int)grp[g].size() != n_in_group) {   /* a strict subset: one launch per axis */
                for (int cond : grp[g]) {
                    cudaError_t e = launch_forward_col(c->gc, dbasis(c), fr, vl, n_views, &ci->all[cond], 1, g,
                                                       ci->magsig, vol, out, mode, c->views_per_cta, storage,
                                                       c->stream, coef, coef_kind, zlo, zhi);
                    if (e != cudaSuccess) return e;
                }
                continue;
            }
        }
        cudaError_t e = launch_forward_col(c->gc, dbasis(c), fr, vl, n_views, dl, (int)grp[g].size(), g, ci->magsig,
                                           vol, out, mode, c->views_per_cta, storage, c->stream, coef, coef_kind, zlo,
                                           zhi);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

/* forwardProjFiber of the listed views of every axis: the column kernel for
 * each group of column-aligned axes, the general kernel per other axis. */
static cudaError_t fiber_forward_dispatch(xr_ctx *c, const int *vl, int n_views, const float *vol, float *out) {
    const ViewFrame *fr = (const ViewFrame *)c->frames.p;
    const ColInfo *ci = dcol(c);
    int n_in_group[3] = {0, 0, 0};
    for (int cond = 0; cond < c->C; cond++) {
        const int g = c->axis_g[cond];
        if (g >= 0) {
            n_in_group[g]++;
            continue;
        }
        cudaError_t e = launch_fiber_forward(c->gc, fr, vl, n_views, &ci->all[cond], 1, vol, out, c->stream);
        if (e != cudaSuccess) return e;
    }
    for (int g = 0; g < 3; g++) {
        if (n_in_group[g] == 0) continue;
        cudaError_t e = launch_fiber_forward_col(c->gc, fr, vl, n_views, ci->group[g], n_in_group[g], g, ci->magsig,
                                                 vol, out, c->stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static std::vector<int> all_conds(const xr_ctx *c) {
    std::vector<int> v(c->C);
    for (int i = 0; i < c->C; i++) v[i] = i;
    return v;
}

/* Frame table for the rotation direction and the normaliser L/(sum c + 1e-5)
 * for every axis and view (geometry only; computed once per context). */
static xr_status ensure_frames(xr_ctx *c, int rotation) {
    xr_status st;
    const size_t nf = (size_t)c->C * c->V;
    if (c->frames_rotation != rotation) {
        std::vector<ViewFrame> h(nf);
        for (int cond = 0; cond < c->C; cond++)
            for (int v = 0; v < c->V; v++) h[(size_t)cond * c->V + v] = make_frame(c, cond, rotation * v, false);
        ColInfo ci;
        std::memset(&ci, 0, sizeof(ci));
        c->axis_g.assign(c->C, -1);
        c->all_aligned = true;
        int ng[3] = {0, 0, 0};
        for (int cond = 0; cond < c->C; cond++) {
            float sg = 1.0f;
            const int g = aligned_axis(h, cond, c->V, &sg);
            c->axis_g[cond] = g;
            ci.axis_g[cond] = g;
            ci.magsig[cond] = sg * c->gc.mag;
            ci.all[cond] = cond;
            if (g < 0) c->all_aligned = false;
            else ci.group[g][ng[g]++] = cond;
        }
        if ((st = ensure(c, c->colinfo, sizeof(ColInfo), "column info"))) return st;
        st = cuda_check(c, cudaMemcpyAsync(c->colinfo.p, &ci, sizeof(ColInfo), cudaMemcpyHostToDevice, c->stream),
                        "upload column info");
        if (st) return st;
        if ((st = ensure(c, c->frames, nf * sizeof(ViewFrame), "frames"))) return st;
        st = cuda_check(c, cudaMemcpyAsync(c->frames.p, h.data(), nf * sizeof(ViewFrame), cudaMemcpyHostToDevice,
                                           c->stream), "upload frames");
        if (st) return st;
        st = cuda_check(c, cudaStreamSynchronize(c->stream), "upload frames");
        if (st) return st;
        c->frames_rotation = rotation;
        c->norm_valid = false;
        c->col_rotation = rotation;
    }
    if (!c->norm_valid) {
        const size_t npx = nf * (size_t)c->Nd * c->Nd;
        if ((st = ensure(c, c->norm, npx * sizeof(float), "normaliser"))) return st;
        std::vector<int> all(c->V);
        for (int v = 0; v < c->V; v++) all[v] = v;
        DevBuf lst;
        if ((st = ensure(c, lst, all.size() * sizeof(int), "view list"))) return st;
        cudaMemcpyAsync(lst.p, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
        {
            Timed t(c, XR_T_SETUP);
            cudaMemsetAsync(c->norm.p, 0, npx * sizeof(float), c->stream);
            st = cuda_check(c, forward_dispatch(c, (const int *)lst.p, c->V, all_conds(c), nullptr,
                                                (float *)c->norm.p, 2, 0), "weight splat");
        }
        if (!st) {
            Timed t(c, XR_T_SETUP);
            st = cuda_check(c, launch_chord(c->gc, (const ViewFrame *)c->frames.p, (float *)c->norm.p, c->C,
                                            c->stream), "chord length");
        }
        cudaStreamSynchronize(c->stream);
        release(lst);
        if (st) return st;
        c->norm_valid = true;
    }
    return XR_OK;
}

static xr_status check_xtt_k(xr_ctx *c) {
    if (c->K > kMaxBasisXTT)
        return fail(c, XR_ERR_ARG, "XTT paths support at most " + std::to_string(kMaxBasisXTT) +
                                       " scattering vectors (got " + std::to_string(c->K) + ")");
    return XR_OK;
}

/* The fiber model reads the fiber vector (mu_0, mu_1, mu_2) and, with K = 4,
 * the isotropic term mu_3 (fiber.cu:19-24 index exactly four planes), all
 * FP32. */
static xr_status check_fiber(xr_ctx *c) {
    if (c->K < 3 || c->K > 4) return fail(c, XR_ERR_CONFIG, "the fiber model needs K = 3 or 4 channels");
    if (c->storage != 0) return fail(c, XR_ERR_CONFIG, "the fiber model needs FP32 volume storage");
    return XR_OK;
}

static xr_status validate_scan(xr_ctx *c) {
    if (!(c->sdd > 0 && c->sod > 0 && c->det > 0)) return fail(c, XR_ERR_ARG, "sdd, sod and det_size must be > 0");
    if (c->N < 1 || c->N > 4096) return fail(c, XR_ERR_ARG, "num_voxel out of range [1, 4096]");
    if (c->Nd < 2 || c->Nd > 16384) return fail(c, XR_ERR_ARG, "num_detect out of range [2, 16384]");
    if (c->V < 1 || c->V > 65535) return fail(c, XR_ERR_ARG, "num_proj out of range [1, 65535]");
    if (c->C < 1 || c->C > kMaxCond) return fail(c, XR_ERR_ARG, "num_cond out of range [1, 32]");
    if (c->K < 1 || c->K > kMaxBasis) return fail(c, XR_ERR_ARG, "num_basis out of range [1, 32]");
    if ((long)c->C * c->V > 65535) return fail(c, XR_ERR_ARG, "num_cond * num_proj must be <= 65535");
    fill_consts(c);
    return XR_OK;
}

/* ---------------------------------------------------------------- settings */

static const JVal *need(const JVal *o, const char *key, std::string &err) {
    const JVal *v = o ? o->get(key) : nullptr;
    if (!v) err = std::string("settings: missing key \"") + key + "\"";
    return v;
}

static bool floats(const JVal *v, std::vector<float> &out) {
    if (!v || v->kind != JVal::Arr) return false;
    out.clear();
    for (const auto &e : v->a) {
        if (e.kind != JVal::Num) return false;
        out.push_back((float)e.n);
    }
    return true;
}

/* Host-call tail, after the last update of z-planes [z0, z1): voxelSqrt of
 * those planes of every channel, their orientation, and the downloads of
 * the slab's volume and orientation planes on the copy stream (session
 * fields vol_dst / md_dst / ev_dst, FP32 storage). */
static cudaError_t tail_slab(xr_ctx *c, int z0, int z1, int i) {
    Session &s = c->sess;
    cudaStream_t str = c->stream, cs = c->copy_stream;
    const size_t NN = (size_t)c->N * c->N, N3 = NN * c->N, n = (size_t)(z1 - z0) * NN, o = (size_t)z0 * NN;
    float *vol = (float *)s.d_vol;
    cudaError_t e = cudaSuccess;
    if (c->xtt_sqrt)   /* reconstruct.cu:919-922 */
        for (int k = 0; k < c->K && e == cudaSuccess; k++) e = launch_sqrt_abs((long)n, vol + k * N3 + o, 0, str);
    if (e == cudaSuccess) e = cudaEventRecord(c->slab_ev[i], str);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, c->slab_ev[i], 0);
    for (int k = 0; k < c->K && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(s.vol_dst[k] + o, vol + k * N3 + o, n * sizeof(float), cudaMemcpyDeviceToHost, cs);
    if (e != cudaSuccess || !s.tail_md) return e;
    e = launch_orientation_range((long)N3, (long)o, (long)(o + n), c->K, dbasis(c), vol, s.tail_md, s.tail_ev, 0, str);
    if (e == cudaSuccess) e = cudaEventRecord(c->tail_ev[i], str);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, c->tail_ev[i], 0);
    for (int k = 0; k < 3 && e == cudaSuccess; k++) {
        e = cudaMemcpyAsync(s.md_dst[k] + o, s.tail_md + k * N3 + o, n * sizeof(float), cudaMemcpyDeviceToHost, cs);
        if (e == cudaSuccess && s.tail_ev && s.ev_dst)
            e = cudaMemcpyAsync(s.ev_dst[k] + o, s.tail_ev + k * N3 + o, n * sizeof(float), cudaMemcpyDeviceToHost,
                                cs);
    }
    return e;
}

/* Enqueue one epoch's device work on the context stream for the given
 * subset orders (XTT: one row; IR: one row per axis). */
static xr_status issue_epoch(xr_ctx *c, const std::vector<int> &orders) {
    Session &s = c->sess;
    xr_status st;
    cudaStream_t str = c->stream;
    const size_t NdNd = (size_t)c->Nd * c->Nd;
    const size_t blk = (size_t)c->V * NdNd;
    const size_t N3 = (size_t)c->N * c->N * c->N;
    const float alpha = s.lambda / (float)s.subset_size;   /* reconstruct.cu:124 / :906 */
    const ViewFrame *fr = (const ViewFrame *)c->frames.p;
    float *proj = (float *)c->proj.p;
    const float *norm = (const float *)c->norm.p;
    double *dl = (double *)c->loss.p;
    cudaMemsetAsync(dl, 0, kMaxCond * sizeof(double), str);
    if (s.xtt) {
        /* XTT::reconstruct epoch, reconstruct.cu:857-917: the ratio images of
         * every axis are cleared once per epoch. */
        cudaMemsetAsync(proj, 0, (size_t)c->C * blk * sizeof(float), str);
        /* ratio_dst: a view's ratio image is final after the last subset of the
         * epoch that holds it (views recur when V % batch != 0) */
        std::vector<int> last;
        if (s.ratio_dst) {
            last.assign(c->V, -1);
            for (int b = 0; b < s.batch; b++)
                for (int j = 0; j < s.subset_size; j++) last[((long)orders[b] + (long)s.batch * j) % c->V] = b;
        }
        for (int b = 0; b < s.batch; b++) {
            const int *vl = (const int *)c->subsets.p + (size_t)orders[b] * s.subset_size;
            {
                Timed t(c, XR_T_FORWARD);
                cudaError_t e = cudaSuccess;
                if (s.vol_slabs > 0 && !s.fiber) {
                    /* the volume arrives by z-slabs: each slab's bricks start as
                     * soon as its upload event has fired (column axes), the
                     * general kernels after the last slab */
                    const int S = s.vol_slabs, zs = ((c->N + S - 1) / S + 15) / 16 * 16;
                    for (int i = 0; i < S && e == cudaSuccess; i++) {
                        e = cudaStreamWaitEvent(str, s.slab_ev[i], 0);
                        if (e == cudaSuccess && c->all_aligned)
                            e = forward_dispatch(c, vl, s.subset_size, all_conds(c), s.d_vol, proj, 1, s.storage,
                                                 s.coef, s.coef_kind, i * zs, i == S - 1 ? (1 << 30) : (i + 1) * zs);
                    }
                    if (e == cudaSuccess && !c->all_aligned)
                        e = forward_dispatch(c, vl, s.subset_size, all_conds(c), s.d_vol, proj, 1, s.storage, s.coef,
                                             s.coef_kind);
                    s.vol_slabs = 0;
                } else {
                    e = s.fiber ? fiber_forward_dispatch(c, vl, s.subset_size, (const float *)s.d_vol, proj)
                                : forward_dispatch(c, vl, s.subset_size, all_conds(c), s.d_vol, proj, 1, s.storage,
                                                   s.coef, s.coef_kind);
                }
                if ((st = cuda_check(c, e, s.fiber ? "fiber forward" : "XTT forward"))) return st;
            }
            {
                Timed t(c, XR_T_RATIO);
                if (s.sino_ready) {
                    if ((st = cuda_check(c, cudaStreamWaitEvent(str, s.sino_ready, 0), "cudaStreamWaitEvent")))
                        return st;
                    s.sino_ready = s.sino_rest;   /* the next subset's ratio waits for the rest */
                    s.sino_rest = nullptr;
                }
                /* the (phi, cos theta) forward is not chord-normalised (forwardOrth ->
                 * projRatio, reconstruct.cu:1086-1099); the main-direction one is
                 * (forwardOrthByMD -> correlationProjByLength, reconstruct.cu:1501-1509) */
                const float *nrm = ((s.coef && s.coef_kind == 0) || s.fiber) ? nullptr : norm;
                if ((st = cuda_check(c, launch_ratio(c->gc, vl, s.subset_size, c->C, proj, nrm,
                                                     s.d_sino, s.art, dl, s.sino_storage, str,
                                                     s.rtex ? c->rsurf : 0), "ratio")))
                    return st;
            }
            if (s.ratio_dst) {
                cudaStream_t cs = c->copy_stream;
                if ((st = cuda_check(c, cudaEventRecord(c->copy_ev[0], str), "cudaEventRecord"))) return st;
                if ((st = cuda_check(c, cudaStreamWaitEvent(cs, c->copy_ev[0], 0), "cudaStreamWaitEvent"))) return st;
                for (int j = 0; j < s.subset_size; j++) {
                    const int n = (int)(((long)orders[b] + (long)s.batch * j) % c->V);
                    if (last[n] != b) continue;
                    for (int cond = 0; cond < c->C; cond++) {
                        const size_t off = (size_t)n * NdNd;
                        if ((st = cuda_check(c, cudaMemcpyAsync(s.ratio_dst[cond] + off, proj + cond * blk + off,
                                                                NdNd * sizeof(float), cudaMemcpyDeviceToHost, cs),
                                             "ratio images")))
                            return st;
                    }
                }
            }
            {
                Timed t(c, XR_T_BACK);
                cudaError_t e;
                if (s.fiber) {
                    const ColInfo *ci = dcol(c);
                    e = launch_fiber_back(c->gc, fr, vl, s.subset_size, c->C, ci->axis_g, ci->magsig, proj,
                                          (float *)s.d_vol, s.art, alpha, (int *)c->fiber_flag.p, str,
                                          s.rtex ? c->rtex : 0);
                } else if (c->all_aligned) {
                    const ColInfo *ci = dcol(c);
                    const float *sens =
                        s.art ? nullptr : (const float *)c->sens.p + (size_t)orders[b] * c->K * N3;
                    const bool tail = s.tail_slabs > 0 && b == s.batch - 1;
                    const int nb8 = (c->N + 7) / 8, S = tail ? s.tail_slabs : 1, zbs = (nb8 + S - 1) / S;
                    e = cudaSuccess;
                    for (int i = 0; i < S && e == cudaSuccess; i++) {
                        const int zb0 = i * zbs, zb1 = tail ? std::min(nb8, zb0 + zbs) : -1;
                        if (tail && zb0 >= zb1) break;
                        e = launch_back_col(c->gc, dbasis(c), fr, vl, s.subset_size, ci->all, c->C, ci->axis_g,
                                            ci->magsig, proj, s.d_vol, sens, nullptr, 1, s.art, alpha,
                                            s.update_storage, str, s.coef, s.coef_kind, s.rtex ? c->rtex : 0, zb0,
                                            zb1);
                        if (e == cudaSuccess && tail) e = tail_slab(c, zb0 * 8, std::min(c->N, zb1 * 8), i);
                    }
                    if (tail && e == cudaSuccess) s.tail_done = true;
                } else {
                    e = launch_back_update(c->gc, dbasis(c), fr, vl, s.subset_size, 0, c->C, proj, s.d_vol, 1, s.art,
                                           alpha, s.update_storage, str, s.coef, s.coef_kind);
                }
                if ((st = cuda_check(c, e, s.fiber ? "fiber back" : "XTT back"))) return st;
            }
        }
    } else {
        /* IR::reconstruct epoch (reconstruct.cu:80-132) of every axis. */
        for (int cond = 0; cond < c->C; cond++) {
            const int *order = &orders[(size_t)cond * s.batch];
            float *pc = proj + (size_t)cond * blk;
            void *vc = (char *)s.d_vol + (size_t)cond * N3 * storage_bytes(s.storage);
            const void *bc = (const char *)s.d_sino + (size_t)cond * blk * storage_bytes(s.sino_storage);
            cudaMemsetAsync(pc, 0, blk * sizeof(float), str);
            for (int b = 0; b < s.batch; b++) {
                const int *vl = (const int *)c->subsets.p + (size_t)order[b] * s.subset_size;
                {
                    Timed t(c, XR_T_FORWARD);
                    if ((st = cuda_check(c, forward_dispatch(c, vl, s.subset_size, std::vector<int>{cond}, vc, proj, 0,
                                                             s.storage), "forward")))
                        return st;
                }
                {
                    Timed t(c, XR_T_RATIO);
                    const bool tex = s.rtex && c->axis_g[cond] >= 0;
                    if ((st = cuda_check(c, launch_ratio(c->gc, vl, s.subset_size, 1, pc, norm + (size_t)cond * blk,
                                                         bc, s.art, dl + cond, s.sino_storage, str,
                                                         tex ? c->rsurf : 0), "ratio")))
                        return st;
                }
                {
                    Timed t(c, XR_T_BACK);
                    cudaError_t e;
                    if (c->axis_g[cond] >= 0) {
                        const ColInfo *ci = dcol(c);
                        e = launch_back_col(c->gc, dbasis(c), fr, vl, s.subset_size, &ci->all[cond], 1, ci->axis_g,
                                            ci->magsig, proj, vc, nullptr, nullptr, 0, s.art, alpha, s.update_storage,
                                            str, nullptr, 0, s.rtex ? c->rtex : 0);
                    } else {
                        e = launch_back_update(c->gc, dbasis(c), fr, vl, s.subset_size, cond, 1, proj, vc, 0, s.art,
                                               alpha, s.update_storage, str);
                    }
                    if ((st = cuda_check(c, e, "back"))) return st;
                }
            }
        }
    }
    return XR_OK;
}

static xr_status epoch_ready(xr_ctx *c) {
    Session &s = c->sess;
    if (!s.active) return fail(c, XR_ERR_STATE, "no active session (call xr_dev_session_begin)");
    if (!s.xtt && s.epoch_done >= s.epochs) return fail(c, XR_ERR_STATE, "IR session: all planned epochs already run");
    return XR_OK;
}

/* Subset orders of the session's next epoch (advances the XTT order). */
static std::vector<int> next_orders(xr_ctx *c) {
    Session &s = c->sess;
    std::vector<int> orders;
    if (s.xtt) {
        /* a fresh default engine shuffles the persistent order (reconstruct.cu:858-859) */
        std::mt19937_64 eng;
        std::shuffle(s.order.begin(), s.order.end(), eng);
        orders = s.order;
    } else {
        for (int cond = 0; cond < c->C; cond++) {
            const int *o = &s.ir_orders[((size_t)cond * s.epochs + s.epoch_done) * s.batch];
            orders.insert(orders.end(), o, o + s.batch);
        }
    }
    return orders;
}

static xr_status loss_copy(xr_ctx *c, cudaStream_t str) {
    return cuda_check(c, cudaMemcpyAsync(c->h_loss, c->loss.p, kMaxCond * sizeof(double), cudaMemcpyDeviceToHost, str),
                      "loss copy");
}

static void loss_read(const xr_ctx *c, double *loss) {
    if (c->sess.xtt) {
        loss[0] = c->h_loss[0];
    } else {
        for (int cond = 0; cond < c->C; cond++) loss[cond] = c->h_loss[cond];
    }
}

static void drop_graphs(xr_ctx *c) {
    for (auto &kv : c->sess.graphs) cudaGraphExecDestroy(kv.second);
    c->sess.graphs.clear();
}

}  // namespace xr

using namespace xr;

extern "C" {

const char *xr_version(void) { return "libxr 0.1 (sm_100a)"; }

xr_status xr_create(const xr_scan *s, int device, xr_ctx **out) {
    if (!s || !out) return XR_ERR_ARG;
    *out = nullptr;
    if (!s->rot || !s->trans || !s->offset || !s->basis) return XR_ERR_ARG;
    if (s->num_cond < 1 || s->num_cond > kMaxCond || s->num_basis < 1 || s->num_basis > kMaxBasis) return XR_ERR_ARG;
    xr_ctx *c = new xr_ctx();
    c->device = device;
    c->sdd = s->sdd;
    c->sod = s->sod;
    c->det = s->det_size;
    c->N = s->num_voxel;
    c->Nd = s->num_detect;
    c->V = s->num_proj;
    c->C = s->num_cond;
    c->K = s->num_basis;
    c->rot.assign(s->rot, s->rot + 9 * c->C);
    c->trans.assign(s->trans, s->trans + 3 * c->C);
    c->offset.assign(s->offset, s->offset + 3 * c->C);
    c->basis.assign(s->basis, s->basis + 3 * c->K);
    c->load_index.resize(c->C);
    for (int i = 0; i < c->C; i++) c->load_index[i] = i + 1;
    const xr_status st = validate_scan(c);
    if (st) {
        delete c;
        return st;
    }
    *out = c;
    return XR_OK;
}

/* init_params, params.cu:42-104. */
xr_status xr_init_params(const char *json_path, const char *tag, int device, xr_ctx **out) {
    if (!json_path || !tag || !out) return XR_ERR_ARG;
    *out = nullptr;
    std::ifstream f(json_path, std::ios::binary);
    if (!f) return XR_ERR_IO;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    JVal root;
    std::string err;
    JParser p(text.data(), text.data() + text.size());
    if (!p.parse(root, err)) return XR_ERR_CONFIG;
    const JVal *rv = need(&root, "recon_variable", err);
    const JVal *t = need(&root, tag, err);
    if (!rv || !t) return XR_ERR_CONFIG;
    auto num = [&](const JVal *o, const char *k, double &d) -> bool {
        const JVal *v = need(o, k, err);
        if (!v || v->kind != JVal::Num) return false;
        d = v->n;
        return true;
    };
    auto str = [&](const JVal *o, const char *k, std::string &s) -> bool {
        const JVal *v = need(o, k, err);
        if (!v || v->kind != JVal::Str) return false;
        s = v->s;
        return true;
    };
    double vec, cond, sod, sdd, proj, ndu, ndv, det, nvox, rot;
    std::string pp, vp, dp;
    if (!str(t, "proj_path", pp) || !str(t, "vol_path", vp) || !str(t, "direc_path", dp)) return XR_ERR_CONFIG;
    if (!num(rv, "vector", vec) || !num(rv, "condition", cond)) return XR_ERR_CONFIG;
    if (!num(t, "sod", sod) || !num(t, "sdd", sdd) || !num(t, "proj", proj) || !num(t, "num_det_u", ndu) ||
        !num(t, "num_det_v", ndv) || !num(t, "det_size", det) || !num(t, "num_voxel", nvox) || !num(t, "rot", rot))
        return XR_ERR_CONFIG;
    std::vector<float> mRot, vTrans, recon, offset, base;
    if (!floats(need(t, "matrixRot", err), mRot) || !floats(need(t, "vecTrans", err), vTrans) ||
        !floats(need(t, "areaTrans", err), recon) || !floats(need(t, "offset", err), offset) ||
        !floats(need(rv, "base", err), base))
        return XR_ERR_CONFIG;
    const JVal *srt = t->get("sorting");
    const bool sorting = srt && srt->kind == JVal::Bool && srt->b;
    const int K = (int)vec, C = (int)cond, proj_cond = (int)rot;
    if (K < 1 || K > kMaxBasis || C < 1 || C > kMaxCond || (int)base.size() < 3 * K || recon.size() < 3 ||
        (int)vTrans.size() < 3 * proj_cond)
        return XR_ERR_CONFIG;
    for (int i = 0; i < proj_cond; i++)
        for (int j = 0; j < 3; j++) vTrans[3 * i + j] += recon[j];
    std::vector<float> R(9 * C), T(3 * C), O(3 * C);
    std::vector<int> li(C);
    if (sorting) {
        std::vector<float> idx;
        if (!floats(need(t, "index", err), idx) || (int)idx.size() < C) return XR_ERR_CONFIG;
        for (int i = 0; i < C; i++) {
            const int k = (int)idx[i];
            if (k < 0 || 9 * k + 9 > (int)mRot.size() || 3 * k + 3 > (int)vTrans.size() ||
                3 * k + 3 > (int)offset.size())
                return XR_ERR_CONFIG;
            li[i] = k + 1;
            std::copy(&mRot[9 * k], &mRot[9 * k + 9], &R[9 * i]);
            std::copy(&vTrans[3 * k], &vTrans[3 * k + 3], &T[3 * i]);
            std::copy(&offset[3 * k], &offset[3 * k + 3], &O[3 * i]);
        }
    } else {
        if ((int)mRot.size() < 9 * C || (int)vTrans.size() < 3 * C || (int)offset.size() < 3 * C)
            return XR_ERR_CONFIG;
        for (int i = 0; i < C; i++) li[i] = i + 1;
        std::copy(mRot.begin(), mRot.begin() + 9 * C, R.begin());
        std::copy(vTrans.begin(), vTrans.begin() + 3 * C, T.begin());
        std::copy(offset.begin(), offset.begin() + 3 * C, O.begin());
    }
    xr_scan s;
    s.sdd = (float)sdd;
    s.sod = (float)sod;
    s.det_size = (float)det;
    s.num_voxel = (int)nvox;
    s.num_detect = (int)ndu;
    s.num_proj = (int)proj;
    s.num_cond = C;
    s.num_basis = K;
    s.rot = R.data();
    s.trans = T.data();
    s.offset = O.data();
    s.basis = base.data();
    const xr_status st = xr_create(&s, device, out);
    if (st) return st;
    (*out)->proj_path = pp;
    (*out)->vol_path = vp;
    (*out)->direc_path = dp;
    (*out)->load_index = li;
    return XR_OK;
}

static void free_ratio_texture(xr_ctx *c);

void xr_destroy(xr_ctx *c) {
    if (!c) return;
    if (c->dev_ready) {
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        drop_graphs(c);
        timing_collect(c);
        for (auto &pr : c->timing.pool) {
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
    }
    release(c->frames);
    release(c->norm);
    release(c->proj);
    release(c->subsets);
    release(c->loss);
    release(c->fiber_flag);
    if (c->dev_ready) free_ratio_texture(c);
    release(c->scratch_vol);
    release(c->scratch_sino);
    release(c->scratch_md);
    release(c->stage);
    release(c->basis_dev);
    release(c->colinfo);
    release(c->sens);
    release(c->fdk_frames);
    release(c->fdk_filt);
    release(c->fdk_weight);
    release(c->fdk_sf);
    if (c->h_loss) cudaFreeHost(c->h_loss);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    for (cudaEvent_t e : c->copy_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->slab_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->tail_ev)
        if (e) cudaEventDestroy(e);
    delete c;
}

const char *xr_last_error(const xr_ctx *c) { return c ? c->err.c_str() : "null context"; }

xr_status xr_get_scan(const xr_ctx *c, xr_scan *out) {
    if (!c || !out) return XR_ERR_ARG;
    out->sdd = c->sdd;
    out->sod = c->sod;
    out->det_size = c->det;
    out->num_voxel = c->N;
    out->num_detect = c->Nd;
    out->num_proj = c->V;
    out->num_cond = c->C;
    out->num_basis = c->K;
    out->rot = c->rot.data();
    out->trans = c->trans.data();
    out->offset = c->offset.data();
    out->basis = c->basis.data();
    return XR_OK;
}

xr_status xr_get_paths(const xr_ctx *c, const char **pp, const char **vp, const char **dp, int *li) {
    if (!c) return XR_ERR_ARG;
    if (pp) *pp = c->proj_path.c_str();
    if (vp) *vp = c->vol_path.c_str();
    if (dp) *dp = c->direc_path.c_str();
    if (li) std::copy(c->load_index.begin(), c->load_index.end(), li);
    return XR_OK;
}

xr_status xr_set_stream(xr_ctx *c, void *stream) {
    if (!c) return XR_ERR_ARG;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return XR_OK;
}

xr_status xr_set_option(xr_ctx *c, int key, int value) {
    if (!c) return XR_ERR_ARG;
    switch (key) {
        case XR_OPT_TIMING: c->timing.on = value != 0; return XR_OK;
        case XR_OPT_FDK_AXIS_BLOCKS: c->fdk_axis_blocks = value != 0; return XR_OK;
        case XR_OPT_VIEWS_PER_CTA:
            if (value < 0 || value > 64) return fail(c, XR_ERR_ARG, "views per CTA must be in [0, 64]");
            c->views_per_cta = value;
            return XR_OK;
        case XR_OPT_GRAPHS: c->use_graphs = value != 0; return XR_OK;
        case XR_OPT_XTT_SQRT: c->xtt_sqrt = value != 0; return XR_OK;
        case XR_OPT_RATIO_TEXTURE:
            if (c->sess.active) return fail(c, XR_ERR_STATE, "the ratio texture cannot change during a session");
            c->ratio_texture = value != 0;
            return XR_OK;
        case XR_OPT_AXES_ONE_LAUNCH:
            if (value < 0 || value > 2) return fail(c, XR_ERR_ARG, "axes per launch must be 0, 1 or 2");
            c->axes_one_launch = value;
            return XR_OK;
        case XR_OPT_ROUNDING:
            if (value < 0 || value > 1) return fail(c, XR_ERR_ARG, "rounding must be 0 (nearest) or 1 (stochastic)");
            if (c->sess.active) return fail(c, XR_ERR_STATE, "rounding cannot change during a session");
            c->stochastic = value != 0;
            return XR_OK;
        case XR_OPT_SINO_STORAGE:
            if (value < -1 || value > 2) return fail(c, XR_ERR_ARG, "sinogram storage must be -1, 0, 1 or 2");
            if (c->sess.active) return fail(c, XR_ERR_STATE, "storage cannot change during a session");
            c->sino_storage = value;
            return XR_OK;
        case XR_OPT_STORAGE:
            if (value < 0 || value > 2) return fail(c, XR_ERR_ARG, "storage must be 0 (FP32), 1 (BF16) or 2 (FP16)");
            if (c->sess.active) return fail(c, XR_ERR_STATE, "storage cannot change during a session");
            c->storage = value;
            return XR_OK;
        default: return fail(c, XR_ERR_ARG, "unknown option " + std::to_string(key));
    }
}

xr_status xr_get_timings(const xr_ctx *cc, xr_timings *out) {
    xr_ctx *c = const_cast<xr_ctx *>(cc);
    if (!c || !out) return XR_ERR_ARG;
    if (c->dev_ready) timing_collect(c);
    for (int k = 0; k < XR_T_COUNT; k++) {
        out->ms[k] = c->timing.ms[k];
        out->launches[k] = c->timing.launches[k];
    }
    return XR_OK;
}

xr_status xr_reset_timings(xr_ctx *c) {
    if (!c) return XR_ERR_ARG;
    if (c->dev_ready) timing_collect(c);
    for (int k = 0; k < XR_T_COUNT; k++) {
        c->timing.ms[k] = 0;
        c->timing.launches[k] = 0;
    }
    return XR_OK;
}

/* ------------------------------------------------------------- sessions */

static void free_layered(cudaArray_t &arr, cudaTextureObject_t &tex, cudaSurfaceObject_t &surf, int &layers,
                         int &nd) {
    if (tex) cudaDestroyTextureObject(tex);
    if (surf) cudaDestroySurfaceObject(surf);
    if (arr) cudaFreeArray(arr);
    tex = 0;
    surf = 0;
    arr = nullptr;
    layers = nd = 0;
}

static void free_ratio_texture(xr_ctx *c) {
    free_layered(c->rarr, c->rtex, c->rsurf, c->rlayers, c->rnd);
    free_layered(c->farr, c->ftex, c->fsurf, c->flayers, c->fnd);
}

/* A 2D-layered array of Nd x Nd float images (`layers` layers) with its
 * texture (point sampling, clamped, unnormalised coordinates) and surface
 * objects; kept while the shape stays.  Leaves tex = 0 (the kernels then load
 * from the linear images) when the device cannot hold that many layers. */
static xr_status ensure_layered(xr_ctx *c, int want, cudaArray_t &arr, cudaTextureObject_t &tex,
                                cudaSurfaceObject_t &surf, int &layers, int &nd, const char *what) {
    if (arr && layers == want && nd == c->Nd) return XR_OK;
    free_layered(arr, tex, surf, layers, nd);
    int max_layers = 0, max_wh = 0;
    cudaDeviceGetAttribute(&max_layers, cudaDevAttrMaxSurface2DLayeredLayers, c->device);
    cudaDeviceGetAttribute(&max_wh, cudaDevAttrMaxSurface2DLayeredWidth, c->device);
    if (want < 1 || want > max_layers || c->Nd > max_wh) return XR_OK;
    const cudaChannelFormatDesc fd = cudaCreateChannelDesc<float>();
    xr_status st = cuda_check(c, cudaMalloc3DArray(&arr, &fd, make_cudaExtent(c->Nd, c->Nd, want),
                                                   cudaArrayLayered | cudaArraySurfaceLoadStore),
                              what);
    if (st) {
        arr = nullptr;
        return st;
    }
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td{};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    if ((st = cuda_check(c, cudaCreateTextureObject(&tex, &rd, &td, nullptr), what)) ||
        (st = cuda_check(c, cudaCreateSurfaceObject(&surf, &rd), what))) {
        free_layered(arr, tex, surf, layers, nd);
        return st;
    }
    layers = want;
    nd = c->Nd;
    return XR_OK;
}

/* The subset's ratio images for the back-projections (layer = axis * subset
 * size + list position). */
static xr_status ensure_ratio_texture(xr_ctx *c, int layers) {
    return ensure_layered(c, layers, c->rarr, c->rtex, c->rsurf, c->rlayers, c->rnd, "ratio image array");
}


static xr_status session_begin_impl(xr_ctx *c, const void *d_sino, void *d_vol, int xtt, int epochs, int batch,
                                    xr_rotate dir, xr_method method, float lambda, const float *coef,
                                    int coef_kind = 0, bool fiber = false) {
    if (!c || !d_sino || !d_vol) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    if (batch < 1 || batch > c->V) return fail(c, XR_ERR_ARG, "batch must be in [1, num_proj]");
    if (method != XR_METHOD_MLEM && method != XR_METHOD_ART && method != XR_METHOD_XTT)
        return fail(c, XR_ERR_ARG, "method must be MLEM or ART");
    if (dir != XR_ROTATE_CW && dir != XR_ROTATE_CCW) return fail(c, XR_ERR_ARG, "bad rotate");
    if (epochs < 0) return fail(c, XR_ERR_ARG, "epochs must be >= 0");
    xr_status st;
    if (fiber) {
        if ((st = check_fiber(c))) return st;
    } else if (xtt && (st = check_xtt_k(c))) {
        return st;
    }
    if ((st = ensure_device(c))) return st;
    const int rotation = dir == XR_ROTATE_CW ? 1 : -1;
    if ((st = ensure_frames(c, rotation))) return st;
    Session &s = c->sess;
    drop_graphs(c);
    s = Session();
    s.xtt = xtt != 0;
    s.epochs = epochs;
    s.batch = batch;
    s.subset_size = (c->V + batch - 1) / batch;      /* reconstruct.cu:61 / :842 */
    s.rotation = rotation;
    s.art = method == XR_METHOD_ART;
    s.lambda = lambda;
    s.d_sino = d_sino;
    s.d_vol = d_vol;
    s.storage = c->storage;
    s.sino_storage = sino_st(c);
    s.update_storage = s.storage | ((c->stochastic && s.storage != 0) ? kStoreStochastic : 0);
    s.coef = coef;
    s.coef_kind = coef_kind;
    s.fiber = fiber;
    std::vector<int> lists((size_t)batch * s.subset_size);
    for (int sub = 0; sub < batch; sub++)
        for (int j = 0; j < s.subset_size; j++)   /* n = (sub + batch*j) % nProj, reconstruct.cu:89 */
            lists[(size_t)sub * s.subset_size + j] = (int)(((long)sub + (long)batch * j) % c->V);
    if ((st = ensure(c, c->subsets, lists.size() * sizeof(int), "subset lists"))) return st;
    st = cuda_check(c, cudaMemcpyAsync(c->subsets.p, lists.data(), lists.size() * sizeof(int),
                                       cudaMemcpyHostToDevice, c->stream), "upload subsets");
    if (st) return st;
    const size_t npx = (size_t)c->C * c->V * c->Nd * c->Nd;
    if ((st = ensure(c, c->proj, npx * sizeof(float), "projections"))) return st;
    s.rtex = false;
    if (c->ratio_texture && (fiber || (s.xtt ? c->all_aligned : true))) {
        /* XTT and fiber: every axis's subset views; IR: one axis at a time */
        if ((st = ensure_ratio_texture(c, (s.xtt || fiber ? c->C : 1) * s.subset_size))) return st;
        s.rtex = c->rtex != 0;
    }
    if (fiber) {
        if ((st = ensure(c, c->fiber_flag, sizeof(int), "fiber flag"))) return st;
        st = cuda_check(c, cudaMemsetAsync(c->fiber_flag.p, 0, sizeof(int), c->stream), "clear fiber flag");
        if (st) return st;
    }
    s.order.resize(batch);
    for (int i = 0; i < batch; i++) s.order[i] = i;
    if (!s.xtt) {
        /* IR: one engine for the whole run, shuffled once per (axis, epoch),
         * axis-major (reconstruct.cu:75-81). */
        std::mt19937_64 eng;
        s.ir_orders.resize((size_t)c->C * epochs * batch);
        std::vector<int> o = s.order;
        for (long r = 0; r < (long)c->C * epochs; r++) {
            std::shuffle(o.begin(), o.end(), eng);
            std::copy(o.begin(), o.end(), s.ir_orders.begin() + r * batch);
        }
    }
    if (s.xtt && !s.fiber && c->all_aligned && !s.art &&
        !(coef == nullptr && c->sens_batch == batch && c->sens_rotation == rotation)) {
        /* factor_k of every subset (geometry only): sum over the subset's views
         * of (|B x S_k| |S_k . G|)^2 (ir.cu:1847), once per session, and kept
         * on the context for the next session of the same subsets and
         * rotation (the rotated-basis variants depend on their planes: not kept). */
        const size_t N3 = (size_t)c->N * c->N * c->N;
        c->sens_batch = 0;
        if ((st = ensure(c, c->sens, (size_t)batch * c->K * N3 * sizeof(float), "sensitivity"))) return st;
        const ColInfo *ci = dcol(c);
        for (int sub = 0; sub < batch; sub++) {
            Timed t(c, XR_T_SETUP);
            st = cuda_check(c, launch_back_col(c->gc, dbasis(c), (const ViewFrame *)c->frames.p,
                                               (const int *)c->subsets.p + (size_t)sub * s.subset_size, s.subset_size,
                                               ci->all, c->C, ci->axis_g, ci->magsig, nullptr, nullptr, nullptr,
                                               (float *)c->sens.p + (size_t)sub * c->K * N3, 2, 0, 0.f, 0, c->stream,
                                               coef, coef_kind),
                            "sensitivity");
            if (st) return st;
        }
        if (!coef) {
            c->sens_batch = batch;
            c->sens_rotation = rotation;
        }
    }
    st = cuda_check(c, cudaStreamSynchronize(c->stream), "session begin");
    if (st) return st;
    s.active = true;
    return XR_OK;
}

xr_status xr_dev_session_begin(xr_ctx *c, const void *d_sino, void *d_vol, int xtt, int epochs, int batch,
                               xr_rotate dir, xr_method method, float lambda) {
    return session_begin_impl(c, d_sino, d_vol, xtt, epochs, batch, dir, method, lambda, nullptr);
}

xr_status xr_dev_session_begin_orth(xr_ctx *c, const void *d_sino, void *d_vol, const float *d_coef, int epochs,
                                    int batch, xr_rotate dir, xr_method method, float lambda) {
    if (!c || !d_coef) return c ? fail(c, XR_ERR_ARG, "null coefficient planes") : XR_ERR_ARG;
    return session_begin_impl(c, d_sino, d_vol, 1, epochs, batch, dir, method, lambda, d_coef);
}

xr_status xr_dev_session_begin_md(xr_ctx *c, const void *d_sino, void *d_vol, const float *d_md, int epochs,
                                  int batch, xr_rotate dir, xr_method method, float lambda) {
    if (!c || !d_md) return c ? fail(c, XR_ERR_ARG, "null main-direction planes") : XR_ERR_ARG;
    return session_begin_impl(c, d_sino, d_vol, 1, epochs, batch, dir, method, lambda, d_md, 1);
}

xr_status xr_dev_session_begin_fiber(xr_ctx *c, const void *d_sino, float *d_vol, int epochs, int batch,
                                     xr_rotate dir, xr_method method, float lambda) {
    return session_begin_impl(c, d_sino, d_vol, 1, epochs, batch, dir, method, lambda, nullptr, 0, true);
}

xr_status xr_dev_session_epoch(xr_ctx *c, double *loss) {
    if (!c) return XR_ERR_ARG;
    Session &s = c->sess;
    xr_status st;
    if ((st = epoch_ready(c))) return st;
    const std::vector<int> orders = next_orders(c);
    cudaStream_t str = c->stream;
    if (c->use_graphs && !c->timing.on) {
        /* one CUDA graph per distinct subset order, captured on first use */
        auto it = s.graphs.find(orders);
        if (it == s.graphs.end()) {
            if ((st = cuda_check(c, cudaStreamBeginCapture(str, cudaStreamCaptureModeRelaxed), "begin capture")))
                return st;
            const xr_status ist = issue_epoch(c, orders);
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(str, &graph);
            if (ist) {
                if (graph) cudaGraphDestroy(graph);
                return ist;
            }
            if ((st = cuda_check(c, ce, "end capture"))) return st;
            cudaGraphExec_t exec = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if ((st = cuda_check(c, ie, "graph instantiate"))) return st;
            it = s.graphs.emplace(orders, exec).first;
        }
        if ((st = cuda_check(c, cudaGraphLaunch(it->second, str), "graph launch"))) return st;
    } else {
        if ((st = issue_epoch(c, orders))) return st;
    }
    s.epoch_done++;
    if (loss) {
        if ((st = loss_copy(c, str))) return st;
        if ((st = cuda_check(c, cudaStreamSynchronize(str), "epoch"))) return st;
        loss_read(c, loss);
    }
    return cuda_check(c, cudaGetLastError(), "epoch");
}

/* Session end; `after` (if set) is called once the volume is final on the
 * compute stream (phase 0, after the voxelSqrt) and once the orientation is
 * (phase 1), before the host waits for the stream. */
static xr_status session_end_impl(xr_ctx *c, float *d_md, float *d_ev,
                                  const std::function<xr_status(int)> &after) {
    if (!c) return XR_ERR_ARG;
    Session &s = c->sess;
    if (!s.active) return fail(c, XR_ERR_STATE, "no active session");
    xr_status st = XR_OK;
    if (s.xtt && !s.fiber && !s.tail_done) {
        const long nvox = (long)c->N * c->N * c->N;
        if (c->xtt_sqrt) {
            Timed t(c, XR_T_ORIENT);
            st = cuda_check(c, launch_sqrt_abs(nvox * c->K, s.d_vol, s.storage, c->stream), "sqrt");   /* reconstruct.cu:919-922 */
        }
        if (!st && after) st = after(0);
        if (!st && d_md) {
            Timed t(c, XR_T_ORIENT);
            st = cuda_check(c, launch_orientation(nvox, c->K, dbasis(c), s.d_vol, d_md, d_ev, s.storage, c->stream),
                            "orientation");
        }
        if (!st && after) st = after(1);
    }
    xr_status st2 = cuda_check(c, cudaStreamSynchronize(c->stream), "session end");
    drop_graphs(c);
    s.active = false;
    return st ? st : st2;
}

xr_status xr_dev_session_end(xr_ctx *c, float *d_md, float *d_ev) {
    return session_end_impl(c, d_md, d_ev, nullptr);
}

xr_status xr_dev_session_proj(xr_ctx *c, const float **d_proj) {
    if (!c || !d_proj) return XR_ERR_ARG;
    *d_proj = (const float *)c->proj.p;
    return XR_OK;
}

/* ---------------------------------------------------- device-buffer calls */

/* forward_into mode of the fiber model's forwardProjFiber */
constexpr int kFiberMode = -1;

static xr_status forward_into(xr_ctx *c, const void *d_vol, float *d_out, int rotation, int mode, bool normalise,
                              int storage, const float *coef = nullptr, int coef_kind = 0) {
    xr_status st;
    if ((st = ensure_frames(c, rotation))) return st;
    const size_t npx = (size_t)c->C * c->V * c->Nd * c->Nd;
    std::vector<int> all(c->V);
    for (int v = 0; v < c->V; v++) all[v] = v;
    DevBuf lst;
    if ((st = ensure(c, lst, all.size() * sizeof(int), "view list"))) return st;
    cudaMemcpyAsync(lst.p, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(d_out, 0, npx * sizeof(float), c->stream);
    {
        Timed t(c, XR_T_FORWARD);
        const cudaError_t e =
            mode == kFiberMode
                ? fiber_forward_dispatch(c, (const int *)lst.p, c->V, (const float *)d_vol, d_out)
                : forward_dispatch(c, (const int *)lst.p, c->V, all_conds(c), d_vol, d_out, mode, storage, coef,
                                   coef_kind);
        st = cuda_check(c, e, "forward");
    }
    if (!st && normalise) {
        Timed t(c, XR_T_OTHER);
        st = cuda_check(c, launch_normalize(c->gc, c->C, d_out, (const float *)c->norm.p, c->stream), "normalise");
    }
    cudaStreamSynchronize(c->stream);
    release(lst);
    return st;
}

xr_status xr_dev_forward_orth(xr_ctx *c, const void *d_vol, const float *d_coef, float *d_sino, xr_rotate dir) {
    if (!c || !d_vol || !d_coef || !d_sino) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if ((st = check_xtt_k(c))) return st;
    if ((st = ensure_device(c))) return st;
    return forward_into(c, d_vol, d_sino, dir == XR_ROTATE_CCW ? -1 : 1, 1, false, c->storage, d_coef);
}

xr_status xr_dev_forward_fiber(xr_ctx *c, const float *d_vol, float *d_sino, xr_rotate dir) {
    if (!c || !d_vol || !d_sino) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    if (dir != XR_ROTATE_CW && dir != XR_ROTATE_CCW) return fail(c, XR_ERR_ARG, "bad rotate");
    xr_status st;
    if ((st = check_fiber(c))) return st;
    if ((st = ensure_device(c))) return st;
    return forward_into(c, d_vol, d_sino, dir == XR_ROTATE_CCW ? -1 : 1, kFiberMode, false, 0);
}

xr_status xr_dev_forward_md(xr_ctx *c, const void *d_vol, const float *d_md, float *d_sino, xr_rotate dir) {
    if (!c || !d_vol || !d_md || !d_sino) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if ((st = check_xtt_k(c))) return st;
    if ((st = ensure_device(c))) return st;
    return forward_into(c, d_vol, d_sino, dir == XR_ROTATE_CCW ? -1 : 1, 1, true, c->storage, d_md, 1);
}

static xr_status md_need3(xr_ctx *c) {
    if (c->K < 3) return fail(c, XR_ERR_CONFIG, "the main-direction steps need three basis vectors");
    return ensure_device(c);
}

xr_status xr_md_filter(xr_ctx *c, float *d_md, float *d_tmp, float weight, int passes) {
    if (!c || !d_md || !d_tmp || passes < 0) return c ? fail(c, XR_ERR_ARG, "bad argument") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    const size_t bytes = 3 * (size_t)c->N * c->N * c->N * sizeof(float);
    Timed t(c, XR_T_ORIENT);
    for (int p = 0; p < passes; p++) {
        if ((st = cuda_check(c, cudaMemcpyAsync(d_tmp, d_md, bytes, cudaMemcpyDeviceToDevice, c->stream), "md copy")))
            return st;
        if ((st = cuda_check(c, launch_md_filter(c->N, d_md, d_tmp, weight, c->stream), "md filter"))) return st;
        if ((st = cuda_check(c, cudaMemcpyAsync(d_md, d_tmp, bytes, cudaMemcpyDeviceToDevice, c->stream), "md copy")))
            return st;
    }
    return cuda_check(c, cudaStreamSynchronize(c->stream), "md filter");
}

xr_status xr_md_main_direction(xr_ctx *c, const float *d_vol, float *d_md, int iter) {
    if (!c || !d_vol || !d_md || iter < 0 || iter > 3) return c ? fail(c, XR_ERR_ARG, "bad argument") : XR_ERR_ARG;
    xr_status st;
    if ((st = md_need3(c))) return st;
    st = cuda_check(c, launch_main_direction(c->N, d_vol, d_md, nullptr, iter, c->stream), "main direction");
    return st ? st : cuda_check(c, cudaStreamSynchronize(c->stream), "main direction");
}

xr_status xr_md_with_estimate(xr_ctx *c, const float *d_vol, float *d_md, const float *d_est) {
    if (!c || !d_vol || !d_md || !d_est) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if ((st = md_need3(c))) return st;
    st = cuda_check(c, launch_main_direction(c->N, d_vol, d_md, d_est, 0, c->stream), "main direction");
    return st ? st : cuda_check(c, cudaStreamSynchronize(c->stream), "main direction");
}

xr_status xr_md_update_estimation(xr_ctx *c, const float *d_vol, float *d_est, int iter) {
    if (!c || !d_vol || !d_est) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if ((st = md_need3(c))) return st;
    st = cuda_check(c, launch_update_estimation(c->N, d_vol, d_est, iter, c->stream), "estimation");
    return st ? st : cuda_check(c, cudaStreamSynchronize(c->stream), "estimation");
}

xr_status xr_dev_fill(xr_ctx *c, float *d, size_t n, float value) {
    if (!c || (!d && n)) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    st = cuda_check(c, launch_fill((long)n, d, value, c->stream), "fill");
    return st ? st : cuda_check(c, cudaStreamSynchronize(c->stream), "fill");
}

xr_status xr_orth_normal_update(xr_ctx *c, const float *d_vol, float *d_coef, float *d_loss, int rot) {
    if (!c || !d_vol || !d_coef || !d_loss) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    if (c->K < 3) return fail(c, XR_ERR_CONFIG, "the normal update needs three basis vectors");
    xr_status st;
    if ((st = ensure_device(c))) return st;
    st = cuda_check(c, launch_normal_three((long)c->N * c->N * c->N, dbasis(c), d_vol, d_coef, d_loss, rot, c->stream),
                    "normal update");
    if (!st) st = cuda_check(c, cudaStreamSynchronize(c->stream), "normal update");
    return st;
}

xr_status xr_orth_normal_update_est(xr_ctx *c, const float *d_vol, float *d_coef, float *d_loss, const float *d_est) {
    if (!c || !d_vol || !d_coef || !d_loss || !d_est) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    if (c->K < 3) return fail(c, XR_ERR_CONFIG, "the normal update needs three basis vectors");
    xr_status st;
    if ((st = ensure_device(c))) return st;
    st = cuda_check(c, launch_normal_three((long)c->N * c->N * c->N, dbasis(c), d_vol, d_coef, d_loss, 0, c->stream,
                                           d_est),
                    "normal update");
    return st ? st : cuda_check(c, cudaStreamSynchronize(c->stream), "normal update");
}

xr_status xr_orth_filter(xr_ctx *c, float *d_coef, float *d_tmp, const float *d_vol, float weight, int passes) {
    if (!c || !d_coef || !d_tmp || !d_vol || passes < 0) return c ? fail(c, XR_ERR_ARG, "bad argument") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    const size_t bytes = 2 * (size_t)c->N * c->N * c->N * sizeof(float);
    Timed t(c, XR_T_ORIENT);
    for (int p = 0; p < passes; p++) {
        if ((st = cuda_check(c, cudaMemcpyAsync(d_tmp, d_coef, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy")))
            return st;
        if ((st = cuda_check(c, launch_coef_filter(c->N, d_coef, d_vol, d_tmp, weight, c->stream), "fiber filter")))
            return st;
        if ((st = cuda_check(c, cudaMemcpyAsync(d_coef, d_tmp, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy")))
            return st;
    }
    return cuda_check(c, cudaStreamSynchronize(c->stream), "fiber filter");
}

xr_status xr_orth_update_estimation(xr_ctx *c, const float *d_vol, float *d_est, int iter) {
    if (!c || !d_vol || !d_est) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    if (c->K < 3) return fail(c, XR_ERR_CONFIG, "the estimation needs three basis vectors");
    xr_status st;
    if ((st = ensure_device(c))) return st;
    st = cuda_check(c, launch_update_estimation_coef((long)c->N * c->N * c->N, dbasis(c), d_vol, d_est, iter,
                                                     c->stream),
                    "estimation");
    return st ? st : cuda_check(c, cudaStreamSynchronize(c->stream), "estimation");
}

xr_status xr_dev_forward(xr_ctx *c, const void *d_vol, float *d_sino, xr_rotate dir, int xtt) {
    if (!c || !d_vol || !d_sino) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if (xtt && (st = check_xtt_k(c))) return st;
    if ((st = ensure_device(c))) return st;
    return forward_into(c, d_vol, d_sino, dir == XR_ROTATE_CCW ? -1 : 1, xtt ? 1 : 0, true, c->storage);
}

xr_status xr_dev_residual(xr_ctx *c, const void *d_vol, const void *d_sino, xr_rotate dir, int xtt,
                          double *rel_l2, double *l1) {
    if (!c || !d_vol || !d_sino) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if (xtt && (st = check_xtt_k(c))) return st;
    if ((st = ensure_device(c))) return st;
    const size_t npx = (size_t)c->C * c->V * c->Nd * c->Nd;
    if ((st = ensure(c, c->scratch_sino, npx * sizeof(float), "residual scratch"))) return st;
    float *p = (float *)c->scratch_sino.p;
    if ((st = forward_into(c, d_vol, p, dir == XR_ROTATE_CCW ? -1 : 1, xtt ? 1 : 0, true, c->storage))) return st;
    double *dl = (double *)c->loss.p + 40;
    cudaMemsetAsync(dl, 0, 3 * sizeof(double), c->stream);
    {
        Timed t(c, XR_T_OTHER);
        if ((st = cuda_check(c, launch_residual((long)npx, p, d_sino, dl, sino_st(c), c->stream), "residual")))
            return st;
    }
    if ((st = cuda_check(c, cudaMemcpyAsync(c->h_loss, dl, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                         "residual copy")))
        return st;
    if ((st = cuda_check(c, cudaStreamSynchronize(c->stream), "residual"))) return st;
    if (rel_l2) *rel_l2 = c->h_loss[1] > 0 ? std::sqrt(c->h_loss[0] / c->h_loss[1]) : 0.0;
    if (l1) *l1 = c->h_loss[2];
    return XR_OK;
}

xr_status xr_dev_orientation(xr_ctx *c, const void *d_mu, float *d_md, float *d_ev) {
    if (!c || !d_mu || !d_md) return c ? fail(c, XR_ERR_ARG, "null buffer") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    {
        Timed t(c, XR_T_ORIENT);
        st = cuda_check(c, launch_orientation((long)c->N * c->N * c->N, c->K, dbasis(c), d_mu, d_md, d_ev,
                                              c->storage, c->stream), "orientation");
    }
    if (!st) st = cuda_check(c, cudaStreamSynchronize(c->stream), "orientation");
    return st;
}

/* ------------------------------------------------------ host-buffer calls */

static xr_status upload_planes_on(xr_ctx *c, DevBuf &b, const float *const *src, int planes, size_t plane_elems,
                                  const char *what, cudaStream_t str) {
    for (int i = 0; i < planes; i++)
        if (!src[i]) return fail(c, XR_ERR_ARG, std::string("null host pointer: ") + what);
    xr_status st;
    if ((st = ensure(c, b, (size_t)planes * plane_elems * sizeof(float), what))) return st;
    for (int i = 0; i < planes; i++) {
        st = cuda_check(c, cudaMemcpyAsync((float *)b.p + i * plane_elems, src[i], plane_elems * sizeof(float),
                                           cudaMemcpyHostToDevice, str), what);
        if (st) return st;
    }
    return XR_OK;
}

static xr_status upload_planes(xr_ctx *c, DevBuf &b, const float *const *src, int planes, size_t plane_elems,
                               const char *what) {
    return upload_planes_on(c, b, src, planes, plane_elems, what, c->stream);
}

/* Device planes into host planes, enqueued on `str` without waiting. */
static xr_status download_planes_async(xr_ctx *c, const float *d, float *const *dst, int planes, size_t plane_elems,
                                       const char *what, cudaStream_t str) {
    for (int i = 0; i < planes; i++) {
        if (!dst[i]) return fail(c, XR_ERR_ARG, std::string("null host pointer: ") + what);
        xr_status st = cuda_check(c, cudaMemcpyAsync(dst[i], d + i * plane_elems, plane_elems * sizeof(float),
                                                     cudaMemcpyDeviceToHost, str), what);
        if (st) return st;
    }
    return XR_OK;
}

static xr_status download_planes(xr_ctx *c, const float *d, float *const *dst, int planes, size_t plane_elems,
                                 const char *what) {
    xr_status st = download_planes_async(c, d, dst, planes, plane_elems, what, c->stream);
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), what);
}

/* Host float planes into `b` in the storage type (through the FP32 staging
 * buffer when the storage is 16-bit), and back. */
static xr_status upload_planes_s_on(xr_ctx *c, DevBuf &b, const float *const *src, int planes, size_t plane_elems,
                                    int storage, const char *what, cudaStream_t str) {
    if (storage == 0) return upload_planes_on(c, b, src, planes, plane_elems, what, str);
    xr_status st;
    const size_t n = (size_t)planes * plane_elems;
    if ((st = upload_planes_on(c, c->stage, src, planes, plane_elems, what, str))) return st;
    if ((st = ensure(c, b, n * storage_bytes(storage), what))) return st;
    return cuda_check(c, launch_convert((long)n, c->stage.p, 0, b.p, storage, str), what);
}

static xr_status upload_planes_s(xr_ctx *c, DevBuf &b, const float *const *src, int planes, size_t plane_elems,
                                 int storage, const char *what) {
    return upload_planes_s_on(c, b, src, planes, plane_elems, storage, what, c->stream);
}

static xr_status download_planes_s_async(xr_ctx *c, const void *d, float *const *dst, int planes,
                                         size_t plane_elems, int storage, const char *what, cudaStream_t str) {
    if (storage == 0) return download_planes_async(c, (const float *)d, dst, planes, plane_elems, what, str);
    xr_status st;
    const size_t n = (size_t)planes * plane_elems;
    if ((st = ensure(c, c->stage, n * sizeof(float), what))) return st;
    if ((st = cuda_check(c, launch_convert((long)n, d, storage, c->stage.p, 0, str), what))) return st;
    return download_planes_async(c, (const float *)c->stage.p, dst, planes, plane_elems, what, str);
}

static xr_status download_planes_s(xr_ctx *c, const void *d, float *const *dst, int planes, size_t plane_elems,
                                   int storage, const char *what) {
    xr_status st = download_planes_s_async(c, d, dst, planes, plane_elems, storage, what, c->stream);
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), what);
}

/* The transfer stream and its events (created on first use). */
static xr_status ensure_copy_stream(xr_ctx *c) {
    xr_status st;
    if (!c->copy_stream &&
        (st = cuda_check(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate")))
        return st;
    for (cudaEvent_t &e : c->copy_ev)
        if (!e && (st = cuda_check(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")))
            return st;
    for (cudaEvent_t &e : c->slab_ev)
        if (!e && (st = cuda_check(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")))
            return st;
    for (cudaEvent_t &e : c->tail_ev)
        if (!e && (st = cuda_check(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")))
            return st;
    return XR_OK;
}

/* Makes `to` wait for the work enqueued on `from` so far. */
static xr_status stream_after(xr_ctx *c, cudaStream_t to, cudaStream_t from, cudaEvent_t e) {
    xr_status st = cuda_check(c, cudaEventRecord(e, from), "cudaEventRecord");
    if (st) return st;
    return cuda_check(c, cudaStreamWaitEvent(to, e, 0), "cudaStreamWaitEvent");
}

xr_status xr_forward(xr_ctx *c, const float *const *voxel, float *const *sino, xr_rotate dir, int xtt) {
    if (!c || !voxel || !sino) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    xr_status st;
    if (xtt && (st = check_xtt_k(c))) return st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N, blk = (size_t)c->V * c->Nd * c->Nd;
    if ((st = upload_planes_s(c, c->scratch_vol, voxel, xtt ? c->K : 1, N3, c->storage, "volume"))) return st;
    if ((st = ensure(c, c->scratch_sino, c->C * blk * sizeof(float), "sinogram"))) return st;
    if ((st = forward_into(c, c->scratch_vol.p, (float *)c->scratch_sino.p, dir == XR_ROTATE_CCW ? -1 : 1,
                           xtt ? 1 : 0, true, c->storage)))
        return st;
    return download_planes(c, (const float *)c->scratch_sino.p, sino, c->C, blk, "sinogram");
}

/* forwardProjOnly, reconstruct.cu:1890-1949: plain splat of channel 0, no
 * normalisation (the reference passes a null weight buffer there, which
 * faults; the weights are simply not accumulated here). */
xr_status xr_forward_proj_only(xr_ctx *c, const float *const *voxel, float *const *sino, xr_rotate dir) {
    if (!c || !voxel || !sino) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N, blk = (size_t)c->V * c->Nd * c->Nd;
    if ((st = upload_planes(c, c->scratch_vol, voxel, 1, N3, "volume"))) return st;
    if ((st = ensure(c, c->scratch_sino, c->C * blk * sizeof(float), "sinogram"))) return st;
    if ((st = forward_into(c, c->scratch_vol.p, (float *)c->scratch_sino.p, dir == XR_ROTATE_CCW ? -1 : 1, 0,
                           false, 0)))
        return st;
    return download_planes(c, (const float *)c->scratch_sino.p, sino, c->C, blk, "sinogram");
}

xr_status xr_ir_reconstruct(xr_ctx *c, float *const *sino, float *const *voxel, int epoch, int batch,
                            xr_rotate dir, xr_method method, float lambda, float *losses) {
    if (!c || !sino || !voxel) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    if (epoch < 0) return fail(c, XR_ERR_ARG, "epoch must be >= 0");
    xr_status st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N, blk = (size_t)c->V * c->Nd * c->Nd;
    if ((st = upload_planes_s(c, c->scratch_sino, sino, c->C, blk, sino_st(c), "sinogram"))) return st;
    if ((st = upload_planes_s(c, c->scratch_vol, voxel, c->C, N3, c->storage, "volume"))) return st;
    if ((st = xr_dev_session_begin(c, c->scratch_sino.p, c->scratch_vol.p, 0, epoch, batch, dir, method, lambda)))
        return st;
    std::vector<double> l(c->C);
    for (int ep = 0; ep < epoch; ep++) {
        if ((st = xr_dev_session_epoch(c, losses ? l.data() : nullptr))) return st;
        if (losses)
            for (int cond = 0; cond < c->C; cond++) losses[(size_t)cond * epoch + ep] = (float)l[cond];
    }
    if ((st = xr_dev_session_end(c, nullptr, nullptr))) return st;
    return download_planes_s(c, c->scratch_vol.p, voxel, c->C, N3, c->storage, "volume");
}

xr_status xr_xtt_reconstruct(xr_ctx *c, float *const *sino, float *const *voxel, float *const *md,
                             float *const *evalue, int epoch, int batch, xr_rotate dir, xr_method method,
                             float lambda, float *losses) {
    if (!c || !sino || !voxel) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    if (epoch < 0) return fail(c, XR_ERR_ARG, "epoch must be >= 0");
    xr_status st;
    if ((st = check_xtt_k(c))) return st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N, blk = (size_t)c->V * c->Nd * c->Nd;
    if ((st = ensure_copy_stream(c))) return st;
    cudaStream_t cs = c->copy_stream;
    /* Transfers run on the copy stream beside the compute stream: the uploads
     * overlap the per-subset sensitivity (geometry only) of the session start,
     * the downloads the voxelSqrt and the orientation of its end.  Every exit
     * waits for the copy stream, so no transfer outlives the call. */
    struct CopyWait {
        cudaStream_t s;
        ~CopyWait() { cudaStreamSynchronize(s); }
    } copy_wait{cs};
    if ((st = stream_after(c, cs, c->stream, c->copy_ev[0]))) return st;   /* earlier work on the buffers */
    /* FP32 storage, direct epochs: the uploads are staged so the first
     * subset's work overlaps them (below); else volume, then sinogram */
    const bool staged = c->storage == 0 && sino_st(c) == 0 && !c->use_graphs && epoch > 0;
    if (!staged) {
        if ((st = upload_planes_s_on(c, c->scratch_vol, voxel, c->K, N3, c->storage, "volume", cs))) return st;
        if ((st = cuda_check(c, cudaEventRecord(c->copy_ev[1], cs), "cudaEventRecord"))) return st;
        if ((st = upload_planes_s_on(c, c->scratch_sino, sino, c->C, blk, sino_st(c), "sinogram", cs))) return st;
        if ((st = cuda_check(c, cudaEventRecord(c->copy_ev[2], cs), "cudaEventRecord"))) return st;
    } else {
        for (int i = 0; i < c->K; i++)
            if (!voxel[i]) return fail(c, XR_ERR_ARG, "null host pointer: volume");
        for (int i = 0; i < c->C; i++)
            if (!sino[i]) return fail(c, XR_ERR_ARG, "null host pointer: sinogram");
        if ((st = ensure(c, c->scratch_vol, (size_t)c->K * N3 * sizeof(float), "volume"))) return st;
        if ((st = ensure(c, c->scratch_sino, (size_t)c->C * blk * sizeof(float), "sinogram"))) return st;
    }
    if ((st = xr_dev_session_begin(c, c->scratch_sino.p, c->scratch_vol.p, 1, epoch, batch, dir, method, lambda)))
        return st;
    if (!staged) {
        /* the first subset's forward needs only the volume; its ratio waits for
         * the sinogram (inside a captured epoch graph the wait comes first) */
        st = cuda_check(c, cudaStreamWaitEvent(c->stream, c->copy_ev[1], 0), "cudaStreamWaitEvent");
        if (!st && (c->use_graphs || epoch == 0))
            st = cuda_check(c, cudaStreamWaitEvent(c->stream, c->copy_ev[2], 0), "cudaStreamWaitEvent");
        else if (!st)
            c->sess.sino_ready = c->copy_ev[2];
    } else {
        /* Order on the copy stream: the first subset's views of the sinogram,
         * the volume in z-slabs (the first forward starts on each slab as it
         * lands), then the rest of the sinogram (waited for by the second
         * subset's ratio).  The first epoch's subset order is the one its
         * epoch call will draw: the persistent order shuffled by a fresh
         * default engine (reconstruct.cu:858-859). */
        std::vector<int> o = c->sess.order;
        {
            std::mt19937_64 eng;
            std::shuffle(o.begin(), o.end(), eng);
        }
        const size_t NdNd = (size_t)c->Nd * c->Nd, NN = (size_t)c->N * c->N;
        std::vector<char> first(c->V, 0);
        for (int j = 0; j < c->sess.subset_size; j++) first[((long)o[0] + (long)batch * j) % c->V] = 1;
        float *dsino = (float *)c->scratch_sino.p, *dvol = (float *)c->scratch_vol.p;
        auto copy_views = [&](char want) -> xr_status {
            for (int cond = 0; cond < c->C; cond++)
                for (int v0 = 0; v0 < c->V;) {
                    if (first[v0] != want) { v0++; continue; }
                    int v1 = v0;
                    while (v1 < c->V && first[v1] == want) v1++;
                    xr_status e2 = cuda_check(c, cudaMemcpyAsync(dsino + cond * blk + v0 * NdNd, sino[cond] + v0 * NdNd,
                                                                 (size_t)(v1 - v0) * NdNd * sizeof(float),
                                                                 cudaMemcpyHostToDevice, cs), "sinogram");
                    if (e2) return e2;
                    v0 = v1;
                }
            return XR_OK;
        };
        st = copy_views(1);
        if (!st) st = cuda_check(c, cudaEventRecord(c->copy_ev[2], cs), "cudaEventRecord");
        const int S = xr_ctx::kSlabs, zs = ((c->N + S - 1) / S + 15) / 16 * 16;
        for (int i = 0; i < S && !st; i++) {
            const int z0 = std::min(c->N, i * zs), z1 = (i == S - 1) ? c->N : std::min(c->N, (i + 1) * zs);
            for (int k = 0; k < c->K && !st && z1 > z0; k++)
                st = cuda_check(c, cudaMemcpyAsync(dvol + k * N3 + z0 * NN, voxel[k] + z0 * NN,
                                                   (size_t)(z1 - z0) * NN * sizeof(float), cudaMemcpyHostToDevice, cs),
                                "volume");
            if (!st) st = cuda_check(c, cudaEventRecord(c->slab_ev[i], cs), "cudaEventRecord");
        }
        if (!st) st = copy_views(0);
        if (!st) st = cuda_check(c, cudaEventRecord(c->copy_ev[1], cs), "cudaEventRecord");
        if (!st) {
            c->sess.sino_ready = c->copy_ev[2];
            c->sess.sino_rest = c->copy_ev[1];
            c->sess.vol_slabs = S;
            c->sess.slab_ev = c->slab_ev;
        }
    }
    if (st) {
        xr_dev_session_end(c, nullptr, nullptr);
        return st;
    }
    float *d_md = nullptr, *d_ev = nullptr;
    if (md) {
        if ((st = ensure(c, c->scratch_md, 6 * N3 * sizeof(float), "orientation"))) return st;
        d_md = (float *)c->scratch_md.p;
        d_ev = evalue ? d_md + 3 * N3 : nullptr;
    }
    /* the last epoch hands each view's final ratio image to the copy stream
     * as soon as its subset is done (not inside a captured epoch graph); with
     * staged transfers its last back-projection also runs by z-slabs, each
     * slab's voxelSqrt, orientation and downloads following at once */
    const bool early = !c->use_graphs && epoch > 0;
    for (int ep = 0; ep < epoch; ep++) {
        double l = 0;
        Session &s = c->sess;
        if (early && ep == epoch - 1) s.ratio_dst = sino;
        if (staged && ep == epoch - 1 && c->all_aligned) {
            s.tail_slabs = xr_ctx::kSlabs;
            s.vol_dst = voxel;
            s.md_dst = md;
            s.ev_dst = evalue;
            s.tail_md = d_md;
            s.tail_ev = d_ev;
        }
        st = xr_dev_session_epoch(c, losses ? &l : nullptr);
        s.ratio_dst = nullptr;
        s.tail_slabs = 0;
        if (st) return st;
        if (losses) losses[ep] = (float)l;
    }
    if (!early) {   /* the ratio images are final after the last epoch */
        if ((st = stream_after(c, cs, c->stream, c->copy_ev[0]))) return st;
        if ((st = download_planes_async(c, (const float *)c->proj.p, sino, c->C, blk, "ratio images", cs)))
            return st;
    }
    const void *d_vol = c->scratch_vol.p;
    auto after = [&](int phase) -> xr_status {
        xr_status s2 = stream_after(c, cs, c->stream, c->copy_ev[1 + phase]);
        if (s2) return s2;
        if (phase == 0) return download_planes_s_async(c, d_vol, voxel, c->K, N3, c->storage, "volume", cs);
        if (!md) return XR_OK;
        if ((s2 = download_planes_async(c, d_md, md, 3, N3, "md", cs))) return s2;
        return evalue ? download_planes_async(c, d_ev, evalue, 3, N3, "evalue", cs) : XR_OK;
    };
    if ((st = session_end_impl(c, d_md, d_ev, after))) return st;
    return cuda_check(c, cudaStreamSynchronize(cs), "downloads");
}

xr_status xr_fiber_reconstruct(xr_ctx *c, float *const *sino, float *const *voxel, int epoch, int batch,
                               xr_rotate dir, xr_method method, float lambda, float *losses) {
    if (!c || !sino || !voxel) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    if (epoch < 0) return fail(c, XR_ERR_ARG, "epoch must be >= 0");
    xr_status st;
    if ((st = check_fiber(c))) return st;
    for (int i = 0; i < c->K; i++)
        if (!voxel[i]) return fail(c, XR_ERR_ARG, "null host pointer: volume");
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N, blk = (size_t)c->V * c->Nd * c->Nd;
    if ((st = upload_planes_s(c, c->scratch_sino, sino, c->C, blk, sino_st(c), "sinogram"))) return st;
    if ((st = ensure(c, c->scratch_vol, (size_t)c->K * N3 * sizeof(float), "volume"))) return st;
    /* every channel starts at 0.01 whatever the caller passed (reconstruct.cu:1245-1247) */
    if ((st = cuda_check(c, launch_fill((long)(c->K * N3), (float *)c->scratch_vol.p, 0.01f, c->stream), "fill")))
        return st;
    if ((st = xr_dev_session_begin_fiber(c, c->scratch_sino.p, (float *)c->scratch_vol.p, epoch, batch, dir, method,
                                         lambda)))
        return st;
    for (int ep = 0; ep < epoch; ep++) {
        double l = 0;
        if ((st = xr_dev_session_epoch(c, losses ? &l : nullptr))) return st;
        if (losses) losses[ep] = (float)l;
    }
    if ((st = xr_dev_session_end(c, nullptr, nullptr))) return st;
    /* with no epoch the reference hands back its never-written devProj; here that is zeros */
    if (epoch == 0 && (st = cuda_check(c, cudaMemsetAsync(c->proj.p, 0, (size_t)c->C * blk * sizeof(float), c->stream),
                                       "clear ratio images")))
        return st;
    if ((st = download_planes_async(c, (const float *)c->proj.p, sino, c->C, blk, "ratio images", c->stream))) return st;
    return download_planes(c, (const float *)c->scratch_vol.p, voxel, c->K, N3, "volume");
}

xr_status xr_orientation(xr_ctx *c, const float *const *mu, float *const *md, float *const *evalue) {
    if (!c || !mu || !md) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N;
    if ((st = upload_planes_s(c, c->scratch_vol, mu, c->K, N3, c->storage, "mu"))) return st;
    if ((st = ensure(c, c->scratch_md, 6 * N3 * sizeof(float), "orientation"))) return st;
    float *d_md = (float *)c->scratch_md.p;
    float *d_ev = evalue ? d_md + 3 * N3 : nullptr;
    if ((st = xr_dev_orientation(c, c->scratch_vol.p, d_md, d_ev))) return st;
    if ((st = download_planes(c, d_md, md, 3, N3, "md"))) return st;
    if (evalue) return download_planes(c, d_ev, evalue, 3, N3, "evalue");
    return XR_OK;
}

xr_status xr_angle_from_md(xr_ctx *c, const float *const *md, float *const *angle) {
    if (!c || !md || !angle) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N;
    if ((st = upload_planes(c, c->scratch_vol, md, 3, N3, "md"))) return st;
    if ((st = ensure(c, c->scratch_md, 6 * N3 * sizeof(float), "angle"))) return st;
    {
        Timed t(c, XR_T_ORIENT);
        if ((st = cuda_check(c, launch_angle_from_md((long)N3, (const float *)c->scratch_vol.p,
                                                     (float *)c->scratch_md.p, c->stream), "angle")))
            return st;
    }
    return download_planes(c, (const float *)c->scratch_md.p, angle, 2, N3, "angle");
}

xr_status xr_direction_normalization(xr_ctx *c, float *const *md) {
    if (!c || !md) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    xr_status st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N;
    if ((st = upload_planes(c, c->scratch_vol, (const float *const *)md, 3, N3, "md"))) return st;
    {
        Timed t(c, XR_T_ORIENT);
        if ((st = cuda_check(c, launch_direction_normalization((long)N3, (float *)c->scratch_vol.p, c->stream),
                             "normalise")))
            return st;
    }
    return download_planes(c, (const float *)c->scratch_vol.p, md, 3, N3, "md");
}

xr_status xr_residual(xr_ctx *c, const float *const *voxel, const float *const *sino, xr_rotate dir, int xtt,
                      double *rel_l2, double *l1) {
    if (!c || !voxel || !sino) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    xr_status st;
    if (xtt && (st = check_xtt_k(c))) return st;
    if ((st = ensure_device(c))) return st;
    const size_t N3 = (size_t)c->N * c->N * c->N, blk = (size_t)c->V * c->Nd * c->Nd;
    if ((st = upload_planes_s(c, c->scratch_vol, voxel, xtt ? c->K : 1, N3, c->storage, "volume"))) return st;
    DevBuf b;
    if ((st = upload_planes_s(c, b, sino, c->C, blk, sino_st(c), "sinogram"))) return st;
    st = xr_dev_residual(c, c->scratch_vol.p, b.p, dir, xtt, rel_l2, l1);
    release(b);
    return st;
}

/* FDK::reconstruct, reconstruct.cu:1651-1724. */
xr_status xr_fdk_reconstruct(xr_ctx *c, float *const *sino, float *const *voxel, xr_rotate dir, xr_filter filter) {
    if (!c || !sino || !voxel) return c ? fail(c, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    if (filter != XR_FILTER_REFERENCE && filter != XR_FILTER_RAMLAK) return fail(c, XR_ERR_ARG, "bad filter");
    xr_status st;
    if ((st = ensure_device(c))) return st;
    xr_ctx &x = *c;
    const int rotation = dir == XR_ROTATE_CCW ? -1 : 1;
    const size_t N3 = (size_t)c->N * c->N * c->N, blk = (size_t)c->V * c->Nd * c->Nd;
    if (x.fdk_rotation != rotation) {
        std::vector<ViewFrame> h((size_t)c->C * c->V);
        for (int cond = 0; cond < c->C; cond++)
            for (int v = 0; v < c->V; v++) h[(size_t)cond * c->V + v] = make_frame(c, cond, rotation * v, true);
        if ((st = ensure(c, x.fdk_frames, h.size() * sizeof(ViewFrame), "fdk frames"))) return st;
        cudaMemcpy(x.fdk_frames.p, h.data(), h.size() * sizeof(ViewFrame), cudaMemcpyHostToDevice);
        x.fdk_rotation = rotation;
        x.fdk_axis_g.assign(c->C, -1);
        x.fdk_magsig.assign(c->C, 0.f);
        for (int cond = 0; cond < c->C; cond++) {
            float sg = 0.f;
            x.fdk_axis_g[cond] = aligned_axis(h, cond, c->V, &sg);
            x.fdk_magsig[cond] = sg * c->gc.mag;
        }
    }
    /* filter table, reconstruct.cu:1694-1698 (or Ram-Lak in the same scaling) */
    std::vector<float> filt(c->Nd);
    const float d = c->det * (c->sod / c->sdd);
    for (int k = 0; k < c->Nd; k++) {
        if (filter == XR_FILTER_REFERENCE) {
            filt[k] = 1.0f / (float)(M_PI * M_PI * d * (1.0f - 4.0f * (float)(k * k)));
        } else {
            if (k == 0) filt[k] = 1.0f / (8.0f * d);
            else if (k % 2) filt[k] = -1.0f / (2.0f * (float)(M_PI * M_PI) * (float)((long)k * k) * d);
            else filt[k] = 0.0f;
        }
    }
    if ((st = ensure(c, x.fdk_filt, filt.size() * sizeof(float), "filter"))) return st;
    cudaMemcpyAsync(x.fdk_filt.p, filt.data(), filt.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    if ((st = ensure(c, x.fdk_weight, (size_t)c->Nd * c->Nd * sizeof(float), "weight"))) return st;
    if ((st = upload_planes(c, c->scratch_sino, (const float *const *)sino, c->C, blk, "sinogram"))) return st;
    if ((st = ensure(c, x.fdk_sf, c->C * blk * sizeof(float), "filtered"))) return st;
    if ((st = ensure(c, c->scratch_vol, c->C * N3 * sizeof(float), "volume"))) return st;
    if (c->ratio_texture &&
        (st = ensure_layered(c, c->C * c->V, x.farr, x.ftex, x.fsurf, x.flayers, x.fnd, "filtered projection array")))
        return st;
    {
        Timed t(c, XR_T_FDK);
        st = cuda_check(c, launch_fdk(c->gc, (const ViewFrame *)x.fdk_frames.p, c->C,
                                      (const float *)c->scratch_sino.p, (float *)x.fdk_sf.p,
                                      (float *)c->scratch_vol.p, (const float *)x.fdk_filt.p,
                                      (float *)x.fdk_weight.p, c->fdk_axis_blocks, c->stream,
                                      x.fdk_axis_g.data(), x.fdk_magsig.data(), c->ratio_texture ? x.fsurf : 0,
                                      c->ratio_texture ? x.ftex : 0), "fdk");
    }
    if (st) return st;
    if ((st = download_planes(c, (const float *)c->scratch_vol.p, voxel, c->C, N3, "volume"))) return st;
    return download_planes(c, (const float *)x.fdk_sf.p, sino, c->C, blk, "filtered sinogram");
}

/* ---------------------------------------------------------------- batches */

struct xr_batch {
    std::vector<xr_ctx *> ctx;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> ev;                          /* fork, then one join per specimen */
    std::map<std::vector<int>, cudaGraphExec_t> graphs;   /* per combination of subset orders */
    std::string err;
};

static xr_status bfail(xr_batch *b, xr_status st, const std::string &m) {
    b->err = m;
    return st;
}

static xr_status bspec(xr_batch *b, int i, xr_status st) {
    return bfail(b, st, "specimen " + std::to_string(i) + ": " + b->ctx[i]->err);
}

static void batch_drop_graphs(xr_batch *b) {
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

xr_status xr_batch_create(xr_ctx *const *ctxs, int n, xr_batch **out) {
    if (!ctxs || n < 1 || !out) return XR_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < n; i++)
        if (!ctxs[i] || ctxs[i]->device != ctxs[0]->device) return XR_ERR_ARG;
    for (int i = 0; i < n; i++) {
        const xr_status st = ensure_device(ctxs[i]);
        if (st) return st;
    }
    xr_batch *b = new xr_batch();
    b->ctx.assign(ctxs, ctxs + n);
    b->device = ctxs[0]->device;
    cudaSetDevice(b->device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    for (int i = 0; i <= n && e == cudaSuccess; i++) {
        cudaEvent_t ev = nullptr;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) b->ev.push_back(ev);
    }
    if (e != cudaSuccess) {
        xr_batch_destroy(b);
        return XR_ERR_CUDA;
    }
    *out = b;
    return XR_OK;
}

void xr_batch_destroy(xr_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graphs(b);
    for (cudaEvent_t ev : b->ev) cudaEventDestroy(ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char *xr_batch_last_error(const xr_batch *b) { return b ? b->err.c_str() : "null batch"; }

xr_status xr_batch_session_begin(xr_batch *b, const void *const *d_sinos, void *const *d_vols, int xtt, int epochs,
                                 int subsets, xr_rotate dir, xr_method method, float lambda) {
    if (!b || !d_sinos || !d_vols) return b ? bfail(b, XR_ERR_ARG, "null argument") : XR_ERR_ARG;
    batch_drop_graphs(b);
    for (size_t i = 0; i < b->ctx.size(); i++) {
        const xr_status st = xr_dev_session_begin(b->ctx[i], d_sinos[i], d_vols[i], xtt, epochs, subsets, dir, method,
                                                  lambda);
        if (st) return bspec(b, (int)i, st);
    }
    return XR_OK;
}

/* Fork every specimen's stream from the batch stream, enqueue its epoch,
 * join it back. */
static xr_status batch_issue(xr_batch *b, const std::vector<std::vector<int>> &orders) {
    if (cudaEventRecord(b->ev[0], b->stream) != cudaSuccess) return bfail(b, XR_ERR_CUDA, "fork event");
    for (size_t i = 0; i < b->ctx.size(); i++) {
        xr_ctx *c = b->ctx[i];
        if (cudaStreamWaitEvent(c->stream, b->ev[0], 0) != cudaSuccess) return bfail(b, XR_ERR_CUDA, "fork wait");
        const xr_status st = issue_epoch(c, orders[i]);
        if (st) return bspec(b, (int)i, st);
        if (cudaEventRecord(b->ev[i + 1], c->stream) != cudaSuccess ||
            cudaStreamWaitEvent(b->stream, b->ev[i + 1], 0) != cudaSuccess)
            return bfail(b, XR_ERR_CUDA, "join");
    }
    return XR_OK;
}

xr_status xr_batch_epoch(xr_batch *b, double *losses) {
    if (!b) return XR_ERR_ARG;
    cudaSetDevice(b->device);
    const size_t n = b->ctx.size();
    xr_status st;
    bool timing = false;
    for (size_t i = 0; i < n; i++) {
        if ((st = epoch_ready(b->ctx[i]))) return bspec(b, (int)i, st);
        timing = timing || b->ctx[i]->timing.on;
    }
    std::vector<std::vector<int>> orders(n);
    std::vector<int> key;
    for (size_t i = 0; i < n; i++) {
        orders[i] = next_orders(b->ctx[i]);
        key.insert(key.end(), orders[i].begin(), orders[i].end());
        key.push_back(-1);
    }
    if (b->ctx[0]->use_graphs && !timing) {
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess)
                return bfail(b, XR_ERR_CUDA, "begin capture");
            const xr_status ist = batch_issue(b, orders);
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
            if (ist) {
                if (graph) cudaGraphDestroy(graph);
                return ist;
            }
            if (ce != cudaSuccess) return bfail(b, XR_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ce));
            cudaGraphExec_t exec = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ie != cudaSuccess) return bfail(b, XR_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ie));
            it = b->graphs.emplace(key, exec).first;
        }
        if (cudaGraphLaunch(it->second, b->stream) != cudaSuccess) return bfail(b, XR_ERR_CUDA, "graph launch");
    } else {
        if ((st = batch_issue(b, orders))) return st;
    }
    for (size_t i = 0; i < n; i++) b->ctx[i]->sess.epoch_done++;
    if (losses) {
        for (size_t i = 0; i < n; i++)
            if ((st = loss_copy(b->ctx[i], b->stream))) return bspec(b, (int)i, st);
    }
    const cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail(b, XR_ERR_CUDA, std::string("epoch: ") + cudaGetErrorString(e));
    if (losses) {
        double tmp[kMaxCond];
        for (size_t i = 0; i < n; i++) {
            loss_read(b->ctx[i], tmp);
            losses[i] = tmp[0];
        }
    }
    return XR_OK;
}

xr_status xr_batch_session_end(xr_batch *b) {
    if (!b) return XR_ERR_ARG;
    batch_drop_graphs(b);
    xr_status first = XR_OK;
    for (size_t i = 0; i < b->ctx.size(); i++) {
        const xr_status st = xr_dev_session_end(b->ctx[i], nullptr, nullptr);
        if (st && !first) first = bspec(b, (int)i, st);
    }
    return first;
}

xr_status xr_batch_autotune_shapes(xr_batch *b, int *chosen, int *shape) {
    if (!b) return XR_ERR_ARG;
    cudaSetDevice(b->device);
    batch_drop_graphs(b);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return bfail(b, XR_ERR_CUDA, "events");
    }
    xr_status st = XR_OK;
    for (size_t i = 0; i < b->ctx.size() && !st; i++) {
        xr_ctx *c = b->ctx[i];
        Session &s = c->sess;
        if (!s.active || !s.xtt) {
            st = bfail(b, XR_ERR_STATE, "autotune needs an active XTT session on every specimen");
            break;
        }
        drop_graphs(c);
        if ((st = ensure(c, c->scratch_sino, (size_t)c->C * c->V * c->Nd * c->Nd * sizeof(float), "autotune"))) {
            st = bspec(b, (int)i, st);
            break;
        }
        const int ss = s.subset_size;
        std::vector<int> cand = {0, ss, (ss + 1) / 2, (ss + 3) / 4, 8, 4};
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        /* launch shapes worth timing: both when several column axes exist */
        int groups = 0;
        for (int g = 0; g < 3; g++) {
            bool any = false;
            for (int cond = 0; cond < c->C; cond++) any = any || c->axis_g[cond] == g;
            groups += any;
        }
        std::vector<int> shapes = {c->axes_one_launch};
        if (shape && c->all_aligned && groups > 1) shapes = {0, 1};
        const int saved = c->views_per_cta, saved_shape = c->axes_one_launch;
        int best = saved, best_shape = saved_shape;
        float best_ms = 1e30f;
        for (int sh : shapes) {
            c->axes_one_launch = sh;
            for (int v : cand) {
                if (v > 64 || (v > ss && v != 0)) continue;
                c->views_per_cta = v;
                float total = 0.f;
                for (int rep = 0; rep < 3 && !st; rep++) {
                    cudaEventRecord(e0, c->stream);
                    st = cuda_check(c, forward_dispatch(c, (const int *)c->subsets.p, ss, all_conds(c), s.d_vol,
                                                        (float *)c->scratch_sino.p, 1, s.storage),
                                    "autotune forward");
                    cudaEventRecord(e1, c->stream);
                    if (!st) st = cuda_check(c, cudaEventSynchronize(e1), "autotune");
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep > 0) total += ms;   /* first run warms up */
                }
                if (st) break;
                if (total < best_ms) {
                    best_ms = total;
                    best = v;
                    best_shape = sh;
                }
            }
            if (st) break;
        }
        if (st) {
            st = bspec(b, (int)i, st);
            c->views_per_cta = saved;
            c->axes_one_launch = saved_shape;
            break;
        }
        c->views_per_cta = best;
        c->axes_one_launch = best_shape;
        if (chosen) chosen[i] = c->views_per_cta;
        if (shape) shape[i] = c->axes_one_launch;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

xr_status xr_batch_autotune(xr_batch *b, int *chosen) { return xr_batch_autotune_shapes(b, chosen, nullptr); }

}  // extern "C"
