/*
 * xr_dev_forward_proj_only_static: the raw forward splat (forwardProjOnly
 * semantics) for callers that cannot allocate device memory — code whose
 * device memory all belongs to another allocator (a framework's caching pool
 * that must see every byte), or a steady-state loop that is not allowed to
 * allocate.  The regular entry points allocate their per-view tables and
 * workspace with cudaMalloc on first use; this one keeps its only scratch —
 * the per-(axis, view) geometry table, the view list and one flag word — in
 * the fixed array below, so it calls no cudaMalloc, cudaFree or other
 * allocating routine.
 *
 * Scratch: kStaticPairs (axis, view) pairs, i.e. num_cond * num_proj <= 4096
 * (4096 * 80 B of frames + 4096 ints + one flag word, about 344 KB).  Every
 * GPU that loads libxr holds this array until the process exits.  All calls
 * share it and it keeps the last call's contents; calls whose work overlaps
 * on the GPU (for instance on two streams at once) race on it and must be
 * serialised by the caller.  The first call on a device resolves the array's
 * device address with cudaGetSymbolAddress (with that device current).  The
 * frames are copied from host stack memory, so no call may be made while its
 * stream is being captured into a CUDA graph: such a call is refused.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "xr_internal.h"

namespace xr {
namespace {

constexpr int kStaticPairs = 4096;
constexpr int kStaticDevices = 64;

struct StaticScratch {
    ViewFrame frames[kStaticPairs];
    int views[kStaticPairs];
    unsigned div_flag;   /* mismatch count of the division check (k_check_div) */
};

/* The fixed scratch.  In host code this name is only a stand-in for the
 * symbol, not a device address: host code passes the address that
 * cudaGetSymbolAddress returns. */
static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

std::mutex g_static_mu;
void *g_static_addr[kStaticDevices] = {};  /* per device ordinal */

/* views[i] = i: the view list of a whole scan, written on the device. */
__global__ void k_identity(int *views, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) views[i] = i;
}

/* Makes the context's device current and gives the caller's current device
 * back on every return. */
struct DeviceScope {
    int prev = -1;
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

/* The per-view frame of rayCasting (ir.cu:1860-1879), computed by the host
 * library code (xr_host.cpp, built with -ffp-contract=off) so the table is
 * bit-identical to the regular entry points'. */
ViewFrame host_view_frame(const xr_ctx *c, int cond, int n, bool fdk);

}  // namespace xr

using namespace xr;

extern "C" xr_status xr_dev_forward_proj_only_static(xr_ctx *c, const float *d_vol, float *d_sino, xr_rotate dir,
                                                     void *stream) {
    if (!c) return XR_ERR_ARG;
    if (!d_vol || !d_sino) return fail(c, XR_ERR_ARG, "xr_dev_forward_proj_only_static: null device buffer");
    if (dir != XR_ROTATE_CW && dir != XR_ROTATE_CCW) return fail(c, XR_ERR_ARG, "bad rotate");
    const long pairs = (long)c->C * c->V;
    if (pairs > kStaticPairs)
        return fail(c, XR_ERR_ARG,
                    "xr_dev_forward_proj_only_static: num_cond * num_proj = " + std::to_string(pairs) +
                        " exceeds the fixed scratch of " + std::to_string(kStaticPairs) + " (axis, view) pairs");
    if (c->device < 0 || c->device >= kStaticDevices) return fail(c, XR_ERR_ARG, "device ordinal out of range");
    /* The device check of the regular entry points, from device attributes
     * alone (no allocation): an sm_100 device or XR_ERR_NODEV. */
    int count = 0, major = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || c->device >= count ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c->device) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, XR_ERR_NODEV, "no CUDA device available (libxr needs a B200, sm_100a)");
    }
    if (major != 10)
        return fail(c, XR_ERR_NODEV, "libxr is built for sm_100a; device " + std::to_string(c->device) +
                                         " has compute capability " + std::to_string(major) + ".x");
    DeviceScope scope;
    xr_status st = cuda_check(c, cudaGetDevice(&scope.prev), "cudaGetDevice");
    if (st) return st;
    if ((st = cuda_check(c, cudaSetDevice(c->device), "cudaSetDevice"))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if ((st = cuda_check(c, cudaStreamIsCapturing(s, &cap), "cudaStreamIsCapturing"))) return st;
    if (cap != cudaStreamCaptureStatusNone)
        return fail(c, XR_ERR_ARG,
                    "xr_dev_forward_proj_only_static cannot be captured into a CUDA graph: it copies its geometry "
                    "table from host stack memory on every call");
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_addr[c->device]) {
            void *p = nullptr;
            st = cuda_check(c, cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress(static scratch)");
            if (st) return st;
            g_static_addr[c->device] = p;
        }
        base = g_static_addr[c->device];
    }
    StaticScratch *dev = (StaticScratch *)base;
    const int rotation = dir == XR_ROTATE_CCW ? -1 : 1;

    /* Division by the detector pitch as a corrected product only where it
     * equals IEEE division bit for bit on this device: the check of the
     * regular entry points, run once per context on a context they have not
     * set up, with the flag word in the fixed scratch. */
    GeomConst gc = c->gc;
    if (!c->dev_ready) {
        if (c->static_rdet < 0) {
            unsigned bad = 1;
            st = cuda_check(c, check_exact_rdet(c->det, gc.rdet, &dev->div_flag, &bad, s), "division check");
            if (st) return st;
            c->static_rdet = (bad == 0) ? 1 : 0;
        }
        gc.exact_rdet = c->static_rdet;
    }

    /* The frames go through a stack buffer; every entry of the used part of
     * the scratch is rewritten, so nothing needs clearing.  (cudaMemcpyAsync
     * from pageable memory returns once the source has been staged, so the
     * buffer can be reused at once.) */
    constexpr int kChunk = 256;
    ViewFrame hf[kChunk];
    for (long i0 = 0; i0 < pairs; i0 += kChunk) {
        const int n = (int)std::min<long>(kChunk, pairs - i0);
        for (int j = 0; j < n; j++) {
            const long i = i0 + j;
            const int cond = (int)(i / c->V), v = (int)(i % c->V);
            hf[j] = host_view_frame(c, cond, rotation * v, false);
        }
        st = cuda_check(c, cudaMemcpyAsync(&dev->frames[i0], hf, n * sizeof(ViewFrame), cudaMemcpyHostToDevice, s),
                        "frames to static scratch");
        if (st) return st;
    }
    k_identity<<<(c->V + 255) / 256, 256, 0, s>>>(dev->views, c->V);
    if ((st = cuda_check(c, cudaGetLastError(), "view list"))) return st;
    /* The output accumulates the splat: it must start at zero. */
    const size_t npx = (size_t)c->C * c->V * c->Nd * c->Nd;
    st = cuda_check(c, cudaMemsetAsync(d_sino, 0, npx * sizeof(float), s), "clear output");
    if (st) return st;
    return cuda_check(c, launch_forward(gc, nullptr, dev->frames, dev->views, c->V, 0, c->C, d_vol, d_sino, 0,
                                        c->views_per_cta, 0, s),
                      "static forward splat");
}
