/*
 * xr_dev_forward_proj_only_static: the raw forward splat (forwardProjOnly
 * semantics) for callers that cannot allocate device memory — code whose
 * device memory all belongs to another allocator (a framework's caching pool
 * that must see every byte), or a steady-state loop that is not allowed to
 * allocate.  The regular entry points allocate their per-view tables and
 * workspace with cudaMalloc on first use; this one keeps its only scratch —
 * the per-(axis, view) geometry table and the view list — in the fixed array
 * below, so it calls no cudaMalloc, cudaFree or other allocating routine.
 *
 * Scratch: kStaticPairs (axis, view) pairs, i.e. num_cond * num_proj <= 4096
 * (4096 * 80 B of frames + 4096 ints = 344 KB).  Every GPU that loads libxr
 * holds this array until the process exits.  All calls share it and it keeps
 * the last call's contents; calls whose work overlaps on the GPU (for
 * instance on two streams at once) race on it and must be serialised by the
 * caller.  The first call on a device resolves the array's device address
 * with cudaGetSymbolAddress (with that device current); make that first call
 * before any stream capture.
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
};

/* The fixed scratch.  In host code this name is only a stand-in for the
 * symbol, not a device address: host code passes the address that
 * cudaGetSymbolAddress returns. */
static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

std::mutex g_static_mu;
void *g_static_addr[kStaticDevices] = {};  /* per device ordinal */

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
    xr_status st = cuda_check(c, cudaSetDevice(c->device), "cudaSetDevice");
    if (st) return st;
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
    cudaStream_t s = (cudaStream_t)stream;
    StaticScratch *dev = (StaticScratch *)base;
    const int rotation = dir == XR_ROTATE_CCW ? -1 : 1;

    /* Frames and the view list go through a small stack buffer: every entry
     * of the used part of the scratch is rewritten, so nothing needs
     * clearing.  (cudaMemcpyAsync from pageable memory returns once the
     * source has been staged, so the buffer can be reused at once.) */
    constexpr int kChunk = 32;
    ViewFrame hf[kChunk];
    int hv[kChunk];
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
    for (long i0 = 0; i0 < c->V; i0 += kChunk) {
        const int n = (int)std::min<long>(kChunk, c->V - i0);
        for (int j = 0; j < n; j++) hv[j] = (int)(i0 + j);
        st = cuda_check(c, cudaMemcpyAsync(&dev->views[i0], hv, n * sizeof(int), cudaMemcpyHostToDevice, s),
                        "views to static scratch");
        if (st) return st;
    }
    /* The output accumulates the splat: it must start at zero. */
    const size_t npx = (size_t)c->C * c->V * c->Nd * c->Nd;
    st = cuda_check(c, cudaMemsetAsync(d_sino, 0, npx * sizeof(float), s), "clear output");
    if (st) return st;
    return cuda_check(c, launch_forward(c->gc, nullptr, dev->frames, dev->views, c->V, 0, c->C, d_vol, d_sino, 0,
                                        c->views_per_cta, 0, s),
                      "static forward splat");
}
