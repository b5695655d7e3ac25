/*
 * The reference's FDK kernels and orientation post-processing compiled for the
 * host (TEST INFRASTRUCTURE ONLY: the checker of the oracle's restatements).
 *
 *   fdk_kernels.inc  reconstruct/src/fdk.cu lines 1-170: calcWeight (:13-26),
 *                    projConv (:28-43), filteredBackProj (:51-60) and its
 *                    backwardonDevice (:62-170).  The file's later lines hold
 *                    the Hilbert variant with a kernel launch (:330), which
 *                    host C++ cannot parse, so oracle/Makefile cuts the slice
 *                    into oracle/_ref/slice at build time.
 *   pca_post.inc     direction/src/pca.cu lines 67-106: calcAngleFromMD and
 *                    directionNormalization (the rest of the file needs Eigen,
 *                    which is absent).
 *
 * The host loop below restates FDK::reconstruct (reconstruct/src/reconstruct.cu:
 * 1651-1724) around the reference's own kernels: the Shepp-Logan-type filter
 * table of :1692-1698, per axis and view the row convolution into the filtered
 * block, then the back-projection of every y slab from the filtered sinogram
 * passed without the axis offset (:1708), into channel `cond` (fdk.cu:163).
 * devSinoFilt and devVoxel start at zero (the reference never clears the
 * former, :1669).  The globals (elemR, elemT, INIT_OFFSET, sizes) are the ones
 * xr_ref_setup sets.
 */
#include "cuda_runtime.h"
#include "params.h"

#include <vector>

#include "fdk_kernels.inc"

#include <volume.h>
#include <cmath>
#include "pca_post.inc"

namespace {

/* Every (block, thread) of a 2-D grid as a plain call.  The FDK kernels write
 * one output element per thread without atomics, so rows may run in parallel
 * and the result is the serial one. */
template <class F, class... A>
void launch_rows(dim3 grid, dim3 block, F kernel, A... args) {
    const long rows = (long)grid.y * block.y;
#pragma omp parallel for schedule(dynamic, 4)
    for (long r = 0; r < rows; ++r) {
        gridDim = grid;
        blockDim = block;
        const unsigned by = (unsigned)(r / block.y), ty = (unsigned)(r % block.y);
        for (unsigned bx = 0; bx < grid.x; ++bx)
            for (unsigned tx = 0; tx < block.x; ++tx) {
                blockIdx = uint3{bx, by, 0};
                threadIdx = uint3{tx, ty, 0};
                kernel(args...);
            }
    }
}

Geometry current_geometry() {
    return Geometry(SRC_DETECT_DISTANCE, SRC_OBJ_DISTANCE, DETECTOR_SIZE, NUM_VOXEL, NUM_DETECT_U, NUM_PROJ);
}

}  // namespace

extern "C" {

/* calcWeight (fdk.cu:13-26) into w (Nd*Nd). */
void xr_ref_fdk_weight(float *w) {
    Geometry geom = current_geometry();
    const int bs = BLOCK_SIZE;
    const dim3 blockD(bs, bs, 1), gridD((geom.detect + bs - 1) / bs, (geom.detect + bs - 1) / bs, 1);
    launch_rows(gridD, blockD, calcWeight, w, (const Geometry *)&geom);
}

/* The host filter table of FDK::reconstruct (reconstruct.cu:1692-1698). */
void xr_ref_fdk_filter(float *filt) {
    Geometry geom = current_geometry();
    float d = geom.detSize * (geom.sod / geom.sdd);
    for (int v = 0; v < geom.detect; v++) filt[v] = 1.0f / (float)(M_PI * M_PI * d * (1.0f - 4.0f * (float)(v * v)));
}

/* FDK::reconstruct (reconstruct.cu:1651-1724) on one scan: sino (C blocks of
 * V*Nd*Nd) in, vol (C channels of N^3) and the filtered sinograms filt_out (C
 * blocks) out. */
void xr_ref_fdk_reconstruct(const float *sino, float *vol, float *filt_out, int rotate_ccw) {
    Geometry geom = current_geometry();
    const int C = NUM_PROJ_COND;
    const long lenV = (long)geom.voxel * geom.voxel * geom.voxel;
    const long lenD = (long)geom.detect * geom.detect * geom.nProj;
    const int rotation = rotate_ccw ? -1 : 1;
    std::vector<float> devSino(sino, sino + lenD * C), devSinoFilt(lenD * C, 0.0f), weight((size_t)geom.detect * geom.detect);
    std::vector<float> filt(geom.detect);
    std::fill(vol, vol + lenV * C, 0.0f);
    const int bs = BLOCK_SIZE;
    const dim3 blockV(bs, bs, 1), gridV((geom.voxel + bs - 1) / bs, (geom.voxel + bs - 1) / bs, 1);
    const dim3 blockD(bs, bs, 1), gridD((geom.detect + bs - 1) / bs, (geom.detect + bs - 1) / bs, 1);
    launch_rows(gridD, blockD, calcWeight, weight.data(), (const Geometry *)&geom);
    xr_ref_fdk_filter(filt.data());
    for (int cond = 0; cond < C; cond++)
        for (int n = 0; n < geom.nProj; n++) {
            launch_rows(gridD, blockD, projConv, &devSinoFilt[lenD * cond], (const float *)&devSino[lenD * cond],
                        (const Geometry *)&geom, n, (const float *)filt.data(), (const float *)weight.data());
            for (int y = 0; y < geom.voxel; y++)
                launch_rows(gridV, blockV, filteredBackProj, devSinoFilt.data(), vol, &geom, cond, y, rotation * n);
        }
    std::copy(devSinoFilt.begin(), devSinoFilt.end(), filt_out);
}

/* calcAngleFromMD (pca.cu:67-83) on planes of nx*ny*nz floats (x fastest). */
void xr_ref_angle_from_md(const float *md, float *angle, int nx, int ny, int nz) {
    const long n = (long)nx * ny * nz;
    Volume<float> m[3] = {Volume<float>(nx, ny, nz), Volume<float>(nx, ny, nz), Volume<float>(nx, ny, nz)};
    Volume<float> a[2] = {Volume<float>(nx, ny, nz), Volume<float>(nx, ny, nz)};
    for (int i = 0; i < 3; i++) std::copy(md + i * n, md + (i + 1) * n, m[i].get());
    calcAngleFromMD(m, a, nx, ny, nz);
    for (int i = 0; i < 2; i++) std::copy(a[i].get(), a[i].get() + n, angle + i * n);
}

/* directionNormalization (pca.cu:85-106), in place. */
void xr_ref_direction_normalization(float *md, int nx, int ny, int nz) {
    const long n = (long)nx * ny * nz;
    Volume<float> m[3] = {Volume<float>(nx, ny, nz), Volume<float>(nx, ny, nz), Volume<float>(nx, ny, nz)};
    for (int i = 0; i < 3; i++) std::copy(md + i * n, md + (i + 1) * n, m[i].get());
    directionNormalization(m);
    for (int i = 0; i < 3; i++) std::copy(m[i].get(), m[i].get() + n, md + i * n);
}

}  // extern "C"
