/*
 * Host driver for the reference's own projector kernels (reconstruct/src/ir.cu),
 * compiled for the CPU through the CUDA shim in this folder.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  The
 * kernels are the reference's, compiled from its source tree in place; the
 * host loops below restate the reference's schedulers:
 *   ref_ir_reconstruct   <- IR::reconstruct   reconstruct/src/reconstruct.cu:23-156
 *   ref_xtt_reconstruct  <- XTT::reconstruct  reconstruct/src/reconstruct.cu:799-927
 *                           (the Eigen orientation step :929-942 is not built:
 *                            Eigen is absent; the oracle's Jacobi replaces it)
 *   ref_fiber_reconstruct <- XTT::fiberModelReconstruct  reconstruct.cu:1242-1371
 *                           (its ratio launches pass a null loss pointer, :1318-1322,
 *                            which projRatio's atomicAdd dereferences, ir.cu:1623:
 *                            the restatement passes a local float instead)
 *   ref_forward_view     <- the forward half of one view of those loops
 *                           (reconstruct.cu:86-98 / :866-878)
 * A "launch" runs every (block, thread) of the grid as a plain call, serially in
 * z-major, x-minor order (deterministic float sums), or under OpenMP with CAS
 * float atomics when xr_ref_set_parallel(1) was called.
 */
#include "cuda_runtime.h"
#include "params.h"
#include <geometry.h>
#include <ir.cuh>
#include <fiber.cuh>

#include <algorithm>
#include <random>
#include <vector>
#include <omp.h>

namespace {

template <class F, class... A>
void launch2d(dim3 grid, dim3 block, F kernel, A... args) {
    if (!xr_shim_parallel) {
        gridDim = grid;
        blockDim = block;
        for (unsigned by = 0; by < grid.y; ++by)
            for (unsigned ty = 0; ty < block.y; ++ty)
                for (unsigned bx = 0; bx < grid.x; ++bx)
                    for (unsigned tx = 0; tx < block.x; ++tx) {
                        blockIdx = uint3{bx, by, 0};
                        threadIdx = uint3{tx, ty, 0};
                        kernel(args...);
                    }
        return;
    }
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

struct Ctx {
    Geometry geom{1.f, 1.f, 1.f, 1, 1, 1};
    int C = 1, K = 1;
    dim3 blockV, gridV, blockD, gridD;
};
Ctx g;

}  // namespace

extern "C" {

/* Mirrors init_params (params.cu:42-104) for an already-parsed scan: sets the
 * globals the kernels read.  trans must already include areaTrans. */
void xr_ref_setup(float sdd, float sod, float det, int N, int Nd, int V, int C, int K,
                  const float *rot, const float *trans, const float *offset, const float *basis) {
    g.geom = Geometry(sdd, sod, det, N, Nd, V);
    g.C = C;
    g.K = K;
    NUM_PROJ_COND = C;
    NUM_BASIS_VECTOR = K;
    SRC_DETECT_DISTANCE = sdd;
    SRC_OBJ_DISTANCE = sod;
    DETECTOR_SIZE = det;
    NUM_VOXEL = N;
    NUM_DETECT_U = NUM_DETECT_V = Nd;
    NUM_PROJ = V;
    std::memcpy(elemR, rot, sizeof(float) * 9 * C);
    std::memcpy(elemT, trans, sizeof(float) * 3 * C);
    std::memcpy(INIT_OFFSET, offset, sizeof(float) * 3 * C);
    std::memcpy(basisVector, basis, sizeof(float) * 3 * K);
    const int bs = BLOCK_SIZE;
    g.blockV = dim3(bs, bs, 1);
    g.gridV = dim3((N + bs - 1) / bs, (N + bs - 1) / bs, 1);
    g.blockD = dim3(bs, bs, 1);
    g.gridD = dim3((Nd + bs - 1) / bs, (Nd + bs - 1) / bs, 1);
}

void xr_ref_set_parallel(int on) { xr_shim_parallel = on; }

float xr_ref_vox_size(void) { return g.geom.voxSize; }

/* One view of the forward: all y slabs of forwardProj / forwardProjXTT
 * (reconstruct.cu:94-97 / :872-877) into proj (C-block base, all views) and
 * the per-view weight image factor (zeroed here, as reconstruct.cu:88/:866). */
void xr_ref_forward_view(int cond, int n, float *vol, float *proj, float *factor, int xtt) {
    Geometry *geom = &g.geom;
    const long Nd = geom->detect;
    std::memset(factor, 0, sizeof(float) * Nd * Nd);
    for (int y = 0; y < geom->voxel; y++) {
        if (xtt)
            launch2d(g.gridV, g.blockV, forwardProjXTT, proj, factor, vol, geom, cond, y, n);
        else
            launch2d(g.gridV, g.blockV, forwardProj, proj, vol, factor, geom, y, n, cond);
    }
}

/* forwardOrth (ir.cu:294-364): one view, every y slab, basis rotated per voxel
 * by the coefficient planes (phi, cos theta); no weight image. */
void xr_ref_forward_orth(int cond, int n, float *vol, const float *coef, float *proj) {
    Geometry *geom = &g.geom;
    for (int y = 0; y < geom->voxel; y++)
        launch2d(g.gridV, g.blockV, forwardOrth, proj, (const float *)vol, coef, cond, y, n, 0, geom);
}

/* backwardOrth (ir.cu:366-423): slab y, view n; tmp / factor K planes of N*N. */
void xr_ref_backward_orth(int cond, int y, int n, const float *proj, const float *coef, float *tmp, float *factor) {
    launch2d(g.gridV, g.blockV, backwardOrth, proj, coef, tmp, factor, (const Geometry *)&g.geom, cond, y, n, 0);
}

/* calcNormalVectorThreeDirec (ir.cu:856-974), every y slab. */
void xr_ref_normal_three(float *vol, float *coef, float *loss, int rot) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, calcNormalVectorThreeDirec, vol, coef, y, (const Geometry *)&g.geom, loss, rot);
}

/* forwardOrthByMD (ir.cu:154-231): one view, every y slab, basis rotated per
 * voxel by its main direction; the weight image factor is zeroed here first
 * (reconstruct.cu:1494). */
void xr_ref_forward_md(int cond, int n, float *vol, const float *md, float *proj, float *factor) {
    Geometry *geom = &g.geom;
    std::memset(factor, 0, sizeof(float) * geom->detect * geom->detect);
    for (int y = 0; y < geom->voxel; y++)
        launch2d(g.gridV, g.blockV, forwardOrthByMD, proj, factor, (const float *)vol, md, geom, cond, 0, n, y);
}

/* backwardOrthByMD (ir.cu:233-292): slab y, view n. */
void xr_ref_backward_md(int cond, int y, int n, const float *proj, const float *md, float *tmp, float *factor) {
    launch2d(g.gridV, g.blockV, backwardOrthByMD, proj, md, tmp, factor, (const Geometry *)&g.geom, cond, y, n, 0);
}

/* meanFiltFiberMD (ir.cu:1304-1363), slab y into out. */
void xr_ref_md_filter(int y, const float *md, float *out, float coef) {
    launch2d(g.gridV, g.blockV, meanFiltFiberMD, md, out, (const Geometry *)&g.geom, y, coef);
}

/* calcMainDirection (ir.cu:624-710), every y slab; loss is the unused
 * norm_loss argument (N^3 floats). */
void xr_ref_main_direction(float *vol, float *md, float *loss, int iter) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, calcMainDirection, vol, md, y, (const Geometry *)&g.geom, loss, iter);
}

/* calcMDWithEst (ir.cu:712-789), every y slab. */
void xr_ref_md_with_estimate(float *vol, float *md, const float *est) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, calcMDWithEst, vol, md, y, (const Geometry *)&g.geom, est);
}

/* updateEstimation (ir.cu:791-844), every y slab. */
void xr_ref_update_estimation(const float *vol, float *md, float *loss, float *est, int iter) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, updateEstimation, vol, md, y, (const Geometry *)&g.geom, loss, est, iter);
}

/* calcNormalVectorThreeDirecWithEst (ir.cu:976-1071), every y slab. */
void xr_ref_normal_three_est(float *vol, float *coef, float *loss, const float *est) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, calcNormalVectorThreeDirecWithEst, vol, coef, y, (const Geometry *)&g.geom, loss,
                 est);
}

/* meanFiltFiber (ir.cu:1231-1302), slab y: coef -> out. */
void xr_ref_coef_filter(int y, const float *coef, float *out, const float *vol, float w) {
    launch2d(g.gridV, g.blockV, meanFiltFiber, coef, out, vol, (const Geometry *)&g.geom, y, w);
}

/* updateEstimationByCoef (ir.cu:1073-1120), every y slab. */
void xr_ref_update_estimation_coef(const float *vol, float *loss, float *est, int iter) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, updateEstimationByCoef, vol, y, (const Geometry *)&g.geom, loss, est, iter);
}

/* forwardProjFiber (fiber.cu:80-153): one view, every y slab. */
void xr_ref_fiber_forward(int cond, int n, float *vol, float *proj) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, forwardProjFiber, proj, vol, &g.geom, cond, y, n);
}

/* backwardProjFiber (fiber.cu:217-226): slab y, view n. */
void xr_ref_fiber_backward(int cond, int y, int n, float *proj, float *vol, float *tmp, float *factor) {
    launch2d(g.gridV, g.blockV, backwardProjFiber, proj, vol, tmp, factor, &g.geom, cond, y, n);
}

void xr_ref_correlation(int cond, int n, float *proj, const float *factor) {
    launch2d(g.gridD, g.blockD, correlationProjByLength, proj, factor, &g.geom, cond, n);
}

/* projRatio / projSubtract (ir.cu:1616-1666); returns the float loss sum. */
float xr_ref_ratio(int n, float *proj, const float *sino, int art) {
    float loss = 0.0f;
    if (art)
        launch2d(g.gridD, g.blockD, projSubtract, proj, sino, (const Geometry *)&g.geom, n, &loss);
    else
        launch2d(g.gridD, g.blockD, projRatio, proj, sino, (const Geometry *)&g.geom, n, &loss);
    return loss;
}

/* One launch of backwardProj / backwardProjXTT (ir.cu:1605-1614 / :143-152). */
void xr_ref_backward_slab(int cond, int y, int n, float *proj, float *tmp, float *factor, int xtt) {
    if (xtt)
        launch2d(g.gridV, g.blockV, backwardProjXTT, proj, tmp, factor, &g.geom, cond, y, n);
    else
        launch2d(g.gridV, g.blockV, backwardProj, proj, tmp, factor, &g.geom, cond, y, n);
}

void xr_ref_voxel_product(int y, float *vol, const float *tmp, const float *factor) {
    launch2d(g.gridV, g.blockV, voxelProduct, vol, tmp, factor, (const Geometry *)&g.geom, y);
}

void xr_ref_voxel_plus(int y, float *vol, const float *tmp, float alpha) {
    launch2d(g.gridV, g.blockV, voxelPlus, vol, tmp, alpha, (const Geometry *)&g.geom, y);
}

void xr_ref_voxel_sqrt(float *vol) {
    for (int y = 0; y < g.geom.voxel; y++)
        launch2d(g.gridV, g.blockV, voxelSqrt, vol, (const Geometry *)&g.geom, y);
}

/* The normalised forward operator of the reconstruction loops (forward +
 * correlationProjByLength for every axis and view, no ratio): the "A" of the
 * data residual.  vol holds K channels; proj holds C blocks of V views. */
void xr_ref_forward_all(float *vol, float *proj, int rotate_ccw, int xtt) {
    const long Nd = g.geom.detect, V = g.geom.nProj;
    const long lenD = Nd * Nd * V;
    const int rotation = rotate_ccw ? -1 : 1;
    std::vector<float> factor(Nd * Nd);
    std::memset(proj, 0, sizeof(float) * lenD * g.C);
    for (int cond = 0; cond < g.C; cond++)
        for (int v = 0; v < V; v++) {
            const int n = rotation * v;
            xr_ref_forward_view(cond, n, vol, proj + lenD * cond, factor.data(), xtt);
            xr_ref_correlation(cond, n, proj + lenD * cond, factor.data());
        }
}

/* IR::reconstruct, reconstruct.cu:23-156.  sino[C] and vol[C] are host volumes
 * (the reference's Volume<float>::get()); losses[epoch] receives the raw float
 * loss sum of the last axis, as the reference's `losses` vector does. */
void xr_ref_ir_reconstruct(float **sino, float **vol, int epoch, int batch, int rotate_ccw,
                           int art, float lambda, float *losses) {
    Geometry *geom = &g.geom;
    const int rotation = rotate_ccw ? -1 : 1;
    const long N = geom->voxel, Nd = geom->detect, nProj = geom->nProj;
    const long lenV = N * N * N, lenD = Nd * Nd * nProj;
    std::vector<float> devSino(lenD), devProj(lenD), devProjFactor(Nd * Nd), devVoxel(lenV),
        devVoxelFactor(N * N), devVoxelTmp(N * N);
    const int subsetSize = (int)((nProj + batch - 1) / batch);
    std::vector<int> subsetOrder(batch);
    for (int i = 0; i < batch; i++) subsetOrder[i] = i;
    std::mt19937_64 get_rand_mt;
    for (int cond = 0; cond < g.C; cond++) {
        std::memcpy(devVoxel.data(), vol[cond], sizeof(float) * lenV);
        std::memcpy(devSino.data(), sino[cond], sizeof(float) * lenD);
        for (int ep = 0; ep < epoch; ep++) {
            std::shuffle(subsetOrder.begin(), subsetOrder.end(), get_rand_mt);
            float loss1 = 0.0f;
            std::fill(devProj.begin(), devProj.end(), 0.0f);
            for (int &sub : subsetOrder) {
                for (int subOrder = 0; subOrder < subsetSize; subOrder++) {
                    std::fill(devProjFactor.begin(), devProjFactor.end(), 0.0f);
                    int n = rotation * (int)((sub + batch * subOrder) % nProj);
                    for (int y = 0; y < N; y++)
                        launch2d(g.gridV, g.blockV, forwardProj, devProj.data(), devVoxel.data(),
                                 devProjFactor.data(), geom, y, n, cond);
                    launch2d(g.gridD, g.blockD, correlationProjByLength, devProj.data(),
                             (const float *)devProjFactor.data(), geom, cond, n);
                    if (art)
                        launch2d(g.gridD, g.blockD, projSubtract, devProj.data(),
                                 (const float *)devSino.data(), (const Geometry *)geom, n, &loss1);
                    else
                        launch2d(g.gridD, g.blockD, projRatio, devProj.data(),
                                 (const float *)devSino.data(), (const Geometry *)geom, n, &loss1);
                }
                for (int y = 0; y < N; y++) {
                    std::fill(devVoxelFactor.begin(), devVoxelFactor.end(), 0.0f);
                    std::fill(devVoxelTmp.begin(), devVoxelTmp.end(), 0.0f);
                    for (int subOrder = 0; subOrder < subsetSize; subOrder++) {
                        int n = rotation * (int)((sub + batch * subOrder) % nProj);
                        launch2d(g.gridV, g.blockV, backwardProj, devProj.data(), devVoxelTmp.data(),
                                 devVoxelFactor.data(), geom, cond, y, n);
                    }
                    if (art)
                        launch2d(g.gridV, g.blockV, voxelPlus, devVoxel.data(),
                                 (const float *)devVoxelTmp.data(), lambda / (float)subsetSize,
                                 (const Geometry *)geom, y);
                    else
                        launch2d(g.gridV, g.blockV, voxelProduct, devVoxel.data(),
                                 (const float *)devVoxelTmp.data(), (const float *)devVoxelFactor.data(),
                                 (const Geometry *)geom, y);
                }
            }
            if (losses) losses[ep] = loss1;
        }
        std::memcpy(vol[cond], devVoxel.data(), sizeof(float) * lenV);
    }
}

/* XTT::reconstruct, reconstruct.cu:799-927 (up to the copies back; the
 * orientation step is left to the caller).  sino[C] is overwritten with the
 * last ratio images, as the reference does (:924-925). */
void xr_ref_xtt_reconstruct(float **sino, float **vol, int epoch, int batch, int rotate_ccw,
                            int art, float lambda, float *losses) {
    Geometry *geom = &g.geom;
    const int rotation = rotate_ccw ? -1 : 1;
    const long N = geom->voxel, Nd = geom->detect;
    const int nProj = geom->nProj;
    const long lenV = N * N * N, lenD = Nd * Nd * (long)nProj, lenP = N * N;
    const int C = g.C, K = g.K;
    std::vector<float> devSino(lenD * C), devProj(lenD * C), devProjFactor(Nd * Nd),
        devVoxel(lenV * K), devVoxelFactor(lenP * K), devVoxelTmp(lenP * K);
    for (int i = 0; i < C; i++) std::memcpy(&devSino[i * lenD], sino[i], sizeof(float) * lenD);
    for (int i = 0; i < K; i++) std::memcpy(&devVoxel[i * lenV], vol[i], sizeof(float) * lenV);
    const int subsetSize = (nProj + batch - 1) / batch;
    std::vector<int> subsetOrder(batch);
    for (int i = 0; i < batch; i++) subsetOrder[i] = i;
    for (int ep = 0; ep < epoch; ep++) {
        std::mt19937_64 get_rand_mt;
        std::shuffle(subsetOrder.begin(), subsetOrder.end(), get_rand_mt);
        float loss1 = 0.0f;
        std::fill(devProj.begin(), devProj.end(), 0.0f);
        for (int &sub : subsetOrder) {
            for (int cond = 0; cond < C; cond++) {
                for (int subOrder = 0; subOrder < subsetSize; subOrder++) {
                    std::fill(devProjFactor.begin(), devProjFactor.end(), 0.0f);
                    int n = rotation * ((sub + batch * subOrder) % nProj);
                    for (int y = 0; y < N; y++)
                        launch2d(g.gridV, g.blockV, forwardProjXTT, &devProj[lenD * cond],
                                 devProjFactor.data(), devVoxel.data(), geom, cond, y, n);
                    launch2d(g.gridD, g.blockD, correlationProjByLength, &devProj[lenD * cond],
                             (const float *)devProjFactor.data(), geom, cond, n);
                    if (art)
                        launch2d(g.gridD, g.blockD, projSubtract, &devProj[lenD * cond],
                                 (const float *)&devSino[lenD * cond], (const Geometry *)geom, n, &loss1);
                    else
                        launch2d(g.gridD, g.blockD, projRatio, &devProj[lenD * cond],
                                 (const float *)&devSino[lenD * cond], (const Geometry *)geom, n, &loss1);
                }
            }
            for (int y = 0; y < N; y++) {
                std::fill(devVoxelFactor.begin(), devVoxelFactor.end(), 0.0f);
                std::fill(devVoxelTmp.begin(), devVoxelTmp.end(), 0.0f);
                for (int cond = 0; cond < C; cond++)
                    for (int subOrder = 0; subOrder < subsetSize; subOrder++) {
                        int n = rotation * ((sub + batch * subOrder) % nProj);
                        launch2d(g.gridV, g.blockV, backwardProjXTT, &devProj[lenD * cond],
                                 devVoxelTmp.data(), devVoxelFactor.data(), geom, cond, y, n);
                    }
                for (int vec = 0; vec < K; vec++) {
                    if (art)
                        launch2d(g.gridV, g.blockV, voxelPlus, &devVoxel[lenV * vec],
                                 (const float *)&devVoxelTmp[lenP * vec], lambda / (float)subsetSize,
                                 (const Geometry *)geom, y);
                    else
                        launch2d(g.gridV, g.blockV, voxelProduct, &devVoxel[lenV * vec],
                                 (const float *)&devVoxelTmp[lenP * vec],
                                 (const float *)&devVoxelFactor[lenP * vec], (const Geometry *)geom, y);
                }
            }
        }
        if (losses) losses[ep] = loss1;
    }
    for (int y = 0; y < N; y++)
        launch2d(g.gridV, g.blockV, voxelSqrt, devVoxel.data(), (const Geometry *)geom, y);
    for (int i = 0; i < C; i++) std::memcpy(sino[i], &devProj[i * lenD], sizeof(float) * lenD);
    for (int i = 0; i < K; i++) std::memcpy(vol[i], &devVoxel[i * lenV], sizeof(float) * lenV);
}

/* XTT::fiberModelReconstruct (reconstruct.cu:1242-1371): the caller's
 * volume is the start (the reference sets every channel to 0.01 first,
 * :1245-1247); per subset forwardProjFiber + projRatio / projSubtract over
 * every axis, then per slab backwardProjFiber over every axis and view and
 * voxelProduct / voxelPlus of channel 0 (the first N^3 of devVoxel,
 * :1341-1345).  sino[C] receives devProj (:1355-1356). */
void xr_ref_fiber_reconstruct(float **sino, float **vol, int epoch, int batch, int rotate_ccw, int art,
                              float lambda, float *losses) {
    Geometry *geom = &g.geom;
    const int rotation = rotate_ccw ? -1 : 1;
    const long N = geom->voxel, Nd = geom->detect;
    const int nProj = geom->nProj;
    const long lenV = N * N * N, lenD = Nd * Nd * (long)nProj, lenP = N * N;
    const int C = g.C, K = g.K;
    std::vector<float> devSino(lenD * C), devProj(lenD * C), devVoxel(lenV * K), devVoxelFactor(lenP * K),
        devVoxelTmp(lenP * K);
    for (int i = 0; i < C; i++) std::memcpy(&devSino[i * lenD], sino[i], sizeof(float) * lenD);
    for (int i = 0; i < K; i++) std::memcpy(&devVoxel[i * lenV], vol[i], sizeof(float) * lenV);
    const int subsetSize = (nProj + batch - 1) / batch;
    std::vector<int> subsetOrder(batch);
    for (int i = 0; i < batch; i++) subsetOrder[i] = i;
    for (int ep = 0; ep < epoch; ep++) {
        std::mt19937_64 get_rand_mt;
        std::shuffle(subsetOrder.begin(), subsetOrder.end(), get_rand_mt);
        float loss1 = 0.0f;
        std::fill(devProj.begin(), devProj.end(), 0.0f);
        for (int &sub : subsetOrder) {
            for (int cond = 0; cond < C; cond++) {
                for (int subOrder = 0; subOrder < subsetSize; subOrder++) {
                    int n = rotation * ((sub + batch * subOrder) % nProj);
                    for (int y = 0; y < N; y++)
                        launch2d(g.gridV, g.blockV, forwardProjFiber, &devProj[lenD * cond], devVoxel.data(), geom,
                                 cond, y, n);
                    if (art)
                        launch2d(g.gridD, g.blockD, projSubtract, &devProj[lenD * cond],
                                 (const float *)&devSino[lenD * cond], (const Geometry *)geom, n, &loss1);
                    else
                        launch2d(g.gridD, g.blockD, projRatio, &devProj[lenD * cond],
                                 (const float *)&devSino[lenD * cond], (const Geometry *)geom, n, &loss1);
                }
            }
            for (int y = 0; y < N; y++) {
                std::fill(devVoxelFactor.begin(), devVoxelFactor.end(), 0.0f);
                std::fill(devVoxelTmp.begin(), devVoxelTmp.end(), 0.0f);
                for (int cond = 0; cond < C; cond++)
                    for (int subOrder = 0; subOrder < subsetSize; subOrder++) {
                        int n = rotation * ((sub + batch * subOrder) % nProj);
                        launch2d(g.gridV, g.blockV, backwardProjFiber, &devProj[lenD * cond], devVoxel.data(),
                                 devVoxelTmp.data(), devVoxelFactor.data(), geom, cond, y, n);
                    }
                if (art)
                    launch2d(g.gridV, g.blockV, voxelPlus, devVoxel.data(), (const float *)devVoxelTmp.data(),
                             lambda / (float)subsetSize, (const Geometry *)geom, y);
                else
                    launch2d(g.gridV, g.blockV, voxelProduct, devVoxel.data(), (const float *)devVoxelTmp.data(),
                             (const float *)devVoxelFactor.data(), (const Geometry *)geom, y);
            }
        }
        if (losses) losses[ep] = loss1;
    }
    for (int i = 0; i < C; i++) std::memcpy(sino[i], &devProj[i * lenD], sizeof(float) * lenD);
    for (int i = 0; i < K; i++) std::memcpy(vol[i], &devVoxel[i * lenV], sizeof(float) * lenV);
}

}  // extern "C"
