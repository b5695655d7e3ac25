/*
 * The reference's own CUDA kernels (reconstruct/src/ir.cu, compiled for
 * sm_100a from the reference's source tree by `make -C oracle ref`) driven
 * the way XTT::reconstruct drives them (reconstruct/src/reconstruct.cu:
 * 799-927): per subset, for every axis and view one forwardProjXTT launch per
 * y slab, each followed by a device synchronize, then correlationProjByLength
 * and projRatio / projSubtract; per y slab the backwardProjXTT launches of
 * every axis and view and the voxelProduct / voxelPlus of every channel;
 * voxelSqrt at the end.  Grids of BLOCK_SIZE x BLOCK_SIZE threads as the
 * reference's (reconstruct.cu:833-836).
 *
 * TEST INFRASTRUCTURE ONLY: the reference's GPU run on the same box, timed
 * beside the product (bench.py), and a second check of the oracle (a GPU
 * test at a small size).  Nothing in the product links or calls it.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

#include <params.h>
#include <geometry.h>
#include <ir.cuh>

int BLOCK_SIZE = 32;
__managed__ int NUM_BASIS_VECTOR = 1;
__managed__ int NUM_PROJ_COND = 1;
float SRC_OBJ_DISTANCE;
float SRC_DETECT_DISTANCE;
int NUM_PROJ;
int NUM_DETECT_U;
int NUM_DETECT_V;
float DETECTOR_SIZE;
int NUM_VOXEL;
__constant__ float elemR[9 * XR_REFGPU_MAX_COND];
__constant__ float elemT[3 * XR_REFGPU_MAX_COND];
__constant__ float INIT_OFFSET[3 * XR_REFGPU_MAX_COND];
__managed__ int proj_arr[20];
__managed__ float basisVector[3 * XR_REFGPU_MAX_BASIS];
__constant__ float fdThresh = 0.99f;
const float scatter_angle_xy = 0.0f;
__managed__ float d_loss_proj;
__managed__ float d_loss_norm;

namespace {

/* device buffers of one run, released on every exit */
struct Buffers {
    std::vector<void *> p;
    float *get(size_t n) {
        void *q = nullptr;
        if (cudaMalloc(&q, n * sizeof(float)) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (float *)q;
    }
    ~Buffers() {
        for (void *q : p) cudaFree(q);
    }
};

}  // namespace

extern "C" {

/* XTT::reconstruct's epochs on the GPU with the reference's kernels.  sino:
 * C blocks of V*Nd*Nd (host, read), vol: K channels of N^3 (host, in/out:
 * the result after voxelSqrt), ratio_out: C blocks (host, may be NULL: the
 * last ratio images), losses: epoch floats (may be NULL), ms_epoch: epoch
 * doubles (may be NULL: each epoch's time by CUDA events).  Returns a CUDA
 * error code (0 on success). */
int xr_refgpu_xtt_reconstruct(float sdd, float sod, float det, int N, int Nd, int V, int C, int K,
                              const float *rot, const float *trans, const float *offset, const float *basis,
                              const float *sino, float *vol, float *ratio_out, int epoch, int batch,
                              int rotate_ccw, int art, float lambda, float *losses, double *ms_epoch) {
    if (C < 1 || C > XR_REFGPU_MAX_COND || K < 1 || K > XR_REFGPU_MAX_BASIS || batch < 1) return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return (int)e;
    NUM_BASIS_VECTOR = K;
    NUM_PROJ_COND = C;
    std::memcpy(basisVector, basis, sizeof(float) * 3 * K);
    if ((e = cudaMemcpyToSymbol(elemR, rot, sizeof(float) * 9 * C)) != cudaSuccess) return (int)e;
    if ((e = cudaMemcpyToSymbol(elemT, trans, sizeof(float) * 3 * C)) != cudaSuccess) return (int)e;
    if ((e = cudaMemcpyToSymbol(INIT_OFFSET, offset, sizeof(float) * 3 * C)) != cudaSuccess) return (int)e;

    Geometry geom(sdd, sod, det, N, Nd, V);
    const long lenV = (long)N * N * N, lenD = (long)Nd * Nd * V, lenP = (long)N * N;
    Buffers B;
    float *devSino = B.get(lenD * C), *devProj = B.get(lenD * C), *devProjFactor = B.get((size_t)Nd * Nd);
    float *devVoxel = B.get(lenV * K), *devVoxelTmp = B.get(lenP * K), *devVoxelFactor = B.get(lenP * K);
    float *loss1 = B.get(1);
    Geometry *devGeom = nullptr;
    if (cudaMalloc(&devGeom, sizeof(Geometry)) != cudaSuccess) return (int)cudaErrorMemoryAllocation;
    B.p.push_back(devGeom);
    if (!devSino || !devProj || !devProjFactor || !devVoxel || !devVoxelTmp || !devVoxelFactor || !loss1)
        return (int)cudaErrorMemoryAllocation;
    cudaMemcpy(devGeom, &geom, sizeof(Geometry), cudaMemcpyHostToDevice);
    cudaMemcpy(devSino, sino, sizeof(float) * lenD * C, cudaMemcpyHostToDevice);
    cudaMemcpy(devVoxel, vol, sizeof(float) * lenV * K, cudaMemcpyHostToDevice);

    const int bs = BLOCK_SIZE;
    const dim3 blockV(bs, bs, 1), gridV((N + bs - 1) / bs, (N + bs - 1) / bs, 1);
    const dim3 blockD(bs, bs, 1), gridD((Nd + bs - 1) / bs, (Nd + bs - 1) / bs, 1);
    const int rotation = rotate_ccw ? -1 : 1;
    const int subsetSize = (V + batch - 1) / batch;
    std::vector<int> subsetOrder(batch);
    for (int i = 0; i < batch; i++) subsetOrder[i] = i;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    for (int ep = 0; ep < epoch; ep++) {
        cudaEventRecord(t0);
        std::mt19937_64 eng;   /* a fresh default engine every epoch, as the reference */
        std::shuffle(subsetOrder.begin(), subsetOrder.end(), eng);
        cudaMemset(loss1, 0, sizeof(float));
        cudaMemset(devProj, 0, sizeof(float) * lenD * C);
        for (const int sub : subsetOrder) {
            for (int cond = 0; cond < C; cond++)
                for (int j = 0; j < subsetSize; j++) {
                    cudaMemset(devProjFactor, 0, sizeof(float) * Nd * Nd);
                    const int n = rotation * ((sub + batch * j) % V);
                    for (int y = 0; y < N; y++) {
                        forwardProjXTT<<<gridV, blockV>>>(&devProj[lenD * cond], devProjFactor, devVoxel, devGeom,
                                                          cond, y, n);
                        cudaDeviceSynchronize();
                    }
                    correlationProjByLength<<<gridD, blockD>>>(&devProj[lenD * cond], devProjFactor, devGeom, cond,
                                                               n);
                    if (art)
                        projSubtract<<<gridD, blockD>>>(&devProj[lenD * cond], &devSino[lenD * cond], devGeom, n,
                                                        loss1);
                    else
                        projRatio<<<gridD, blockD>>>(&devProj[lenD * cond], &devSino[lenD * cond], devGeom, n, loss1);
                    cudaDeviceSynchronize();
                }
            for (int y = 0; y < N; y++) {
                cudaMemset(devVoxelFactor, 0, sizeof(float) * lenP * K);
                cudaMemset(devVoxelTmp, 0, sizeof(float) * lenP * K);
                for (int cond = 0; cond < C; cond++)
                    for (int j = 0; j < subsetSize; j++) {
                        const int n = rotation * ((sub + batch * j) % V);
                        backwardProjXTT<<<gridV, blockV>>>(&devProj[lenD * cond], devVoxelTmp, devVoxelFactor, devGeom,
                                                           cond, y, n);
                        cudaDeviceSynchronize();
                    }
                for (int k = 0; k < K; k++) {
                    if (art)
                        voxelPlus<<<gridV, blockV>>>(&devVoxel[lenV * k], &devVoxelTmp[lenP * k],
                                                     lambda / (float)subsetSize, devGeom, y);
                    else
                        voxelProduct<<<gridV, blockV>>>(&devVoxel[lenV * k], &devVoxelTmp[lenP * k],
                                                        &devVoxelFactor[lenP * k], devGeom, y);
                }
                cudaDeviceSynchronize();
            }
        }
        cudaEventRecord(t1);
        cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        if (ms_epoch) ms_epoch[ep] = ms;
        if (losses) cudaMemcpy(losses + ep, loss1, sizeof(float), cudaMemcpyDeviceToHost);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    for (int y = 0; y < N; y++) {
        voxelSqrt<<<gridV, blockV>>>(devVoxel, devGeom, y);
        cudaDeviceSynchronize();
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    if (ratio_out) cudaMemcpy(ratio_out, devProj, sizeof(float) * lenD * C, cudaMemcpyDeviceToHost);
    e = cudaMemcpy(vol, devVoxel, sizeof(float) * lenV * K, cudaMemcpyDeviceToHost);
    return (int)e;
}

}  // extern "C"
