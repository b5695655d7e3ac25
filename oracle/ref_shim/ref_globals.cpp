/*
 * Definitions of the reference's configuration globals for the host shim build
 * (the reference defines them in reconstruct/src/params.cu:14-40; sizes here
 * follow ref_shim/params.h).  Test infrastructure only.
 */
#include "cuda_runtime.h"
#include "params.h"

int BLOCK_SIZE = 32;
int NUM_BASIS_VECTOR = 1;
int NUM_PROJ_COND = 1;

float SRC_OBJ_DISTANCE;
float SRC_DETECT_DISTANCE;
int NUM_PROJ;
int NUM_DETECT_U;
int NUM_DETECT_V;
float DETECTOR_SIZE;
int NUM_VOXEL;

float elemR[9 * XR_REF_MAX_COND];
float elemT[3 * XR_REF_MAX_COND];
float INIT_OFFSET[3 * XR_REF_MAX_COND];
int proj_arr[20];
float basisVector[3 * XR_REF_MAX_BASIS];
float fdThresh = 0.99f;
const float scatter_angle_xy = 0.0f;
float d_loss_proj;
float d_loss_norm;

thread_local uint3 blockIdx;
thread_local uint3 threadIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
int xr_shim_parallel = 0;
