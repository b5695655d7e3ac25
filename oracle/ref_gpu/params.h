/*
 * Declarations of the reference's configuration globals
 * (reconstruct/include/params.h:9-37, defined in reconstruct/src/params.cu:14-40)
 * for the build of the reference's own CUDA kernels on the B200, with
 * capacities for 13 scattering vectors and 32 rotation axes (the reference
 * sizes basisVector for 7 vectors, params.cu:36, and elemR for 13 axes,
 * params.cu:31).  Found before the reference's params.h on the include path
 * (same include guard).  Definitions: ref_gpu_driver.cu.  Test
 * infrastructure only.
 */
#ifndef CUDA_EXAMPLE_PARAMS_H
#define CUDA_EXAMPLE_PARAMS_H
#include <string>

#define XR_REFGPU_MAX_COND 32
#define XR_REFGPU_MAX_BASIS 32

extern int BLOCK_SIZE;
extern __managed__ int NUM_BASIS_VECTOR;
extern __managed__ int NUM_PROJ_COND;

extern float SRC_OBJ_DISTANCE;
extern float SRC_DETECT_DISTANCE;
extern int NUM_PROJ;
extern int NUM_DETECT_U;
extern int NUM_DETECT_V;
extern float DETECTOR_SIZE;
extern int NUM_VOXEL;

extern __constant__ float elemR[9 * XR_REFGPU_MAX_COND];
extern __constant__ float elemT[3 * XR_REFGPU_MAX_COND];
extern __constant__ float INIT_OFFSET[3 * XR_REFGPU_MAX_COND];
extern __managed__ int proj_arr[20];
extern __managed__ float basisVector[3 * XR_REFGPU_MAX_BASIS];
extern __constant__ float fdThresh;

extern const float scatter_angle_xy;
extern __managed__ float d_loss_proj;
extern __managed__ float d_loss_norm;

#endif
