/*
 * Declarations of the reference's configuration globals
 * (reconstruct/include/params.h:9-37, defined in reconstruct/src/params.cu:14-40)
 * with capacities large enough for 13 scattering vectors and 32 rotation axes.
 *
 * The reference sizes basisVector for 7 vectors (params.cu:36) and elemR for
 * 13 axes (params.cu:31).  This header is found before the reference's own
 * params.h on the include path of the shim build, so ir.cu sees these sizes;
 * the definitions live in ref_globals.cpp.  Test infrastructure only.
 */
#ifndef CUDA_EXAMPLE_PARAMS_H
#define CUDA_EXAMPLE_PARAMS_H
#include <string>

#define XR_REF_MAX_COND 32
#define XR_REF_MAX_BASIS 32

extern int BLOCK_SIZE;
extern int NUM_BASIS_VECTOR;
extern int NUM_PROJ_COND;

extern float SRC_OBJ_DISTANCE;
extern float SRC_DETECT_DISTANCE;
extern int NUM_PROJ;
extern int NUM_DETECT_U;
extern int NUM_DETECT_V;
extern float DETECTOR_SIZE;
extern int NUM_VOXEL;

extern float elemR[9 * XR_REF_MAX_COND];
extern float elemT[3 * XR_REF_MAX_COND];
extern float INIT_OFFSET[3 * XR_REF_MAX_COND];
extern int proj_arr[20];
extern float basisVector[3 * XR_REF_MAX_BASIS];
extern float fdThresh;

extern const float scatter_angle_xy;
extern float d_loss_proj;
extern float d_loss_norm;

#endif
