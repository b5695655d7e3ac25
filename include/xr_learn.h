/*
 * libxr learned warm start: a small 3D convolutional network that maps an
 * early OS-EM iterate of a K-channel XTT volume to a warm start for further
 * OS-EM epochs, trained and run on sm_100a tensor cores (BF16 operands, FP32
 * accumulation).
 *
 * The reference has no learned component; these entry points are an
 * extension beside its reconstruct/direction path and replace nothing in it.
 *
 * Network (depth D >= 2, width W <= 32, K <= 16 channels):
 *   h_1 = relu(conv(s * x, W_1) + b_1), h_i = relu(conv(h_{i-1}, W_i) + b_i),
 *   y = x + (conv(h_{D-1}, W_D) + b_D) / s,
 * with 3x3x3 kernels and zero padding; x, y are K planes of nx*ny*nz voxels
 * (x fastest), s the caller's input scale.  Weights W_i[tap][cout][cin]
 * (tap = 9*(dz+1) + 3*(dy+1) + (dx+1)), all layers in order, each followed by
 * its bias, form the flat FP32 parameter vector.
 *
 * Training: loss = mean over K*nvox of (y - target)^2; Adam on FP32 master
 * parameters, BF16 copies for the tensor cores.
 */
#ifndef XR_LEARN_H
#define XR_LEARN_H

#include <stddef.h>
#include <stdint.h>

#include "xr.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xr_net xr_net;

/* New network on `device` with He-initialised weights (the last layer scaled
 * by 0.1, so the map starts close to the identity). */
xr_status xr_net_create(int device, int channels, int width, int depth, unsigned long long seed, xr_net **out);
void xr_net_destroy(xr_net *net);
const char *xr_net_last_error(const xr_net *net);
/* Stream for every later call (cudaStream_t; NULL = the legacy default stream). */
xr_status xr_net_set_stream(xr_net *net, void *stream);
size_t xr_net_num_params(const xr_net *net);
xr_status xr_net_get_params(xr_net *net, float *host, size_t n);
xr_status xr_net_set_params(xr_net *net, const float *host, size_t n);
/* Raw file: "XRNET1\0\0", int32 channels, width, depth, then the FP32 parameters. */
xr_status xr_net_save(xr_net *net, const char *path);
xr_status xr_net_load(xr_net *net, const char *path);

/* y = net(x) for device volumes of `storage` type (0 FP32, 1 BF16, 2 FP16),
 * K planes each; y = max(y, floor_value).  d_out may equal d_in (in place). */
xr_status xr_net_infer(xr_net *net, const void *d_in, void *d_out, int storage, int nx, int ny, int nz,
                       float in_scale, float floor_value);
/* Loss of the FP32 device volumes (no clamp) and its gradient, kept for the
 * next xr_net_adam_step; host_grad (xr_net_num_params floats) may be NULL. */
xr_status xr_net_loss_grad(xr_net *net, const float *d_in, const float *d_target, int nx, int ny, int nz,
                           float in_scale, double *loss, float *host_grad);
xr_status xr_net_adam_step(xr_net *net, float lr, float beta1, float beta2, float eps);
/* Orientation term of the training loss (0 = off, the default): xr_net_loss_grad
 * then minimises sum_c (pred - target)_c^2 + weight * ||T(pred) - T(target)||_F^2
 * per voxel (over K * voxels), T(mu) = sum_k mu_k S_k S_k^T the tensor whose
 * smallest-eigenvalue eigenvector is the voxel's main direction (calcEigenVector,
 * direction/src/pca.cu:12-55, on sqrt|mu|); basis: K rows of S_k (host). */
xr_status xr_net_set_tensor_loss(xr_net *net, const float *basis, float weight);

/* Layer-level tensor-core operators on device buffers (BF16 as uint16 bits,
 * channels-last: element [v][c], v = x + nx*(y + ny*z)); cin, cout in {16, 32}.
 * fprop:  y[v][n] = epi(sum_{tap,k} x[v + d(tap)][k] * w[tap][n][k]),
 *         epilogue 0: + bias; 1: relu(+ bias); 2: * (mask[v][n] > 0).
 * wgrad:  dw[tap][n][k] += sum_v dy[v][n] * x[v + d(tap)][k]   (FP32). */
xr_status xr_conv3d_fprop(void *stream, const uint16_t *x, int cin, const uint16_t *w, const float *bias,
                          const uint16_t *mask, uint16_t *y, int cout, int nx, int ny, int nz, int epilogue);
xr_status xr_conv3d_wgrad(void *stream, const uint16_t *x, int cin, const uint16_t *dy, int cout, float *dw, int nx,
                          int ny, int nz);

/* Training-data synthesis: K planes of an N^3 fiber phantom into d_out
 * (FP32).  fibers: n_fib <= 32 rows of (f_x, f_y, f_z, p0_x, p0_y, p0_z, r),
 * f a unit direction, p0 a point on the axis (voxel units from the volume
 * centre, voxel i at i - (N-1)/2), r the radius; inside a fiber channel k is
 * |S_k x f|^2 (basis: K rows of S_k), outside 0; later fibers overwrite
 * earlier ones.  Asynchronous on `stream`. */
xr_status xr_dev_fiber_phantom(void *stream, int N, int K, const float *basis, int n_fib, const float *fibers,
                               float *d_out);

#ifdef __cplusplus
}
#endif

#endif
