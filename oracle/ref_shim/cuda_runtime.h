/*
 * Host shim standing in for the CUDA runtime header so that the reference's
 * device code (reconstruct/src/ir.cu) compiles as ordinary host C++ with g++.
 *
 * TEST INFRASTRUCTURE ONLY: this builds the checker (oracle/_ref), never the
 * product.  Kernels become plain functions; the launch helper in
 * ref_driver.cpp sets the thread-local blockIdx/threadIdx before each call.
 */
#ifndef XR_REF_SHIM_CUDA_RUNTIME_H
#define XR_REF_SHIM_CUDA_RUNTIME_H

#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <cstdlib>
#include <atomic>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __managed__
#define __shared__
#define __forceinline__ inline

/* Float overloads of the C math names must win over ::abs(int) and friends,
 * exactly as CUDA's device overloads do inside the kernels. */
using std::abs;
using std::sqrt;
using std::floor;
using std::isnan;
using std::cos;
using std::sin;

struct uint3 { unsigned int x, y, z; };
struct dim3 {
    unsigned int x, y, z;
    dim3(unsigned int x_ = 1, unsigned int y_ = 1, unsigned int z_ = 1) : x(x_), y(y_), z(z_) {}
};

extern thread_local uint3 blockIdx;
extern thread_local uint3 threadIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

/* When set (OpenMP timing runs), float atomics use a CAS loop; the serial
 * golden-vector runs use a plain add so the summation order is fixed. */
extern int xr_shim_parallel;

inline float atomicAdd(float *addr, float val) {
    if (!xr_shim_parallel) {
        float old = *addr;
        *addr = old + val;
        return old;
    }
    std::atomic_ref<float> ref(*addr);
    return ref.fetch_add(val, std::memory_order_relaxed);
}

typedef int cudaError_t;
#define cudaSuccess 0
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost,
                      cudaMemcpyDeviceToDevice, cudaMemcpyDefault };

inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }

#endif
