/*
 * Host shim that lets the reference's hot-path CUDA sources (gpu-vh rhic/src/*.cu)
 * compile with g++ as plain C++, so the reference itself can be run on the CPU as the
 * pinning oracle. Test infrastructure only: nothing in the product links this.
 *
 * It is reached through the reference's own `#include <cuda.h>` / `<cuda_runtime.h>`
 * (this directory is first on the include path). It does two things:
 *   1. (guarded) defines the CUDA keywords away and gives the kernels a thread-local
 *      threadIdx/blockIdx/blockDim so a driver can call a __global__ kernel as a function
 *      once per thread id;
 *   2. (NOT guarded, re-run at every inclusion) applies the compile-time overlays the
 *      reference exposes as macros: PRECISION (DynamicalVariables.cuh:44), bulk on/off
 *      (PI, DynamicalVariables.cuh:14-21), ideal (DynamicalVariables.cuh:37-39). Because
 *      DynamicalVariables.cuh includes <cuda.h> right after it defines PRECISION and the
 *      component counts (DynamicalVariables.cuh:44-47), re-running this block there
 *      overrides them before any struct or kernel is declared.
 * With GVH_REF_FP64 the single-precision intrinsics the reference calls are remapped to
 * their double versions, otherwise they would silently truncate to float.
 */
#ifndef GVH_REF_SHIM_TYPES_
#define GVH_REF_SHIM_TYPES_

#include <math.h>
#include <cmath>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__
#define __forceinline__ inline

struct dim3 {
	unsigned int x, y, z;
	dim3(unsigned int x_ = 1, unsigned int y_ = 1, unsigned int z_ = 1) : x(x_), y(y_), z(z_) {}
};
extern thread_local dim3 threadIdx;
extern thread_local dim3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

typedef int cudaError_t;
typedef void *cudaStream_t;

#ifndef GVH_REF_FP64
static inline float fdividef(float a, float b) { return a / b; }
static inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
#else
static inline double gvh_ref_rsqrt(double x) { return 1.0 / sqrt(x); }
#endif

#endif /* GVH_REF_SHIM_TYPES_ */

/* ---- overlays: evaluated at every inclusion (shared with the nvcc build) ---------- */
#include "gvh_ref_overlays.h"
