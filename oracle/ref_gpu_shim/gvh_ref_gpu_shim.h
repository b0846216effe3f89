/*
 * nvcc shim for the reference's own CUDA sources (gpu-vh rhic/src), reached through the
 * reference's `#include <cuda.h>` / `<cuda_runtime.h>` (this directory is first on the
 * include path; the real headers come in through #include_next). It adds nothing to the
 * CUDA build except the compile-time overlays of oracle/ref_shim/gvh_ref_overlays.h, so
 * the same sources build as shipped (FP32) or with PRECISION double. Test and measurement
 * infrastructure only.
 */
#ifndef GVH_REF_GPU_SHIM_
#define GVH_REF_GPU_SHIM_
#ifdef GVH_REF_FP64
/* rsqrtf (RegulateDissipativeCurrents.cu) in double */
static __device__ __forceinline__ double gvh_ref_rsqrt(double x) { return rsqrt(x); }
#endif
#endif
#include "../ref_shim/gvh_ref_overlays.h"
