/*
 * Compile-time overlays the reference exposes as macros, applied at every inclusion of
 * <cuda.h> / <cuda_runtime.h> through the shim directories (oracle/ref_shim for the g++
 * build, oracle/ref_gpu_shim for the nvcc build). No include guard on purpose:
 * DynamicalVariables.cuh includes <cuda.h> right after it defines PRECISION and the
 * component counts (DynamicalVariables.cuh:44-47), so re-running this block there overrides
 * them before any struct or kernel is declared. Test infrastructure only.
 *
 *   GVH_REF_FP64     PRECISION double (DynamicalVariables.cuh:44) and the single-precision
 *                    intrinsics remapped to their double versions, which would otherwise
 *                    silently truncate to float (gvh_ref_rsqrt is defined by each shim)
 *   GVH_REF_NO_BULK  PI off (DynamicalVariables.cuh:14-21): 14 components
 *   GVH_REF_IDEAL    PIMUNU off as well: 4 components, IDEAL (DynamicalVariables.cuh:37-39)
 */
#ifdef GVH_REF_FP64
#undef PRECISION
#define PRECISION double
#undef fminf
#define fminf fmin
#undef fmaxf
#define fmaxf fmax
#undef fabsf
#define fabsf fabs
#undef sqrtf
#define sqrtf sqrt
#undef fmaf
#define fmaf fma
#undef tanhf
#define tanhf tanh
#undef powf
#define powf pow
#undef rsqrtf
#define rsqrtf gvh_ref_rsqrt
#undef fdividef
#define fdividef(a, b) ((a) / (b))
#endif

#if defined(GVH_REF_NO_BULK) || defined(GVH_REF_IDEAL)
#undef PI
#undef NUMBER_PI_COMPONENTS
#define NUMBER_PI_COMPONENTS 0
#endif

#ifdef GVH_REF_IDEAL
#undef PIMUNU
#undef NUMBER_PROPAGATED_PIMUNU_COMPONENTS
#define NUMBER_PROPAGATED_PIMUNU_COMPONENTS 0
#ifndef IDEAL
#define IDEAL
#endif
#endif
