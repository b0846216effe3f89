// twoStepRungeKutta_gvh.cu -- drop-in for gpu-vh's FullyDiscreteKurganovTadmorScheme.cu.
//
// Build it inside the gpu-vh tree in place of rhic/src/FullyDiscreteKurganovTadmorScheme.cu
// and link libgvh.so (gpu-vh_b200/libgvh.so; include/gvh.h). It defines twoStepRungeKutta
// with the reference's signature (FullyDiscreteKurganovTadmorScheme.cuh:18) and leaves the
// reference's device globals as the reference's own step does (FullyDiscreteKurganovTadmorScheme
// .cu:109-139): d_Q holds the new conserved variables, d_e / d_p the new e and p, d_u the new
// u^mu and d_up the previous one (after the same swapFluidVelocity), ghost cells filled.
//
// Per call: one gather launch (the reference's arrays of its PRECISION -> the handle, converted
// to double), the handle's two fused stage launches, one scatter launch back (ghost cells
// filled), all on the legacy default stream the reference launches on, then the
// cudaDeviceSynchronize the reference ends its step with. The pointers behind the reference's
// device-resident CONSERVED_VARIABLES / FLUID_VELOCITY structs are read once per struct and
// cached (the structs never change after allocateDeviceMemory; the step loop only swaps which
// struct d_q, d_Q, d_u and d_up point to).
//
// Compile-time settings follow the reference's: CONFORMAL_EOS, the PIMUNU / PI component count
// (NUMBER_CONSERVED_VARIABLES) and PRECISION come from its headers; the limiter slope is
// GVH_THETA (default 2.0, the reference's THETA, FluxLimiter.cu:15). The validity
// diagnostics the reference computes at the end of its step (checkValidity) are not computed
// here; the reference's run loop does not read them.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/DynamicalVariables.cuh"
#include "../include/CudaConfiguration.cuh"
#include "../include/FullyDiscreteKurganovTadmorScheme.cuh"
#include "gvh.h"

#ifndef GVH_THETA
#define GVH_THETA 2.0
#endif

namespace {

gvh_handle *g_handle = nullptr;

// device address of a reference struct -> the component pointers stored in it
struct CachedStruct {
  const void *dev;
  PRECISION *ptr[NUMBER_CONSERVED_VARIABLES > 4 ? NUMBER_CONSERVED_VARIABLES : 4];
};
CachedStruct g_cache[8];
int g_ncache = 0;

void die(const char *what) {
  fprintf(stderr, "twoStepRungeKutta (libgvh): %s: %s\n", what, gvh_last_error());
  exit(-1);
}

template <class S>
PRECISION *const *struct_pointers(const S *dev_struct) {
  for (int c = 0; c < g_ncache; ++c)
    if (g_cache[c].dev == dev_struct) return g_cache[c].ptr;
  if (g_ncache == 8) {
    fprintf(stderr, "twoStepRungeKutta (libgvh): more state structs than expected\n");
    exit(-1);
  }
  S host;
  if (cudaMemcpy(&host, dev_struct, sizeof host, cudaMemcpyDeviceToHost) != cudaSuccess) die("reading a state struct");
  CachedStruct &e = g_cache[g_ncache++];
  e.dev = dev_struct;
  // both structs are plain sequences of PRECISION pointers (DynamicalVariables.cuh:50-80)
  memcpy(e.ptr, &host, sizeof host);
  return e.ptr;
}

}  // namespace

void twoStepRungeKutta(PRECISION t, PRECISION dt, CONSERVED_VARIABLES *__restrict__ d_q,
                       CONSERVED_VARIABLES *__restrict__ d_Q, PRECISION T_reg) {
  const int nq = NUMBER_CONSERVED_VARIABLES;
  if (!g_handle) {
    int nx, ny, nz;
    PRECISION ddt, dx, dy, dz, etabar;
    cudaMemcpyFromSymbol(&nx, d_nx, sizeof nx);
    cudaMemcpyFromSymbol(&ny, d_ny, sizeof ny);
    cudaMemcpyFromSymbol(&nz, d_nz, sizeof nz);
    cudaMemcpyFromSymbol(&ddt, d_dt, sizeof ddt);
    cudaMemcpyFromSymbol(&dx, d_dx, sizeof dx);
    cudaMemcpyFromSymbol(&dy, d_dy, sizeof dy);
    cudaMemcpyFromSymbol(&dz, d_dz, sizeof dz);
    cudaMemcpyFromSymbol(&etabar, d_etabar, sizeof etabar);
    gvh_lattice_params L = {nx, ny, nz, nx + 4, ny + 4, nz + 4, 0, dx, dy, dz, ddt};
    gvh_hydro_params H = {0.0, etabar, 0.0, 0, 0.0};
    gvh_options o;
    gvh_default_options(&o);
#ifdef CONFORMAL_EOS
    o.eos = GVH_EOS_CONFORMAL;
#endif
#ifdef USE_CARTESIAN_COORDINATES
    o.coordinates = GVH_COORDINATES_CARTESIAN;
#endif
    o.shear = NUMBER_CONSERVED_VARIABLES >= 14;
    o.bulk = NUMBER_CONSERVED_VARIABLES == 15;
    o.theta = GVH_THETA;
    if (gvh_create(&L, &H, &o, &g_handle)) die("gvh_create");
    // the reference's kernels and copies run on the legacy default stream: queue ours there too
    if (gvh_set_stream(g_handle, (void *)cudaStreamLegacy)) die("gvh_set_stream");
  }
  const void *in[32];
  PRECISION *const *q = struct_pointers(d_q);
  for (int c = 0; c < nq; ++c) in[c] = q[c];
  in[nq] = d_e;
  in[nq + 1] = d_p;
  PRECISION *const *u = struct_pointers(d_u);
  PRECISION *const *up = struct_pointers(d_up);
  for (int m = 0; m < 4; ++m) in[nq + 2 + m] = u[m];
  for (int m = 0; m < 4; ++m) in[nq + 6 + m] = up[m];
  if (gvh_gather_state_device(g_handle, in, nq + 10, (int)sizeof(PRECISION))) die("gvh_gather_state_device");
  if (gvh_rk2_step(g_handle, t, dt, T_reg)) die("gvh_rk2_step");
  // the reference swaps u and up inside the step (FullyDiscreteKurganovTadmorScheme.cu:131):
  // the new u^mu goes to the buffer that held u one step earlier, and d_up keeps u^n
  swapFluidVelocity(&d_up, &d_u);
  void *out[32];
  PRECISION *const *Q = struct_pointers(d_Q);
  for (int c = 0; c < nq; ++c) out[c] = Q[c];
  out[nq] = d_e;
  out[nq + 1] = d_p;
  PRECISION *const *un = struct_pointers(d_u);
  for (int m = 0; m < 4; ++m) out[nq + 2 + m] = un[m];
  for (int m = 0; m < 4; ++m) out[nq + 6 + m] = nullptr;  // d_up already holds u^n
  if (gvh_scatter_state_device(g_handle, out, nq + 10, (int)sizeof(PRECISION))) die("gvh_scatter_state_device");
  cudaDeviceSynchronize();  // as the reference's step ends (FullyDiscreteKurganovTadmorScheme.cu:138)
}

// The convex combination kernel the reference declares in the same header (its launch
// set-up queries its occupancy, CudaConfiguration.cu:78); unused here.
__global__ void convexCombinationEulerStepKernel(const CONSERVED_VARIABLES *const __restrict__,
                                                 CONSERVED_VARIABLES *const __restrict__) {}
