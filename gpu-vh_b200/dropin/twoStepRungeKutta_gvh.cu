// twoStepRungeKutta_gvh.cu -- drop-in for gpu-vh's FullyDiscreteKurganovTadmorScheme.cu.
//
// Build it inside the gpu-vh tree in place of rhic/src/FullyDiscreteKurganovTadmorScheme.cu
// and link libgvh.so (gpu-vh_b200/libgvh.so; include/gvh.h). It defines twoStepRungeKutta with the reference's
// signature (FullyDiscreteKurganovTadmorScheme.cuh:18) and leaves the reference's device
// globals exactly as the reference's own step would (FullyDiscreteKurganovTadmorScheme.cu
// :109-139): d_Q holds the new conserved variables, d_e/d_p the new e and p, d_u the new
// u^mu and d_up the previous one (after the same swapFluidVelocity), ghost cells filled.
// Every call copies the full state into libgvh and back (device to device, with the
// reference's PRECISION converted to double); an integration that keeps the state inside
// libgvh (gvh_run, or a gvh_handle across the time loop) avoids those copies.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#include "../include/DynamicalVariables.cuh"
#include "../include/CudaConfiguration.cuh"
#include "../include/FullyDiscreteKurganovTadmorScheme.cuh"
#include "gvh.h"

namespace {

gvh_handle *g_handle = nullptr;
double *g_stage = nullptr;  // (nq + 10) ghosted fields in double
long long g_ng = 0;

__global__ void widen(const PRECISION *src, double *dst, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}
__global__ void narrow(const double *src, PRECISION *dst, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (PRECISION)src[i];
}

void die(const char *what) {
  fprintf(stderr, "twoStepRungeKutta (libgvh): %s: %s\n", what, gvh_last_error());
  exit(-1);
}

int component_pointers(const CONSERVED_VARIABLES *dq, PRECISION **out) {
  CONSERVED_VARIABLES hq;
  cudaMemcpy(&hq, dq, sizeof hq, cudaMemcpyDeviceToHost);
  PRECISION **slots = reinterpret_cast<PRECISION **>(&hq);
  for (int c = 0; c < NUMBER_CONSERVED_VARIABLES; ++c) out[c] = slots[c];
  return NUMBER_CONSERVED_VARIABLES;
}

void velocity_pointers(const FLUID_VELOCITY *du, PRECISION **out) {
  FLUID_VELOCITY hu;
  cudaMemcpy(&hu, du, sizeof hu, cudaMemcpyDeviceToHost);
  out[0] = hu.ut; out[1] = hu.ux; out[2] = hu.uy; out[3] = hu.un;
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
    o.shear = NUMBER_CONSERVED_VARIABLES >= 14;
    o.bulk = NUMBER_CONSERVED_VARIABLES == 15;
    if (gvh_create(&L, &H, &o, &g_handle)) die("gvh_create");
    g_ng = (long long)(nx + 4) * (ny + 4) * (nz + 4);
    if (cudaMalloc(&g_stage, (size_t)(nq + 10) * g_ng * sizeof(double)) != cudaSuccess) die("cudaMalloc");
  }
  const unsigned blocks = (unsigned)((g_ng + 255) / 256);
  PRECISION *src[32];
  component_pointers(d_q, src);
  src[nq] = d_e;
  src[nq + 1] = d_p;
  velocity_pointers(d_u, src + nq + 2);
  velocity_pointers(d_up, src + nq + 6);
  const double *fields_in[32];
  double *fields_out[32];
  for (int f = 0; f < nq + 10; ++f) {
    double *stage = g_stage + f * g_ng;
    widen<<<blocks, 256>>>(src[f], stage, g_ng);
    fields_in[f] = stage;
    fields_out[f] = stage;
  }
  if (gvh_set_state(g_handle, fields_in, nq + 10)) die("gvh_set_state");
  if (gvh_rk2_step(g_handle, t, dt, T_reg)) die("gvh_rk2_step");
  if (gvh_get_state(g_handle, fields_out, nq + 10)) die("gvh_get_state");
  // the reference swaps u and up inside the step (FullyDiscreteKurganovTadmorScheme.cu:131)
  swapFluidVelocity(&d_up, &d_u);
  PRECISION *dst[32];
  component_pointers(d_Q, dst);
  dst[nq] = d_e;
  dst[nq + 1] = d_p;
  velocity_pointers(d_u, dst + nq + 2);
  velocity_pointers(d_up, dst + nq + 6);
  for (int f = 0; f < nq + 10; ++f) narrow<<<blocks, 256>>>(g_stage + f * g_ng, dst[f], g_ng);
  cudaDeviceSynchronize();
}

// The convex combination kernel the reference declares in the same header; unused here.
__global__ void convexCombinationEulerStepKernel(const CONSERVED_VARIABLES *const __restrict__,
                                                 CONSERVED_VARIABLES *const __restrict__) {}
