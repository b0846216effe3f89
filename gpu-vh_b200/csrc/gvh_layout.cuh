// gvh_layout.cuh -- conversion between the reference's ghosted SoA layout (what the C ABI
// takes and returns) and the interior-only layout the stage kernels use, and the initial
// T^{tau mu} from primitive fields. Internal linkage: each translation unit gets its copy.
#pragma once

#include <cuda_runtime.h>

#include "../../include/gvh.h"
#include "gvh_physics.cuh"

namespace {

using namespace gvh;

struct Pack {
  int nx, ny, nz;
  long long sy, sz;   // internal strides
  long long ng;       // ghosted size (field stride in staging)
};

__device__ __forceinline__ long long ref_index(const Pack &p, int i, int j, int k) {
  return (long long)(i + 2) + (long long)(p.nx + 4) * ((j + 2) + (long long)(p.ny + 4) * (k + 2));
}

// Field pointers passed by value: no table has to reach the device before a launch, so the
// conversions can be queued without waiting (the asynchronous set/get of the C ABI).
struct FieldTable {
  double *p[32];
};

// staging (nf fields, ghosted) -> internal fields dst.p[f] (interior); null entries are skipped
__global__ void pack_kernel(Pack p, int nf, const double *__restrict__ staging, FieldTable dst) {
  long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)p.nx * p.ny * p.nz;
  if (id >= n) return;
  int i = id % p.nx, j = (id / p.nx) % p.ny, k = id / ((long long)p.nx * p.ny);
  long long r = ref_index(p, i, j, k), s = i + p.sy * j + p.sz * k;
  for (int f = 0; f < nf; ++f)
    if (dst.p[f]) dst.p[f][s] = staging[f * p.ng + r];
}

// internal fields src.p[f] -> staging (ghosted, every ghost cell filled from the nearest
// interior cell: the reference's zero-gradient faces, edges and corners alike); null entries
// are skipped
__global__ void unpack_kernel(Pack p, int nf, FieldTable src, double *__restrict__ staging) {
  long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = p.ng;
  if (id >= n) return;
  int gi = id % (p.nx + 4), gj = (id / (p.nx + 4)) % (p.ny + 4), gk = id / ((long long)(p.nx + 4) * (p.ny + 4));
  int i = min(max(gi - 2, 0), p.nx - 1), j = min(max(gj - 2, 0), p.ny - 1), k = min(max(gk - 2, 0), p.nz - 1);
  long long s = i + p.sy * j + p.sz * k;
  for (int f = 0; f < nf; ++f)
    if (src.p[f]) staging[f * p.ng + id] = src.p[f][s];
}

// Arrays in the element type of the caller (the reference's PRECISION: float as shipped,
// double in its FP64 build), passed by value like FieldTable.
struct RefTable {
  void *p[32];
};

// The reference's ghosted device arrays (type T) -> internal fields dst.p[f] (interior),
// converted to double; one launch for every field. Null entries on either side are skipped.
template <class T>
__global__ void gather_ref_kernel(Pack p, int nf, RefTable src, FieldTable dst) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)p.nx * p.ny * p.nz;
  if (id >= n) return;
  const int i = id % p.nx, j = (id / p.nx) % p.ny, k = id / ((long long)p.nx * p.ny);
  const long long r = ref_index(p, i, j, k), s = i + p.sy * j + p.sz * k;
  for (int f = 0; f < nf; ++f)
    if (dst.p[f] && src.p[f]) dst.p[f][s] = (double)static_cast<const T *>(src.p[f])[r];
}

// Internal fields src.p[f] -> the reference's ghosted device arrays (type T), every ghost
// cell filled from the nearest interior cell (GhostCells.cu:15-144 fills the faces; edges and
// corners get the same clamped value); null entries are skipped.
template <class T>
__global__ void scatter_ref_kernel(Pack p, int nf, FieldTable src, RefTable dst) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= p.ng) return;
  const int gi = id % (p.nx + 4), gj = (id / (p.nx + 4)) % (p.ny + 4);
  const int gk = id / ((long long)(p.nx + 4) * (p.ny + 4));
  const int i = min(max(gi - 2, 0), p.nx - 1), j = min(max(gj - 2, 0), p.ny - 1), k = min(max(gk - 2, 0), p.nz - 1);
  const long long s = i + p.sy * j + p.sz * k;
  for (int f = 0; f < nf; ++f)
    if (dst.p[f] && src.p[f]) static_cast<T *>(dst.p[f])[id] = (T)src.p[f][s];
}

// T^{tau mu} from primitives (DynamicalVariables.cu:349-392 with EnergyMomentumTensor.cu
// :159-177) and p = p(e) (InitialConditions.cpp:124-127), in the internal layout.
template <int EOS>
// p_given: the initial-condition reader supplied p (type 11, InitialConditions.cpp:29-97) and
// p already holds it; otherwise p = p(e) of the EoS (type 10).
__global__ void init_conserved_kernel(long long n, int nq, long long cs, double *q, double *e, double *p,
                                      double *u, double *up, int p_given) {
  long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  double es = e[s];
  double ps = p_given ? p[s] : eq_pressure<EOS>(es);
  p[s] = ps;
  double ut = u[s], ux = u[cs + s], uy = u[2 * cs + s], un = u[3 * cs + s];
  double pitt = 0, pitx = 0, pity = 0, pitn = 0, Pi = 0;
  if (nq >= 14) { pitt = q[4 * cs + s]; pitx = q[5 * cs + s]; pity = q[6 * cs + s]; pitn = q[7 * cs + s]; }
  if (nq == 15) Pi = q[14 * cs + s];
  double pp = ps + Pi;
  q[s] = (es + pp) * ut * ut - pp + pitt;
  q[cs + s] = (es + pp) * ut * ux + pitx;
  q[2 * cs + s] = (es + pp) * ut * uy + pity;
  q[3 * cs + s] = (es + pp) * ut * un + pitn;
  for (int m = 0; m < 4; ++m) up[m * cs + s] = u[m * cs + s];
}

// ---- Glauber-hotspot initial state on the device ----------------------------------------
// e(x, y, eta) = fz(eta) * scale * sum_p w_p gy_p gx_p + background, gx_p = exp(-(x - x_p)^2 / s2),
// fz = exp(-max(|eta| - eta_flat, 0)^2 / s2_eta), rounded to float and + 1e-3 as the type-10
// reader stores a value written to its files (InitialConditions.cpp:106, 122-124). Every
// operation is rounded on its own (no multiply-add contraction), in the order of the host
// generator (gvh/workloads.py hotspot_field), so the two agree wherever the device's exp
// agrees with the host's. Cell centres x_i = (i - (nx - 1)/2) dx (the centred grid).
struct HotspotArgs {
  int nx, ny, nz;
  long long sy, sz;    // internal strides
  double dx, dy, dz;
  int n;               // sources: x[n], y[n], w[n] back to back in src
  const double *src;
  double s2, scale, eta_flat, s2_eta, background;
};

// The kernels' arguments for a lattice (internal strides sy, sz) and a gvh_hotspots whose
// sources have been copied to src (x, y, w back to back). s2 = 2 sigma^2 as the host generator
// forms it.
inline HotspotArgs hotspot_args(int nx, int ny, int nz, long long sy, long long sz, const gvh_lattice_params *L,
                                const gvh_hotspots *hs, const double *src) {
  HotspotArgs a;
  a.nx = nx; a.ny = ny; a.nz = nz; a.sy = sy; a.sz = sz;
  a.dx = L->latticeSpacingX; a.dy = L->latticeSpacingY; a.dz = L->latticeSpacingRapidity;
  a.n = hs->n;
  a.src = src;
  a.s2 = 2.0 * (hs->sigma * hs->sigma);
  a.scale = hs->scale;
  a.eta_flat = hs->eta_flat;
  a.s2_eta = 2.0 * (hs->sigma_eta * hs->sigma_eta);
  a.background = hs->background;
  return a;
}

// The transverse profile scale * sum_p (w_p gy_p) gx_p, one thread per (i, j), into plane.
__global__ void hotspot_plane_kernel(HotspotArgs h, double *__restrict__ plane) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= h.nx * h.ny) return;
  const int i = id % h.nx, j = id / h.nx;
  const double x = __dmul_rn((double)i - (h.nx - 1) / 2.0, h.dx);
  const double y = __dmul_rn((double)j - (h.ny - 1) / 2.0, h.dy);
  const double *xs = h.src, *ys = h.src + h.n, *ws = h.src + 2 * h.n;
  double T = 0.0;
  for (int p = 0; p < h.n; ++p) {
    const double ddx = __dsub_rn(x, xs[p]), ddy = __dsub_rn(y, ys[p]);
    const double gx = exp(-__dmul_rn(ddx, ddx) / h.s2);
    const double gy = exp(-__dmul_rn(ddy, ddy) / h.s2);
    T = __dadd_rn(T, __dmul_rn(__dmul_rn(ws[p], gy), gx));
  }
  plane[id] = __dmul_rn(T, h.scale);
}

// Every interior cell: e from the plane and the eta profile, u = (1, 0, 0, 0) and the
// dissipative components (q[4..nq)) zero, in the internal layout; init_conserved_kernel then
// builds p and T^{tau mu} as for any primitive initial state.
__global__ void hotspot_fill_kernel(HotspotArgs h, const double *__restrict__ plane, double *e, double *u, long long cs,
                                    double *q, int nq) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)h.nx * h.ny * h.nz;
  if (id >= n) return;
  const int i = id % h.nx, j = (id / h.nx) % h.ny, k = id / ((long long)h.nx * h.ny);
  const long long s = i + h.sy * j + h.sz * k;
  const double z = __dmul_rn((double)k - (h.nz - 1) / 2.0, h.dz);
  const double m = fmax(__dsub_rn(fabs(z), h.eta_flat), 0.0);
  const double fz = exp(-__dmul_rn(m, m) / h.s2_eta);
  const double v = __dadd_rn(__dmul_rn(fz, plane[i + h.nx * j]), h.background);
  e[s] = __dadd_rn((double)__double2float_rn(v), 1.0e-3);
  u[s] = 1.0;
  u[cs + s] = 0.0;
  u[2 * cs + s] = 0.0;
  u[3 * cs + s] = 0.0;
  for (int c = 4; c < nq; ++c) q[c * cs + s] = 0.0;
}

// Max of a non-negative double array (interior energy densities), as the bit pattern of a
// double: for non-negative values the integer order of the bits is the numeric order.
__global__ void max_e_kernel(const double *e, long long n, unsigned long long *out) {
  unsigned long long b = 0ull;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
    b = max(b, (unsigned long long)__double_as_longlong(fmax(e[s], 0.0)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, b);
}

// One word to (mapped) host memory.
__global__ void word_to_host_kernel(const unsigned long long *src, unsigned long long *dst) { *dst = *src; }

}  // namespace
