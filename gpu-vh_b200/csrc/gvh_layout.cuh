// gvh_layout.cuh -- conversion between the reference's ghosted SoA layout (what the C ABI
// takes and returns) and the interior-only layout the stage kernels use, and the initial
// T^{tau mu} from primitive fields. Internal linkage: each translation unit gets its copy.
#pragma once

#include <cuda_runtime.h>

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
