// gvh_handle.h -- the single-lattice handle behind the gvh_* C ABI (shared by the
// translation units of libgvh.so; not part of the public interface).
#pragma once

#include <cuda_runtime.h>

struct gvh_handle {
  int nx, ny, nz, nq;
  long long ncells, ng;     // interior cells, ghosted cells
  long long sy, sz, cs;     // internal strides
  double dx, dy, dz, dt_lattice, etabar, theta;
  int eos, shear, bulk, precision, device;
  cudaStream_t stream;      // where work is queued (own_stream unless the caller set one)
  cudaStream_t own_stream;
  double *block;
  double *qA, *qB, *e, *pA, *pB, *u[3];
  int ucur, uprev, ufree;
  unsigned *status;
  double *staging;          // reference-layout fields for set/get, allocated on first use
  double *diag;             // validity diagnostics (allocated by gvh_enable_validity)
  int validity_on;
};

// The current time level's fields in the handle's interior-only layout (cell
// s = i + nx * (j + ny * k), component stride cs).
inline const double *gvh_current_q(const gvh_handle *h) { return h->qA; }
inline const double *gvh_current_u(const gvh_handle *h) { return h->u[h->ucur]; }
