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
  int cartesian;            // GVH_COORDINATES_CARTESIAN
  long long split_below;    // lattices with fewer cells take the split stage kernel
  cudaStream_t stream;      // where work is queued (own_stream unless the caller set one)
  cudaStream_t own_stream;
  double *block;
  double *qA, *qB, *e, *pA, *pB, *u[3];
  int ucur, uprev, ufree;
  unsigned *status;
  double *staging;          // reference-layout fields for set/get, allocated on first use
  double *diag;             // validity diagnostics (allocated by gvh_enable_validity)
  int validity_on;
  // asynchronous set/get (allocated on first use): two input and two output staging areas
  // used in turn (a copy into one overlaps the pack of the other; an unpack into one overlaps
  // the copy out of the other), one copy stream each way, events that order them with the
  // handle's stream; in_slot / out_slot are the areas the next calls use
  double *staging_in[2], *staging_out[2];
  cudaStream_t s_h2d, s_d2h;
  cudaEvent_t ev_in_ready, ev_in_free[2], ev_out_ready, ev_out_free[2], ev_fence;
  int in_slot, out_slot;
  int async_ready;
  // mapped pinned word for small results read on the host (allocated on first use): a
  // kernel writes it, so the read needs no copy that could queue behind another stream's
  // large copy to the host
  unsigned long long *host_word, *host_word_dev;
};

// The current time level's fields in the handle's interior-only layout (cell
// s = i + nx * (j + ny * k), component stride cs).
inline const double *gvh_current_q(const gvh_handle *h) { return h->qA; }
inline const double *gvh_current_u(const gvh_handle *h) { return h->u[h->ucur]; }
