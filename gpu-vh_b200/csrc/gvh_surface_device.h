// gvh_surface_device.h -- the device half of the surface rows (gvh_surface_rows.cu), as
// gvh_surface.cu drives it.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "gvh_surface_rows.hpp"

namespace gvh {
namespace surface {

struct DeviceRows {
  RowGeometry g;
  long long ncubes, npoints;
  const int *cube_key;      // crossed hypercubes in the reference's loop order
  const int *point_cell;    // lattice cell of each point
  const double *point_vals; // per point: kRowVars values at the lower level, then the upper
  int *c2p;                 // lattice cell -> point (scratch, nx ny nz ints)
  double *slot_rows;        // scratch: iso::kMaxElements rows per hypercube
  int *slot_n, *offsets;    // scratch: rows per hypercube, and their exclusive offsets
  long long *totals;        // scratch: [0] rows, [1] hypercubes where cornelius stopped
  double *rows;             // out (mapped pinned host memory): the slab's rows, in order, room
                            // for the slots' worth
  long long *host_totals;   // out (mapped pinned host memory): totals, written last
};

// Bytes of device scratch per batch of ncubes hypercubes: slot_rows + slot_n + offsets (the
// host's mapped row buffer needs the slot rows' worth too).
size_t device_rows_slot_bytes(long long ncubes);

cudaError_t launch_device_rows(const DeviceRows &d, cudaStream_t st);

}  // namespace surface
}  // namespace gvh
