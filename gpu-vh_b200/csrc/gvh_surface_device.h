// gvh_surface_device.h -- the device half of the surface rows (gvh_surface_rows.cu), as
// gvh_surface.cu drives it.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "gvh_surface_rows.hpp"

namespace gvh {
namespace surface {

// A row's text holds 20 numbers of at most 12 characters ("-1.23456e+27", "-0.000123456":
// the fast path of %g takes exponents in [-17, 27]) and 20 separators.
constexpr int kTextSlot = 288;

struct DeviceRows {
  RowGeometry g;
  long long ncubes, npoints;
  const int *cube_key;      // crossed hypercubes in the reference's loop order
  const int *point_cell;    // lattice cell of each point
  const double *point_vals; // per point: kRowVars values at the lower level, then the upper
  int *c2p;                 // lattice cell -> point (scratch, nx ny nz ints)
  // scratch, per slot (hypercube c, element i: slot c kMaxElements + i; the rows are the
  // filled slots in slot order)
  double *slot_rows;        // kRowColumns values per slot
  int *slot_n, *offsets;    // rows per hypercube (+1 entry), and their exclusive offsets
  long long *slot_len;      // text bytes per slot (+1 entry; 0 for an empty slot or a host row)
  long long *text_off;      // their exclusive offsets
  unsigned char *slot_host; // 1 for a host row
  char *text_slots;         // kTextSlot bytes per slot
  void *scan_temp;          // the scans' work space
  size_t scan_temp_bytes;
  long long *totals;        // [0] rows, [1] hypercubes where cornelius stopped, [2] text bytes,
                            // [3] host rows
  // out
  long long *host_totals;   // mapped pinned host memory: totals, written last
  char *text;               // device: the slab's text (rows in order, host rows left out), or
                            // nullptr for no text
  HostRow *host_rows;       // mapped: the host rows, in no particular order
  long long host_rows_cap;
  double *rows;             // device: every row, in order (slot_rows' worth of room), when
                            // keep_rows, when there is no text, or when the host rows
                            // overflow host_rows_cap (then the host copies them)
  bool keep_rows;
};

// Bytes of device scratch for cap hypercubes (slots, their text, scan space; 256-byte
// aligned pieces), and the carving of one such allocation into d's scratch pointers.
size_t device_rows_scratch_bytes(long long cap);
void device_rows_carve(DeviceRows &d, char *base, long long cap);

// The rows (and text) of d's slab, queued on st. d.totals must be the carve's.
cudaError_t launch_device_rows(const DeviceRows &d, cudaStream_t st);

}  // namespace surface
}  // namespace gvh
