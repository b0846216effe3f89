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
  double *slot_rows;        // scratch: iso::kMaxElements rows per hypercube
  int *slot_n, *offsets;    // scratch: rows per hypercube, and their exclusive offsets
  long long *totals;        // scratch: [0] rows, [1] hypercubes where cornelius stopped, [2] text
                            // bytes, [3] 1 when the text fits text_cap, [4] rows without text
  double *rows;             // out (mapped pinned host memory): the slab's rows, in order, room
                            // for the slots' worth. With text, only the rows the host formats
                            // itself are written, unless keep_rows
  long long *host_totals;   // out (mapped pinned host memory): totals, written last
  // The rows' text as the reference's ofstream writes it (printf's %g), made with the fast
  // path of gvh_format.hpp. A row with a number the fast path leaves to the exact one gets
  // no text (length 0), and its values go to rows for the host to format. text == nullptr:
  // no text, every row to rows.
  char *text_slots;         // scratch: kTextSlot bytes per row slot
  int *row_len;             // scratch: text bytes per row, -1 for a row the host formats
  long long *text_off;      // scratch: exclusive offsets of the rows' text, rows + 1 entries
  char *text;               // out (mapped): the rows' text, concatenated
  long long text_cap;       // bytes text can hold; when the text is longer, every row goes to
                            // rows and no text is written (totals[3] = 0)
  long long *host_text_off; // out (mapped): text_off
  bool keep_rows;           // every row to rows, text or not
};

// Bytes of device scratch per hypercube (the slots, their counts and offsets, the text
// slots, lengths and offsets); the host's mapped row buffer needs the slot rows' worth.
size_t device_rows_slot_bytes(long long ncubes);

// Carves the scratch for cap hypercubes out of one allocation of device_rows_slot_bytes(cap)
// + 1024 bytes at base (256-byte aligned) into d's scratch pointers.
void device_rows_carve(DeviceRows &d, char *base, long long cap);

cudaError_t launch_device_rows(const DeviceRows &d, cudaStream_t st);

}  // namespace surface
}  // namespace gvh
