// Host check of the stage kernels' per-cell index check (cell_stencil_ok, gvh_stage.cuh),
// which the bounds-checked build (GVH_BOUNDS_CHECK) runs before any load of a cell: on
// consistent lattices every cell passes; a row or plane stride that does not match the
// lattice, a component stride shorter than the lattice, or a cell outside it fails. Built
// with nvcc and run on the CPU (no device code runs).
#include <stdio.h>
#include <string.h>

#include "gvh_stage.cuh"

using gvh::StageArgs;

static StageArgs lattice(int nx, int ny, int nz) {
  StageArgs a;
  memset(&a, 0, sizeof a);
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.sy = nx; a.sz = (long long)nx * ny;
  a.ncells = (long long)nx * ny * nz;
  a.cs = (a.ncells + 31) / 32 * 32;
  return a;
}

static long long failing(const StageArgs &a) {
  long long bad = 0;
  for (int k = 0; k < a.nz; ++k)
    for (int j = 0; j < a.ny; ++j)
      for (int i = 0; i < a.nx; ++i) bad += !gvh::cell_stencil_ok(a, i, j, k);
  return bad;
}

int main() {
  int errors = 0;
  const int shapes[][3] = {{1, 1, 1}, {1, 1, 12}, {9, 8, 1}, {12, 10, 6}, {33, 33, 17}, {131, 7, 3}};
  for (const auto &sh : shapes) {
    StageArgs a = lattice(sh[0], sh[1], sh[2]);
    if (failing(a)) { printf("consistent %dx%dx%d flagged\n", sh[0], sh[1], sh[2]); ++errors; }
  }
  StageArgs a = lattice(12, 10, 6);
  StageArgs b = a;
  b.sy = a.sy + 3;  // rows too far apart: the last planes reach past the arrays
  if (!failing(b)) { printf("bad row stride not flagged\n"); ++errors; }
  b = a;
  b.sz = a.sz * 2;
  if (!failing(b)) { printf("bad plane stride not flagged\n"); ++errors; }
  b = a;
  b.cs = a.ncells - 7;  // component arrays shorter than the lattice
  if (!failing(b)) { printf("short component stride not flagged\n"); ++errors; }
  if (gvh::cell_stencil_ok(a, 12, 0, 0) || gvh::cell_stencil_ok(a, 0, -1, 0) || gvh::cell_stencil_ok(a, 0, 0, 6)) {
    printf("cell outside the lattice not flagged\n");
    ++errors;
  }
  printf("%d errors\n", errors);
  return errors ? 1 : 0;
}
