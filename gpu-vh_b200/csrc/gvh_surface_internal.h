// gvh_surface_internal.h -- what the device side of the freeze-out surface hands to the host.
#pragma once

#include <string>
#include <vector>

namespace gvh {
namespace surface {

constexpr int kVars = 10;     // u^x u^y u^eta e pi^xx pi^xy pi^x eta pi^yy pi^y eta Pi (FreezeOut.cpp:73-86)
constexpr int kColumns = 20;  // one surface.dat row (HydroPlugin.cpp:315-372)

// One slab of the evolution: two consecutive stored time levels ("lo", "hi") of the
// interior lattice, of which the device copied back only what the crossed hypercubes need.
struct Slab {
  int dim;                  // 4 (3+1D) or 3 (2+1D, nz == 1)
  int nx, ny, nz;           // interior points
  double dt, dx, dy, dz;    // hypercube edges (tau, x, y, eta)
  double iso;               // e at freeze-out
  int eos;                  // EoS of T(e), p(e) in the rows
  long long ncubes;         // crossed hypercubes, in the reference's loop order
  const int *cube_key;      // (ix * (ny-1) + iy) * nzc + iz, nzc = nz-1 (4D) or 1 (3D)
  long long npoints;        // lattice points that are corners of crossed hypercubes
  const int *point_cell;    // ix + nx * (iy + ny * iz)
  const double *point_vals; // per point: kVars values at lo, then kVars at hi
};

// How the reference labels a slab's rows: the proper time added to the centroid's tau and
// the factor that multiplies the normal (HydroPlugin.cpp:298-314).
struct Labels {
  double tau_label;
  double tau_scale;
};

struct Result {
  std::vector<double> rows;  // kColumns per element
  std::string text;          // the same rows formatted as the reference writes them
  long long elements = 0;
  long long errors = 0;      // hypercubes where the algorithm stops (the reference exits)
};

// Runs the surface finder on every crossed hypercube of the slab with nthreads host threads,
// in order. cell_to_point is scratch of at least nx*ny*nz entries kept by the caller.
void process_slab(const Slab &s, const Labels &lab, int nthreads, bool want_text, std::vector<int> &cell_to_point,
                  Result &out);

}  // namespace surface
}  // namespace gvh
