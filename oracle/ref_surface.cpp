// ref_surface.cpp -- test infrastructure: the freeze-out part of the reference's run loop,
// replayed on the state of the CPU build of the reference (ref_driver.cpp), with the
// reference's own FreezeOut.cpp, Memory.cpp and cornelius (included from the reference tree
// as HydroPlugin.cpp:21-23 includes them). The surface.dat it writes is the checker for the
// library's gvh_surface_* / gvh_run output.
//
// Restated from HydroPlugin.cpp: the set-up of lines 155-211 and, per loop iteration n, the
// block of lines 256-393 (store the level, run the finder every FOFREQ steps, write rows).
#include <fstream>

#include "DynamicalVariables.cuh"
#include "EquationOfState.cuh"
#include "cornelius-c++-1.3/cornelius.cpp"
#include "FreezeOut.cpp"
#include "Memory.cpp"

void gvh_ref_current(CONSERVED_VARIABLES **q, PRECISION **e, FLUID_VELOCITY **u);  // ref_driver.cpp

namespace {

const int kFoFreq = 10;  // FOFREQ, HydroPlugin.cpp:40

struct Replay {
  int nx, ny, nz, dim;
  double t0, dt, dx, dy, dz;
  double lattice_spacing[4];
  Cornelius cor;
  double ****eev;
  double *****hev;
  double ****hc4;
  double ***hc3;
  std::ofstream out;
  long long rows;
};

}  // namespace

extern "C" {

/* The lattice of the last gvh_ref_init; spacings as run() takes them from LatticeParameters
 * (HydroPlugin.cpp:124-128), e_fo = e(T_fo) (HydroPlugin.cpp:135). */
void *gvh_ref_surface_begin(int nx, int ny, int nz, double t0, double dt, double dx, double dy, double dz,
                            double e_fo, const char *path) {
  Replay *r = new Replay();
  r->nx = nx; r->ny = ny; r->nz = nz;
  r->t0 = t0; r->dt = dt; r->dx = dx; r->dy = dy; r->dz = dz;
  r->rows = 0;
  if (r->nx > 1 && r->ny > 1 && r->nz > 1) {
    r->dim = 4;
    double ls[4] = {r->dt, r->dx, r->dy, r->dz};
    for (int k = 0; k < 4; ++k) r->lattice_spacing[k] = ls[k];
  } else if (r->nx > 1 && r->ny > 1 && r->nz < 2) {
    r->dim = 3;
    double ls[3] = {r->dt, r->dx, r->dy};
    for (int k = 0; k < 3; ++k) r->lattice_spacing[k] = ls[k];
  } else {
    delete r;
    return nullptr;
  }
  r->cor.init(r->dim, e_fo, r->lattice_spacing);
  r->eev = calloc4dArray(r->eev, kFoFreq + 1, r->nx, r->ny, r->nz);
  r->hev = calloc5dArray(r->hev, 10, kFoFreq + 1, r->nx, r->ny, r->nz);
  r->hc4 = calloc4dArray(r->hc4, 2, 2, 2, 2);
  r->hc3 = calloc3dArray(r->hc3, 2, 2, 2);
  r->out.open(path, std::ios::out);
  return r;
}

/* Iteration n of the loop (state = level n-1, t = t0 + (n-1) dt as the loop keeps it). */
long long gvh_ref_surface_iteration(void *handle, int n, double t) {
  Replay *r = static_cast<Replay *>(handle);
  CONSERVED_VARIABLES *q;
  PRECISION *e;
  FLUID_VELOCITY *u;
  gvh_ref_current(&q, &e, &u);
  const int nx = r->nx, ny = r->ny, nz = r->nz, dim = r->dim;
  const double t0 = r->t0, dt = r->dt, dx = r->dx, dy = r->dy, dz = r->dz;
  int nFO = n % kFoFreq;
  if (nFO == 0) swapAndSetHydroVariables(r->eev, r->hev, q, e, u, nx, ny, nz, kFoFreq);
  else setHydroVariables(r->eev, r->hev, q, e, u, nx, ny, nz, kFoFreq, n);
  int start = (n <= kFoFreq) ? 2 : 0;
  long long written = 0;
  if (nFO == kFoFreq - 1) {
    int dimZ = dim == 4 ? nz - 1 : 1;
    for (int it = start; it < kFoFreq; it++)
      for (int ix = 0; ix < nx - 1; ix++)
        for (int iy = 0; iy < ny - 1; iy++)
          for (int iz = 0; iz < dimZ; iz++) {
            if (dim == 4) writeEnergyDensityToHypercube4D(r->hc4, r->eev, it, ix, iy, iz);
            else writeEnergyDensityToHypercube3D(r->hc3, r->eev, it, ix, iy);
            if (dim == 4) r->cor.find_surface_4d(r->hc4);
            else r->cor.find_surface_3d(r->hc3);
            for (int i = 0; i < r->cor.get_Nelements(); i++) {
              double cell_tau;
              if (n <= kFoFreq) cell_tau = t0 + ((double)(n - kFoFreq + (it - 1))) * dt;
              else cell_tau = t0 + ((double)(n - kFoFreq + it)) * dt;
              double cell_x = (double)ix * dx - (((double)(nx - 1)) / 2.0 * dx);
              double cell_y = (double)iy * dy - (((double)(ny - 1)) / 2.0 * dy);
              double cell_z = (double)iz * dz - (((double)(nz - 1)) / 2.0 * dz);
              double tau_frac = r->cor.get_centroid_elem(i, 0) / r->lattice_spacing[0];
              double x_frac = r->cor.get_centroid_elem(i, 1) / r->lattice_spacing[1];
              double y_frac = r->cor.get_centroid_elem(i, 2) / r->lattice_spacing[2];
              double z_frac = dim == 4 ? r->cor.get_centroid_elem(i, 3) / r->lattice_spacing[3] : 0.0;
              std::ofstream &f = r->out;
              f << r->cor.get_centroid_elem(i, 0) + cell_tau << " ";
              f << r->cor.get_centroid_elem(i, 1) + cell_x << " ";
              f << r->cor.get_centroid_elem(i, 2) + cell_y << " ";
              if (dim == 4) f << r->cor.get_centroid_elem(i, 3) + cell_z << " ";
              else f << cell_z << " ";
              f << t * r->cor.get_normal_elem(i, 0) << " ";
              f << t * r->cor.get_normal_elem(i, 1) << " ";
              f << t * r->cor.get_normal_elem(i, 2) << " ";
              if (dim == 4) f << t * r->cor.get_normal_elem(i, 3) << " ";
              else f << 0.0 << " ";
              double v;
              for (int ivar = 0; ivar < 3; ivar++) {
                v = dim == 4 ? interpolateVariable4D(r->hev, ivar, it, ix, iy, iz, tau_frac, x_frac, y_frac, z_frac)
                             : interpolateVariable3D(r->hev, ivar, it, ix, iy, tau_frac, x_frac, y_frac);
                f << v << " ";
              }
              v = dim == 4 ? interpolateVariable4D(r->hev, 3, it, ix, iy, iz, tau_frac, x_frac, y_frac, z_frac)
                           : interpolateVariable3D(r->hev, 3, it, ix, iy, tau_frac, x_frac, y_frac);
              f << v << " ";
              f << effectiveTemperature(v) << " ";
              f << equilibriumPressure(v) << " ";
              for (int ivar = 4; ivar < 9; ivar++) {
                v = dim == 4 ? interpolateVariable4D(r->hev, ivar, it, ix, iy, iz, tau_frac, x_frac, y_frac, z_frac)
                             : interpolateVariable3D(r->hev, ivar, it, ix, iy, tau_frac, x_frac, y_frac);
                f << v << " ";
              }
              v = dim == 4 ? interpolateVariable4D(r->hev, 9, it, ix, iy, iz, tau_frac, x_frac, y_frac, z_frac)
                           : interpolateVariable3D(r->hev, 9, it, ix, iy, tau_frac, x_frac, y_frac);
              f << v << std::endl;
              ++written;
            }
          }
  }
  r->rows += written;
  return written;
}

long long gvh_ref_surface_end(void *handle) {
  Replay *r = static_cast<Replay *>(handle);
  if (!r) return -1;
  long long rows = r->rows;
  r->out.close();
  delete r;  // the host arrays are left to the process (the reference never frees them either)
  return rows;
}

}  // extern "C"
