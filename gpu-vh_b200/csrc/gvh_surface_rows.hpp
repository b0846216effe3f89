// gvh_surface_rows.hpp -- the surface.dat rows of one crossed hypercube, on the host or on
// the device: cornelius on the corner energies, the reference's interpolation of the fluid
// fields to each element's centroid and its row (HydroPlugin.cpp:283-372, FreezeOut.cpp:1-43,
// 242-280). The host pool (gvh_surface_host.cpp) and the device kernel (gvh_surface_rows.cu)
// run this same code; both are compiled without FMA contraction, so their rows are the same
// to the last bit.
#pragma once

#include <math.h>

#include "gvh_cornelius.hpp"

namespace gvh {
namespace surface {

constexpr int kRowVars = 10;     // u^x u^y u^eta e pi^xx pi^xy pi^x eta pi^yy pi^y eta Pi (FreezeOut.cpp:73-86)
constexpr int kRowColumns = 20;  // one surface.dat row (HydroPlugin.cpp:315-372)
constexpr int kEosConformal = 1; // GVH_EOS_CONFORMAL

// A row whose text the host makes (a number the device's fast %g leaves to the exact path):
// its values, its row index and where its text goes in the slab's text (before byte
// text_off of the device's text).
struct HostRow {
  long long text_off;
  long long row;
  double v[kRowColumns];
};

// What a row needs to know about the slab.
struct RowGeometry {
  int dim;                // 4 (3+1D) or 3 (2+1D)
  int nx, ny, nz;
  double dt, dx, dy, dz;  // hypercube edges (tau, x, y, eta)
  double iso;             // e at freeze-out
  int eos;
  double tau_label;       // added to the centroid's tau (HydroPlugin.cpp:298-314)
  double tau_scale;       // multiplies the normal
};

// p(e), T(e) of the rows in the reference's own host forms (EquationOfState.cu:30-80 and
// 118-148: explicit powers, nested fma for p, a plain sum for T), so that the row columns
// are the values the reference's FP64 build writes.
GVH_HD inline double row_pressure(int eos, double e) {
  if (eos == kEosConformal) return e / 3;
  const double e1 = e, e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e, e7 = e6 * e, e8 = e7 * e;
  const double e9 = e8 * e, e10 = e9 * e, e11 = e10 * e, e12 = e11 * e;
  const double A[13] = {-0.25181736420168666, 9737.845799644809, 1.077580993288114e6,
                        3.1729694865420084e6, 1.6357487344679043e6, 334334.4309240126,
                        41913.439282708554, 6340.448389300905, 141.5073484468774,
                        0.7158279081255019, 0.0009417586777847889, 3.1188455176941583e-7,
                        1.9531729608963267e-11};
  const double B[13] = {45829.44617893836, 4.0574329080826794e6, 2.0931169138134286e7,
                        1.3512402226067686e7, 1.7851642641834426e6, 278581.2989342773,
                        26452.34905933697, 499.04919730607065, 2.3405487982094204,
                        0.002962497695527404, 9.601103399348206e-7, 5.928138360995685e-11,
                        3.2581066229887368e-18};
  const double pw[13] = {1.0, e1, e2, e3, e4, e5, e6, e7, e8, e9, e10, e11, e12};
  double a = A[0], b = B[0];
  for (int k = 1; k <= 12; ++k) {
    a = fma(A[k], pw[k], a);
    b = fma(B[k], pw[k], b);
  }
  return a / b;
}

GVH_HD inline double row_temperature(int eos, double e) {
  if (eos == kEosConformal) return pow(e / 13.8997, 0.25);
  const double e1 = e, e2 = e * e1, e3 = e2 * e1, e4 = e3 * e1, e5 = e4 * e1, e6 = e5 * e1, e7 = e6 * e1;
  const double e8 = e7 * e1, e9 = e8 * e1, e10 = e9 * e1, e11 = e10 * e1;
  return (1.510073201405604e-29 + 8.014062800678687e-18 * e + 2.4954778310451065e-10 * e2 +
          0.000063810382643387 * e3 + 0.4873490574161924 * e4 + 207.48582344326206 * e5 + 6686.07424325115 * e6 +
          14109.766109389702 * e7 + 1471.6180520527757 * e8 + 14.055788949565482 * e9 +
          0.015421252394182246 * e10 + 1.5780479034557783e-6 * e11) /
         (7.558667139355393e-28 + 1.3686372302041508e-16 * e + 2.998130743142826e-9 * e2 +
          0.0005036835870305458 * e3 + 2.316902328874072 * e4 + 578.0778724946719 * e5 +
          11179.193315394154 * e6 + 17965.67607192861 * e7 + 1051.0730543534657 * e8 +
          5.916312075925817 * e9 + 0.003778342768228011 * e10 + 1.8472801679382593e-7 * e11);
}

// Multilinear interpolation inside the hypercube with the term order of FreezeOut.cpp:5-29
// (4D) and :31-43 (3D). a[t][x][y][z] (4D) or a[t][x][y] (3D, packed as a[t][x][y][0]).
GVH_HD inline double row_interp4(double x0, double x1, double x2, double x3, const double a[2][2][2][2]) {
  const double y0 = 1 - x0, y1 = 1 - x1, y2 = 1 - x2, y3 = 1 - x3;
  return (y0 * y1 * y2 * y3 * a[0][0][0][0]) + (x0 * y1 * y2 * y3 * a[1][0][0][0]) +
         (y0 * x1 * y2 * y3 * a[0][1][0][0]) + (y0 * y1 * x2 * y3 * a[0][0][1][0]) +
         (y0 * y1 * y2 * x3 * a[0][0][0][1]) + (x0 * x1 * y2 * y3 * a[1][1][0][0]) +
         (x0 * y1 * x2 * y3 * a[1][0][1][0]) + (x0 * y1 * y2 * x3 * a[1][0][0][1]) +
         (y0 * x1 * x2 * y3 * a[0][1][1][0]) + (y0 * x1 * y2 * x3 * a[0][1][0][1]) +
         (y0 * y1 * x2 * x3 * a[0][0][1][1]) + (x0 * x1 * x2 * y3 * a[1][1][1][0]) +
         (x0 * x1 * y2 * x3 * a[1][1][0][1]) + (x0 * y1 * x2 * x3 * a[1][0][1][1]) +
         (y0 * x1 * x2 * x3 * a[0][1][1][1]) + (x0 * x1 * x2 * x3 * a[1][1][1][1]);
}

GVH_HD inline double row_interp3(double x0, double x1, double x2, const double a[2][2][2][2]) {
  const double y0 = 1 - x0, y1 = 1 - x1, y2 = 1 - x2;
  return (y0 * y1 * y2 * a[0][0][0][0]) + (x0 * y1 * y2 * a[1][0][0][0]) + (y0 * x1 * y2 * a[0][1][0][0]) +
         (y0 * y1 * x2 * a[0][0][1][0]) + (x0 * x1 * y2 * a[1][1][0][0]) + (x0 * y1 * x2 * a[1][0][1][0]) +
         (y0 * x1 * x2 * a[0][1][1][0]) + (x0 * x1 * x2 * a[1][1][1][0]);
}

// Work space of one hypercube (fixed size; on the device it lives in the thread's local
// memory).
struct RowWork {
  iso::Result res;
  // the corner (a, b, k)'s kRowVars values at the lower then the upper time level, read in
  // place from the slab's point table; null for the absent eta layer of a 3-cube
  const double *corner[2][2][2];
  iso::HypercubeWork hw;  // a 3-cube uses its first cube's work space
};

// Field q at the corners, as f[t][a][b][k] (0 for an absent corner).
GVH_HD inline void corner_field(const RowWork &w, int q, double f[2][2][2][2]) {
  for (int t = 0; t < 2; ++t)
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 2; ++k) f[t][a][b][k] = w.corner[a][b][k] ? w.corner[a][b][k][t * kRowVars + q] : 0.0;
}

// The rows of hypercube `key` ((ix (ny-1) + iy) nzc + iz) whose corners the caller has set
// (gather_corners). Writes up to kMaxElements rows of kRowColumns values to rows and returns
// how many, or a negative cornelius error.
GVH_HD inline int cube_rows(const RowGeometry &g, int key, RowWork &w, double *rows) {
  const int nzc = g.dim == 4 ? g.nz - 1 : 1;
  const int iz = key % nzc;
  const int iy = (key / nzc) % (g.ny - 1);
  const int ix = key / nzc / (g.ny - 1);
  int rc;
  double e4[2][2][2][2];
  corner_field(w, 3, e4);
  if (g.dim == 4) {
    const double dx4[4] = {g.dt, g.dx, g.dy, g.dz};
    rc = iso::find_4d(e4, dx4, g.iso, w.res, w.hw);
  } else {
    double v3[2][2][2];
    for (int t = 0; t < 2; ++t)
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) v3[t][a][b] = e4[t][a][b][0];
    // cornelius is set up with the spacings of the dimensions in use (HydroPlugin.cpp
    // :155-182); in 3D its first axis has unit length and is not used
    const double dx3[4] = {1.0, g.dt, g.dx, g.dy};
    rc = iso::find_3d(v3, dx3, g.iso, w.res, w.hw.cube[0]);
  }
  if (rc) return rc;
  const double cell_x = (double)ix * g.dx - (((double)(g.nx - 1)) / 2.0 * g.dx);
  const double cell_y = (double)iy * g.dy - (((double)(g.ny - 1)) / 2.0 * g.dy);
  const double cell_z = (double)iz * g.dz - (((double)(g.nz - 1)) / 2.0 * g.dz);
  const iso::Result &res = w.res;
  for (int i = 0; i < res.n; ++i) {
    // element components in the frame of the cube's own axes (tau, x, y[, eta])
    double cen[4], nrm[4];
    if (g.dim == 4) {
      for (int k = 0; k < 4; ++k) { cen[k] = res.centroid[i][k]; nrm[k] = res.normal[i][k]; }
    } else {
      for (int k = 0; k < 3; ++k) { cen[k] = res.centroid[i][k + 1]; nrm[k] = res.normal[i][k + 1]; }
      cen[3] = 0.0;
      nrm[3] = 0.0;
    }
    const double tf = cen[0] / g.dt, xf = cen[1] / g.dx, yf = cen[2] / g.dy;
    const double zf = g.dim == 4 ? cen[3] / g.dz : 0.0;
    double *row = rows + i * kRowColumns;
    row[0] = cen[0] + g.tau_label;
    row[1] = cen[1] + cell_x;
    row[2] = cen[2] + cell_y;
    row[3] = g.dim == 4 ? cen[3] + cell_z : cell_z;
    for (int k = 0; k < 3; ++k) row[4 + k] = g.tau_scale * nrm[k];
    row[7] = g.dim == 4 ? g.tau_scale * nrm[3] : 0.0;
    double val[kRowVars];
    for (int q = 0; q < kRowVars; ++q) {
      double f[2][2][2][2];
      corner_field(w, q, f);
      val[q] = g.dim == 4 ? row_interp4(tf, xf, yf, zf, f) : row_interp3(tf, xf, yf, f);
    }
    row[8] = val[0];
    row[9] = val[1];
    row[10] = val[2];
    row[11] = val[3];
    row[12] = row_temperature(g.eos, val[3]);
    row[13] = row_pressure(g.eos, val[3]);
    for (int q = 4; q < kRowVars; ++q) row[10 + q] = val[q];
  }
  return res.n;
}

// Points w's corners of hypercube `key` at the slab's point table: c2p maps a lattice cell
// to its point, point_vals holds kRowVars values at the lower then the upper level per point.
GVH_HD inline void gather_corners(const RowGeometry &g, int key, const int *c2p, const double *point_vals,
                                  RowWork &w) {
  const int nzc = g.dim == 4 ? g.nz - 1 : 1;
  const int iz = key % nzc;
  const int iy = (key / nzc) % (g.ny - 1);
  const int ix = key / nzc / (g.ny - 1);
  const int nzk = g.dim == 4 ? 2 : 1;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int k = 0; k < 2; ++k) {
        if (k >= nzk) {
          w.corner[a][b][k] = nullptr;
          continue;
        }
        const int cell = (ix + a) + g.nx * ((iy + b) + g.ny * (iz + k));
        w.corner[a][b][k] = point_vals + (size_t)c2p[cell] * (2 * kRowVars);
      }
}

}  // namespace surface
}  // namespace gvh
