// gvh_surface_host.cpp -- host half of the freeze-out hypersurface: cornelius on the
// hypercubes the device marked, the reference's interpolation of the fluid fields to each
// element's centroid, and the surface.dat row (HydroPlugin.cpp:283-393, FreezeOut.cpp:1-43,
// 242-280). Also the stand-alone gvh_cornelius entry point.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <charconv>
#include <thread>

#include "../../include/gvh.h"
#include "gvh_cornelius.hpp"
#include "gvh_format.hpp"
#include "gvh_surface_internal.h"

namespace gvh {
namespace surface {
namespace {

// p(e), T(e) of the rows in the reference's own host forms (EquationOfState.cu:30-80 and
// 118-148: explicit powers, nested fma for p, a plain sum for T), so that the row columns
// are the values the reference's FP64 build writes.
double eos_pressure(int eos, double e) {
  if (eos == GVH_EOS_CONFORMAL) return e / 3;
  const double e1 = e, e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e, e7 = e6 * e, e8 = e7 * e;
  const double e9 = e8 * e, e10 = e9 * e, e11 = e10 * e, e12 = e11 * e;
  static const double A[13] = {-0.25181736420168666, 9737.845799644809, 1.077580993288114e6,
                               3.1729694865420084e6, 1.6357487344679043e6, 334334.4309240126,
                               41913.439282708554, 6340.448389300905, 141.5073484468774,
                               0.7158279081255019, 0.0009417586777847889, 3.1188455176941583e-7,
                               1.9531729608963267e-11};
  static const double B[13] = {45829.44617893836, 4.0574329080826794e6, 2.0931169138134286e7,
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

double eos_temperature(int eos, double e) {
  if (eos == GVH_EOS_CONFORMAL) return pow(e / 13.8997, 0.25);
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
double interp4(double x0, double x1, double x2, double x3, const double a[2][2][2][2]) {
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

double interp3(double x0, double x1, double x2, const double a[2][2][2][2]) {
  const double y0 = 1 - x0, y1 = 1 - x1, y2 = 1 - x2;
  return (y0 * y1 * y2 * a[0][0][0][0]) + (x0 * y1 * y2 * a[1][0][0][0]) + (y0 * x1 * y2 * a[0][1][0][0]) +
         (y0 * y1 * x2 * a[0][0][1][0]) + (x0 * x1 * y2 * a[1][1][0][0]) + (x0 * y1 * x2 * a[1][0][1][0]) +
         (y0 * x1 * x2 * a[0][1][1][0]) + (x0 * x1 * x2 * a[1][1][1][0]);
}

// One row as the reference's ofstream writes it: default format (%g, 6 significant digits),
// values separated by spaces, a newline after the last (gvh_format.hpp: the same characters
// as printf's %g).
void append_row_text(std::string &out, const double *row) {
  char buf[kColumns * 32];
  char *p = buf;
  for (int c = 0; c < kColumns; ++c) {
    p = fmt::g6(p, buf + sizeof buf, row[c]);
    *p++ = c + 1 < kColumns ? ' ' : '\n';
  }
  out.append(buf, p - buf);
}

void process_range(const Slab &s, const Labels &lab, int outputs, const std::vector<int> &c2p, long long c0,
                   long long c1, Part &part) {
  const bool want_rows = outputs & OUT_ROWS, want_text = outputs & OUT_TEXT;
  part.rows.clear();
  part.text.clear();
  part.elements = part.errors = 0;
  const size_t expect = (size_t)((c1 - c0) * 5 / 4 + 8);  // about one element per hypercube
  if (want_rows) part.rows.reserve(expect * kColumns);
  if (want_text) part.text.reserve(expect * 240);
  const int nzc = s.dim == 4 ? s.nz - 1 : 1;
  const double dx4[4] = {s.dt, s.dx, s.dy, s.dim == 4 ? s.dz : 1.0};
  // cornelius is set up with the spacings of the dimensions in use (HydroPlugin.cpp:155-182);
  // in 3D its first axis has unit length and is not used
  const double dx3[4] = {1.0, s.dt, s.dx, s.dy};
  iso::Result res;
  iso::HypercubeWork hw;
  iso::CubeWork cw;
  double v4[2][2][2][2];
  double v3[2][2][2];
  double f[kVars][2][2][2][2];
  for (long long c = c0; c < c1; ++c) {
    const int key = s.cube_key[c];
    const int iz = key % nzc;
    const int iy = (key / nzc) % (s.ny - 1);
    const int ix = key / nzc / (s.ny - 1);
    const int nzk = s.dim == 4 ? 2 : 1;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 2; ++k) {
          if (k >= nzk) {
            for (int t = 0; t < 2; ++t)
              for (int q = 0; q < kVars; ++q) f[q][t][a][b][k] = 0.0;
            continue;
          }
          const int cell = (ix + a) + s.nx * ((iy + b) + s.ny * (iz + k));
          const double *pv = s.point_vals + (size_t)c2p[cell] * (2 * kVars);
          for (int t = 0; t < 2; ++t)
            for (int q = 0; q < kVars; ++q) f[q][t][a][b][k] = pv[t * kVars + q];
        }
    int rc;
    if (s.dim == 4) {
      for (int t = 0; t < 2; ++t)
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 2; ++k) v4[t][a][b][k] = f[3][t][a][b][k];
      rc = iso::find_4d(v4, dx4, s.iso, res, hw);
    } else {
      for (int t = 0; t < 2; ++t)
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) v3[t][a][b] = f[3][t][a][b][0];
      rc = iso::find_3d(v3, dx3, s.iso, res, cw);
    }
    if (rc) {
      ++part.errors;
      continue;
    }
    const double cell_x = (double)ix * s.dx - (((double)(s.nx - 1)) / 2.0 * s.dx);
    const double cell_y = (double)iy * s.dy - (((double)(s.ny - 1)) / 2.0 * s.dy);
    const double cell_z = (double)iz * s.dz - (((double)(s.nz - 1)) / 2.0 * s.dz);
    for (int i = 0; i < res.n; ++i) {
      // element components in the frame of the cube's own axes (tau, x, y[, eta])
      double cen[4], nrm[4];
      if (s.dim == 4) {
        for (int k = 0; k < 4; ++k) { cen[k] = res.centroid[i][k]; nrm[k] = res.normal[i][k]; }
      } else {
        for (int k = 0; k < 3; ++k) { cen[k] = res.centroid[i][k + 1]; nrm[k] = res.normal[i][k + 1]; }
        cen[3] = 0.0;
        nrm[3] = 0.0;
      }
      const double tf = cen[0] / s.dt, xf = cen[1] / s.dx, yf = cen[2] / s.dy;
      const double zf = s.dim == 4 ? cen[3] / s.dz : 0.0;
      double row[kColumns];
      row[0] = cen[0] + lab.tau_label;
      row[1] = cen[1] + cell_x;
      row[2] = cen[2] + cell_y;
      row[3] = s.dim == 4 ? cen[3] + cell_z : cell_z;
      for (int k = 0; k < 3; ++k) row[4 + k] = lab.tau_scale * nrm[k];
      row[7] = s.dim == 4 ? lab.tau_scale * nrm[3] : 0.0;
      double val[kVars];
      for (int q = 0; q < kVars; ++q) val[q] = s.dim == 4 ? interp4(tf, xf, yf, zf, f[q]) : interp3(tf, xf, yf, f[q]);
      row[8] = val[0];
      row[9] = val[1];
      row[10] = val[2];
      row[11] = val[3];
      row[12] = eos_temperature(s.eos, val[3]);
      row[13] = eos_pressure(s.eos, val[3]);
      for (int q = 4; q < kVars; ++q) row[10 + q] = val[q];
      if (want_rows) part.rows.insert(part.rows.end(), row, row + kColumns);
      if (want_text) append_row_text(part.text, row);
      ++part.elements;
    }
  }
}

}  // namespace

Pool::Pool(int nthreads) {
  for (int i = 1; i < nthreads; ++i) workers_.emplace_back([this] { loop(); });
}

Pool::~Pool() {
  {
    std::lock_guard<std::mutex> lock(mu_);
    stop_ = true;
  }
  wake_.notify_all();
  for (auto &t : workers_) t.join();
}

void Pool::loop() {
  long long seen = 0;
  std::unique_lock<std::mutex> lock(mu_);
  for (;;) {
    wake_.wait(lock, [&] { return stop_ || generation_ != seen; });
    if (stop_) return;
    seen = generation_;
    while (next_ < njobs_) {
      const int i = next_++;
      const std::function<void(int)> *f = job_;
      lock.unlock();
      (*f)(i);
      lock.lock();
      if (--pending_ == 0) done_.notify_all();
    }
  }
}

void Pool::run(int n, const std::function<void(int)> &f) {
  if (n <= 0) return;
  std::unique_lock<std::mutex> lock(mu_);
  job_ = &f;
  njobs_ = n;
  next_ = 0;
  pending_ = n;
  ++generation_;
  wake_.notify_all();
  while (next_ < njobs_) {  // the calling thread works too
    const int i = next_++;
    lock.unlock();
    f(i);
    lock.lock();
    --pending_;
  }
  done_.wait(lock, [&] { return pending_ == 0; });
  job_ = nullptr;
}

void process_slab(const Slab &s, const Labels &lab, Pool &pool, int outputs, std::vector<int> &c2p, Result &out) {
  out.elements = 0;
  out.errors = 0;
  out.joined_valid = false;
  if (s.ncubes == 0) {
    out.parts.clear();
    return;
  }
  const size_t ncells = (size_t)s.nx * s.ny * s.nz;
  if (c2p.size() < ncells) c2p.assign(ncells, 0);
  for (long long p = 0; p < s.npoints; ++p) c2p[s.point_cell[p]] = (int)p;
  // a few contiguous ranges per thread for balance; range i becomes part i, so order is kept
  const long long min_range = 256;
  const int nparts = (int)std::max<long long>(1, std::min<long long>(4ll * pool.size(), s.ncubes / min_range));
  out.parts.resize(nparts);
  pool.run(nparts, [&](int i) {
    const long long c0 = s.ncubes * i / nparts, c1 = s.ncubes * (i + 1) / nparts;
    process_range(s, lab, outputs, c2p, c0, c1, out.parts[i]);
  });
  for (auto &p : out.parts) {
    out.elements += p.elements;
    out.errors += p.errors;
  }
}

}  // namespace surface
}  // namespace gvh

extern "C" {

int gvh_cornelius(int dim, const double *corners, const double *dx, double iso_value, double *centroids,
                  double *normals, int max_elements, int *n_elements) {
  if (!corners || !dx || !n_elements || (dim != 2 && dim != 3 && dim != 4)) return GVH_ERR_INVALID;
  *n_elements = 0;
  double dx4[4] = {1.0, 1.0, 1.0, 1.0};
  for (int k = 0; k < dim; ++k) dx4[4 - dim + k] = dx[k];
  gvh::iso::Result r;
  int rc;
  if (dim == 2) {
    double v[2][2];
    memcpy(v, corners, sizeof v);
    rc = gvh::iso::find_2d(v, dx4, iso_value, r);
  } else if (dim == 3) {
    double v[2][2][2];
    memcpy(v, corners, sizeof v);
    gvh::iso::CubeWork cw;
    rc = gvh::iso::find_3d(v, dx4, iso_value, r, cw);
  } else {
    double v[2][2][2][2];
    memcpy(v, corners, sizeof v);
    static thread_local gvh::iso::HypercubeWork hw;
    rc = gvh::iso::find_4d(v, dx4, iso_value, r, hw);
  }
  if (rc == gvh::iso::ERR_OVERFLOW) return GVH_ERR_INVALID;
  if (rc) return GVH_ERR_NUMERIC;
  if (r.n > max_elements || (r.n > 0 && (!centroids || !normals))) {
    *n_elements = r.n;
    return GVH_ERR_INVALID;
  }
  for (int i = 0; i < r.n; ++i)
    for (int k = 0; k < dim; ++k) {
      centroids[i * dim + k] = r.centroid[i][4 - dim + k];
      normals[i * dim + k] = r.normal[i][4 - dim + k];
    }
  *n_elements = r.n;
  return GVH_OK;
}

}  // extern "C"
