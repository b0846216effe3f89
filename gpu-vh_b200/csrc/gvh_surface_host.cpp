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
#include "gvh_surface_rows.hpp"
#include "gvh_surface_internal.h"

namespace gvh {
namespace surface {
namespace {

static_assert(kVars == kRowVars && kColumns == kRowColumns, "row layout");

RowGeometry row_geometry(const Slab &s, const Labels &lab) {
  RowGeometry g;
  g.dim = s.dim;
  g.nx = s.nx; g.ny = s.ny; g.nz = s.nz;
  g.dt = s.dt; g.dx = s.dx; g.dy = s.dy; g.dz = s.dz;
  g.iso = s.iso;
  g.eos = s.eos;
  g.tau_label = lab.tau_label;
  g.tau_scale = lab.tau_scale;
  return g;
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
  const RowGeometry g = row_geometry(s, lab);
  RowWork w;
  double rows[iso::kMaxElements * kColumns];
  for (long long c = c0; c < c1; ++c) {
    const int key = s.cube_key[c];
    gather_corners(g, key, c2p.data(), s.point_vals, w);
    const int n = cube_rows(g, key, w, rows);
    if (n < 0) {
      ++part.errors;
      continue;
    }
    for (int i = 0; i < n; ++i) {
      const double *row = rows + i * kColumns;
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

void Pool::start(int n, std::function<void(int)> f) {
  if (n <= 0) return;
  if (workers_.empty()) {  // no workers: do it now
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::unique_lock<std::mutex> lock(mu_);
  owned_ = std::move(f);
  job_ = &owned_;
  njobs_ = n;
  next_ = 0;
  pending_ = n;
  ++generation_;
  wake_.notify_all();
}

void Pool::wait() {
  std::unique_lock<std::mutex> lock(mu_);
  done_.wait(lock, [&] { return pending_ == 0; });
  job_ = nullptr;
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

void format_rows(const double *rows, long long n, Pool &pool, int outputs, Result &out, bool async,
                 const DeviceText &dt) {
  out.elements = n;
  out.errors = 0;
  out.joined_valid = false;
  if (n == 0) {
    out.parts.clear();
    return;
  }
  const bool text = outputs & OUT_TEXT, device_text = text && dt.text;
  const long long work = device_text ? (dt.bytes + dt.n_host * 240) / 65536 : n / 256;
  const int nparts = (int)std::max<long long>(1, std::min<long long>(4ll * pool.size(), work));
  out.parts.resize(nparts);
  Result *res = &out;
  DeviceText d = dt;
  auto job = [rows, n, nparts, outputs, res, text, device_text, d](int i) {
    if (d.ready) d.ready();
    Part &part = res->parts[i];
    part.rows.clear();
    part.text.clear();
    const long long r0 = n * i / nparts, r1 = n * (i + 1) / nparts;
    part.elements = r1 - r0;
    part.errors = 0;
    if (outputs & OUT_ROWS) part.rows.assign(rows + r0 * kColumns, rows + r1 * kColumns);
    if (!text) return;
    if (!device_text) {
      part.text.reserve((size_t)(r1 - r0) * 240);
      for (long long r = r0; r < r1; ++r) append_row_text(part.text, rows + r * kColumns);
      return;
    }
    // bytes [lo, hi) of the device's text, with the host rows that go before byte lo .. hi - 1
    // (and, in the last part, those at the end)
    const long long lo = d.bytes * i / nparts, hi = d.bytes * (i + 1) / nparts;
    const HostRow *hb = d.host_rows, *he = d.host_rows + d.n_host;
    auto first_at = [](const HostRow *b, const HostRow *e, long long off) {
      return std::lower_bound(b, e, off, [](const HostRow &h, long long o) { return h.text_off < o; });
    };
    const HostRow *h0 = first_at(hb, he, lo), *h1 = i + 1 == nparts ? he : first_at(hb, he, hi);
    part.text.reserve((size_t)(hi - lo) + (size_t)(h1 - h0) * 240);
    long long pos = lo;
    for (const HostRow *h = h0; h < h1; ++h) {
      part.text.append(d.text + pos, (size_t)(h->text_off - pos));
      append_row_text(part.text, h->v);
      pos = h->text_off;
    }
    part.text.append(d.text + pos, (size_t)(hi - pos));
  };
  if (async) pool.start(nparts, job);
  else pool.run(nparts, job);
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
