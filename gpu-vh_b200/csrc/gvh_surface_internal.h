// gvh_surface_internal.h -- what the device side of the freeze-out surface hands to the host.
#pragma once

#include <condition_variable>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gvh_surface_rows.hpp"

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

enum : int { OUT_ROWS = 1, OUT_TEXT = 2 };

// One thread's share of a slab's rows, in order.
struct Part {
  std::vector<double> rows;  // kColumns per element
  std::string text;          // the same rows formatted as the reference writes them
  long long elements = 0;
  long long errors = 0;      // hypercubes where the algorithm stops (the reference exits)
};

struct Result {
  std::vector<Part> parts;
  long long elements = 0, errors = 0;
  std::string joined;        // the parts' text in one piece, made on first request
  bool joined_valid = false;
  const std::string &text() {
    if (!joined_valid) {
      size_t n = 0;
      for (auto &p : parts) n += p.text.size();
      joined.clear();
      joined.reserve(n);
      for (auto &p : parts) joined += p.text;
      joined_valid = true;
    }
    return joined;
  }
};

// Persistent host worker threads: run(n, f) calls f(0..n-1) on the workers and waits.
class Pool {
 public:
  explicit Pool(int nthreads);
  ~Pool();
  int size() const { return (int)workers_.size() + 1; }
  void run(int n, const std::function<void(int)> &f);
  // start(): f(0..n-1) on the workers only, returning at once (inline when there are no
  // workers); wait(): until a started job is done. A pool runs one job at a time.
  void start(int n, std::function<void(int)> f);
  void wait();

 private:
  void loop();
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable wake_, done_;
  const std::function<void(int)> *job_ = nullptr;
  std::function<void(int)> owned_;  // the started job
  int njobs_ = 0, next_ = 0, pending_ = 0;
  long long generation_ = 0;
  bool stop_ = false;
};

// The device's text of a slab (gvh_surface_rows.cu): its rows' text in order with the host
// rows left out, and the host rows, sorted by row.
struct DeviceText {
  const char *text = nullptr;
  long long bytes = 0;
  const HostRow *host_rows = nullptr;
  long long n_host = 0;
  std::function<void()> ready;  // each job calls it before reading text (the copy's wait)
};

// Formats rows the device produced (n rows of kColumns) into out's parts on the pool, in
// order; keeps the rows too when outputs has OUT_ROWS. With dt.text the text is the device's,
// with the host rows formatted here and spliced in (rows may then be null unless OUT_ROWS).
// Each job calls dt.ready first, when set. With async the work is started on the pool's
// workers and format_rows returns at once: pool.wait() before reading out or reusing rows or
// the device text.
void format_rows(const double *rows, long long n, Pool &pool, int outputs, Result &out, bool async,
                 const DeviceText &dt);

// Runs the surface finder on every crossed hypercube of the slab on the pool, in order.
// outputs: OUT_ROWS and/or OUT_TEXT. cell_to_point is scratch of at least nx*ny*nz entries
// kept by the caller.
void process_slab(const Slab &s, const Labels &lab, Pool &pool, int outputs, std::vector<int> &cell_to_point,
                  Result &out);

}  // namespace surface
}  // namespace gvh

struct gvh_surface;

namespace gvh {
namespace surface {
// Moves the last slab's text, part by part and in order, to the end of out (for writers that
// keep a chunk of slabs before writing, as gvh_run does); the slab's text is empty afterwards.
void take_text(gvh_surface *s, std::vector<std::string> &out);
}  // namespace surface
}  // namespace gvh
