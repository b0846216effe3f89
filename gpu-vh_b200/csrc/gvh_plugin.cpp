// gvh_plugin.cpp -- the host side around the KT step: the reference's run-time inputs and
// its run loop, in C++ over the C ABI of gvh.h.
//
//   gvh_read_lattice_parameters / gvh_read_hydro_parameters / gvh_read_ic_parameters
//       the positional .properties readers (LatticeParameters.cpp:65-138,
//       HydroParameters.cpp:49-98, InitialConditionParameters.cpp:65-149): line n is field
//       n, whitespace is dropped, the value is what follows '='; missing lines leave 0.
//   gvh_read_ic_files
//       the type-10 initial-condition reader (InitialConditions.cpp:98-489): one
//       "x y z value" file per field under <root>/input/, i outermost and k innermost, each
//       value scanned as a float; e gets +1e-3 (InitialConditions.cpp:124).
//   gvh_run
//       HydroPlugin.cpp:107-434 for initial-condition type 10: set-up, then per step the
//       field dump every FREQ = 10 steps (FileIO.cpp:15-60 format), the stop test (11
//       checks with every cell at or below e(T_fo), HydroPlugin.cpp:396-413) and one RK2
//       step. The state stays on the device: the stop test is a device reduction and only
//       dumps copy fields back (the reference copies 30 arrays back every step).
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <fstream>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gvh.h"
#include "gvh_handle.h"
#include "gvh_surface_internal.h"

namespace {

thread_local std::string g_plugin_error;

int pfail(int code, const std::string &msg) {
  g_plugin_error = msg;
  return code;
}

// One positional .properties file: the value of each line (text after '=', whitespace
// removed), in order.
bool read_properties(const std::string &path, std::vector<std::string> &values) {
  std::ifstream in(path);
  if (!in.is_open()) return false;
  std::string line;
  while (std::getline(in, line)) {
    line.erase(std::remove_if(line.begin(), line.end(), [](unsigned char c) { return std::isspace(c); }),
               line.end());
    size_t pos = line.find('=');
    values.push_back(pos == std::string::npos ? line : line.substr(pos + 1));
  }
  return true;
}

double num(const std::vector<std::string> &v, size_t i) { return i < v.size() ? atof(v[i].c_str()) : 0.0; }
int inum(const std::vector<std::string> &v, size_t i) { return i < v.size() ? atoi(v[i].c_str()) : 0; }

constexpr double kHbarc = 0.197326938;  // HydroPlugin.cpp:132
constexpr int kFreq = 10;                // HydroPlugin.cpp:39
constexpr int kFreezeoutChecks = 11;     // FOFREQ + 1, HydroPlugin.cpp:409

long long ghost_index(int i, int j, int k, int nx, int ny) {
  return (long long)i + (long long)(nx + 4) * (j + (long long)(ny + 4) * k);
}

}  // namespace

extern "C" {

const char *gvh_plugin_last_error(void) { return g_plugin_error.c_str(); }

int gvh_read_lattice_parameters(const char *config_dir, gvh_lattice_params *out) {
  if (!config_dir || !out) return pfail(GVH_ERR_INVALID, "null argument");
  std::vector<std::string> v;
  if (!read_properties(std::string(config_dir) + "/lattice.properties", v))
    return pfail(GVH_ERR_INVALID, std::string("cannot open ") + config_dir + "/lattice.properties");
  out->numLatticePointsX = inum(v, 0);
  out->numLatticePointsY = inum(v, 1);
  out->numLatticePointsRapidity = inum(v, 2);
  out->numProperTimePoints = inum(v, 3);
  out->latticeSpacingX = num(v, 4);
  out->latticeSpacingY = num(v, 5);
  out->latticeSpacingRapidity = num(v, 6);
  out->latticeSpacingProperTime = num(v, 7);
  out->numComputationalLatticePointsX = out->numLatticePointsX + 4;  // N_GHOST_CELLS
  out->numComputationalLatticePointsY = out->numLatticePointsY + 4;
  out->numComputationalLatticePointsRapidity = out->numLatticePointsRapidity + 4;
  return GVH_OK;
}

int gvh_read_hydro_parameters(const char *config_dir, gvh_hydro_params *out) {
  if (!config_dir || !out) return pfail(GVH_ERR_INVALID, "null argument");
  std::vector<std::string> v;
  if (!read_properties(std::string(config_dir) + "/hydro.properties", v))
    return pfail(GVH_ERR_INVALID, std::string("cannot open ") + config_dir + "/hydro.properties");
  out->initialProperTimePoint = num(v, 0);
  out->shearViscosityToEntropyDensity = num(v, 1);
  out->freezeoutTemperatureGeV = num(v, 2);
  out->initializePimunuNavierStokes = inum(v, 3);
  out->regulationTemperatureGeV = num(v, 4);  // absent in the shipped file: stays 0
  return GVH_OK;
}

int gvh_read_ic_parameters(const char *config_dir, gvh_ic_params *out) {
  if (!config_dir || !out) return pfail(GVH_ERR_INVALID, "null argument");
  std::vector<std::string> v;
  if (!read_properties(std::string(config_dir) + "/ic.properties", v))
    return pfail(GVH_ERR_INVALID, std::string("cannot open ") + config_dir + "/ic.properties");
  // line order of InitialConditionParameters.cpp:65-149 (not the struct's member order)
  out->initialConditionType = inum(v, 0);
  out->numberOfSourceFiles = inum(v, 1);
  out->numberOfNucleonsPerNuclei = inum(v, 2);
  out->initialEnergyDensity = num(v, 3);
  out->scatteringCrossSectionNN = num(v, 4);
  out->impactParameter = num(v, 5);
  out->fractionOfBinaryCollisions = num(v, 6);
  out->rapidityVariance = num(v, 7);
  out->rapidityMean = num(v, 8);
  out->sourceType = inum(v, 9);
  return GVH_OK;
}

int gvh_read_ic_files(const char *root_dir, const gvh_lattice_params *L, int shear, int bulk, double *const *prim,
                      int n_prim) {
  if (!root_dir || !L || !prim) return pfail(GVH_ERR_INVALID, "null argument");
  const int want = 5 + (shear ? 10 : 0) + (bulk ? 1 : 0);
  if (n_prim != want) return pfail(GVH_ERR_INVALID, "wrong number of primitive arrays");
  const int nx = L->numLatticePointsX, ny = L->numLatticePointsY, nz = L->numLatticePointsRapidity;
  std::vector<std::string> names = {"e", "ut", "ux", "uy", "un"};
  if (shear)
    for (const char *c : {"pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn", "pinn"})
      names.push_back(c);
  if (bulk) names.push_back("bulk");
  const long long ng = (long long)(nx + 4) * (ny + 4) * (nz + 4);
  for (int f = 0; f < n_prim; ++f) {
    if (!prim[f]) return pfail(GVH_ERR_INVALID, "null primitive array");
    std::fill(prim[f], prim[f] + ng, 0.0);
    const std::string path = std::string(root_dir) + "/input/" + names[f] + ".dat";
    FILE *fp = fopen(path.c_str(), "r");
    if (!fp) return pfail(GVH_ERR_INVALID, "cannot open " + path);
    for (int i = 2; i < nx + 2; ++i)
      for (int j = 2; j < ny + 2; ++j)
        for (int k = 2; k < nz + 2; ++k) {
          float x, y, z, value;
          if (fscanf(fp, "%f %f %f %f", &x, &y, &z, &value) != 4) {
            fclose(fp);
            return pfail(GVH_ERR_INVALID, "short or malformed file " + path);
          }
          double v = (double)value;
          if (f == 0) v += 1.0e-3;
          prim[f][ghost_index(i, j, k, nx, ny)] = v;
        }
    fclose(fp);
  }
  return GVH_OK;
}

// setInitialTmunuFromFile (InitialConditions.cpp:29-97): one file <root>/input/Tmunu.dat, lines
// "x y z e p ut ux uy un pitt pitx pity pitn pixx pixy pixn piyy piyn pinn Pi" scanned as floats,
// i outermost and k innermost; e gets +1e-3; p is taken from the file; the dissipative
// currents are kept when evolved.
int gvh_read_ic_tmunu(const char *root_dir, const gvh_lattice_params *L, int shear, int bulk, double *const *prim,
                      int n_prim, double *p_out) {
  if (!root_dir || !L || !prim || !p_out) return pfail(GVH_ERR_INVALID, "null argument");
  const int want = 5 + (shear ? 10 : 0) + (bulk ? 1 : 0);
  if (n_prim != want) return pfail(GVH_ERR_INVALID, "wrong number of primitive arrays");
  for (int f = 0; f < n_prim; ++f)
    if (!prim[f]) return pfail(GVH_ERR_INVALID, "null primitive array");
  const int nx = L->numLatticePointsX, ny = L->numLatticePointsY, nz = L->numLatticePointsRapidity;
  const long long ng = (long long)(nx + 4) * (ny + 4) * (nz + 4);
  for (int f = 0; f < n_prim; ++f) std::fill(prim[f], prim[f] + ng, 0.0);
  std::fill(p_out, p_out + ng, 0.0);
  const std::string path = std::string(root_dir) + "/input/Tmunu.dat";
  FILE *fp = fopen(path.c_str(), "r");
  if (!fp) return pfail(GVH_ERR_INVALID, "cannot open " + path);
  for (int i = 2; i < nx + 2; ++i)
    for (int j = 2; j < ny + 2; ++j)
      for (int k = 2; k < nz + 2; ++k) {
        float v[20];
        int got = fscanf(fp, "%f %f %f %f %f %f %f %f %f %f %f %f %f %f %f %f %f %f %f %f", &v[0], &v[1], &v[2], &v[3],
                         &v[4], &v[5], &v[6], &v[7], &v[8], &v[9], &v[10], &v[11], &v[12], &v[13], &v[14], &v[15],
                         &v[16], &v[17], &v[18], &v[19]);
        if (got != 20) {
          fclose(fp);
          return pfail(GVH_ERR_INVALID, "short or malformed file " + path);
        }
        const long long s = ghost_index(i, j, k, nx, ny);
        prim[0][s] = (double)v[3] + 1.0e-3;
        p_out[s] = (double)v[4];
        for (int m = 0; m < 4; ++m) prim[1 + m][s] = (double)v[5 + m];
        if (shear)
          for (int m = 0; m < 10; ++m) prim[5 + m][s] = (double)v[9 + m];
        if (bulk) prim[15][s] = (double)v[19];
      }
  fclose(fp);
  return GVH_OK;
}

// FileIO.cpp:15-60: <dir>/<name>_<t %.3f>.dat, k outermost, "x y z value" lines.
int gvh_write_field(const char *output_dir, const char *name, double t, const gvh_lattice_params *L,
                    const double *field) {
  if (!output_dir || !name || !L || !field) return pfail(GVH_ERR_INVALID, "null argument");
  char fname[1024];
  snprintf(fname, sizeof fname, "%s/%s_%.3f.dat", output_dir, name, t);
  FILE *fp = fopen(fname, "w");
  if (!fp) return pfail(GVH_ERR_INVALID, std::string("cannot write ") + fname);
  const int nx = L->numLatticePointsX, ny = L->numLatticePointsY, nz = L->numLatticePointsRapidity;
  const double dx = L->latticeSpacingX, dy = L->latticeSpacingY, dz = L->latticeSpacingRapidity;
  for (int k = 2; k < nz + 2; ++k) {
    double z = (k - 2 - (nz - 1) / 2.) * dz;
    for (int j = 2; j < ny + 2; ++j) {
      double y = (j - 2 - (ny - 1) / 2.) * dy;
      for (int i = 2; i < nx + 2; ++i) {
        double x = (i - 2 - (nx - 1) / 2.) * dx;
        fprintf(fp, "%.3f\t%.3f\t%.3f\t%.8f\n", x, y, z, field[ghost_index(i, j, k, nx, ny)]);
      }
    }
  }
  fclose(fp);
  return GVH_OK;
}

void gvh_surface_slab_labels(long long k, double tau0, double dtau, double *tau_label, double *tau_scale,
                             long long *flush_iteration) {
  // Levels are stored at iteration n = level + 1; the finder runs at iterations n with
  // n % 10 == 9 over the slabs stored since the last run (HydroPlugin.cpp:262-287). The first
  // chunk labels a slab with its lower level's time, later ones with its upper level's
  // (HydroPlugin.cpp:298-299); the normal is scaled by the loop's t of the flush iteration.
  long long flush;
  double label;
  if (k <= 7) {
    flush = 9;
    label = tau0 + ((double)k) * dtau;
  } else {
    flush = 10 * ((k + 2) / 10) + 9;
    label = tau0 + ((double)(k + 1)) * dtau;
  }
  if (tau_label) *tau_label = label;
  if (tau_scale) *tau_scale = tau0 + (double)(flush - 1) * dtau;
  if (flush_iteration) *flush_iteration = flush;
}

int gvh_run(const gvh_lattice_params *L, const gvh_ic_params *ic, const gvh_hydro_params *H, const char *root_dir,
            const char *output_dir, const gvh_options *opts, int outputs, gvh_run_report *report) {
  g_plugin_error.clear();
  if (!L || !ic || !H || !root_dir) return pfail(GVH_ERR_INVALID, "null argument");
  const int ic_type = ic->initialConditionType;
  if (ic_type != 10 && ic_type != 11)
    return pfail(GVH_ERR_INVALID, "gvh_run reads initial-condition types 10 (input/*.dat files) and 11 "
                                  "(input/Tmunu.dat); type " + std::to_string(ic_type) + " is generated by the "
                                  "reference's own initial-condition code, which is outside this library");
  gvh_options o;
  if (opts) o = *opts; else gvh_default_options(&o);
  gvh_handle *h = nullptr;
  int rc = gvh_create(L, H, &o, &h);
  if (rc) return pfail(rc, std::string("gvh_create: ") + gvh_last_error());
  const int nx = L->numLatticePointsX, ny = L->numLatticePointsY, nz = L->numLatticePointsRapidity;
  const long long ng = (long long)(nx + 4) * (ny + 4) * (nz + 4);
  const int n_prim = 5 + (o.shear ? 10 : 0) + (o.bulk ? 1 : 0);
  std::vector<std::vector<double>> prim(n_prim, std::vector<double>(ng));
  std::vector<double *> pp(n_prim);
  for (int f = 0; f < n_prim; ++f) pp[f] = prim[f].data();
  if (ic_type == 10) {
    rc = gvh_read_ic_files(root_dir, L, o.shear, o.bulk, pp.data(), n_prim);
    if (!rc) rc = gvh_set_primitive_state(h, pp.data(), n_prim);
  } else {
    std::vector<double> p_in(ng);
    rc = gvh_read_ic_tmunu(root_dir, L, o.shear, o.bulk, pp.data(), n_prim, p_in.data());
    if (!rc) rc = gvh_set_primitive_state_p(h, pp.data(), n_prim, p_in.data());
  }
  if (rc) {
    std::string msg = g_plugin_error.empty() ? gvh_last_error() : g_plugin_error;
    gvh_destroy(h);
    return pfail(rc, msg);
  }
  prim.clear();

  rc = gvh_run_loop(h, L, H, output_dir, outputs, report);
  gvh_destroy(h);
  return rc;
}

namespace {

// Writes surface.dat chunks on a thread of its own, in the order they are handed over, so
// that the file writes overlap the host half of the next slabs. At most two chunks wait.
class ChunkWriter {
 public:
  explicit ChunkWriter(FILE *fp) : fp_(fp) { th_ = std::thread([this] { loop(); }); }
  ~ChunkWriter() { finish(); }
  // false once a write has failed
  bool push(std::vector<std::string> &&chunk) {
    std::unique_lock<std::mutex> lock(mu_);
    space_.wait(lock, [&] { return q_.size() < kMaxQueued || failed_; });
    if (failed_) return false;
    q_.push_back(std::move(chunk));
    ready_.notify_one();
    return true;
  }
  // waits until every chunk handed over is written; false if a write failed
  bool finish() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    ready_.notify_one();
    if (th_.joinable()) th_.join();
    return !failed_;
  }

 private:
  void loop() {
    std::unique_lock<std::mutex> lock(mu_);
    for (;;) {
      ready_.wait(lock, [&] { return stop_ || !q_.empty(); });
      if (q_.empty()) return;
      std::vector<std::string> chunk = std::move(q_.front());
      q_.pop_front();
      space_.notify_one();
      lock.unlock();
      bool ok = true;
      for (const std::string &part : chunk) ok = ok && fwrite(part.data(), 1, part.size(), fp_) == part.size();
      chunk.clear();
      lock.lock();
      if (!ok) {
        failed_ = true;
        space_.notify_all();
      }
    }
  }
  static constexpr size_t kMaxQueued = 2;
  FILE *fp_;
  std::mutex mu_;
  std::condition_variable ready_, space_;
  std::deque<std::vector<std::string>> q_;
  bool stop_ = false, failed_ = false;
  std::thread th_;
};

}  // namespace

int gvh_run_loop(gvh_handle *h, const gvh_lattice_params *L, const gvh_hydro_params *H, const char *output_dir,
                 int outputs, gvh_run_report *report) {
  if (!h || !L || !H) return pfail(GVH_ERR_INVALID, "gvh_run_loop: null argument");
  if (L->numLatticePointsX != h->nx || L->numLatticePointsY != h->ny || L->numLatticePointsRapidity != h->nz)
    return pfail(GVH_ERR_INVALID, "gvh_run_loop: lattice parameters do not match the handle");
  g_plugin_error.clear();
  const bool dump_fields = (outputs & GVH_RUN_FIELDS) != 0 && output_dir;
  const bool want_surface = (outputs & GVH_RUN_SURFACE) != 0 && output_dir;
  const int nx = L->numLatticePointsX, ny = L->numLatticePointsY, nz = L->numLatticePointsRapidity;
  const long long ng = (long long)(nx + 4) * (ny + 4) * (nz + 4);
  int rc = GVH_OK;
  const double t0 = H->initialProperTimePoint, dt = L->latticeSpacingProperTime;
  const double T_reg = H->regulationTemperatureGeV / kHbarc;
  // e(T_fo), HydroPlugin.cpp:131-135
  const double e_fo = gvh_energy_density_of_temperature(h->eos, H->freezeoutTemperatureGeV);

  // freeze-out surface (HydroPlugin.cpp:155-211 set-up, 255-393 per iteration)
  gvh_surface *surf = nullptr;
  FILE *surf_file = nullptr;
  std::vector<std::string> chunk_text;
  long long surf_rows = 0, chunk_rows = 0;
  double surf_seconds = 0.0;
  if (want_surface) {
    const std::string path = std::string(output_dir) + "/surface.dat";
    surf_file = fopen(path.c_str(), "w");
    if (!surf_file) {
      return pfail(GVH_ERR_INVALID, "cannot open " + path);
    }
    // the reference's finder handles 3+1D and 2+1D lattices only (HydroPlugin.cpp:157-182)
    if (L->numLatticePointsX > 1 && L->numLatticePointsY > 1) {
      if ((rc = gvh_surface_create(h, e_fo, &surf)) || (rc = gvh_surface_set_outputs(surf, GVH_SURFACE_TEXT)) ||
          (rc = gvh_surface_set_lower(surf))) {
        std::string msg = gvh_surface_last_error();
        gvh_surface_destroy(surf);
        fclose(surf_file);
        return pfail(rc, msg);
      }
    }
  }

  std::unique_ptr<ChunkWriter> writer;
  if (surf_file) writer.reset(new ChunkWriter(surf_file));
  // the slab found last, whose text is taken at the next slab (or at the end)
  struct DeferredSlab {
    bool active;
    long long flush, n, elements;
  } deferred{false, -1, -1, 0};
  auto take_deferred = [&]() -> int {
    if (!deferred.active) return GVH_OK;
    deferred.active = false;
    const auto s0 = std::chrono::steady_clock::now();
    gvh::surface::take_text(surf, chunk_text);  // waits for its formatting
    chunk_rows += deferred.elements;
    if (deferred.flush == deferred.n) {
      if (!writer->push(std::move(chunk_text))) {
        g_plugin_error = "writing surface.dat failed";
        return GVH_ERR_INVALID;
      }
      surf_rows += chunk_rows;
      chunk_text.clear();
      chunk_rows = 0;
    }
    surf_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
    return GVH_OK;
  };

  const int nf = gvh_num_fields(h), nq = gvh_num_conserved(h);
  std::vector<std::vector<double>> fields;
  std::vector<double *> fp;
  double total_ms = 0.0;
  long long steps = 0;
  int frozen = 0;
  double t = t0;
  const int nt = L->numProperTimePoints;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
  cudaSetDevice(h->device);
  // the wait for each step blocks the thread instead of spinning on a core: the surface's
  // formatting threads and the file writer need the host cores meanwhile
  if (cudaEventCreate(&ev_begin) != cudaSuccess ||
      cudaEventCreateWithFlags(&ev_end, surf ? cudaEventBlockingSync : cudaEventDefault) != cudaSuccess) {
    gvh_surface_destroy(surf);
    if (surf_file) fclose(surf_file);
    return pfail(GVH_ERR_CUDA, "gvh_run_loop: event creation failed");
  }
  for (int n = 1; n <= nt + 1; ++n) {
    if (dump_fields && output_dir && (n - 1) % kFreq == 0) {
      if (fields.empty()) {
        fields.assign(nf, std::vector<double>(ng));
        for (int f = 0; f < nf; ++f) fp.push_back(fields[f].data());
      }
      if ((rc = gvh_get_state(h, fp.data(), nf))) break;
      static const char *qn[15] = {"ttt", "ttx", "tty", "ttn", "pitt", "pitx", "pity", "pitn",
                                   "pixx", "pixy", "pixn", "piyy", "piyn", "pinn", "Pi"};
      // HydroPlugin.cpp:44-70: e, p, u and the dissipative components
      const int base = nq;
      gvh_write_field(output_dir, "e", t, L, fp[base]);
      gvh_write_field(output_dir, "p", t, L, fp[base + 1]);
      gvh_write_field(output_dir, "ux", t, L, fp[base + 3]);
      gvh_write_field(output_dir, "uy", t, L, fp[base + 4]);
      gvh_write_field(output_dir, "un", t, L, fp[base + 5]);
      gvh_write_field(output_dir, "ut", t, L, fp[base + 2]);
      for (int c = 4; c < nq; ++c) gvh_write_field(output_dir, qn[c], t, L, fp[c]);
    }
    // the stop test's reduction first: it waits for its result, which must not queue behind
    // the surface's device work
    double emax = 0.0;
    if ((rc = gvh_max_energy_density(h, &emax))) break;
    // The slab (n-2, n-1) is marked now and its rows made on the surface's stream beside the
    // next step; its host half runs while the GPU takes that step.
    bool surf_pending = false;
    long long flush = -1;
    if (surf && n >= 2) {
      const auto s0 = std::chrono::steady_clock::now();
      double label, scale;
      gvh_surface_slab_labels(n - 2, t0, dt, &label, &scale, &flush);
      if ((rc = gvh_surface_find_begin(surf, label, scale))) {
        g_plugin_error = gvh_surface_last_error();
        break;
      }
      surf_pending = true;
      surf_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
    }
    // the host half: this slab's elements are counted now and its rows formatted on the
    // surface's thread pool while the loop goes on; its text joins the chunk one iteration
    // later, which is written at the reference's iteration (HydroPlugin.cpp:287)
    auto finish_surface = [&]() -> int {
      if (!surf_pending) return GVH_OK;
      surf_pending = false;
      const auto s0 = std::chrono::steady_clock::now();
      int r = take_deferred();
      if (r) return r;
      long long nel = 0;
      r = gvh_surface_find_end(surf, &nel);
      if (r) {
        g_plugin_error = gvh_surface_last_error();
        return r;
      }
      deferred = DeferredSlab{true, flush, n, nel};
      surf_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
      return GVH_OK;
    };
    if (emax <= e_fo) ++frozen;
    if (frozen >= kFreezeoutChecks) {
      rc = finish_surface();
      break;
    }
    // device time of one step (the reference's Stopwatch brackets twoStepRungeKutta,
    // HydroPlugin.cpp:414-420), taken with events so the host half of the slab overlaps it
    if (cudaEventRecord(ev_begin, h->stream) != cudaSuccess || (rc = gvh_rk2_step(h, t, dt, T_reg)) ||
        cudaEventRecord(ev_end, h->stream) != cudaSuccess) {
      if (!rc) rc = GVH_ERR_CUDA;
      break;
    }
    if ((rc = finish_surface())) break;
    float ms = 0.f;
    if (cudaEventSynchronize(ev_end) != cudaSuccess || cudaEventElapsedTime(&ms, ev_begin, ev_end) != cudaSuccess) {
      rc = GVH_ERR_CUDA;
      break;
    }
    total_ms += ms;
    ++steps;
    t = t0 + n * dt;
  }
  if (!rc) rc = take_deferred();
  cudaEventDestroy(ev_begin);
  cudaEventDestroy(ev_end);
  unsigned flags = 0;
  gvh_status(h, &flags);
  if (report) {
    report->steps = steps;
    report->tau_end = t;
    report->average_ms_per_step = steps ? total_ms / steps : 0.0;
    report->frozen_out = frozen >= kFreezeoutChecks;
    report->status = flags;
    report->freezeout_energy_density = e_fo;
    report->surface_elements = surf_rows;
    report->surface_seconds = surf_seconds;
    gvh_surface_info si;
    memset(&si, 0, sizeof si);
    if (surf) gvh_surface_get_info(surf, &si);
    report->surface_hypercubes = si.hypercubes_total;
    report->surface_bytes_to_host = si.bytes_to_host_total;
    report->surface_host_seconds = si.host_seconds_total;
  }
  if (writer && !writer->finish() && !rc) {
    g_plugin_error = "writing surface.dat failed";
    rc = GVH_ERR_INVALID;
  }
  writer.reset();
  gvh_surface_destroy(surf);
  if (surf_file) fclose(surf_file);
  if (rc) return pfail(rc, g_plugin_error.empty() ? gvh_last_error() : g_plugin_error);
  return GVH_OK;
}

}  // extern "C"
