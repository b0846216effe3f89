// gvh_surface.cu -- freeze-out hypersurface of a handle's evolution: device marking of the
// hypercubes the iso-surface e = e_fo crosses, compacted copy to the host, host cornelius.
//
// The reference copies every field of the whole lattice to the host every step
// (HydroPlugin.cpp:264), keeps FOFREQ + 1 host copies of ten fields
// (FreezeOut.cpp:45-160) and scans every hypercube on the host (HydroPlugin.cpp:283-305).
// Here the fields of one time level stay on the device as a snapshot (u^x, u^y, u^eta, e,
// pi^{xx,xy,x eta,yy,y eta}, Pi; cell-major per field), and each call of gvh_surface_find
// takes the slab between the lower snapshot and the handle's current level:
//
//   fo_snapshot      current level -> the upper snapshot                   (all cells)
//   fo_mark          16 (8 in 2+1D) corner energies per hypercube -> crossed? (memory order)
//   fo_count         crossed hypercubes per block, in the reference's loop order
//                    (x outer, eta inner); per block, the lattice points that are corners of
//                    a crossed hypercube
//   fo_scan          block offsets (one block)
//   fo_write         ordered hypercube keys; the points' 2 x 10 values
//
// and then, for the QCD EoS (the default), the rows themselves are made on the device
// (gvh_surface_rows.cu: cornelius, interpolation and the row, one thread per crossed
// hypercube, the host's code without FMA contraction), and with them their surface.dat text,
// which the copy engine brings to the host; the host formats only the few rows whose numbers
// the device's fast %g leaves to the exact path. Otherwise the host receives the keys and points (about 170 bytes per
// crossed hypercube instead of ~160 bytes per lattice cell per level) and runs the same code
// with a pool of host threads (gvh_surface_host.cpp).
#include <cuda_runtime.h>
#include <limits.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gvh.h"
#include "gvh_handle.h"
#include "gvh_surface_device.h"
#include "gvh_nvtx.h"
#include "gvh_surface_internal.h"

using gvh::surface::kVars;

namespace {

constexpr int kFoThreads = 256;

thread_local std::string g_surface_error;

int sfail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_surface_error = buf;
  return code;
}

#define SF_CUDA(call)                                                                             \
  do {                                                                                            \
    cudaError_t err_ = (call);                                                                    \
    if (err_ != cudaSuccess) return sfail(GVH_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(err_)); \
  } while (0)

struct Geometry {
  int nx, ny, nz, nzc;  // nzc: hypercubes along eta (nz-1 in 3+1D, 1 in 2+1D)
  int kz;               // corner layers along eta (2 in 3+1D, 1 in 2+1D)
  long long ncells, ncubes;
};

__global__ void fo_snapshot(long long n, long long cs, const double *__restrict__ e, const double *__restrict__ u,
                            const double *__restrict__ q, int shear, int bulk, double *__restrict__ snap) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  snap[0 * n + i] = u[1 * cs + i];
  snap[1 * n + i] = u[2 * cs + i];
  snap[2 * n + i] = u[3 * cs + i];
  snap[3 * n + i] = e[i];
  // pi^{xx}, pi^{xy}, pi^{x eta}, pi^{yy}, pi^{y eta} are conserved components 8..12, Pi is 14
  for (int c = 0; c < 5; ++c) snap[(4 + c) * n + i] = shear ? q[(8 + c) * cs + i] : 0.0;
  snap[9 * n + i] = bulk ? q[14 * cs + i] : 0.0;
}

// Hypercube cm (memory order: x fastest) is crossed when its corners' energies are neither all
// >= iso nor all < iso (the test of cornelius.cpp:2202-2217 and :2152-2165).
__global__ void fo_mark(Geometry g, const double *__restrict__ elo, const double *__restrict__ ehi, double iso,
                        unsigned char *__restrict__ flag) {
  const long long cm = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cm >= g.ncubes) return;
  const int ix = (int)(cm % (g.nx - 1));
  const long long r = cm / (g.nx - 1);
  const int iy = (int)(r % (g.ny - 1));
  const int iz = (int)(r / (g.ny - 1));
  int high = 0;
  for (int k = 0; k < g.kz; ++k)
    for (int b = 0; b < 2; ++b) {
      const long long s = ix + (long long)g.nx * ((iy + b) + (long long)g.ny * (iz + k));
      high += (elo[s] >= iso) + (elo[s + 1] >= iso) + (ehi[s] >= iso) + (ehi[s + 1] >= iso);
    }
  flag[cm] = (high != 0 && high != 8 * g.kz);
}

__device__ __forceinline__ void cube_of_key(const Geometry &g, long long key, int &ix, int &iy, int &iz) {
  iz = (int)(key % g.nzc);
  const long long r = key / g.nzc;
  iy = (int)(r % (g.ny - 1));
  ix = (int)(r / (g.ny - 1));
}

__device__ __forceinline__ bool point_needed(const Geometry &g, const unsigned char *flag, long long p) {
  const int ix = (int)(p % g.nx);
  const long long r = p / g.nx;
  const int iy = (int)(r % g.ny);
  const int iz = (int)(r / g.ny);
  bool need = false;
  for (int c = 0; c < g.kz; ++c)
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        const int cx = ix - a, cy = iy - b, cz = iz - c;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx - 1 || cy >= g.ny - 1 || cz >= g.nzc) continue;
        need |= flag[cx + (long long)(g.nx - 1) * (cy + (long long)(g.ny - 1) * cz)] != 0;
      }
  return need;
}

// Blocks [0, nbc) count crossed hypercubes in key order; blocks [nbc, nbc + nbp) count the
// points needed, in memory order.
__global__ void fo_count(Geometry g, int nbc, const unsigned char *__restrict__ flag,
                         unsigned char *__restrict__ pflag, int *__restrict__ counts) {
  const int b = blockIdx.x;
  int f = 0;
  if (b < nbc) {
    const long long key = (long long)b * kFoThreads + threadIdx.x;
    if (key < g.ncubes) {
      int ix, iy, iz;
      cube_of_key(g, key, ix, iy, iz);
      f = flag[ix + (long long)(g.nx - 1) * (iy + (long long)(g.ny - 1) * iz)];
    }
  } else {
    const long long p = (long long)(b - nbc) * kFoThreads + threadIdx.x;
    if (p < g.ncells) {
      f = point_needed(g, flag, p);
      pflag[p] = (unsigned char)f;
    }
  }
  const int total = __syncthreads_count(f);
  if (threadIdx.x == 0) counts[b] = total;
}

// Exclusive offsets of the two count segments, and the two totals at the end (also written to
// mapped host memory: the host reads them without a copy, which could queue behind another
// stream's large copy to the host).
__global__ void fo_scan(int nbc, int nbp, int *__restrict__ counts, int *__restrict__ totals,
                        volatile int *__restrict__ host_totals) {
  __shared__ int part[1024];
  for (int seg = 0; seg < 2; ++seg) {
    int *c = counts + (seg ? nbc : 0);
    const int n = seg ? nbp : nbc;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int lo = min(n, (int)threadIdx.x * per), hi = min(n, lo + per);
    int sum = 0;
    for (int i = lo; i < hi; ++i) sum += c[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
      const int v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
      __syncthreads();
      part[threadIdx.x] += v;
      __syncthreads();
    }
    int run = part[threadIdx.x] - sum;
    for (int i = lo; i < hi; ++i) {
      const int v = c[i];
      c[i] = run;
      run += v;
    }
    if (threadIdx.x == blockDim.x - 1) {
      totals[seg] = part[threadIdx.x];
      host_totals[seg] = part[threadIdx.x];
    }
    __syncthreads();
  }
}

// Rank of this thread's flag among the block's set flags, in thread order.
__device__ __forceinline__ int block_rank(int f) {
  __shared__ int warp_base[kFoThreads / 32];
  const unsigned ballot = __ballot_sync(0xffffffffu, f);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_base[w] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int i = 0; i < kFoThreads / 32; ++i) {
      const int v = warp_base[i];
      warp_base[i] = run;
      run += v;
    }
  }
  __syncthreads();
  return warp_base[w] + __popc(ballot & ((1u << lane) - 1u));
}

__global__ void fo_write(Geometry g, int nbc, const unsigned char *__restrict__ flag,
                         const unsigned char *__restrict__ pflag, const int *__restrict__ offsets,
                         const double *__restrict__ lo, const double *__restrict__ hi, int *__restrict__ cube_key,
                         int *__restrict__ point_cell, double *__restrict__ point_vals) {
  const int b = blockIdx.x;
  if (b < nbc) {
    const long long key = (long long)b * kFoThreads + threadIdx.x;
    int f = 0;
    if (key < g.ncubes) {
      int ix, iy, iz;
      cube_of_key(g, key, ix, iy, iz);
      f = flag[ix + (long long)(g.nx - 1) * (iy + (long long)(g.ny - 1) * iz)];
    }
    const int rank = block_rank(f);
    if (f) cube_key[offsets[b] + rank] = (int)key;
  } else {
    const long long p = (long long)(b - nbc) * kFoThreads + threadIdx.x;
    const int f = p < g.ncells ? pflag[p] : 0;
    const int rank = block_rank(f);
    if (f) {
      const long long o = offsets[b] + rank;
      point_cell[o] = (int)p;
      double *dst = point_vals + o * (2 * kVars);
      for (int v = 0; v < kVars; ++v) dst[v] = lo[v * g.ncells + p];
      for (int v = 0; v < kVars; ++v) dst[kVars + v] = hi[v * g.ncells + p];
    }
  }
}

template <class T>
int grow_pinned(T **buf, long long *cap, long long need) {
  if (need <= *cap) return GVH_OK;
  long long n = std::max<long long>(need, *cap * 3 / 2 + 1024);
  if (*buf) cudaFreeHost(*buf);
  *buf = nullptr;
  *cap = 0;
  if (cudaHostAlloc(reinterpret_cast<void **>(buf), (size_t)n * sizeof(T), cudaHostAllocDefault) != cudaSuccess)
    return sfail(GVH_ERR_NOMEM, "gvh_surface: cannot pin %lld bytes of host memory", n * (long long)sizeof(T));
  *cap = n;
  return GVH_OK;
}

// Mapped pinned host memory: the device writes into it directly.
template <class T>
int grow_mapped(T **buf, T **dev, long long *cap, long long need) {
  if (need <= *cap) return GVH_OK;
  long long n = std::max<long long>(need, *cap * 3 / 2 + 1024);
  if (*buf) cudaFreeHost(*buf);
  *buf = nullptr;
  *dev = nullptr;
  *cap = 0;
  if (cudaHostAlloc(reinterpret_cast<void **>(buf), (size_t)n * sizeof(T), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void **>(dev), *buf, 0) != cudaSuccess)
    return sfail(GVH_ERR_NOMEM, "gvh_surface: cannot map %lld bytes of host memory", n * (long long)sizeof(T));
  *cap = n;
  return GVH_OK;
}

}  // namespace

struct gvh_surface {
  gvh_handle *h;
  int device;        // the handle's device, kept so that destroying needs no handle
  Geometry g;
  double iso;
  int dim, nthreads;
  int nbc, nbp;
  int lower;         // snapshot holding the lower time level
  bool have_lower;
  char *dev;         // one device allocation for everything below
  double *snap[2];
  unsigned char *flag, *pflag;
  int *counts, *totals, *cube_key, *point_cell;
  double *point_vals;
  int *h_totals, *d_totals_mapped;  // mapped pinned: crossed hypercubes, points
  int *h_cube_key, *h_point_cell;
  double *h_point_vals;
  long long cap_cubes, cap_points, cap_vals;
  std::vector<int> c2p;
  std::unique_ptr<gvh::surface::Pool> pool;
  int outputs;       // gvh::surface::OUT_ROWS | OUT_TEXT
  // rows made on the device (gvh_surface_rows.cu; the default for the QCD EoS): scratch and
  // output grown to the largest slab, the rows' copy on the host
  bool device_rows;
  int *d_c2p;
  char *rowdev;
  long long rowdev_cap;
  long long *h_rowtot, *d_rowtot_mapped;  // mapped pinned: rows, errors, text bytes, host rows
  // two sets of host buffers, alternating by slab: the host assembles one slab's text on the
  // pool's workers while the device makes the next slab's. The device's text, and all rows
  // when they are kept (or the host rows overflow), come by copy into pinned memory; the host
  // rows are written by the device into mapped pinned memory.
  double *h_rows[2];
  long long cap_rows[2];
  gvh::surface::HostRow *h_hrows[2], *d_hrows_mapped[2];
  long long cap_hrows[2];
  char *h_text[2];
  long long cap_text[2];
  cudaEvent_t copied_out[2];  // after a slab's copies of text and rows
  int rbuf;             // buffer of the slab begun last
  bool formatting;      // a slab's rows are being formatted on the pool (format_rows async)
  long long p_nrows, p_errors, p_text_bytes, p_host_rows;
  bool p_all_rows;
  gvh::surface::Result last;
  gvh_surface_info info;
  // a slab between gvh_surface_find_begin and _end: its copies to the pinned buffers are in
  // flight on the handle's stream, ordered before whatever the caller queues next
  bool pending;
  // an internal consistency check failed in gvh_surface_find_end: the last slab's rows are
  // dropped and every later call on this surface is refused
  bool failed;
  long long p_ncubes, p_npoints;
  double p_label, p_scale;
  cudaEvent_t copied;
  cudaStream_t rows_stream;  // the device rows run here, beside the handle's next step
  std::chrono::steady_clock::time_point p_t0;
};

extern "C" {

const char *gvh_surface_last_error(void) { return g_surface_error.c_str(); }

int gvh_surface_create(gvh_handle *h, double e_freezeout, gvh_surface **out) {
  if (!h || !out) return sfail(GVH_ERR_INVALID, "gvh_surface_create: null argument");
  *out = nullptr;
  if (h->nx < 2 || h->ny < 2)
    return sfail(GVH_ERR_INVALID, "gvh_surface_create: the surface finder works in 3+1D or 2+1D (nx, ny > 1); "
                                  "lattice is %dx%dx%d", h->nx, h->ny, h->nz);
  if (!(e_freezeout > 0)) return sfail(GVH_ERR_INVALID, "gvh_surface_create: e_freezeout must be > 0");
  if (h->ncells >= (1ll << 31)) return sfail(GVH_ERR_INVALID, "gvh_surface_create: lattice too large");
  SF_CUDA(cudaSetDevice(h->device));
  gvh_surface *s = new gvh_surface();
  s->h = h;
  s->device = h->device;
  s->iso = e_freezeout;
  s->dim = h->nz > 1 ? 4 : 3;
  Geometry &g = s->g;
  g.nx = h->nx; g.ny = h->ny; g.nz = h->nz;
  g.nzc = s->dim == 4 ? h->nz - 1 : 1;
  g.kz = s->dim == 4 ? 2 : 1;
  g.ncells = h->ncells;
  g.ncubes = (long long)(g.nx - 1) * (g.ny - 1) * g.nzc;
  s->nbc = (int)((g.ncubes + kFoThreads - 1) / kFoThreads);
  s->nbp = (int)((g.ncells + kFoThreads - 1) / kFoThreads);
  s->nthreads = (int)std::min(64u, std::max(1u, std::thread::hardware_concurrency()));
  s->outputs = gvh::surface::OUT_ROWS | gvh::surface::OUT_TEXT;
  const long long n = g.ncells;
  auto al = [](long long b) { return (b + 255) / 256 * 256; };
  const long long bytes = 2 * al(kVars * n * 8) + al(g.ncubes) + al(n) + al(4 * (s->nbc + s->nbp + 2)) +
                          al(4 * g.ncubes) + al(4 * n) + al(2 * kVars * n * 8) + al(4 * n);
  if (cudaMalloc(&s->dev, (size_t)bytes) != cudaSuccess) {
    delete s;
    return sfail(GVH_ERR_NOMEM, "gvh_surface_create: cannot allocate %lld bytes", bytes);
  }
  char *p = s->dev;
  s->snap[0] = reinterpret_cast<double *>(p); p += al(kVars * n * 8);
  s->snap[1] = reinterpret_cast<double *>(p); p += al(kVars * n * 8);
  s->flag = reinterpret_cast<unsigned char *>(p); p += al(g.ncubes);
  s->pflag = reinterpret_cast<unsigned char *>(p); p += al(n);
  s->counts = reinterpret_cast<int *>(p); p += al(4 * (s->nbc + s->nbp + 2));
  s->totals = s->counts + s->nbc + s->nbp;
  s->cube_key = reinterpret_cast<int *>(p); p += al(4 * g.ncubes);
  s->point_cell = reinterpret_cast<int *>(p); p += al(4 * n);
  s->point_vals = reinterpret_cast<double *>(p); p += al(2 * kVars * n * 8);
  s->d_c2p = reinterpret_cast<int *>(p);
  // the device rows repeat the host's arithmetic exactly for the QCD EoS; the conformal T(e)
  // is a pow, which the device does not evaluate as the host's libm does
  s->device_rows = h->eos == GVH_EOS_QCD;
  if (cudaHostAlloc(reinterpret_cast<void **>(&s->h_totals), 4 * sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void **>(&s->d_totals_mapped), s->h_totals, 0) != cudaSuccess ||
      cudaHostAlloc(reinterpret_cast<void **>(&s->h_rowtot), 8 * sizeof(long long), cudaHostAllocMapped) !=
          cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void **>(&s->d_rowtot_mapped), s->h_rowtot, 0) != cudaSuccess) {
    if (s->h_rowtot) cudaFreeHost(s->h_rowtot);
    if (s->h_totals) cudaFreeHost(s->h_totals);
    cudaFree(s->dev);
    delete s;
    return sfail(GVH_ERR_NOMEM, "gvh_surface_create: cannot pin host memory");
  }
  memset(&s->info, 0, sizeof s->info);
  // waited on by blocking, not spinning: the pool's formatting threads need the cores
  if (cudaEventCreateWithFlags(&s->copied, cudaEventDisableTiming | cudaEventBlockingSync) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->copied_out[0], cudaEventDisableTiming | cudaEventBlockingSync) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->copied_out[1], cudaEventDisableTiming | cudaEventBlockingSync) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->rows_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFreeHost(s->h_totals);
    cudaFreeHost(s->h_rowtot);
    cudaFree(s->dev);
    delete s;
    return sfail(GVH_ERR_CUDA, "gvh_surface_create: event creation failed");
  }
  *out = s;
  return GVH_OK;
}

// Waits for the pool's formatting of the last slab (format_rows async), if any.
static void wait_format(gvh_surface *s) {
  if (s->formatting) {
    const auto t0 = std::chrono::steady_clock::now();
    s->pool->wait();
    s->info.host_seconds_total += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    s->formatting = false;
  }
}

int gvh_surface_destroy(gvh_surface *s) {
  if (!s) return GVH_OK;
  wait_format(s);
  // touches nothing of the handle, which may be gone already; cudaFree waits for the
  // device work that uses the buffers
  cudaSetDevice(s->device);
  cudaEventSynchronize(s->copied);
  cudaStreamSynchronize(s->rows_stream);
  cudaEventDestroy(s->copied);
  for (int b = 0; b < 2; ++b)
    if (s->copied_out[b]) cudaEventDestroy(s->copied_out[b]);
  cudaStreamDestroy(s->rows_stream);
  cudaFree(s->dev);
  if (s->rowdev) cudaFree(s->rowdev);
  cudaFreeHost(s->h_totals);
  if (s->h_rowtot) cudaFreeHost(s->h_rowtot);
  for (int b = 0; b < 2; ++b) {
    if (s->h_rows[b]) cudaFreeHost(s->h_rows[b]);
    if (s->h_text[b]) cudaFreeHost(s->h_text[b]);
    if (s->h_hrows[b]) cudaFreeHost(s->h_hrows[b]);
  }
  if (s->h_cube_key) cudaFreeHost(s->h_cube_key);
  if (s->h_point_cell) cudaFreeHost(s->h_point_cell);
  if (s->h_point_vals) cudaFreeHost(s->h_point_vals);
  delete s;
  return GVH_OK;
}

int gvh_surface_set_threads(gvh_surface *s, int nthreads) {
  if (!s || nthreads < 1) return sfail(GVH_ERR_INVALID, "gvh_surface_set_threads: bad argument");
  wait_format(s);
  s->nthreads = nthreads;
  s->pool.reset();
  return GVH_OK;
}

int gvh_surface_set_device_rows(gvh_surface *s, int on) {
  if (!s) return sfail(GVH_ERR_INVALID, "gvh_surface_set_device_rows: null argument");
  wait_format(s);
  if (s->pending) return sfail(GVH_ERR_INVALID, "gvh_surface_set_device_rows: a slab is in flight");
  if (on && s->h->eos != GVH_EOS_QCD)
    return sfail(GVH_ERR_INVALID, "gvh_surface_set_device_rows: the device rows are for the QCD EoS only "
                                  "(the conformal T(e) is a pow, evaluated on the host)");
  s->device_rows = on != 0;
  return GVH_OK;
}

int gvh_surface_set_outputs(gvh_surface *s, int outputs) {
  if (!s || (outputs & ~(GVH_SURFACE_ROWS | GVH_SURFACE_TEXT)))
    return sfail(GVH_ERR_INVALID, "gvh_surface_set_outputs: bad argument");
  wait_format(s);
  s->outputs = (outputs & GVH_SURFACE_ROWS ? gvh::surface::OUT_ROWS : 0) |
               (outputs & GVH_SURFACE_TEXT ? gvh::surface::OUT_TEXT : 0);
  return GVH_OK;
}

static int snapshot(gvh_surface *s, int which) {
  gvh_handle *h = s->h;
  const unsigned blocks = (unsigned)((h->ncells + kFoThreads - 1) / kFoThreads);
  fo_snapshot<<<blocks, kFoThreads, 0, h->stream>>>(h->ncells, h->cs, h->e, gvh_current_u(h), gvh_current_q(h),
                                                     h->shear, h->bulk, s->snap[which]);
  SF_CUDA(cudaGetLastError());
  return GVH_OK;
}

int gvh_surface_set_lower(gvh_surface *s) {
  if (!s) return sfail(GVH_ERR_INVALID, "gvh_surface_set_lower: null argument");
  SF_CUDA(cudaSetDevice(s->h->device));
  int rc = snapshot(s, s->lower);
  if (rc) return rc;
  s->have_lower = true;
  return GVH_OK;
}

// The slab's rows and text on the device (gvh_surface_rows.cu), queued on the surface's
// stream; the counts and the host rows land in mapped pinned host memory, the text (and the
// rows, when needed) stay on the device for find_end to copy, so nothing here waits.
static int device_rows_begin(gvh_surface *s, long long ncubes, long long npoints, double tau_label,
                             double tau_scale) {
  gvh_handle *h = s->h;
  // The marking kernels are complete (find_begin read their totals); the rows run on the
  // surface's own stream, so the handle's next step does not wait for them. The previous
  // slab's rows are complete too (find_end waited for them), so the buffers are free.
  cudaStream_t st = s->rows_stream;
  // the scans count slots in int
  if (ncubes >= (long long)(INT_MAX / gvh::iso::kMaxElements) - 1)
    return sfail(GVH_ERR_INVALID, "gvh_surface: %lld crossed hypercubes in one slab are more than the device rows "
                                  "handle", ncubes);
  if (ncubes > s->rowdev_cap) {
    const long long cap = std::max<long long>(ncubes, s->rowdev_cap * 3 / 2 + 1024);
    if (s->rowdev) {
      SF_CUDA(cudaStreamSynchronize(st));
      cudaFree(s->rowdev);
      s->rowdev = nullptr;
      s->rowdev_cap = 0;
    }
    const size_t bytes = gvh::surface::device_rows_scratch_bytes(cap);
    if (cudaMalloc(&s->rowdev, bytes) != cudaSuccess)
      return sfail(GVH_ERR_NOMEM, "gvh_surface: cannot allocate %zu bytes for the device rows", bytes);
    s->rowdev_cap = cap;
  }
  // room for every crossed hypercube's largest number of rows, and for host rows up to a
  // sixteenth of the slots (more send every row instead); the slab before the last one is
  // formatted by now, so its buffers are free
  const long long slots = std::max(1ll, ncubes) * gvh::iso::kMaxElements;
  s->rbuf = 1 - s->rbuf;
  const int b = s->rbuf;
  int rc;
  const bool text = s->outputs & gvh::surface::OUT_TEXT;
  if (text && (rc = grow_mapped(&s->h_hrows[b], &s->d_hrows_mapped[b], &s->cap_hrows[b], slots / 16 + 1024)))
    return rc;
  for (int i = 0; i < 4; ++i) s->h_rowtot[i] = 0;
  const long long cap = s->rowdev_cap;
  gvh::surface::DeviceRows d;
  d.g.dim = s->dim;
  d.g.nx = s->g.nx; d.g.ny = s->g.ny; d.g.nz = s->g.nz;
  d.g.dt = h->dt_lattice; d.g.dx = h->dx; d.g.dy = h->dy; d.g.dz = h->dz;
  d.g.iso = s->iso;
  d.g.eos = h->eos;
  d.g.tau_label = tau_label;
  d.g.tau_scale = tau_scale;
  d.ncubes = ncubes;
  d.npoints = npoints;
  d.cube_key = s->cube_key;
  d.point_cell = s->point_cell;
  d.point_vals = s->point_vals;
  d.c2p = s->d_c2p;
  gvh::surface::device_rows_carve(d, s->rowdev, cap);
  d.host_totals = s->d_rowtot_mapped;
  if (!text) d.text = nullptr;
  d.host_rows = text ? s->d_hrows_mapped[b] : nullptr;
  d.host_rows_cap = text ? s->cap_hrows[b] : 0;
  d.keep_rows = s->outputs & gvh::surface::OUT_ROWS;
  SF_CUDA(gvh::surface::launch_device_rows(d, st));
  return GVH_OK;
}

int gvh_surface_find_begin(gvh_surface *s, double tau_label, double tau_scale) {
  gvh::NvtxRange range("gvh surface slab (device)");
  if (!s) return sfail(GVH_ERR_INVALID, "gvh_surface_find_begin: null argument");
  if (!s->have_lower) return sfail(GVH_ERR_INVALID, "gvh_surface_find_begin: no lower time level (gvh_surface_set_lower)");
  if (s->pending) return sfail(GVH_ERR_INVALID, "gvh_surface_find_begin: the previous slab has not been ended");
  if (s->failed) return sfail(GVH_ERR_INTERNAL, "gvh_surface_find_begin: an earlier slab failed");
  gvh_handle *h = s->h;
  SF_CUDA(cudaSetDevice(h->device));
  s->p_t0 = std::chrono::steady_clock::now();
  const int upper = 1 - s->lower;
  int rc = snapshot(s, upper);
  if (rc) return rc;
  const Geometry &g = s->g;
  cudaStream_t st = h->stream;
  const double *lo = s->snap[s->lower], *hi = s->snap[upper];
  fo_mark<<<(unsigned)((g.ncubes + kFoThreads - 1) / kFoThreads), kFoThreads, 0, st>>>(g, lo + 3 * g.ncells,
                                                                                       hi + 3 * g.ncells, s->iso,
                                                                                       s->flag);
  fo_count<<<s->nbc + s->nbp, kFoThreads, 0, st>>>(g, s->nbc, s->flag, s->pflag, s->counts);
  fo_scan<<<1, 1024, 0, st>>>(s->nbc, s->nbp, s->counts, s->totals, s->d_totals_mapped);
  fo_write<<<s->nbc + s->nbp, kFoThreads, 0, st>>>(g, s->nbc, s->flag, s->pflag, s->counts, lo, hi, s->cube_key,
                                                   s->point_cell, s->point_vals);
  SF_CUDA(cudaGetLastError());
  SF_CUDA(cudaStreamSynchronize(st));
  const long long ncubes = reinterpret_cast<volatile int *>(s->h_totals)[0];
  const long long npoints = reinterpret_cast<volatile int *>(s->h_totals)[1];
  if (s->device_rows) {
    if ((rc = device_rows_begin(s, ncubes, npoints, tau_label, tau_scale))) return rc;
    SF_CUDA(cudaEventRecord(s->copied, s->rows_stream));
    s->lower = upper;
    s->pending = true;
    s->p_ncubes = ncubes;
    s->p_npoints = npoints;
    s->p_label = tau_label;
    s->p_scale = tau_scale;
    return GVH_OK;
  }
  if ((rc = grow_pinned(&s->h_cube_key, &s->cap_cubes, std::max(1ll, ncubes))) ||
      (rc = grow_pinned(&s->h_point_cell, &s->cap_points, std::max(1ll, npoints))) ||
      (rc = grow_pinned(&s->h_point_vals, &s->cap_vals, std::max(1ll, npoints * 2 * kVars))))
    return rc;
  if (ncubes) {
    SF_CUDA(cudaMemcpyAsync(s->h_cube_key, s->cube_key, ncubes * sizeof(int), cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaMemcpyAsync(s->h_point_cell, s->point_cell, npoints * sizeof(int), cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaMemcpyAsync(s->h_point_vals, s->point_vals, npoints * 2 * kVars * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  }
  SF_CUDA(cudaEventRecord(s->copied, st));
  s->lower = upper;
  s->pending = true;
  s->p_ncubes = ncubes;
  s->p_npoints = npoints;
  s->p_label = tau_label;
  s->p_scale = tau_scale;
  return GVH_OK;
}

int gvh_surface_find_end(gvh_surface *s, long long *n_elements) {
  gvh::NvtxRange range("gvh surface slab (host)");
  if (!s) return sfail(GVH_ERR_INVALID, "gvh_surface_find_end: null argument");
  if (!s->pending) return sfail(GVH_ERR_INVALID, "gvh_surface_find_end: no slab begun");
  gvh_handle *h = s->h;
  SF_CUDA(cudaSetDevice(h->device));
  s->pending = false;
  SF_CUDA(cudaEventSynchronize(s->copied));
  const auto t1 = std::chrono::steady_clock::now();
  const Geometry &g = s->g;
  const long long ncubes = s->p_ncubes, npoints = s->p_npoints;
  gvh::surface::Slab slab;
  slab.dim = s->dim;
  slab.nx = g.nx; slab.ny = g.ny; slab.nz = g.nz;
  slab.dt = h->dt_lattice; slab.dx = h->dx; slab.dy = h->dy; slab.dz = h->dz;
  slab.iso = s->iso;
  slab.eos = h->eos;
  slab.ncubes = ncubes;
  slab.cube_key = s->h_cube_key;
  slab.npoints = npoints;
  slab.point_cell = s->h_point_cell;
  slab.point_vals = s->h_point_vals;
  if (!s->pool) s->pool.reset(new gvh::surface::Pool(s->nthreads));
  wait_format(s);
  if (s->device_rows) {
    s->p_nrows = s->h_rowtot[0];
    s->p_errors = s->h_rowtot[1];
    const int b = s->rbuf;
    const bool text = (s->outputs & gvh::surface::OUT_TEXT) && s->p_nrows > 0;
    const long long bytes = s->h_rowtot[2], nhost = s->h_rowtot[3];
    // the device's text, unless its host rows overflowed (then every row came as values)
    const bool device_text = text && nhost <= s->cap_hrows[b];
    // every row comes as values when they are kept, when there is no text or when the host
    // rows overflowed
    const bool all_rows = s->p_nrows > 0 && (!device_text || (s->outputs & gvh::surface::OUT_ROWS));
    // the copy engine brings the text and rows while the caller goes on; the copies are
    // queued on the rows' stream before the next slab's kernels, which reuse the device buffers
    gvh::surface::DeviceRows d;
    gvh::surface::device_rows_carve(d, s->rowdev, s->rowdev_cap);
    int rc;
    if (all_rows) {
      const long long values = s->p_nrows * gvh::surface::kRowColumns;
      if ((rc = grow_pinned(&s->h_rows[b], &s->cap_rows[b], values))) return rc;
      SF_CUDA(cudaMemcpyAsync(s->h_rows[b], d.rows, (size_t)values * sizeof(double), cudaMemcpyDeviceToHost,
                              s->rows_stream));
    }
    gvh::surface::DeviceText dt;
    if (device_text) {
      if ((rc = grow_pinned(&s->h_text[b], &s->cap_text[b], std::max(1ll, bytes)))) return rc;
      if (bytes)
        SF_CUDA(cudaMemcpyAsync(s->h_text[b], d.text, (size_t)bytes, cudaMemcpyDeviceToHost, s->rows_stream));
      gvh::surface::HostRow *hr = s->h_hrows[b];
      std::sort(hr, hr + nhost, [](const gvh::surface::HostRow &x, const gvh::surface::HostRow &y) {
        return x.row < y.row;
      });
      // the splice needs the places in row order, within the text
      for (long long i = 0; i < nhost; ++i)
        if (hr[i].row < 0 || hr[i].row >= s->p_nrows || hr[i].text_off < (i ? hr[i - 1].text_off : 0) ||
            hr[i].text_off > bytes) {
          // the copies just queued still land in h_text[b] / h_rows[b]: mark them, so that
          // nothing reuses those buffers before they finish, and drop the previous slab's
          // rows so that no later call hands them out as this slab's
          cudaEventRecord(s->copied_out[b], s->rows_stream);
          s->last = gvh::surface::Result();
          s->failed = true;
          return sfail(GVH_ERR_INTERNAL, "gvh_surface_find_end: the device's host rows are inconsistent");
        }
      dt.text = s->h_text[b];
      dt.bytes = bytes;
      dt.host_rows = hr;
      dt.n_host = nhost;
    }
    SF_CUDA(cudaEventRecord(s->copied_out[b], s->rows_stream));
    cudaEvent_t ev = s->copied_out[b];
    const int dev = s->device;
    dt.ready = [ev, dev] {
      cudaSetDevice(dev);
      cudaEventSynchronize(ev);
    };
    // assembled (the device's text) or formatted (rows) on the pool's workers while the
    // caller goes on (the next step, the next slab's device work); anything that reads the
    // rows or text waits for it
    gvh::surface::format_rows(all_rows ? s->h_rows[b] : nullptr, s->p_nrows, *s->pool, s->outputs, s->last, true,
                              dt);
    s->p_text_bytes = device_text ? bytes : 0;
    s->p_host_rows = device_text ? nhost : 0;
    s->p_all_rows = all_rows;
    s->formatting = s->p_nrows > 0;
    s->last.errors = s->p_errors;
  } else {
    gvh::surface::process_slab(slab, gvh::surface::Labels{s->p_label, s->p_scale}, *s->pool, s->outputs, s->c2p,
                               s->last);
  }
  const auto t2 = std::chrono::steady_clock::now();
  gvh_surface_info &in = s->info;
  in.slabs += 1;
  in.hypercubes_last = ncubes;
  in.hypercubes_total += ncubes;
  in.points_last = npoints;
  in.elements_last = s->last.elements;
  in.elements_total += s->last.elements;
  in.errors_total += s->last.errors;
  in.bytes_to_host_total += s->device_rows ? (double)s->p_text_bytes +
                                                 (double)s->p_host_rows * sizeof(gvh::surface::HostRow) +
                                                 (s->p_all_rows ? (double)s->p_nrows * gvh::surface::kRowColumns * 8 : 0.0) +
                                                 32
                                           : (double)ncubes * 4 + (double)npoints * (4 + 2 * kVars * 8) + 8;
  in.device_seconds_total += std::chrono::duration<double>(t1 - s->p_t0).count();
  in.host_seconds_total += std::chrono::duration<double>(t2 - t1).count();
  if (n_elements) *n_elements = s->last.elements;
  return GVH_OK;
}

int gvh_surface_find(gvh_surface *s, double tau_label, double tau_scale, long long *n_elements) {
  int rc = gvh_surface_find_begin(s, tau_label, tau_scale);
  if (rc) return rc;
  return gvh_surface_find_end(s, n_elements);
}

int gvh_surface_get_rows(gvh_surface *s, double *rows, long long max_rows) {
  if (!s || (!rows && max_rows > 0)) return sfail(GVH_ERR_INVALID, "gvh_surface_get_rows: bad argument");
  if (s->failed) return sfail(GVH_ERR_INTERNAL, "gvh_surface_get_rows: the last slab failed");
  wait_format(s);
  if (max_rows < s->last.elements)
    return sfail(GVH_ERR_INVALID, "gvh_surface_get_rows: %lld rows do not fit in %lld", s->last.elements, max_rows);
  if (s->last.elements && !(s->outputs & gvh::surface::OUT_ROWS))
    return sfail(GVH_ERR_INVALID, "gvh_surface_get_rows: rows are not kept (gvh_surface_set_outputs)");
  for (auto &p : s->last.parts) {
    if (!p.rows.empty()) memcpy(rows, p.rows.data(), p.rows.size() * sizeof(double));
    rows += p.rows.size();
  }
  return GVH_OK;
}

int gvh_surface_get_text(gvh_surface *s, const char **text, long long *length) {
  if (!s || !text || !length) return sfail(GVH_ERR_INVALID, "gvh_surface_get_text: null argument");
  if (s->failed) return sfail(GVH_ERR_INTERNAL, "gvh_surface_get_text: the last slab failed");
  wait_format(s);
  const std::string &t = s->last.text();
  *text = t.c_str();
  *length = (long long)t.size();
  return GVH_OK;
}

int gvh_surface_get_info(const gvh_surface *s, gvh_surface_info *info) {
  if (!s || !info) return sfail(GVH_ERR_INVALID, "gvh_surface_get_info: null argument");
  *info = s->info;
  return GVH_OK;
}

}  // extern "C"

namespace gvh {
namespace surface {
void take_text(gvh_surface *s, std::vector<std::string> &out) {
  wait_format(s);
  if (s->failed) return;  // nothing of a failed slab is handed out
  for (auto &p : s->last.parts) {
    out.emplace_back(std::move(p.text));
    p.text.clear();
  }
  s->last.joined.clear();
  s->last.joined_valid = false;
}
}  // namespace surface
}  // namespace gvh
