// gvh_noalloc.cu -- one RK2 step on caller-owned device arrays that allocates nothing.
//
// Who needs it: a caller that already owns all of its device memory and may not (or cannot)
// allocate at step time -- a simulation embedding the KT step into its own run loop with a
// fixed memory plan (the way the reference preallocates once and then calls
// twoStepRungeKutta every step), a framework with its own pool allocator that forbids
// foreign cudaMalloc calls, or code stepping from inside a region where allocation would
// synchronise the device. gvh_create allocates the lattice and its intermediate buffers;
// this entry point takes the state in and out of the caller's arrays and keeps the only
// storage it needs -- the intermediate RK stage q*, p*, u* and a status word -- in a
// fixed-size array compiled into the library (kNoallocScratchBytes). Every GPU that loads
// the library holds that array until the process exits.
//
// Rules of use:
//  * the lattice must fit the array: (nq + 5) * 8 bytes per interior cell plus 256; larger
//    lattices are rejected with GVH_ERR_INVALID and nothing runs;
//  * the first call on a device looks up the array's device address and raises the stage
//    kernels' shared-memory limit (once per device, with that device current); make that
//    first call before any stream capture;
//  * with opts->device >= 0 the call runs on that device and makes the caller's current
//    device current again before it returns (on every path, errors included);
//  * every call shares the one array and it keeps the last call's contents: the status word
//    is cleared at the start of each call, and two calls whose work overlaps on the GPU
//    (different streams, or host threads without ordering) race on it -- order them.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <string>

#include "../../include/gvh.h"
#include "gvh_physics.cuh"
#include "gvh_stage.cuh"

using namespace gvh;

namespace {

constexpr size_t kNoallocScratchBytes = 32u << 20;  // 32 MiB
constexpr int kMaxDevices = 64;

// The scratch: [status word, padded to 256 B][q* (nq x n)][p* (n)][u* (4 x n)].
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_setup_mutex;
std::atomic<unsigned char *> g_scratch_ptr[kMaxDevices];

thread_local std::string g_noalloc_error;

int nfail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_noalloc_error = buf;
  return code;
}

// Device address of the scratch on the current device (looked up once per device).
int scratch_address(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return nfail(GVH_ERR_INVALID, "device ordinal %d out of range", dev);
  unsigned char *p = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    p = g_scratch_ptr[dev].load(std::memory_order_relaxed);
    if (!p) {
      cudaError_t err = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_scratch);
      if (err != cudaSuccess)
        return nfail(GVH_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", dev, cudaGetErrorString(err));
      // the stage kernels' shared-memory limit, part of the same one-time set-up
      err = allow_all_stage_kernels();
      if (err != cudaSuccess)
        return nfail(GVH_ERR_CUDA, "stage kernel set-up on device %d: %s", dev, cudaGetErrorString(err));
      g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return GVH_OK;
}

// Puts the caller's current device back when the call returns (the entry point makes
// opts->device current for its work and must not leave the calling thread switched).
struct DeviceRestore {
  int saved = -1;
  ~DeviceRestore() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};

template <int EOS, bool SHEAR, bool BULK, bool MIXED>
void launch_pair(const StageArgs &a1, const StageArgs &a2, long long, cudaStream_t st) {
  const dim3 grid = stage_grid(a1.ncells);
  const size_t smem = stage_smem_bytes<SHEAR, BULK>();
  kt_stage_kernel<EOS, SHEAR, BULK, false, MIXED><<<grid, kBlock, smem, st>>>(a1);
  kt_stage_kernel<EOS, SHEAR, BULK, true, MIXED><<<grid, kBlock, smem, st>>>(a2);
}

template <int EOS, bool MIXED>
void dispatch_physics(int shear, int bulk, const StageArgs &a1, const StageArgs &a2, long long n, cudaStream_t st) {
  if (!shear) launch_pair<EOS, false, false, MIXED>(a1, a2, n, st);
  else if (!bulk) launch_pair<EOS, true, false, MIXED>(a1, a2, n, st);
  else launch_pair<EOS, true, true, MIXED>(a1, a2, n, st);
}

}  // namespace

extern "C" {

long long gvh_rk2_step_noalloc_max_bytes(void) { return (long long)kNoallocScratchBytes; }

const char *gvh_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

int gvh_rk2_step_noalloc(const gvh_lattice_params *L, const gvh_hydro_params *H, const gvh_options *opts, double t,
                         double dt, double T_reg, double *q, double *e, double *p, const double *u_prev,
                         const double *u, double *u_next, unsigned *status_out, void *stream) {
  if (!L || !H || !q || !e || !p || !u_prev || !u || !u_next)
    return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: null argument");
  gvh_options o;
  if (opts) o = *opts; else gvh_default_options(&o);
  const int nx = L->numLatticePointsX, ny = L->numLatticePointsY, nz = L->numLatticePointsRapidity;
  if (nx < 1 || ny < 1 || nz < 1) return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: lattice sizes must be >= 1");
  if (!(L->latticeSpacingX > 0 && L->latticeSpacingY > 0 && L->latticeSpacingRapidity > 0 &&
        L->latticeSpacingProperTime > 0))
    return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: lattice spacings must be > 0");
  if (o.bulk && !o.shear) return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: bulk needs shear");
  if (o.eos != GVH_EOS_QCD && o.eos != GVH_EOS_CONFORMAL)
    return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: unknown eos");
  if (o.precision != GVH_PRECISION_FP64 && o.precision != GVH_PRECISION_MIXED)
    return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: unknown precision");
  if (!(o.theta > 0)) return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: the limiter's theta must be > 0");
  if (o.coordinates != GVH_COORDINATES_MILNE && o.coordinates != GVH_COORDINATES_CARTESIAN)
    return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: unknown coordinates %d", o.coordinates);
  if (u_next == u || u_next == u_prev)
    return nfail(GVH_ERR_INVALID, "gvh_rk2_step_noalloc: u_next must not alias u or u_prev");
  const int nq = 4 + (o.shear ? 10 : 0) + (o.bulk ? 1 : 0);
  const long long n = (long long)nx * ny * nz;
  const unsigned long long need = 256ull + (unsigned long long)(nq + 5) * (unsigned long long)n * sizeof(double);
  if (need > kNoallocScratchBytes)
    return nfail(GVH_ERR_INVALID,
                 "gvh_rk2_step_noalloc: a %dx%dx%d lattice needs %llu bytes of intermediate storage, more than the "
                 "%zu-byte static scratch; use gvh_create/gvh_rk2_step for lattices this large",
                 nx, ny, nz, need, kNoallocScratchBytes);
  int dev = o.device, caller_dev = -1;
  {
    cudaError_t err = cudaGetDevice(&caller_dev);
    if (err != cudaSuccess) return nfail(GVH_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(err));
  }
  DeviceRestore restore;
  if (dev < 0) {
    dev = caller_dev;
  } else if (dev != caller_dev) {
    cudaError_t err = cudaSetDevice(dev);
    if (err != cudaSuccess) return nfail(GVH_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(err));
    restore.saved = caller_dev;  // every return from here on switches back
  }
  unsigned char *scratch = nullptr;
  int rc = scratch_address(dev, &scratch);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned *status = reinterpret_cast<unsigned *>(scratch);
  double *qS = reinterpret_cast<double *>(scratch + 256);
  double *pS = qS + (size_t)nq * n;
  double *uS = pS + n;
  cudaError_t err = cudaMemsetAsync(status, 0, sizeof(unsigned), st);  // the status word starts at zero
  if (err != cudaSuccess) return nfail(GVH_ERR_CUDA, "clearing the status word: %s", cudaGetErrorString(err));

  StageArgs a;
  memset(&a, 0, sizeof a);
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.sy = nx; a.sz = (long long)nx * ny; a.cs = n; a.ncells = n;
  a.dx = L->latticeSpacingX; a.dy = L->latticeSpacingY; a.dz = L->latticeSpacingRapidity;
  a.dt = L->latticeSpacingProperTime;
  set_inverse_spacings(a);
  a.etabar = H->shearViscosityToEntropyDensity;
  a.theta = o.theta;
  a.cartesian = o.coordinates == GVH_COORDINATES_CARTESIAN;
  a.e_reg = (o.eos == GVH_EOS_CONFORMAL) ? energy_density_of_T<EOS_CONFORMAL>(T_reg) : energy_density_of_T<EOS_QCD>(T_reg);
  a.status = status;
  a.e = e;
  const double t1 = t + dt;
  StageArgs a1 = a, a2 = a;
  // stage 1: q^n, p^n, u^n, u^{n-1} -> q*, p*, u* (all three in the scratch), e in place
  a1.t_euler = t; a1.t_after = t1;
  a1.qin = q; a1.qn = nullptr; a1.qout = qS;
  a1.pin = p; a1.pout = pS;
  a1.uin = u; a1.uprev = u_prev; a1.uout = uS;
  // stage 2: q*, p*, u*, u^n, q^n -> q^{n+1} (over q^n), p^{n+1} (over p^n), u^{n+1}
  a2.t_euler = t1; a2.t_after = t1;
  a2.qin = qS; a2.qn = q; a2.qout = q;
  a2.pin = pS; a2.pout = p;
  a2.uin = uS; a2.uprev = u; a2.uout = u_next;
  const bool mixed = o.precision == GVH_PRECISION_MIXED;
  if (o.eos == GVH_EOS_CONFORMAL) {
    if (mixed) dispatch_physics<EOS_CONFORMAL, true>(o.shear, o.bulk, a1, a2, n, st);
    else dispatch_physics<EOS_CONFORMAL, false>(o.shear, o.bulk, a1, a2, n, st);
  } else {
    if (mixed) dispatch_physics<EOS_QCD, true>(o.shear, o.bulk, a1, a2, n, st);
    else dispatch_physics<EOS_QCD, false>(o.shear, o.bulk, a1, a2, n, st);
  }
  err = cudaGetLastError();
  if (err != cudaSuccess) return nfail(GVH_ERR_CUDA, "stage launch: %s", cudaGetErrorString(err));
  if (status_out) {
    err = cudaMemcpyAsync(status_out, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) return nfail(GVH_ERR_CUDA, "reading the status word: %s", cudaGetErrorString(err));
  }
  return GVH_OK;
}

}  // extern "C"
