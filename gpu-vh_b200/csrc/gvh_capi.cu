// gvh_capi.cu -- libgvh.so: the C ABI declared in include/gvh.h.
//
// A handle owns one lattice in HBM (interior cells only, component-major SoA, see
// gvh_stage.cuh) and a CUDA stream. gvh_rk2_step launches two fused stage kernels; the
// reference issues ~21 launches, 12 stream creations/destructions and a device-wide
// synchronisation for the same step (FullyDiscreteKurganovTadmorScheme.cu:109-139,
// GhostCells.cu:19-28).
//
// Buffers (one allocation): qA, qB (conserved, nq each), e, pA, pB, u[3] (4 each).
//   stage 1: q^n=qA -> q*=qB,  p^n=pA -> p*=pB,  u^n, u^{n-1} -> u* (over u^{n-1}), e in place
//   stage 2: q*=qB, q^n=qA -> q^{n+1}=qA (in place: q^n is read at the centre only),
//            p* -> pA,  u*, u^n -> u^{n+1} (third buffer), e in place
// after the step u^{n+1} is current and u^n previous, as after the reference's
// swapFluidVelocity (FullyDiscreteKurganovTadmorScheme.cu:131).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/gvh.h"
#include "gvh_handle.h"
#include "gvh_layout.cuh"
#include "gvh_nvtx.h"
#include "gvh_stage.cuh"
#include "gvh_validity.cuh"

using namespace gvh;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define GVH_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t err_ = (call);                                                                  \
    if (err_ != cudaSuccess) return fail(GVH_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(err_)); \
  } while (0)

constexpr int kThreads = gvh::kBlock;

}  // namespace


namespace {

template <int EOS, bool SHEAR, bool BULK, bool MIXED>
int launch_stage_p(const gvh_handle *h, const StageArgs &a, bool stage2) {
  const size_t smem = stage_smem_bytes<SHEAR, BULK>();
  if (h->ncells < h->split_below) {
    // fewer cells than one wave of the one-thread-per-cell kernel: four warps per 32 cells
    const dim3 grid = split_grid(h->ncells);
    if (stage2) kt_stage_split_kernel<EOS, SHEAR, BULK, true, MIXED><<<grid, kThreads, smem, h->stream>>>(a);
    else kt_stage_split_kernel<EOS, SHEAR, BULK, false, MIXED><<<grid, kThreads, smem, h->stream>>>(a);
    GVH_CUDA(cudaGetLastError());
    return GVH_OK;
  }
  const dim3 grid = stage_grid(h->ncells);
  if (stage2) kt_stage_kernel<EOS, SHEAR, BULK, true, MIXED><<<grid, kThreads, smem, h->stream>>>(a);
  else kt_stage_kernel<EOS, SHEAR, BULK, false, MIXED><<<grid, kThreads, smem, h->stream>>>(a);
  GVH_CUDA(cudaGetLastError());
  return GVH_OK;
}

template <int EOS, bool SHEAR, bool BULK>
int launch_stage(const gvh_handle *h, const StageArgs &a, bool stage2) {
  if (h->precision == GVH_PRECISION_MIXED) return launch_stage_p<EOS, SHEAR, BULK, true>(h, a, stage2);
  return launch_stage_p<EOS, SHEAR, BULK, false>(h, a, stage2);
}

template <int EOS>
int dispatch_physics(const gvh_handle *h, const StageArgs &a, bool stage2) {
  if (!h->shear) return launch_stage<EOS, false, false>(h, a, stage2);
  if (!h->bulk) return launch_stage<EOS, true, false>(h, a, stage2);
  return launch_stage<EOS, true, true>(h, a, stage2);
}

int dispatch(const gvh_handle *h, const StageArgs &a, bool stage2) {
  if (h->eos == GVH_EOS_CONFORMAL) return dispatch_physics<EOS_CONFORMAL>(h, a, stage2);
  return dispatch_physics<EOS_QCD>(h, a, stage2);
}

// checkValidity after the step (FullyDiscreteKurganovTadmorScheme.cu:137): t + dt, the new
// e, p and u, and u one step earlier.
int launch_validity(const gvh_handle *h, double t_new, const double *u_new, const double *u_old) {
  ValidityArgs v;
  v.nx = h->nx; v.ny = h->ny; v.nz = h->nz;
  v.sy = h->sy; v.sz = h->sz; v.cs = h->cs; v.ncells = h->ncells;
  v.dx = h->dx; v.dy = h->dy; v.dz = h->dz; v.dt = h->dt_lattice; v.etabar = h->etabar;
  v.t = t_new;
  v.e = h->e; v.p = h->pA; v.u = u_new; v.up = u_old;
  v.diag = h->diag;
  const unsigned blocks = (unsigned)((h->ncells + 255) / 256);
  const bool conf = h->eos == GVH_EOS_CONFORMAL;
  if (!h->shear) {
    if (conf) validity_kernel<EOS_CONFORMAL, false, false><<<blocks, 256, 0, h->stream>>>(v);
    else validity_kernel<EOS_QCD, false, false><<<blocks, 256, 0, h->stream>>>(v);
  } else if (!h->bulk) {
    if (conf) validity_kernel<EOS_CONFORMAL, true, false><<<blocks, 256, 0, h->stream>>>(v);
    else validity_kernel<EOS_QCD, true, false><<<blocks, 256, 0, h->stream>>>(v);
  } else {
    if (conf) validity_kernel<EOS_CONFORMAL, true, true><<<blocks, 256, 0, h->stream>>>(v);
    else validity_kernel<EOS_QCD, true, true><<<blocks, 256, 0, h->stream>>>(v);
  }
  GVH_CUDA(cudaGetLastError());
  return GVH_OK;
}

Pack make_pack(const gvh_handle *h) { return Pack{h->nx, h->ny, h->nz, h->sy, h->sz, h->ng}; }

int ensure_staging(gvh_handle *h) {
  if (h->staging) return GVH_OK;
  size_t bytes = (size_t)(h->nq + 10) * h->ng * sizeof(double);
  if (cudaMalloc(&h->staging, bytes) != cudaSuccess) return fail(GVH_ERR_NOMEM, "staging allocation failed");
  return GVH_OK;
}

// Releases whatever ensure_async made (null members are skipped), so a failed set-up leaves
// the handle as it was and the next call starts over.
void release_async(gvh_handle *h) {
  for (int a = 0; a < 2; ++a) {
    if (h->staging_in[a]) cudaFree(h->staging_in[a]);
    if (h->staging_out[a]) cudaFree(h->staging_out[a]);
    if (h->ev_in_free[a]) cudaEventDestroy(h->ev_in_free[a]);
    if (h->ev_out_free[a]) cudaEventDestroy(h->ev_out_free[a]);
    h->staging_in[a] = h->staging_out[a] = nullptr;
    h->ev_in_free[a] = h->ev_out_free[a] = nullptr;
  }
  if (h->s_h2d) cudaStreamDestroy(h->s_h2d);
  if (h->s_d2h) cudaStreamDestroy(h->s_d2h);
  if (h->ev_in_ready) cudaEventDestroy(h->ev_in_ready);
  if (h->ev_out_ready) cudaEventDestroy(h->ev_out_ready);
  if (h->ev_fence) cudaEventDestroy(h->ev_fence);
  h->s_h2d = h->s_d2h = nullptr;
  h->ev_in_ready = h->ev_out_ready = h->ev_fence = nullptr;
  h->async_ready = 0;
}

int ensure_async(gvh_handle *h) {
  if (h->async_ready) return GVH_OK;
  const size_t bytes = (size_t)(h->nq + 10) * h->ng * sizeof(double);
  bool ok = true;
  for (int a = 0; a < 2; ++a) {
    ok = ok && cudaMalloc(&h->staging_in[a], bytes) == cudaSuccess;
    ok = ok && cudaMalloc(&h->staging_out[a], bytes) == cudaSuccess;
  }
  if (!ok) {
    release_async(h);
    cudaGetLastError();
    return fail(GVH_ERR_NOMEM, "async staging allocation failed");
  }
  h->in_slot = h->out_slot = 0;
  cudaError_t ec = cudaSuccess;
  auto step = [&ec](cudaError_t e) {
    if (ec == cudaSuccess) ec = e;
  };
  step(cudaStreamCreateWithFlags(&h->s_h2d, cudaStreamNonBlocking));
  step(cudaStreamCreateWithFlags(&h->s_d2h, cudaStreamNonBlocking));
  step(cudaEventCreateWithFlags(&h->ev_in_ready, cudaEventDisableTiming));
  step(cudaEventCreateWithFlags(&h->ev_out_ready, cudaEventDisableTiming));
  step(cudaEventCreateWithFlags(&h->ev_fence, cudaEventDisableTiming));
  for (int a = 0; a < 2; ++a) {
    step(cudaEventCreateWithFlags(&h->ev_in_free[a], cudaEventDisableTiming));
    step(cudaEventCreateWithFlags(&h->ev_out_free[a], cudaEventDisableTiming));
  }
  // the events start recorded (complete), so the first waits pass
  if (ec == cudaSuccess) {
    for (int a = 0; a < 2; ++a) {
      step(cudaEventRecord(h->ev_in_free[a], h->stream));
      step(cudaEventRecord(h->ev_out_free[a], h->stream));
    }
    step(cudaEventRecord(h->ev_in_ready, h->stream));
    step(cudaEventRecord(h->ev_out_ready, h->stream));
  }
  if (ec != cudaSuccess) {
    release_async(h);
    return fail(GVH_ERR_CUDA, "async set-up: %s", cudaGetErrorString(ec));
  }
  h->async_ready = 1;
  return GVH_OK;
}

void internal_fields(const gvh_handle *h, double **f) {
  for (int n = 0; n < h->nq; ++n) f[n] = h->qA + n * h->cs;
  f[h->nq] = h->e;
  f[h->nq + 1] = h->pA;
  for (int m = 0; m < 4; ++m) f[h->nq + 2 + m] = h->u[h->ucur] + m * h->cs;
  for (int m = 0; m < 4; ++m) f[h->nq + 6 + m] = h->u[h->uprev] + m * h->cs;
}

int set_device(const gvh_handle *h) {
  GVH_CUDA(cudaSetDevice(h->device));
  return GVH_OK;
}

}  // namespace

extern "C" {

void gvh_default_options(gvh_options *o) {
  if (!o) return;
  o->eos = GVH_EOS_QCD;
  o->shear = 1;
  o->bulk = 1;
  o->precision = GVH_PRECISION_FP64;
  o->theta = 2.0;
  o->device = -1;
  o->coordinates = GVH_COORDINATES_MILNE;
}

const char *gvh_last_error(void) { return g_last_error.c_str(); }

int gvh_create(const gvh_lattice_params *L, const gvh_hydro_params *H, const gvh_options *opts, gvh_handle **out) {
  if (!L || !H || !out) return fail(GVH_ERR_INVALID, "gvh_create: null argument");
  *out = nullptr;
  gvh_options o;
  if (opts) o = *opts; else gvh_default_options(&o);
  if (L->numLatticePointsX < 1 || L->numLatticePointsY < 1 || L->numLatticePointsRapidity < 1)
    return fail(GVH_ERR_INVALID, "gvh_create: lattice sizes must be >= 1");
  if (!(L->latticeSpacingX > 0) || !(L->latticeSpacingY > 0) || !(L->latticeSpacingRapidity > 0) ||
      !(L->latticeSpacingProperTime > 0))
    return fail(GVH_ERR_INVALID, "gvh_create: lattice spacings must be > 0");
  if (o.eos != GVH_EOS_QCD && o.eos != GVH_EOS_CONFORMAL) return fail(GVH_ERR_INVALID, "gvh_create: unknown eos");
  if (o.bulk && !o.shear) return fail(GVH_ERR_INVALID, "gvh_create: bulk needs shear (component 14 layout)");
  if (o.precision != GVH_PRECISION_FP64 && o.precision != GVH_PRECISION_MIXED)
    return fail(GVH_ERR_INVALID, "gvh_create: unknown precision mode %d", o.precision);
  if (o.shear && !(H->shearViscosityToEntropyDensity > 0))
    return fail(GVH_ERR_INVALID, "gvh_create: eta/s must be > 0 with shear");
  if (!(o.theta > 0)) return fail(GVH_ERR_INVALID, "gvh_create: the limiter's theta must be > 0");
  if (o.coordinates != GVH_COORDINATES_MILNE && o.coordinates != GVH_COORDINATES_CARTESIAN)
    return fail(GVH_ERR_INVALID, "gvh_create: unknown coordinates %d", o.coordinates);
  int dev = o.device;
  if (dev < 0) GVH_CUDA(cudaGetDevice(&dev));
  GVH_CUDA(cudaSetDevice(dev));
  {
    // the stage kernels' shared-memory limit, once per device (kernel attributes are per device)
    static std::mutex mu;
    static unsigned long long prepared = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && !(prepared & (1ull << dev))) {
      GVH_CUDA(allow_all_stage_kernels());
      GVH_CUDA(allow_all_split_kernels());
      prepared |= 1ull << dev;
    }
  }

  int sms = 0;
  GVH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  gvh_handle *h = new gvh_handle();
  memset(h, 0, sizeof(*h));
  h->nx = L->numLatticePointsX; h->ny = L->numLatticePointsY; h->nz = L->numLatticePointsRapidity;
  h->nq = 4 + (o.shear ? 10 : 0) + (o.bulk ? 1 : 0);
  h->ncells = (long long)h->nx * h->ny * h->nz;
  h->ng = (long long)(h->nx + 4) * (h->ny + 4) * (h->nz + 4);
  h->sy = h->nx;
  h->sz = (long long)h->nx * h->ny;
  h->cs = (h->ncells + 31) / 32 * 32;  // 256-byte aligned components
  h->dx = L->latticeSpacingX; h->dy = L->latticeSpacingY; h->dz = L->latticeSpacingRapidity;
  h->dt_lattice = L->latticeSpacingProperTime;
  h->etabar = H->shearViscosityToEntropyDensity;
  h->theta = o.theta;
  h->cartesian = o.coordinates == GVH_COORDINATES_CARTESIAN;
  h->eos = o.eos; h->shear = o.shear; h->bulk = o.bulk; h->precision = o.precision; h->device = dev;
  // one wave of the one-thread-per-cell stage kernel: below it the split kernel runs
  h->split_below = (long long)sms * GVH_MIN_BLOCKS * kThreads;
  h->ucur = 0; h->uprev = 1; h->ufree = 2;

  size_t nbuf = 2 * (size_t)h->nq + 3 + 12;
  size_t bytes = nbuf * h->cs * sizeof(double) + 256;
  if (cudaMalloc(&h->block, bytes) != cudaSuccess) {
    delete h;
    return fail(GVH_ERR_NOMEM, "gvh_create: cannot allocate %zu bytes", bytes);
  }
  cudaMemset(h->block, 0, bytes);
  double *b = h->block;
  h->qA = b; b += h->nq * h->cs;
  h->qB = b; b += h->nq * h->cs;
  h->e = b; b += h->cs;
  h->pA = b; b += h->cs;
  h->pB = b; b += h->cs;
  for (int m = 0; m < 3; ++m) { h->u[m] = b; b += 4 * h->cs; }
  h->status = reinterpret_cast<unsigned *>(b);
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(h->block);
    delete h;
    return fail(GVH_ERR_CUDA, "gvh_create: stream creation failed");
  }
  h->stream = h->own_stream;
  *out = h;
  return GVH_OK;
}

int gvh_destroy(gvh_handle *h) {
  if (!h) return GVH_OK;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  cudaStreamSynchronize(h->own_stream);
  cudaStreamDestroy(h->own_stream);
  cudaFree(h->block);
  if (h->staging) cudaFree(h->staging);
  if (h->diag) cudaFree(h->diag);
  if (h->host_word) cudaFreeHost(h->host_word);
  if (h->async_ready) {
    cudaStreamSynchronize(h->s_h2d);
    cudaStreamSynchronize(h->s_d2h);
    release_async(h);
  }
  delete h;
  return GVH_OK;
}

int gvh_num_conserved(const gvh_handle *h) { return h ? h->nq : GVH_ERR_INVALID; }
int gvh_num_fields(const gvh_handle *h) { return h ? h->nq + 10 : GVH_ERR_INVALID; }
long long gvh_num_lattice_cells(const gvh_handle *h) { return h ? h->ng : GVH_ERR_INVALID; }
int gvh_launches_per_step(const gvh_handle *h) { return h ? 2 : GVH_ERR_INVALID; }

int gvh_set_state(gvh_handle *h, const double *const *fields, int n_fields) {
  if (!h || !fields) return fail(GVH_ERR_INVALID, "gvh_set_state: null argument");
  if (n_fields != h->nq + 10) return fail(GVH_ERR_INVALID, "gvh_set_state: expected %d fields", h->nq + 10);
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_staging(h))) return rc;
  const size_t fb = h->ng * sizeof(double);
  for (int f = 0; f < n_fields; ++f) {
    const double *src = fields[f];
    if (!src && f >= h->nq + 6) src = fields[f - 4];  // up defaults to u
    if (!src) return fail(GVH_ERR_INVALID, "gvh_set_state: field %d is null", f);
    GVH_CUDA(cudaMemcpyAsync(h->staging + f * h->ng, src, fb, cudaMemcpyDefault, h->stream));
  }
  FieldTable dst = {};
  internal_fields(h, dst.p);
  pack_kernel<<<(unsigned)((h->ncells + 255) / 256), 256, 0, h->stream>>>(make_pack(h), n_fields, h->staging, dst);
  GVH_CUDA(cudaGetLastError());
  GVH_CUDA(cudaStreamSynchronize(h->stream));  // the caller may reuse its arrays on return
  return GVH_OK;
}

int gvh_get_state(gvh_handle *h, double *const *fields, int n_fields) {
  if (!h || !fields) return fail(GVH_ERR_INVALID, "gvh_get_state: null argument");
  if (n_fields != h->nq + 10) return fail(GVH_ERR_INVALID, "gvh_get_state: expected %d fields", h->nq + 10);
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_staging(h))) return rc;
  FieldTable src = {};
  internal_fields(h, src.p);
  for (int f = 0; f < n_fields; ++f)
    if (!fields[f]) src.p[f] = nullptr;
  unpack_kernel<<<(unsigned)((h->ng + 255) / 256), 256, 0, h->stream>>>(make_pack(h), n_fields, src, h->staging);
  GVH_CUDA(cudaGetLastError());
  const size_t fb = h->ng * sizeof(double);
  for (int f = 0; f < n_fields; ++f)
    if (fields[f]) GVH_CUDA(cudaMemcpyAsync(fields[f], h->staging + f * h->ng, fb, cudaMemcpyDefault, h->stream));
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  return GVH_OK;
}

int gvh_gather_state_device(gvh_handle *h, const void *const *fields, int n_fields, int elem_bytes) {
  if (!h || !fields) return fail(GVH_ERR_INVALID, "gvh_gather_state_device: null argument");
  if (n_fields != h->nq + 10)
    return fail(GVH_ERR_INVALID, "gvh_gather_state_device: expected %d fields", h->nq + 10);
  if (elem_bytes != 4 && elem_bytes != 8)
    return fail(GVH_ERR_INVALID, "gvh_gather_state_device: elem_bytes must be 4 or 8");
  RefTable src = {};
  for (int f = 0; f < n_fields; ++f) {
    const void *a = fields[f];
    if (!a && f >= h->nq + 6) a = fields[f - 4];  // up defaults to u
    if (!a) return fail(GVH_ERR_INVALID, "gvh_gather_state_device: field %d is null", f);
    src.p[f] = const_cast<void *>(a);
  }
  int rc;
  if ((rc = set_device(h))) return rc;
  FieldTable dst = {};
  internal_fields(h, dst.p);
  const unsigned blocks = (unsigned)((h->ncells + 255) / 256);
  if (elem_bytes == 4) gather_ref_kernel<float><<<blocks, 256, 0, h->stream>>>(make_pack(h), n_fields, src, dst);
  else gather_ref_kernel<double><<<blocks, 256, 0, h->stream>>>(make_pack(h), n_fields, src, dst);
  GVH_CUDA(cudaGetLastError());
  return GVH_OK;
}

int gvh_scatter_state_device(gvh_handle *h, void *const *fields, int n_fields, int elem_bytes) {
  if (!h || !fields) return fail(GVH_ERR_INVALID, "gvh_scatter_state_device: null argument");
  if (n_fields != h->nq + 10)
    return fail(GVH_ERR_INVALID, "gvh_scatter_state_device: expected %d fields", h->nq + 10);
  if (elem_bytes != 4 && elem_bytes != 8)
    return fail(GVH_ERR_INVALID, "gvh_scatter_state_device: elem_bytes must be 4 or 8");
  int rc;
  if ((rc = set_device(h))) return rc;
  RefTable dst = {};
  for (int f = 0; f < n_fields; ++f) dst.p[f] = fields[f];
  FieldTable src = {};
  internal_fields(h, src.p);
  const unsigned blocks = (unsigned)((h->ng + 255) / 256);
  if (elem_bytes == 4) scatter_ref_kernel<float><<<blocks, 256, 0, h->stream>>>(make_pack(h), n_fields, src, dst);
  else scatter_ref_kernel<double><<<blocks, 256, 0, h->stream>>>(make_pack(h), n_fields, src, dst);
  GVH_CUDA(cudaGetLastError());
  return GVH_OK;
}

int gvh_set_primitive_state_p(gvh_handle *h, const double *const *prim, int n_prim, const double *p_ghosted) {
  if (!h || !prim) return fail(GVH_ERR_INVALID, "gvh_set_primitive_state: null argument");
  const int want = 5 + (h->nq - 4);
  if (n_prim != want) return fail(GVH_ERR_INVALID, "gvh_set_primitive_state: expected %d arrays", want);
  for (int f = 0; f < n_prim; ++f)
    if (!prim[f]) return fail(GVH_ERR_INVALID, "gvh_set_primitive_state: array %d is null", f);
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_staging(h))) return rc;
  const size_t fb = h->ng * sizeof(double);
  for (int f = 0; f < n_prim; ++f)
    GVH_CUDA(cudaMemcpyAsync(h->staging + f * h->ng, prim[f], fb, cudaMemcpyDefault, h->stream));
  if (p_ghosted)
    GVH_CUDA(cudaMemcpyAsync(h->staging + n_prim * h->ng, p_ghosted, fb, cudaMemcpyDefault, h->stream));
  FieldTable dst = {};
  dst.p[0] = h->e;
  for (int m = 0; m < 4; ++m) dst.p[1 + m] = h->u[h->ucur] + m * h->cs;
  for (int n = 4; n < h->nq; ++n) dst.p[5 + n - 4] = h->qA + n * h->cs;
  dst.p[n_prim] = h->pA;
  const int n_pack = n_prim + (p_ghosted ? 1 : 0);
  pack_kernel<<<(unsigned)((h->ncells + 255) / 256), 256, 0, h->stream>>>(make_pack(h), n_pack, h->staging, dst);
  GVH_CUDA(cudaGetLastError());
  const unsigned blocks = (unsigned)((h->ncells + 255) / 256);
  if (h->eos == GVH_EOS_CONFORMAL)
    init_conserved_kernel<EOS_CONFORMAL><<<blocks, 256, 0, h->stream>>>(h->ncells, h->nq, h->cs, h->qA, h->e, h->pA,
                                                                        h->u[h->ucur], h->u[h->uprev], p_ghosted != nullptr);
  else
    init_conserved_kernel<EOS_QCD><<<blocks, 256, 0, h->stream>>>(h->ncells, h->nq, h->cs, h->qA, h->e, h->pA,
                                                                  h->u[h->ucur], h->u[h->uprev], p_ghosted != nullptr);
  GVH_CUDA(cudaGetLastError());
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  return GVH_OK;
}

int gvh_set_hotspot_state(gvh_handle *h, const gvh_hotspots *hs) {
  if (!h || !hs) return fail(GVH_ERR_INVALID, "gvh_set_hotspot_state: null argument");
  if (hs->n < 1 || !hs->x || !hs->y || !hs->w || !(hs->sigma > 0) || !(hs->sigma_eta > 0))
    return fail(GVH_ERR_INVALID, "gvh_set_hotspot_state: n >= 1 sources with positions and weights, sigma > 0 and "
                                 "sigma_eta > 0");
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_staging(h))) return rc;
  // sources and the transverse plane in the staging area
  if (3ll * hs->n + (long long)h->nx * h->ny > (long long)(h->nq + 10) * h->ng)
    return fail(GVH_ERR_INVALID, "gvh_set_hotspot_state: too many sources for this lattice (%d)", hs->n);
  const size_t nb = hs->n * sizeof(double);
  GVH_CUDA(cudaMemcpyAsync(h->staging, hs->x, nb, cudaMemcpyHostToDevice, h->stream));
  GVH_CUDA(cudaMemcpyAsync(h->staging + hs->n, hs->y, nb, cudaMemcpyHostToDevice, h->stream));
  GVH_CUDA(cudaMemcpyAsync(h->staging + 2 * hs->n, hs->w, nb, cudaMemcpyHostToDevice, h->stream));
  gvh_lattice_params L = {h->nx, h->ny, h->nz, h->nx + 4, h->ny + 4, h->nz + 4, 0, h->dx, h->dy, h->dz,
                          h->dt_lattice};
  const HotspotArgs ha = hotspot_args(h->nx, h->ny, h->nz, h->sy, h->sz, &L, hs, h->staging);
  double *plane = h->staging + 3 * hs->n;
  hotspot_plane_kernel<<<(unsigned)((h->nx * h->ny + 255) / 256), 256, 0, h->stream>>>(ha, plane);
  const unsigned blocks = (unsigned)((h->ncells + 255) / 256);
  hotspot_fill_kernel<<<blocks, 256, 0, h->stream>>>(ha, plane, h->e, h->u[h->ucur], h->cs, h->qA, h->nq);
  if (h->eos == GVH_EOS_CONFORMAL)
    init_conserved_kernel<EOS_CONFORMAL><<<blocks, 256, 0, h->stream>>>(h->ncells, h->nq, h->cs, h->qA, h->e, h->pA,
                                                                        h->u[h->ucur], h->u[h->uprev], 0);
  else
    init_conserved_kernel<EOS_QCD><<<blocks, 256, 0, h->stream>>>(h->ncells, h->nq, h->cs, h->qA, h->e, h->pA,
                                                                  h->u[h->ucur], h->u[h->uprev], 0);
  GVH_CUDA(cudaGetLastError());
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  return GVH_OK;
}

int gvh_set_primitive_state(gvh_handle *h, const double *const *prim, int n_prim) {
  return gvh_set_primitive_state_p(h, prim, n_prim, nullptr);
}

int gvh_rk2_step(gvh_handle *h, double t, double dt, double T_reg) {
  if (!h) return fail(GVH_ERR_INVALID, "gvh_rk2_step: null handle");
  int rc;
  if ((rc = set_device(h))) return rc;
  StageArgs a;
  memset(&a, 0, sizeof a);
  a.nx = h->nx; a.ny = h->ny; a.nz = h->nz;
  a.sy = h->sy; a.sz = h->sz; a.cs = h->cs; a.ncells = h->ncells;
  a.dx = h->dx; a.dy = h->dy; a.dz = h->dz; a.dt = h->dt_lattice;
  set_inverse_spacings(a);
  a.etabar = h->etabar; a.theta = h->theta;
  a.cartesian = h->cartesian;
  a.e_reg = (h->eos == GVH_EOS_CONFORMAL) ? energy_density_of_T<EOS_CONFORMAL>(T_reg)
                                          : energy_density_of_T<EOS_QCD>(T_reg);
  a.status = h->status;
  a.e = h->e;
  const double t1 = t + dt;
  // stage 1 (predictor); it also keeps the running maximum of the propagation speed
  // (gvh_max_propagation_speed) in the third 8-byte word after the status word
  a.speed_max = reinterpret_cast<unsigned long long *>(h->status) + 2;
  a.t_euler = t; a.t_after = t1;
  a.qin = h->qA; a.qn = nullptr; a.qout = h->qB;
  a.pin = h->pA; a.pout = h->pB;
  a.uin = h->u[h->ucur]; a.uprev = h->u[h->uprev]; a.uout = h->u[h->uprev];
  {
    NvtxRange r("gvh stage 1 (predictor)");
    if ((rc = dispatch(h, a, false))) return rc;
  }
  // stage 2 (corrector + Heun combination)
  a.speed_max = nullptr;
  a.t_euler = t1; a.t_after = t1;
  a.qin = h->qB; a.qn = h->qA; a.qout = h->qA;
  a.pin = h->pB; a.pout = h->pA;
  a.uin = h->u[h->uprev]; a.uprev = h->u[h->ucur]; a.uout = h->u[h->ufree];
  a.diag = h->validity_on ? h->diag : nullptr;
  {
    NvtxRange r("gvh stage 2 (corrector)");
    if ((rc = dispatch(h, a, true))) return rc;
  }
  if (h->validity_on && (rc = launch_validity(h, t1, h->u[h->ufree], h->u[h->ucur]))) return rc;
  const int nc = h->ufree, np = h->ucur, nf = h->uprev;
  h->ucur = nc; h->uprev = np; h->ufree = nf;
  return GVH_OK;
}

int gvh_enable_validity(gvh_handle *h, int on) {
  if (!h) return fail(GVH_ERR_INVALID, "null handle");
  int rc;
  if ((rc = set_device(h))) return rc;
  if (on && !h->diag) {
    const size_t bytes = (size_t)(kValidityFields + kValiditySaved) * h->cs * sizeof(double);
    if (cudaMalloc(&h->diag, bytes) != cudaSuccess) {
      h->diag = nullptr;
      return fail(GVH_ERR_NOMEM, "gvh_enable_validity: cannot allocate %zu bytes", bytes);
    }
    GVH_CUDA(cudaMemsetAsync(h->diag, 0, bytes, h->stream));
  }
  h->validity_on = on ? 1 : 0;
  return GVH_OK;
}

int gvh_get_validity(gvh_handle *h, double *const *fields, int n_fields) {
  if (!h || !fields) return fail(GVH_ERR_INVALID, "gvh_get_validity: null argument");
  if (n_fields != kValidityFields) return fail(GVH_ERR_INVALID, "gvh_get_validity: expected %d fields", kValidityFields);
  if (!h->diag) return fail(GVH_ERR_INVALID, "gvh_get_validity: diagnostics not enabled (gvh_enable_validity)");
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_staging(h))) return rc;
  FieldTable src = {};
  for (int f = 0; f < kValidityFields; ++f) src.p[f] = fields[f] ? h->diag + (size_t)f * h->cs : nullptr;
  unpack_kernel<<<(unsigned)((h->ng + 255) / 256), 256, 0, h->stream>>>(make_pack(h), n_fields, src, h->staging);
  GVH_CUDA(cudaGetLastError());
  const size_t fb = h->ng * sizeof(double);
  for (int f = 0; f < n_fields; ++f)
    if (fields[f]) GVH_CUDA(cudaMemcpyAsync(fields[f], h->staging + f * h->ng, fb, cudaMemcpyDefault, h->stream));
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  return GVH_OK;
}

// ---- checkpoint / resume ----------------------------------------------------------------
// File: a fixed header (magic, version, lattice sizes, options, spacings, the caller's time
// and step), then the nq + 10 fields of the interior lattice (field order of gvh_set_state,
// cell s = i + nx (j + ny k)) as native doubles, then an FNV-1a 64 checksum of those bytes.
namespace {

struct SnapshotHeader {
  char magic[8];          // "GVHSTATE"
  unsigned version;       // 1
  int nx, ny, nz, nq;
  int eos, shear, bulk, precision;
  double theta, dx, dy, dz, dt, etabar;
  double tau;
  long long step;
};

unsigned long long fnv1a(const void *data, size_t n, unsigned long long h) {
  const unsigned char *p = static_cast<const unsigned char *>(data);
  for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
  return h;
}

}  // namespace

int gvh_save_state(gvh_handle *h, const char *path, double tau, long long step) {
  if (!h || !path) return fail(GVH_ERR_INVALID, "gvh_save_state: null argument");
  int rc;
  if ((rc = set_device(h))) return rc;
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  SnapshotHeader hd;
  memset(&hd, 0, sizeof hd);
  memcpy(hd.magic, "GVHSTATE", 8);
  hd.version = 1;
  hd.nx = h->nx; hd.ny = h->ny; hd.nz = h->nz; hd.nq = h->nq;
  hd.eos = h->eos; hd.shear = h->shear; hd.bulk = h->bulk; hd.precision = h->precision;
  hd.theta = h->theta; hd.dx = h->dx; hd.dy = h->dy; hd.dz = h->dz; hd.dt = h->dt_lattice; hd.etabar = h->etabar;
  hd.tau = tau;
  hd.step = step;
  FILE *f = fopen(path, "wb");
  if (!f) return fail(GVH_ERR_INVALID, "gvh_save_state: cannot open %s", path);
  double *fields[32];
  internal_fields(h, fields);
  std::string buf((size_t)h->ncells * sizeof(double), '\0');
  unsigned long long sum = 0xcbf29ce484222325ull;
  bool ok = fwrite(&hd, sizeof hd, 1, f) == 1;
  for (int k = 0; ok && k < h->nq + 10; ++k) {
    cudaError_t e = cudaMemcpy(&buf[0], fields[k], buf.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      fclose(f);
      return fail(GVH_ERR_CUDA, "gvh_save_state: %s", cudaGetErrorString(e));
    }
    sum = fnv1a(buf.data(), buf.size(), sum);
    ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  }
  ok = ok && fwrite(&sum, sizeof sum, 1, f) == 1;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(GVH_ERR_INVALID, "gvh_save_state: writing %s failed", path);
  return GVH_OK;
}

int gvh_load_state(gvh_handle *h, const char *path, double *tau, long long *step) {
  if (!h || !path) return fail(GVH_ERR_INVALID, "gvh_load_state: null argument");
  int rc;
  if ((rc = set_device(h))) return rc;
  FILE *f = fopen(path, "rb");
  if (!f) return fail(GVH_ERR_INVALID, "gvh_load_state: cannot open %s", path);
  SnapshotHeader hd;
  if (fread(&hd, sizeof hd, 1, f) != 1 || memcmp(hd.magic, "GVHSTATE", 8) != 0 || hd.version != 1) {
    fclose(f);
    return fail(GVH_ERR_INVALID, "gvh_load_state: %s is not a state snapshot", path);
  }
  if (hd.nx != h->nx || hd.ny != h->ny || hd.nz != h->nz || hd.nq != h->nq || hd.eos != h->eos ||
      hd.shear != h->shear || hd.bulk != h->bulk) {
    fclose(f);
    return fail(GVH_ERR_INVALID, "gvh_load_state: %s holds a %dx%dx%d lattice with %d components, eos %d; the handle "
                                 "has %dx%dx%d, %d, eos %d", path, hd.nx, hd.ny, hd.nz, hd.nq, hd.eos, h->nx, h->ny,
                h->nz, h->nq, h->eos);
  }
  // read and check everything before the device state changes
  const size_t fb = (size_t)h->ncells * sizeof(double);
  std::string data((size_t)(h->nq + 10) * fb, '\0');
  unsigned long long sum_file = 0;
  const bool got = fread(&data[0], 1, data.size(), f) == data.size() && fread(&sum_file, sizeof sum_file, 1, f) == 1;
  fclose(f);
  if (!got) return fail(GVH_ERR_INVALID, "gvh_load_state: %s is truncated", path);
  if (fnv1a(data.data(), data.size(), 0xcbf29ce484222325ull) != sum_file)
    return fail(GVH_ERR_INVALID, "gvh_load_state: %s fails its checksum", path);
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  double *fields[32];
  internal_fields(h, fields);
  for (int k = 0; k < h->nq + 10; ++k) GVH_CUDA(cudaMemcpy(fields[k], data.data() + k * fb, fb, cudaMemcpyHostToDevice));
  if (tau) *tau = hd.tau;
  if (step) *step = hd.step;
  return GVH_OK;
}

int gvh_set_stream(gvh_handle *h, void *stream) {
  if (!h) return fail(GVH_ERR_INVALID, "null handle");
  GVH_CUDA(cudaSetDevice(h->device));
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  h->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : h->own_stream;
  return GVH_OK;
}

int gvh_max_propagation_speed(gvh_handle *h, double *out) {
  if (!h || !out) return fail(GVH_ERR_INVALID, "null argument");
  GVH_CUDA(cudaSetDevice(h->device));
  unsigned long long *word = reinterpret_cast<unsigned long long *>(h->status) + 2;
  unsigned long long bits = 0;
  GVH_CUDA(cudaMemcpyAsync(&bits, word, sizeof bits, cudaMemcpyDeviceToHost, h->stream));
  GVH_CUDA(cudaMemsetAsync(word, 0, sizeof bits, h->stream));
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  memcpy(out, &bits, sizeof bits);
  return GVH_OK;
}

int gvh_max_energy_density(gvh_handle *h, double *out) {
  if (!h || !out) return fail(GVH_ERR_INVALID, "null argument");
  GVH_CUDA(cudaSetDevice(h->device));
  unsigned long long *scratch = reinterpret_cast<unsigned long long *>(h->status) + 1;
  GVH_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), h->stream));
  const unsigned blocks = (unsigned)std::min<long long>(1024, (h->ncells + 255) / 256);
  max_e_kernel<<<blocks, 256, 0, h->stream>>>(h->e, h->ncells, scratch);
  GVH_CUDA(cudaGetLastError());
  if (!h->host_word) {
    if (cudaHostAlloc(reinterpret_cast<void **>(&h->host_word), 64, cudaHostAllocMapped) != cudaSuccess)
      return fail(GVH_ERR_NOMEM, "gvh_max_energy_density: cannot map host memory");
    GVH_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&h->host_word_dev), h->host_word, 0));
  }
  word_to_host_kernel<<<1, 1, 0, h->stream>>>(scratch, h->host_word_dev);
  GVH_CUDA(cudaGetLastError());
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  const unsigned long long bits = *reinterpret_cast<volatile unsigned long long *>(h->host_word);
  memcpy(out, &bits, sizeof *out);
  return GVH_OK;
}

double gvh_energy_density_of_temperature(int eos, double T_GeV) {
  const double T = T_GeV / 0.197326938;  // hbarc, HydroPlugin.cpp:132
  return eos == GVH_EOS_CONFORMAL ? energy_density_of_T<EOS_CONFORMAL>(T) : energy_density_of_T<EOS_QCD>(T);
}

int gvh_synchronize(gvh_handle *h) {
  if (!h) return fail(GVH_ERR_INVALID, "null handle");
  GVH_CUDA(cudaSetDevice(h->device));
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  if (h->async_ready) {
    GVH_CUDA(cudaStreamSynchronize(h->s_h2d));
    GVH_CUDA(cudaStreamSynchronize(h->s_d2h));
  }
  return GVH_OK;
}

int gvh_set_state_async(gvh_handle *h, const double *const *fields, int n_fields) {
  if (!h || !fields) return fail(GVH_ERR_INVALID, "gvh_set_state_async: null argument");
  if (n_fields != h->nq + 10) return fail(GVH_ERR_INVALID, "gvh_set_state_async: expected %d fields", h->nq + 10);
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_async(h))) return rc;
  FieldTable dst = {};
  internal_fields(h, dst.p);
  const size_t fb = h->ng * sizeof(double);
  // this call's staging area is free once the pack that last read it (two calls back) is done
  const int slot = h->in_slot;
  double *const staging = h->staging_in[slot];
  GVH_CUDA(cudaStreamWaitEvent(h->s_h2d, h->ev_in_free[slot], 0));
  const double *srcs[32];
  for (int f = 0; f < n_fields; ++f) {
    const double *src = fields[f];
    if (!src && f >= h->nq + 6) src = fields[f - 4];  // up defaults to u
    if (!src) return fail(GVH_ERR_INVALID, "gvh_set_state_async: field %d is null", f);
    srcs[f] = src;
  }
  // one copy per run of fields that follow each other in host memory (a caller's
  // [n_fields][ng] block is one copy): fewer, larger transfers share the link better with the
  // copies going the other way
  for (int f = 0; f < n_fields;) {
    int g = f + 1;
    while (g < n_fields && srcs[g] == srcs[f] + (size_t)(g - f) * h->ng) ++g;
    GVH_CUDA(cudaMemcpyAsync(staging + f * h->ng, srcs[f], (g - f) * fb, cudaMemcpyDefault, h->s_h2d));
    f = g;
  }
  GVH_CUDA(cudaEventRecord(h->ev_in_ready, h->s_h2d));
  GVH_CUDA(cudaStreamWaitEvent(h->stream, h->ev_in_ready, 0));
  pack_kernel<<<(unsigned)((h->ncells + 255) / 256), 256, 0, h->stream>>>(make_pack(h), n_fields, staging, dst);
  GVH_CUDA(cudaGetLastError());
  GVH_CUDA(cudaEventRecord(h->ev_in_free[slot], h->stream));
  h->in_slot = slot ^ 1;
  return GVH_OK;
}

int gvh_get_state_async(gvh_handle *h, double *const *fields, int n_fields) {
  if (!h || !fields) return fail(GVH_ERR_INVALID, "gvh_get_state_async: null argument");
  if (n_fields != h->nq + 10) return fail(GVH_ERR_INVALID, "gvh_get_state_async: expected %d fields", h->nq + 10);
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_async(h))) return rc;
  FieldTable src = {};
  internal_fields(h, src.p);
  for (int f = 0; f < n_fields; ++f)
    if (!fields[f]) src.p[f] = nullptr;
  // this call's staging area is free once the copy to the host that last read it (two calls
  // back) is done
  const int slot = h->out_slot;
  double *const staging = h->staging_out[slot];
  GVH_CUDA(cudaStreamWaitEvent(h->stream, h->ev_out_free[slot], 0));
  unpack_kernel<<<(unsigned)((h->ng + 255) / 256), 256, 0, h->stream>>>(make_pack(h), n_fields, src, staging);
  GVH_CUDA(cudaGetLastError());
  GVH_CUDA(cudaEventRecord(h->ev_out_ready, h->stream));
  GVH_CUDA(cudaStreamWaitEvent(h->s_d2h, h->ev_out_ready, 0));
  const size_t fb = h->ng * sizeof(double);
  for (int f = 0; f < n_fields;) {  // runs of adjacent host fields, as in gvh_set_state_async
    if (!fields[f]) { ++f; continue; }
    int g = f + 1;
    while (g < n_fields && fields[g] && fields[g] == fields[f] + (size_t)(g - f) * h->ng) ++g;
    GVH_CUDA(cudaMemcpyAsync(fields[f], staging + f * h->ng, (g - f) * fb, cudaMemcpyDefault, h->s_d2h));
    f = g;
  }
  GVH_CUDA(cudaEventRecord(h->ev_out_free[slot], h->s_d2h));
  h->out_slot = slot ^ 1;
  return GVH_OK;
}

int gvh_join_async(gvh_handle *h) {
  if (!h) return fail(GVH_ERR_INVALID, "null handle");
  if (!h->async_ready) return GVH_OK;
  GVH_CUDA(cudaSetDevice(h->device));
  // the handle's stream waits for every queued copy, then the copy streams wait for
  // everything queued on the handle's stream up to here
  // (each copy stream runs in order, so its last recorded event covers all its copies)
  GVH_CUDA(cudaStreamWaitEvent(h->stream, h->ev_in_ready, 0));
  GVH_CUDA(cudaStreamWaitEvent(h->stream, h->ev_out_free[h->out_slot ^ 1], 0));
  GVH_CUDA(cudaEventRecord(h->ev_fence, h->stream));
  GVH_CUDA(cudaStreamWaitEvent(h->s_h2d, h->ev_fence, 0));
  GVH_CUDA(cudaStreamWaitEvent(h->s_d2h, h->ev_fence, 0));
  return GVH_OK;
}

int gvh_status(gvh_handle *h, unsigned *flags) {
  if (!h) return fail(GVH_ERR_INVALID, "null handle");
  GVH_CUDA(cudaSetDevice(h->device));
  unsigned v = 0;
  GVH_CUDA(cudaMemcpyAsync(&v, h->status, sizeof v, cudaMemcpyDeviceToHost, h->stream));
  GVH_CUDA(cudaStreamSynchronize(h->stream));
  if (flags) *flags = v;
  return (v & GVH_STATUS_ERRORS) ? GVH_ERR_NUMERIC : GVH_OK;
}

int gvh_clear_status(gvh_handle *h) {
  if (!h) return fail(GVH_ERR_INVALID, "null handle");
  GVH_CUDA(cudaSetDevice(h->device));
  GVH_CUDA(cudaMemsetAsync(h->status, 0, sizeof(unsigned), h->stream));
  return GVH_OK;
}

}  // extern "C"
