// gvh_batch.cu -- many events advanced together (the batched and serving forms of the KT
// step; the reference runs one event per process, HydroPlugin.cpp:107-434).
//
// Design:
//  * One HBM arena per batch, carved first-fit into per-event lattices (each event: qA, qB,
//    e, pA, pB, u[3] in the interior-only layout of gvh_stage.cuh). No cudaMalloc happens
//    while the batch runs; admission fails cleanly (GVH_ERR_NOMEM) when the arena is full.
//  * Every event's scalars, buffer pointers, time, step count, status word and freeze-out
//    bookkeeping live in a device array of EventDev. A persistent stage kernel walks a packed
//    queue of 128-cell tiles (tile -> event table, also on the device) with a grid sized to
//    the GPU, so one launch covers every event whatever its lattice.
//  * One RK2 step is three launches -- stage 1 over all tiles, stage 2 over all tiles, a
//    per-event finish kernel (advance time, rotate the u buffers, freeze-out count) --
//    captured once into a CUDA graph and replayed every step. Pointers in the graph never
//    change: admissions and retirements only rewrite the device tables between replays.
//  * Freeze-out follows the reference's stop rule (HydroPlugin.cpp:396-413): after every
//    step the maximum interior e is compared with e(T_fo); an event is finished once that
//    has held FOFREQ+1 = 11 times (the reference's counter is cumulative, never reset).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gvh.h"
#include "gvh_layout.cuh"
#include "gvh_stage.cuh"

using namespace gvh;

namespace {

constexpr int kMaxEvents = 4096;
constexpr int kFreezeoutChecks = 11;   // FOFREQ + 1 (HydroPlugin.cpp:409)
constexpr double kHbarc = 0.197326938;  // HydroPlugin.cpp:132

thread_local std::string g_batch_error;

int bfail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_batch_error = buf;
  return code;
}

#define BCUDA(call)                                                                              \
  do {                                                                                           \
    cudaError_t err_ = (call);                                                                   \
    if (err_ != cudaSuccess) return bfail(GVH_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(err_)); \
  } while (0)

// Device-resident state of one event.
struct EventDev {
  int nx, ny, nz, active;
  long long sy, sz, cs, ncells;
  double dx, dy, dz, dt, etabar, theta, e_reg, e_fo;
  double inv_dx, inv_dy, inv_dz, inv_dt;  // reciprocals, computed on the host at admission
  double t0;            // initial proper time; the step from t0 + n dt is step n + 1
  long long step;       // completed steps
  double *qA, *qB, *e, *pA, *pB, *u[3];
  int ucur, uprev, ufree, first_tile;
  unsigned status;
  int frozen_checks;
  unsigned long long emax_bits;  // running max of e during stage 2 (bit pattern of e >= 0)
  double emax_last;              // max e after the last completed step
};

__device__ __forceinline__ StageArgs make_args(EventDev &E, bool stage2) {
  StageArgs a;
  a.nx = E.nx; a.ny = E.ny; a.nz = E.nz;
  a.sy = E.sy; a.sz = E.sz; a.cs = E.cs; a.ncells = E.ncells;
  a.dx = E.dx; a.dy = E.dy; a.dz = E.dz; a.dt = E.dt;
  a.inv_dx = E.inv_dx; a.inv_dy = E.inv_dy; a.inv_dz = E.inv_dz; a.inv_dt = E.inv_dt;
  a.etabar = E.etabar; a.theta = E.theta; a.e_reg = E.e_reg;
  a.status = &E.status;
  a.diag = nullptr;       // validity diagnostics are a single-lattice option
  a.speed_max = nullptr;  // so is the propagation-speed maximum
  a.e = E.e;
  // twoStepRungeKutta receives t = t0 + n dt (HydroPlugin.cpp:424) and advances it by dt
  const double t = E.t0 + (double)E.step * E.dt;
  const double t1 = t + E.dt;
  if (!stage2) {
    a.t_euler = t; a.t_after = t1;
    a.qin = E.qA; a.qn = nullptr; a.qout = E.qB;
    a.pin = E.pA; a.pout = E.pB;
    a.uin = E.u[E.ucur]; a.uprev = E.u[E.uprev]; a.uout = E.u[E.uprev];
  } else {
    a.t_euler = t1; a.t_after = t1;
    a.qin = E.qB; a.qn = E.qA; a.qout = E.qA;
    a.pin = E.pB; a.pout = E.pA;
    a.uin = E.u[E.uprev]; a.uprev = E.u[E.ucur]; a.uout = E.u[E.ufree];
  }
  return a;
}

// Persistent stage kernel over the packed tile queue of every active event.
template <int EOS, bool SHEAR, bool BULK, bool STAGE2, bool MIXED>
__global__ void __launch_bounds__(kBlock, GVH_MIN_BLOCKS)
    batch_stage_kernel(EventDev *ev, const int *__restrict__ tile_event, const int *__restrict__ ntiles_p) {
  const int ntiles = *ntiles_p;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    EventDev &E = ev[tile_event[tile]];
    if (!E.active) continue;
    const StageArgs a = make_args(E, STAGE2);
    const long long id = (long long)(tile - E.first_tile) * kBlock + threadIdx.x;
    double en = 0.0, speed;
    if (id < a.ncells) en = stage_cell<EOS, SHEAR, BULK, STAGE2, MIXED>(a, id, speed);
    if (STAGE2) {
      unsigned long long b = __double_as_longlong(fmax(en, 0.0));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
      if ((threadIdx.x & 31) == 0) atomicMax(&E.emax_bits, b);
    }
  }
}

// After stage 2: advance time, rotate the u buffers (u^{n+1} current, u^n previous, as the
// reference's swapFluidVelocity), freeze-out bookkeeping.
__global__ void batch_finish_kernel(EventDev *ev, int nslots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  EventDev &E = ev[i];
  if (!E.active) return;
  E.step += 1;
  const int nc = E.ufree, np = E.ucur, nf = E.uprev;
  E.ucur = nc; E.uprev = np; E.ufree = nf;
  E.emax_last = __longlong_as_double(E.emax_bits);
  E.emax_bits = 0ull;
  if (E.emax_last <= E.e_fo) E.frozen_checks += 1;
}

struct HostEvent {
  bool used = false;
  size_t off = 0, bytes = 0;
  int nx = 0, ny = 0, nz = 0;
  long long ncells = 0, ng = 0, cs = 0;
  int ntiles = 0;
};

}  // namespace

struct gvh_batch {
  gvh_options opts;
  int nq = 0, device = 0, num_sms = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  char *arena = nullptr;
  size_t arena_bytes = 0;
  std::map<size_t, size_t> free_blocks;  // offset -> size
  std::vector<HostEvent> ev;             // slot = event id
  EventDev *d_ev = nullptr;
  int *d_tile_event = nullptr, *d_ntiles = nullptr;
  int tile_capacity = 0;
  double *staging = nullptr;
  size_t staging_bytes = 0;
  unsigned long long *d_scratch = nullptr;
  cudaGraphExec_t graph = nullptr;
  int grid = 0;                          // persistent grid (blocks); 0 = one block per tile
  int ntiles = 0;                        // tiles of the admitted events
  int active_slots = 0;                  // slots the finish kernel scans
};

namespace {

size_t event_bytes(const gvh_batch *b, long long ncells, long long *cs_out) {
  const long long cs = (ncells + 31) / 32 * 32;
  if (cs_out) *cs_out = cs;
  return (size_t)(2 * b->nq + 15) * cs * sizeof(double);
}

bool arena_alloc(gvh_batch *b, size_t bytes, size_t *off) {
  bytes = (bytes + 255) / 256 * 256;
  for (auto it = b->free_blocks.begin(); it != b->free_blocks.end(); ++it) {
    if (it->second >= bytes) {
      *off = it->first;
      size_t rest = it->second - bytes;
      size_t roff = it->first + bytes;
      b->free_blocks.erase(it);
      if (rest) b->free_blocks[roff] = rest;
      return true;
    }
  }
  return false;
}

void arena_free(gvh_batch *b, size_t off, size_t bytes) {
  bytes = (bytes + 255) / 256 * 256;
  auto it = b->free_blocks.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != b->free_blocks.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    b->free_blocks.erase(nx);
  }
  if (it != b->free_blocks.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      b->free_blocks.erase(it);
    }
  }
}

int rebuild_graph(gvh_batch *b);

int rebuild_tiles(gvh_batch *b) {
  std::vector<int> table;
  int slots = 0;
  for (size_t i = 0; i < b->ev.size(); ++i) {
    if (!b->ev[i].used) continue;
    slots = (int)i + 1;
    const int first = (int)table.size();
    for (int t = 0; t < b->ev[i].ntiles; ++t) table.push_back((int)i);
    BCUDA(cudaMemcpyAsync(&b->d_ev[i].first_tile, &first, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  }
  if ((int)table.size() > b->tile_capacity) return bfail(GVH_ERR_NOMEM, "tile table full");
  const int n = (int)table.size();
  if (n) BCUDA(cudaMemcpyAsync(b->d_tile_event, table.data(), n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaMemcpyAsync(b->d_ntiles, &n, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  // pageable sources: wait so the host vectors may go out of scope
  BCUDA(cudaStreamSynchronize(b->stream));
  b->active_slots = slots;
  const bool regrid = b->grid == 0 && n != b->ntiles;
  b->ntiles = n;
  if (regrid) return rebuild_graph(b);
  return GVH_OK;
}

template <int EOS, bool SHEAR, bool BULK, bool MIXED>
int launch_step_t(gvh_batch *b) {
  // grid 0: one block per tile (the hardware block scheduler balances the uneven per-tile
  // cost; measured 2.3-2.5x faster than a persistent grid of 3 blocks per SM on 8-24
  // events); otherwise a persistent grid of that many blocks
  const int g = b->grid > 0 ? b->grid : (b->ntiles > 0 ? b->ntiles : 1);
  const size_t smem = stage_smem_bytes<SHEAR, BULK>();
  batch_stage_kernel<EOS, SHEAR, BULK, false, MIXED><<<g, kBlock, smem, b->stream>>>(b->d_ev, b->d_tile_event,
                                                                                     b->d_ntiles);
  batch_stage_kernel<EOS, SHEAR, BULK, true, MIXED><<<g, kBlock, smem, b->stream>>>(b->d_ev, b->d_tile_event,
                                                                                    b->d_ntiles);
  batch_finish_kernel<<<(kMaxEvents + 127) / 128, 128, 0, b->stream>>>(b->d_ev, kMaxEvents);
  BCUDA(cudaGetLastError());
  return GVH_OK;
}

template <int EOS, bool MIXED>
int launch_step_p(gvh_batch *b) {
  if (!b->opts.shear) return launch_step_t<EOS, false, false, MIXED>(b);
  if (!b->opts.bulk) return launch_step_t<EOS, true, false, MIXED>(b);
  return launch_step_t<EOS, true, true, MIXED>(b);
}

int launch_step(gvh_batch *b) {
  const bool mixed = b->opts.precision == GVH_PRECISION_MIXED;
  if (b->opts.eos == GVH_EOS_CONFORMAL)
    return mixed ? launch_step_p<EOS_CONFORMAL, true>(b) : launch_step_p<EOS_CONFORMAL, false>(b);
  return mixed ? launch_step_p<EOS_QCD, true>(b) : launch_step_p<EOS_QCD, false>(b);
}

int rebuild_graph(gvh_batch *b) {
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaGraph_t g;
  BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = launch_step(b);
  cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
  if (rc) return rc;
  if (ec != cudaSuccess) return bfail(GVH_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
  ec = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (ec != cudaSuccess) return bfail(GVH_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ec));
  return GVH_OK;
}

int ensure_staging(gvh_batch *b, size_t fields, long long ng) {
  size_t need = fields * (size_t)ng * sizeof(double);
  if (need <= b->staging_bytes) return GVH_OK;
  if (b->staging) cudaFree(b->staging);
  b->staging = nullptr;
  b->staging_bytes = 0;
  if (cudaMalloc(&b->staging, need) != cudaSuccess) return bfail(GVH_ERR_NOMEM, "staging allocation failed");
  b->staging_bytes = need;
  return GVH_OK;
}

void event_pointers(gvh_batch *b, const HostEvent &h, double **qA, double **qB, double **e, double **pA,
                    double **pB, double **u) {
  double *p = reinterpret_cast<double *>(b->arena + h.off);
  *qA = p; p += b->nq * h.cs;
  *qB = p; p += b->nq * h.cs;
  *e = p; p += h.cs;
  *pA = p; p += h.cs;
  *pB = p; p += h.cs;
  for (int m = 0; m < 3; ++m) { u[m] = p; p += 4 * h.cs; }
}

}  // namespace

extern "C" {

const char *gvh_batch_last_error(void) { return g_batch_error.c_str(); }

long long gvh_batch_event_bytes(const gvh_lattice_params *L, const gvh_options *opts) {
  if (!L || !opts) return GVH_ERR_INVALID;
  gvh_batch tmp;
  tmp.nq = 4 + (opts->shear ? 10 : 0) + (opts->bulk ? 1 : 0);
  long long n = (long long)L->numLatticePointsX * L->numLatticePointsY * L->numLatticePointsRapidity;
  return (long long)event_bytes(&tmp, n, nullptr);
}

int gvh_batch_create(const gvh_options *opts, long long arena_bytes, gvh_batch **out) {
  if (!out) return bfail(GVH_ERR_INVALID, "null out");
  *out = nullptr;
  gvh_options o;
  if (opts) o = *opts; else gvh_default_options(&o);
  if (o.bulk && !o.shear) return bfail(GVH_ERR_INVALID, "bulk needs shear");
  if (o.eos != GVH_EOS_QCD && o.eos != GVH_EOS_CONFORMAL) return bfail(GVH_ERR_INVALID, "unknown eos");
  if (o.precision != GVH_PRECISION_FP64 && o.precision != GVH_PRECISION_MIXED)
    return bfail(GVH_ERR_INVALID, "unknown precision");
  if (arena_bytes <= 0) return bfail(GVH_ERR_INVALID, "arena_bytes must be > 0");
  if (!(o.theta > 0)) return bfail(GVH_ERR_INVALID, "the limiter's theta must be > 0");
  int dev = o.device;
  if (dev < 0) BCUDA(cudaGetDevice(&dev));
  BCUDA(cudaSetDevice(dev));
  {
    // the batched stage kernels' shared-memory limit, once per device, before any capture
    static std::mutex mu;
    static unsigned long long prepared = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && !(prepared & (1ull << dev))) {
      cudaError_t e = cudaSuccess;
#define GVH_ALLOW_B(EOS_, SH, BU, MX)                                                                           \
  if (e == cudaSuccess)                                                                                         \
    e = allow_stage_smem(batch_stage_kernel<EOS_, SH, BU, false, MX>, stage_smem_bytes<SH, BU>());             \
  if (e == cudaSuccess) e = allow_stage_smem(batch_stage_kernel<EOS_, SH, BU, true, MX>, stage_smem_bytes<SH, BU>());
      GVH_ALLOW_B(EOS_QCD, false, false, false) GVH_ALLOW_B(EOS_QCD, true, false, false)
      GVH_ALLOW_B(EOS_QCD, true, true, false) GVH_ALLOW_B(EOS_CONFORMAL, false, false, false)
      GVH_ALLOW_B(EOS_CONFORMAL, true, false, false) GVH_ALLOW_B(EOS_CONFORMAL, true, true, false)
      GVH_ALLOW_B(EOS_QCD, false, false, true) GVH_ALLOW_B(EOS_QCD, true, false, true)
      GVH_ALLOW_B(EOS_QCD, true, true, true) GVH_ALLOW_B(EOS_CONFORMAL, false, false, true)
      GVH_ALLOW_B(EOS_CONFORMAL, true, false, true) GVH_ALLOW_B(EOS_CONFORMAL, true, true, true)
#undef GVH_ALLOW_B
      if (e != cudaSuccess) return bfail(GVH_ERR_CUDA, "stage kernel set-up: %s", cudaGetErrorString(e));
      prepared |= 1ull << dev;
    }
  }
  gvh_batch *b = new gvh_batch();
  b->opts = o;
  b->device = dev;
  b->nq = 4 + (o.shear ? 10 : 0) + (o.bulk ? 1 : 0);
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev);
  b->arena_bytes = (size_t)arena_bytes;
  bool ok = cudaMalloc(&b->arena, b->arena_bytes) == cudaSuccess;
  b->tile_capacity = (int)(b->arena_bytes / ((2 * b->nq + 15) * sizeof(double) * kBlock) + kMaxEvents);
  ok = ok && cudaMalloc(&b->d_ev, kMaxEvents * sizeof(EventDev)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_tile_event, (size_t)b->tile_capacity * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_ntiles, sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_scratch, sizeof(unsigned long long)) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) == cudaSuccess;
  if (!ok) {
    gvh_batch_destroy(b);
    return bfail(GVH_ERR_NOMEM, "gvh_batch_create: cannot allocate %lld bytes", arena_bytes);
  }
  b->stream = b->own_stream;
  cudaMemsetAsync(b->d_ev, 0, kMaxEvents * sizeof(EventDev), b->stream);
  cudaMemsetAsync(b->d_ntiles, 0, sizeof(int), b->stream);
  b->free_blocks[0] = b->arena_bytes / 256 * 256;
  b->grid = 0;
  int rc = rebuild_graph(b);
  if (rc) {
    gvh_batch_destroy(b);
    return rc;
  }
  *out = b;
  return GVH_OK;
}

int gvh_batch_destroy(gvh_batch *b) {
  if (!b) return GVH_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->arena);
  cudaFree(b->d_ev);
  cudaFree(b->d_tile_event);
  cudaFree(b->d_ntiles);
  cudaFree(b->d_scratch);
  if (b->staging) cudaFree(b->staging);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
  return GVH_OK;
}

int gvh_batch_set_stream(gvh_batch *b, void *stream) {
  if (!b) return bfail(GVH_ERR_INVALID, "null batch");
  BCUDA(cudaSetDevice(b->device));
  BCUDA(cudaStreamSynchronize(b->stream));
  b->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : b->own_stream;
  return GVH_OK;
}

int gvh_batch_add_event(gvh_batch *b, const gvh_lattice_params *L, const gvh_hydro_params *H,
                        const double *const *prim, int n_prim, int *event_id) {
  if (!b || !L || !H || !prim || !event_id) return bfail(GVH_ERR_INVALID, "null argument");
  *event_id = -1;
  const int want = 5 + (b->nq - 4);
  if (n_prim != want) return bfail(GVH_ERR_INVALID, "expected %d primitive arrays", want);
  for (int f = 0; f < n_prim; ++f)
    if (!prim[f]) return bfail(GVH_ERR_INVALID, "primitive array %d is null", f);
  if (L->numLatticePointsX < 1 || L->numLatticePointsY < 1 || L->numLatticePointsRapidity < 1)
    return bfail(GVH_ERR_INVALID, "lattice sizes must be >= 1");
  if (!(L->latticeSpacingX > 0 && L->latticeSpacingY > 0 && L->latticeSpacingRapidity > 0 &&
        L->latticeSpacingProperTime > 0))
    return bfail(GVH_ERR_INVALID, "lattice spacings must be > 0");
  if (b->opts.shear && !(H->shearViscosityToEntropyDensity > 0)) return bfail(GVH_ERR_INVALID, "eta/s must be > 0");
  BCUDA(cudaSetDevice(b->device));
  int slot = -1;
  for (size_t i = 0; i < b->ev.size(); ++i)
    if (!b->ev[i].used) { slot = (int)i; break; }
  if (slot < 0) {
    if ((int)b->ev.size() >= kMaxEvents) return bfail(GVH_ERR_NOMEM, "too many events");
    b->ev.emplace_back();
    slot = (int)b->ev.size() - 1;
  }
  HostEvent h;
  h.nx = L->numLatticePointsX; h.ny = L->numLatticePointsY; h.nz = L->numLatticePointsRapidity;
  h.ncells = (long long)h.nx * h.ny * h.nz;
  h.ng = (long long)(h.nx + 4) * (h.ny + 4) * (h.nz + 4);
  h.bytes = event_bytes(b, h.ncells, &h.cs);
  h.ntiles = (int)((h.ncells + kBlock - 1) / kBlock);
  if (!arena_alloc(b, h.bytes, &h.off)) return bfail(GVH_ERR_NOMEM, "arena full (%zu bytes needed)", h.bytes);
  h.used = true;
  int rc = ensure_staging(b, n_prim, h.ng);
  if (rc) { arena_free(b, h.off, h.bytes); return rc; }

  double *qA, *qB, *e, *pA, *pB, *u[3];
  event_pointers(b, h, &qA, &qB, &e, &pA, &pB, u);
  BCUDA(cudaMemsetAsync(b->arena + h.off, 0, h.bytes, b->stream));
  const size_t fb = h.ng * sizeof(double);
  for (int f = 0; f < n_prim; ++f)
    BCUDA(cudaMemcpyAsync(b->staging + f * h.ng, prim[f], fb, cudaMemcpyDefault, b->stream));
  FieldTable dst = {};
  dst.p[0] = e;
  for (int m = 0; m < 4; ++m) dst.p[1 + m] = u[0] + m * h.cs;
  for (int n = 4; n < b->nq; ++n) dst.p[5 + n - 4] = qA + n * h.cs;
  Pack pk{h.nx, h.ny, h.nz, (long long)h.nx, (long long)h.nx * h.ny, h.ng};
  const unsigned blocks = (unsigned)((h.ncells + 255) / 256);
  pack_kernel<<<blocks, 256, 0, b->stream>>>(pk, n_prim, b->staging, dst);
  if (b->opts.eos == GVH_EOS_CONFORMAL)
    init_conserved_kernel<EOS_CONFORMAL><<<blocks, 256, 0, b->stream>>>(h.ncells, b->nq, h.cs, qA, e, pA, u[0], u[1], 0);
  else
    init_conserved_kernel<EOS_QCD><<<blocks, 256, 0, b->stream>>>(h.ncells, b->nq, h.cs, qA, e, pA, u[0], u[1], 0);
  BCUDA(cudaGetLastError());
  // initial freeze-out check (the reference tests the state before every step, the first
  // one included: HydroPlugin.cpp:396-408)
  BCUDA(cudaMemsetAsync(b->d_scratch, 0, sizeof(unsigned long long), b->stream));
  max_e_kernel<<<min(1024u, blocks), 256, 0, b->stream>>>(e, h.ncells, b->d_scratch);
  unsigned long long emax_bits = 0;
  BCUDA(cudaMemcpyAsync(&emax_bits, b->d_scratch, sizeof emax_bits, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  double emax0;
  memcpy(&emax0, &emax_bits, sizeof emax0);

  EventDev E;
  memset(&E, 0, sizeof E);
  E.nx = h.nx; E.ny = h.ny; E.nz = h.nz; E.active = 1;
  E.sy = h.nx; E.sz = (long long)h.nx * h.ny; E.cs = h.cs; E.ncells = h.ncells;
  E.dx = L->latticeSpacingX; E.dy = L->latticeSpacingY; E.dz = L->latticeSpacingRapidity;
  E.dt = L->latticeSpacingProperTime;
  E.inv_dx = 1.0 / E.dx; E.inv_dy = 1.0 / E.dy; E.inv_dz = 1.0 / E.dz; E.inv_dt = 1.0 / E.dt;
  E.etabar = H->shearViscosityToEntropyDensity;
  E.theta = b->opts.theta;
  const double T_reg = H->regulationTemperatureGeV / kHbarc;
  const double T_fo = H->freezeoutTemperatureGeV / kHbarc;
  if (b->opts.eos == GVH_EOS_CONFORMAL) {
    E.e_reg = energy_density_of_T<EOS_CONFORMAL>(T_reg);
    E.e_fo = energy_density_of_T<EOS_CONFORMAL>(T_fo);
  } else {
    E.e_reg = energy_density_of_T<EOS_QCD>(T_reg);
    E.e_fo = energy_density_of_T<EOS_QCD>(T_fo);
  }
  E.t0 = H->initialProperTimePoint;
  E.step = 0;
  E.qA = qA; E.qB = qB; E.e = e; E.pA = pA; E.pB = pB;
  for (int m = 0; m < 3; ++m) E.u[m] = u[m];
  E.ucur = 0; E.uprev = 1; E.ufree = 2;
  E.emax_last = emax0;
  E.frozen_checks = emax0 <= E.e_fo ? 1 : 0;
  BCUDA(cudaMemcpyAsync(b->d_ev + slot, &E, sizeof E, cudaMemcpyHostToDevice, b->stream));
  b->ev[slot] = h;
  rc = rebuild_tiles(b);
  if (rc) return rc;
  *event_id = slot;
  return GVH_OK;
}

int gvh_batch_remove_event(gvh_batch *b, int id) {
  if (!b || id < 0 || id >= (int)b->ev.size() || !b->ev[id].used) return bfail(GVH_ERR_INVALID, "bad event id");
  BCUDA(cudaSetDevice(b->device));
  const int zero = 0;
  BCUDA(cudaMemcpyAsync(&b->d_ev[id].active, &zero, sizeof zero, cudaMemcpyHostToDevice, b->stream));
  arena_free(b, b->ev[id].off, b->ev[id].bytes);
  b->ev[id] = HostEvent();
  return rebuild_tiles(b);
}

int gvh_batch_num_events(const gvh_batch *b) {
  if (!b) return GVH_ERR_INVALID;
  int n = 0;
  for (const auto &h : b->ev) n += h.used ? 1 : 0;
  return n;
}

long long gvh_batch_free_bytes(const gvh_batch *b) {
  if (!b) return GVH_ERR_INVALID;
  long long f = 0;
  for (const auto &kv : b->free_blocks) f += (long long)kv.second;
  return f;
}

long long gvh_batch_active_cells(const gvh_batch *b) {
  if (!b) return GVH_ERR_INVALID;
  long long n = 0;
  for (const auto &h : b->ev) n += h.used ? h.ncells : 0;
  return n;
}

int gvh_batch_step(gvh_batch *b, int nsteps) {
  if (!b || nsteps < 0) return bfail(GVH_ERR_INVALID, "bad arguments");
  BCUDA(cudaSetDevice(b->device));
  for (int n = 0; n < nsteps; ++n) BCUDA(cudaGraphLaunch(b->graph, b->stream));
  return GVH_OK;
}

int gvh_batch_synchronize(gvh_batch *b) {
  if (!b) return bfail(GVH_ERR_INVALID, "null batch");
  BCUDA(cudaSetDevice(b->device));
  BCUDA(cudaStreamSynchronize(b->stream));
  return GVH_OK;
}

int gvh_batch_event_info(gvh_batch *b, int id, gvh_event_info *info) {
  if (!b || !info || id < 0 || id >= (int)b->ev.size() || !b->ev[id].used)
    return bfail(GVH_ERR_INVALID, "bad event id");
  BCUDA(cudaSetDevice(b->device));
  EventDev E;
  BCUDA(cudaMemcpyAsync(&E, b->d_ev + id, sizeof E, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  info->step = E.step;
  info->tau = E.t0 + (double)E.step * E.dt;
  info->max_energy_density = E.emax_last;
  info->freezeout_energy_density = E.e_fo;
  info->frozen_checks = E.frozen_checks;
  info->frozen_out = E.frozen_checks >= kFreezeoutChecks;
  info->status = E.status;
  info->cells = E.ncells;
  return GVH_OK;
}

int gvh_batch_get_state(gvh_batch *b, int id, double *const *fields, int n_fields) {
  if (!b || !fields || id < 0 || id >= (int)b->ev.size() || !b->ev[id].used)
    return bfail(GVH_ERR_INVALID, "bad arguments");
  if (n_fields != b->nq + 10) return bfail(GVH_ERR_INVALID, "expected %d fields", b->nq + 10);
  BCUDA(cudaSetDevice(b->device));
  const HostEvent &h = b->ev[id];
  int rc = ensure_staging(b, n_fields, h.ng);
  if (rc) return rc;
  EventDev E;
  BCUDA(cudaMemcpyAsync(&E, b->d_ev + id, sizeof E, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  FieldTable src = {};
  for (int n = 0; n < b->nq; ++n) src.p[n] = fields[n] ? E.qA + n * h.cs : nullptr;
  src.p[b->nq] = fields[b->nq] ? E.e : nullptr;
  src.p[b->nq + 1] = fields[b->nq + 1] ? E.pA : nullptr;
  for (int m = 0; m < 4; ++m) src.p[b->nq + 2 + m] = fields[b->nq + 2 + m] ? E.u[E.ucur] + m * h.cs : nullptr;
  for (int m = 0; m < 4; ++m) src.p[b->nq + 6 + m] = fields[b->nq + 6 + m] ? E.u[E.uprev] + m * h.cs : nullptr;
  Pack pk{h.nx, h.ny, h.nz, (long long)h.nx, (long long)h.nx * h.ny, h.ng};
  unpack_kernel<<<(unsigned)((h.ng + 255) / 256), 256, 0, b->stream>>>(pk, n_fields, src, b->staging);
  BCUDA(cudaGetLastError());
  const size_t fb = h.ng * sizeof(double);
  for (int f = 0; f < n_fields; ++f)
    if (fields[f]) BCUDA(cudaMemcpyAsync(fields[f], b->staging + f * h.ng, fb, cudaMemcpyDefault, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  return GVH_OK;
}

int gvh_batch_launch_config(const gvh_batch *b, int *grid_blocks, int *block_threads) {
  if (!b) return GVH_ERR_INVALID;
  if (grid_blocks) *grid_blocks = b->grid;  // 0 = one block per tile
  if (block_threads) *block_threads = kBlock;
  return GVH_OK;
}

int gvh_batch_set_grid(gvh_batch *b, int grid_blocks) {
  if (!b || grid_blocks < 0) return bfail(GVH_ERR_INVALID, "bad grid");
  BCUDA(cudaSetDevice(b->device));
  BCUDA(cudaStreamSynchronize(b->stream));
  b->grid = grid_blocks;
  return rebuild_graph(b);
}

// Times `steps` real RK2 steps (the events do advance) with each candidate grid -- one
// block per tile (0) and persistent grids of 1..GVH_MIN_BLOCKS blocks per SM -- and keeps
// the fastest. Every candidate computes the same values; only the schedule differs.
int gvh_batch_autotune(gvh_batch *b, int steps, int *chosen_grid) {
  if (!b || steps < 1) return bfail(GVH_ERR_INVALID, "bad arguments");
  BCUDA(cudaSetDevice(b->device));
  int ntiles = 0;
  for (const auto &h : b->ev) ntiles += h.used ? h.ntiles : 0;
  std::vector<int> cands{0};
  for (int k = 1; k <= GVH_MIN_BLOCKS; ++k) cands.push_back(b->num_sms * k);
  cudaEvent_t e0, e1;
  BCUDA(cudaEventCreate(&e0));
  BCUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_grid = b->grid;
  for (int g : cands) {
    int rc = gvh_batch_set_grid(b, g);
    if (rc) return rc;
    BCUDA(cudaGraphLaunch(b->graph, b->stream));  // warm
    BCUDA(cudaEventRecord(e0, b->stream));
    for (int n = 0; n < steps; ++n) BCUDA(cudaGraphLaunch(b->graph, b->stream));
    BCUDA(cudaEventRecord(e1, b->stream));
    BCUDA(cudaEventSynchronize(e1));
    float ms = 0;
    BCUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      best_grid = g;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int rc = gvh_batch_set_grid(b, best_grid);
  if (chosen_grid) *chosen_grid = best_grid;
  return rc;
}

}  // extern "C"
