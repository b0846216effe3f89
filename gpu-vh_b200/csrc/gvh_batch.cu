// gvh_batch.cu -- many events advanced together (the batched and serving forms of the KT
// step; the reference runs one event per process, HydroPlugin.cpp:107-434).
//
// Design:
//  * One HBM arena per batch, carved first-fit into per-event lattices (each event: qA, qB,
//    e, pA, pB, u[3] in the interior-only layout of gvh_stage.cuh). No cudaMalloc happens
//    while the batch runs; admission fails cleanly (GVH_ERR_NOMEM) when the arena is full.
//  * Every event's scalars, buffer pointers, time, step count, status word and freeze-out
//    bookkeeping live in a device array of EventDev. The stage kernel walks a packed queue
//    of 128-cell tiles (tile -> event table, also on the device), so one launch covers every
//    event whatever its lattice. A tile is 128 consecutive cells of its event, or a block of
//    TX x (128 / TX) cells of one eta plane (the tile shape, chosen by the autotuner).
//  * One RK2 step is three launches -- stage 1 over all tiles, stage 2 over all tiles, a
//    per-event finish kernel (advance time, rotate the u buffers, freeze-out count) --
//    captured once into a CUDA graph and replayed every step. Pointers in the graph never
//    change: admissions and retirements only rewrite the device tables between replays.
//  * Freeze-out follows the reference's stop rule (HydroPlugin.cpp:396-413): after every
//    step the maximum interior e is compared with e(T_fo); an event is finished once that
//    has held FOFREQ+1 = 11 times (the reference's counter is cumulative, never reset), and
//    from then on it is not advanced (the reference's loop ends there).
//  * Nothing in admission, retirement or a serving round waits for the device: the initial
//    state goes through a pinned staging ring, table updates through pinned buffers or
//    kernel parameters, and a round ends with a kernel that copies every event's bookkeeping
//    into mapped host memory, so the host reads round k while round k+1 runs.
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
#include "gvh_nvtx.h"
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
  int cartesian;        // the batch's coordinates (GVH_COORDINATES_CARTESIAN)
  double t0;            // initial proper time; the step from t0 + n dt is step n + 1
  long long step;       // completed steps
  double *qA, *qB, *e, *pA, *pB, *u[3];
  int ucur, uprev, ufree, first_tile;
  unsigned status;
  int frozen_checks;
  unsigned long long emax_bits;  // running max of e during stage 2 (bit pattern of e >= 0)
  double emax_last;              // max e after the last completed step
  int done;                      // frozen out: no further steps
};

__device__ __forceinline__ StageArgs make_args(EventDev &E, bool stage2) {
  StageArgs a;
  a.nx = E.nx; a.ny = E.ny; a.nz = E.nz;
  a.sy = E.sy; a.sz = E.sz; a.cs = E.cs; a.ncells = E.ncells;
  a.dx = E.dx; a.dy = E.dy; a.dz = E.dz; a.dt = E.dt;
  a.inv_dx = E.inv_dx; a.inv_dy = E.inv_dy; a.inv_dz = E.inv_dz; a.inv_dt = E.inv_dt;
  a.etabar = E.etabar; a.theta = E.theta; a.e_reg = E.e_reg;
  a.cartesian = E.cartesian;
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

// The cell of thread t in local tile lt of an event: tile_x == 0, 128 consecutive cells
// (interior index order); tile_x > 0, a tile_x x (kBlock / tile_x) block of one eta plane.
__device__ __forceinline__ bool tile_cell(const EventDev &E, int tile_x, int lt, int t, int &i, int &j, int &k) {
  if (tile_x == 0) {
    const long long id = (long long)lt * kBlock + t;
    i = (int)(id % E.nx);
    j = (int)((id / E.nx) % E.ny);
    k = (int)(id / ((long long)E.nx * E.ny));
    return id < E.ncells;
  }
  const int tile_y = kBlock / tile_x;
  const int tx = (E.nx + tile_x - 1) / tile_x, ty = (E.ny + tile_y - 1) / tile_y;
  i = (lt % tx) * tile_x + t % tile_x;
  j = ((lt / tx) % ty) * tile_y + t / tile_x;
  k = lt / (tx * ty);
  return i < E.nx && j < E.ny;
}

// Stage kernel over the packed tile queue of every active event (one block per tile, or a
// persistent grid walking the queue).
template <int EOS, bool SHEAR, bool BULK, bool STAGE2, bool MIXED>
__global__ void __launch_bounds__(kBlock, GVH_MIN_BLOCKS)
    batch_stage_kernel(EventDev *ev, const int *__restrict__ tile_event, const int *__restrict__ ntiles_p,
                       int tile_x) {
  const int ntiles = *ntiles_p;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    EventDev &E = ev[tile_event[tile]];
    if (!E.active || E.done) continue;
    const StageArgs a = make_args(E, STAGE2);
    int i, j, k;
    double en = 0.0, speed;
    if (tile_cell(E, tile_x, tile - E.first_tile, threadIdx.x, i, j, k))
      en = stage_cell_ijk<EOS, SHEAR, BULK, STAGE2, MIXED>(a, i, j, k, speed);
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
  if (!E.active || E.done) return;
  E.step += 1;
  const int nc = E.ufree, np = E.ucur, nf = E.uprev;
  E.ucur = nc; E.uprev = np; E.ufree = nf;
  E.emax_last = __longlong_as_double(E.emax_bits);
  E.emax_bits = 0ull;
  if (E.emax_last <= E.e_fo) E.frozen_checks += 1;
  if (E.frozen_checks >= kFreezeoutChecks) E.done = 1;
}

// Table updates as kernels (their arguments travel with the launch, so nothing on the host
// has to outlive the call and nothing waits for the device).
__global__ void event_write_kernel(EventDev *ev, int slot, EventDev E) { ev[slot] = E; }

// The initial freeze-out check (the reference tests the state before every step, the first
// one included: HydroPlugin.cpp:396-408), from the max-e reduction of the initial state.
__global__ void event_first_check_kernel(EventDev *ev, int slot, const unsigned long long *emax_bits) {
  EventDev &E = ev[slot];
  E.emax_last = __longlong_as_double(*emax_bits);
  E.frozen_checks = E.emax_last <= E.e_fo ? 1 : 0;
}

__global__ void event_deactivate_kernel(EventDev *ev, int slot) { ev[slot].active = 0; }

// first_tile of every event from the tile -> event table (events' tiles are contiguous).
__global__ void first_tiles_kernel(EventDev *ev, const int *__restrict__ tile_event, const int *__restrict__ ntiles_p) {
  const int n = *ntiles_p;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    if (t == 0 || tile_event[t] != tile_event[t - 1]) ev[tile_event[t]].first_tile = t;
}

// The end of a serving round: every slot's bookkeeping into mapped host memory, then the
// round's ticket (after a system-scope fence, so a host that sees the ticket sees the rows).
__global__ void publish_kernel(const EventDev *ev, int nslots, gvh_event_info *out, volatile long long *ticket_out,
                               long long ticket) {
  for (int i = threadIdx.x; i < nslots; i += blockDim.x) {
    const EventDev &E = ev[i];
    gvh_event_info r;
    r.step = E.step;
    r.tau = E.t0 + (double)E.step * E.dt;
    r.max_energy_density = E.emax_last;
    r.freezeout_energy_density = E.e_fo;
    r.frozen_checks = E.frozen_checks;
    r.frozen_out = E.frozen_checks >= kFreezeoutChecks;
    r.status = E.status;
    r.cells = E.ncells;
    out[i] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence_system();
    *ticket_out = ticket;
  }
}

struct HostEvent {
  bool used = false;
  size_t off = 0, bytes = 0;
  int nx = 0, ny = 0, nz = 0;
  long long ncells = 0, ng = 0, cs = 0;
  long long serial = 0;  // admission number: tells a re-used slot's events apart
};

// Tiles of an nx x ny x nz lattice for tile shape tile_x (see tile_cell).
int tiles_of(int nx, int ny, int nz, int tile_x) {
  if (tile_x == 0) return (int)(((long long)nx * ny * nz + kBlock - 1) / kBlock);
  const int tile_y = kBlock / tile_x;
  return ((nx + tile_x - 1) / tile_x) * ((ny + tile_y - 1) / tile_y) * nz;
}

// A pinned host buffer that the device copies from asynchronously, with the event that
// marks the end of the last copy (the buffer is reused only after it).
struct PinnedBuf {
  void *h = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;
  bool pending = false;
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
  int tile_x = 0;                        // tile shape (tile_cell): 0 = 128 consecutive cells
  int ntiles = 0;                        // tiles of the admitted events
  int active_slots = 0;                  // slots the finish kernel scans
  long long next_serial = 1;
  // initial states and tile tables on their way to the device: rings deep enough that the
  // admissions and retirements of one serving iteration do not wait for a copy that is queued
  // behind the rounds in flight
  static constexpr int kPrimRing = 4, kTileRing = 8;
  PinnedBuf prim_stage[kPrimRing];
  int prim_next = 0;
  PinnedBuf tile_stage[kTileRing];
  int tile_next = 0;
  // serving rounds: two snapshots in mapped host memory, alternating by ticket
  gvh_event_info *snap_h[2] = {nullptr, nullptr}, *snap_d[2] = {nullptr, nullptr};
  long long *ticket_h = nullptr, *ticket_d = nullptr;  // [2]: last ticket written per snapshot
  cudaEvent_t round_start[2] = {nullptr, nullptr}, round_end[2] = {nullptr, nullptr};
  long long next_ticket = 0;
  std::vector<std::pair<int, long long>> round_events[2];  // (slot, serial) when queued
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

// Makes a pinned buffer at least `bytes` long and free for reuse (its last copy finished).
int pinned_reserve(PinnedBuf &p, size_t bytes) {
  if (p.pending) {
    BCUDA(cudaEventSynchronize(p.done));
    p.pending = false;
  }
  if (p.cap >= bytes) return GVH_OK;
  if (p.h) cudaFreeHost(p.h);
  p.h = nullptr;
  p.cap = 0;
  if (cudaHostAlloc(&p.h, bytes, cudaHostAllocDefault) != cudaSuccess)
    return bfail(GVH_ERR_NOMEM, "cannot allocate %zu bytes of pinned host memory", bytes);
  p.cap = bytes;
  if (!p.done) BCUDA(cudaEventCreateWithFlags(&p.done, cudaEventDisableTiming));
  return GVH_OK;
}

int pinned_mark(gvh_batch *b, PinnedBuf &p) {
  BCUDA(cudaEventRecord(p.done, b->stream));
  p.pending = true;
  return GVH_OK;
}

// The tile -> event table of the admitted events (each event's tiles contiguous, events in
// slot order) and its count go to the device through a pinned buffer; first_tile of every
// event is derived on the device. Nothing waits for the device unless the tile count changes
// under a one-block-per-tile grid, which re-captures the step's graph.
int rebuild_tiles(gvh_batch *b) {
  int slots = 0, n = 0;
  for (size_t i = 0; i < b->ev.size(); ++i)
    if (b->ev[i].used) {
      slots = (int)i + 1;
      n += tiles_of(b->ev[i].nx, b->ev[i].ny, b->ev[i].nz, b->tile_x);
    }
  if (n > b->tile_capacity) return bfail(GVH_ERR_NOMEM, "tile table full");
  PinnedBuf &pb = b->tile_stage[b->tile_next];
  b->tile_next = (b->tile_next + 1) % gvh_batch::kTileRing;
  int rc = pinned_reserve(pb, (size_t)(n + 1) * sizeof(int));
  if (rc) return rc;
  int *table = static_cast<int *>(pb.h);
  int t = 0;
  for (size_t i = 0; i < b->ev.size(); ++i) {
    if (!b->ev[i].used) continue;
    const int m = tiles_of(b->ev[i].nx, b->ev[i].ny, b->ev[i].nz, b->tile_x);
    for (int k = 0; k < m; ++k) table[t++] = (int)i;
  }
  table[n] = n;
  if (n) BCUDA(cudaMemcpyAsync(b->d_tile_event, table, n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaMemcpyAsync(b->d_ntiles, table + n, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  if (n) {
    first_tiles_kernel<<<(unsigned)std::min(1024, (n + 255) / 256), 256, 0, b->stream>>>(b->d_ev, b->d_tile_event,
                                                                                         b->d_ntiles);
    BCUDA(cudaGetLastError());
  }
  if ((rc = pinned_mark(b, pb))) return rc;
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
                                                                                     b->d_ntiles, b->tile_x);
  batch_stage_kernel<EOS, SHEAR, BULK, true, MIXED><<<g, kBlock, smem, b->stream>>>(b->d_ev, b->d_tile_event,
                                                                                    b->d_ntiles, b->tile_x);
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
  if (o.coordinates != GVH_COORDINATES_MILNE && o.coordinates != GVH_COORDINATES_CARTESIAN)
    return bfail(GVH_ERR_INVALID, "unknown coordinates %d", o.coordinates);
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
  for (int r = 0; r < 2 && ok; ++r) {
    ok = cudaHostAlloc(&b->snap_h[r], kMaxEvents * sizeof(gvh_event_info), cudaHostAllocMapped) == cudaSuccess;
    ok = ok && cudaHostGetDevicePointer(&b->snap_d[r], b->snap_h[r], 0) == cudaSuccess;
    ok = ok && cudaEventCreate(&b->round_start[r]) == cudaSuccess;
    ok = ok && cudaEventCreate(&b->round_end[r]) == cudaSuccess;
  }
  ok = ok && cudaHostAlloc(&b->ticket_h, 2 * sizeof(long long), cudaHostAllocMapped) == cudaSuccess;
  ok = ok && cudaHostGetDevicePointer(&b->ticket_d, b->ticket_h, 0) == cudaSuccess;
  if (ok) b->ticket_h[0] = b->ticket_h[1] = -1;
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
  for (PinnedBuf &pb : b->prim_stage) {
    if (pb.h) cudaFreeHost(pb.h);
    if (pb.done) cudaEventDestroy(pb.done);
  }
  for (PinnedBuf &pb : b->tile_stage) {
    if (pb.h) cudaFreeHost(pb.h);
    if (pb.done) cudaEventDestroy(pb.done);
  }
  for (int r = 0; r < 2; ++r) {
    if (b->snap_h[r]) cudaFreeHost(b->snap_h[r]);
    if (b->round_start[r]) cudaEventDestroy(b->round_start[r]);
    if (b->round_end[r]) cudaEventDestroy(b->round_end[r]);
  }
  if (b->ticket_h) cudaFreeHost(b->ticket_h);
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

}  // extern "C"

namespace {

// Admission of an event whose initial state is given either as primitive arrays (prim) or as
// hotspot sources (hs) filled in on the device.
int admit_event(gvh_batch *b, const gvh_lattice_params *L, const gvh_hydro_params *H, const double *const *prim,
                int n_prim, const gvh_hotspots *hs, int *event_id) {
  NvtxRange range("gvh batch admission");
  if (!b || !L || !H || (!prim && !hs) || !event_id) return bfail(GVH_ERR_INVALID, "null argument");
  *event_id = -1;
  if (prim) {
    const int want = 5 + (b->nq - 4);
    if (n_prim != want) return bfail(GVH_ERR_INVALID, "expected %d primitive arrays", want);
    for (int f = 0; f < n_prim; ++f)
      if (!prim[f]) return bfail(GVH_ERR_INVALID, "primitive array %d is null", f);
  } else if (hs->n < 1 || !hs->x || !hs->y || !hs->w || !(hs->sigma > 0) || !(hs->sigma_eta > 0)) {
    return bfail(GVH_ERR_INVALID, "hotspots: n >= 1 sources with positions and weights, sigma > 0, sigma_eta > 0");
  }
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
  if (!arena_alloc(b, h.bytes, &h.off)) return bfail(GVH_ERR_NOMEM, "arena full (%zu bytes needed)", h.bytes);
  h.used = true;
  h.serial = b->next_serial++;
  const long long hs_doubles = hs ? 3ll * hs->n + (long long)h.nx * h.ny : 0;
  int rc = prim ? ensure_staging(b, n_prim, h.ng) : ensure_staging(b, 1, hs_doubles);
  if (rc) { arena_free(b, h.off, h.bytes); return rc; }
  // the initial state (or its sources) goes to the device through a pinned buffer: the host
  // copy happens here, the transfer is queued behind the work in flight and nothing waits
  PinnedBuf &pb = b->prim_stage[b->prim_next];
  b->prim_next = (b->prim_next + 1) % gvh_batch::kPrimRing;
  const size_t fb = h.ng * sizeof(double);
  if ((rc = pinned_reserve(pb, prim ? n_prim * fb : 3 * hs->n * sizeof(double)))) {
    arena_free(b, h.off, h.bytes);
    return rc;
  }
  double *qA, *qB, *e, *pA, *pB, *u[3];
  event_pointers(b, h, &qA, &qB, &e, &pA, &pB, u);
  BCUDA(cudaMemsetAsync(b->arena + h.off, 0, h.bytes, b->stream));
  const unsigned blocks = (unsigned)((h.ncells + 255) / 256);
  if (hs) {
    double *src = static_cast<double *>(pb.h);
    memcpy(src, hs->x, hs->n * sizeof(double));
    memcpy(src + hs->n, hs->y, hs->n * sizeof(double));
    memcpy(src + 2 * hs->n, hs->w, hs->n * sizeof(double));
    BCUDA(cudaMemcpyAsync(b->staging, src, 3 * hs->n * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    if ((rc = pinned_mark(b, pb))) return rc;
    const HotspotArgs ha = hotspot_args(h.nx, h.ny, h.nz, h.nx, (long long)h.nx * h.ny, L, hs, b->staging);
    double *plane = b->staging + 3 * hs->n;
    hotspot_plane_kernel<<<(unsigned)((h.nx * h.ny + 255) / 256), 256, 0, b->stream>>>(ha, plane);
    hotspot_fill_kernel<<<blocks, 256, 0, b->stream>>>(ha, plane, e, u[0], h.cs, qA, b->nq);
  }
  for (int f = 0; prim && f < n_prim; ++f) {
    cudaPointerAttributes at;
    const bool on_device = cudaPointerGetAttributes(&at, prim[f]) == cudaSuccess &&
                           (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
    cudaGetLastError();  // a plain host pointer is not an error
    if (on_device) {
      BCUDA(cudaMemcpyAsync(b->staging + f * h.ng, prim[f], fb, cudaMemcpyDeviceToDevice, b->stream));
    } else {
      memcpy(static_cast<char *>(pb.h) + f * fb, prim[f], fb);
      BCUDA(cudaMemcpyAsync(b->staging + f * h.ng, static_cast<char *>(pb.h) + f * fb, fb, cudaMemcpyHostToDevice,
                            b->stream));
    }
  }
  if (prim) {
    if ((rc = pinned_mark(b, pb))) return rc;
    FieldTable dst = {};
    dst.p[0] = e;
    for (int m = 0; m < 4; ++m) dst.p[1 + m] = u[0] + m * h.cs;
    for (int n = 4; n < b->nq; ++n) dst.p[5 + n - 4] = qA + n * h.cs;
    Pack pk{h.nx, h.ny, h.nz, (long long)h.nx, (long long)h.nx * h.ny, h.ng};
    pack_kernel<<<blocks, 256, 0, b->stream>>>(pk, n_prim, b->staging, dst);
  }
  if (b->opts.eos == GVH_EOS_CONFORMAL)
    init_conserved_kernel<EOS_CONFORMAL><<<blocks, 256, 0, b->stream>>>(h.ncells, b->nq, h.cs, qA, e, pA, u[0], u[1], 0);
  else
    init_conserved_kernel<EOS_QCD><<<blocks, 256, 0, b->stream>>>(h.ncells, b->nq, h.cs, qA, e, pA, u[0], u[1], 0);
  BCUDA(cudaGetLastError());

  EventDev E;
  memset(&E, 0, sizeof E);
  E.nx = h.nx; E.ny = h.ny; E.nz = h.nz; E.active = 1;
  E.sy = h.nx; E.sz = (long long)h.nx * h.ny; E.cs = h.cs; E.ncells = h.ncells;
  E.dx = L->latticeSpacingX; E.dy = L->latticeSpacingY; E.dz = L->latticeSpacingRapidity;
  E.dt = L->latticeSpacingProperTime;
  E.inv_dx = 1.0 / E.dx; E.inv_dy = 1.0 / E.dy; E.inv_dz = 1.0 / E.dz; E.inv_dt = 1.0 / E.dt;
  E.etabar = H->shearViscosityToEntropyDensity;
  E.theta = b->opts.theta;
  E.cartesian = b->opts.coordinates == GVH_COORDINATES_CARTESIAN;
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
  event_write_kernel<<<1, 1, 0, b->stream>>>(b->d_ev, slot, E);
  // initial freeze-out check, on the device
  BCUDA(cudaMemsetAsync(b->d_scratch, 0, sizeof(unsigned long long), b->stream));
  max_e_kernel<<<min(1024u, blocks), 256, 0, b->stream>>>(e, h.ncells, b->d_scratch);
  event_first_check_kernel<<<1, 1, 0, b->stream>>>(b->d_ev, slot, b->d_scratch);
  BCUDA(cudaGetLastError());
  b->ev[slot] = h;
  rc = rebuild_tiles(b);
  if (rc) return rc;
  *event_id = slot;
  return GVH_OK;
}

}  // namespace

extern "C" {

int gvh_batch_add_event(gvh_batch *b, const gvh_lattice_params *L, const gvh_hydro_params *H,
                        const double *const *prim, int n_prim, int *event_id) {
  if (!prim) return bfail(GVH_ERR_INVALID, "null argument");
  return admit_event(b, L, H, prim, n_prim, nullptr, event_id);
}

int gvh_batch_add_event_hotspots(gvh_batch *b, const gvh_lattice_params *L, const gvh_hydro_params *H,
                                 const gvh_hotspots *hs, int *event_id) {
  if (!hs) return bfail(GVH_ERR_INVALID, "null argument");
  return admit_event(b, L, H, nullptr, 0, hs, event_id);
}

int gvh_batch_remove_event(gvh_batch *b, int id) {
  if (!b || id < 0 || id >= (int)b->ev.size() || !b->ev[id].used) return bfail(GVH_ERR_INVALID, "bad event id");
  BCUDA(cudaSetDevice(b->device));
  // queued behind the work in flight, which may still read or write the event's memory; the
  // memory's next user is queued after this, so reusing it at once is safe
  event_deactivate_kernel<<<1, 1, 0, b->stream>>>(b->d_ev, id);
  BCUDA(cudaGetLastError());
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
  NvtxRange r("gvh batch steps");
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

int gvh_batch_set_tile_shape(gvh_batch *b, int tile_x) {
  if (!b || tile_x < 0 || tile_x > kBlock || (tile_x && kBlock % tile_x))
    return bfail(GVH_ERR_INVALID, "tile_x must be 0 or a divisor of %d", kBlock);
  BCUDA(cudaSetDevice(b->device));
  b->tile_x = tile_x;
  int rc = rebuild_tiles(b);
  if (rc) return rc;
  return rebuild_graph(b);  // the shape is a kernel argument of the captured step
}

int gvh_batch_tile_shape(const gvh_batch *b, int *tile_x, int *tile_y) {
  if (!b) return GVH_ERR_INVALID;
  if (tile_x) *tile_x = b->tile_x;
  if (tile_y) *tile_y = b->tile_x ? kBlock / b->tile_x : 1;
  return GVH_OK;
}

// Times `steps` real RK2 steps (the events do advance) with each candidate schedule -- tile
// shapes 128 consecutive cells, 32 x 4 and 16 x 8 cells of an eta plane, each with one block
// per tile (grid 0) and persistent grids of 1..GVH_MIN_BLOCKS blocks per SM -- and keeps the
// fastest. Every candidate computes the same values; only the schedule differs.
int gvh_batch_autotune(gvh_batch *b, int steps, int *chosen_grid) {
  if (!b || steps < 1) return bfail(GVH_ERR_INVALID, "bad arguments");
  BCUDA(cudaSetDevice(b->device));
  std::vector<int> grids{0};
  for (int k = 1; k <= GVH_MIN_BLOCKS; ++k) grids.push_back(b->num_sms * k);
  const int shapes[] = {0, 32, 16};
  cudaEvent_t e0, e1;
  BCUDA(cudaEventCreate(&e0));
  BCUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_grid = b->grid, best_shape = b->tile_x;
  for (int shape : shapes) {
    b->tile_x = shape;
    int rc = rebuild_tiles(b);
    if (rc) return rc;
    for (int g : grids) {
      if ((rc = gvh_batch_set_grid(b, g))) return rc;
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
        best_shape = shape;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tile_x = best_shape;
  int rc = rebuild_tiles(b);
  if (rc) return rc;
  rc = gvh_batch_set_grid(b, best_grid);
  if (chosen_grid) *chosen_grid = best_grid;
  return rc;
}

int gvh_batch_round(gvh_batch *b, int nsteps, long long *ticket) {
  if (!b || nsteps < 0 || !ticket) return bfail(GVH_ERR_INVALID, "bad arguments");
  NvtxRange range("gvh batch round");
  BCUDA(cudaSetDevice(b->device));
  const long long t = b->next_ticket++;
  const int r = (int)(t & 1);
  // the snapshot this round writes belongs to round t - 2: that round has finished (its copy
  // to the host is in the stream before this one) once its end event has
  if (t >= 2) BCUDA(cudaEventSynchronize(b->round_end[r]));
  b->round_events[r].clear();
  for (size_t i = 0; i < b->ev.size(); ++i)
    if (b->ev[i].used) b->round_events[r].emplace_back((int)i, b->ev[i].serial);
  BCUDA(cudaEventRecord(b->round_start[r], b->stream));
  for (int n = 0; n < nsteps; ++n) BCUDA(cudaGraphLaunch(b->graph, b->stream));
  publish_kernel<<<1, 256, 0, b->stream>>>(b->d_ev, std::max(1, b->active_slots), b->snap_d[r], b->ticket_d + r, t);
  BCUDA(cudaGetLastError());
  BCUDA(cudaEventRecord(b->round_end[r], b->stream));
  *ticket = t;
  return GVH_OK;
}

int gvh_batch_poll(gvh_batch *b, long long ticket, int max_events, int *event_ids, gvh_event_info *infos,
                   int *n_events, double *round_ms) {
  if (!b || !n_events || ticket < 0 || ticket >= b->next_ticket || max_events < 0 ||
      (max_events > 0 && (!event_ids || !infos)))
    return bfail(GVH_ERR_INVALID, "bad arguments");
  if (ticket + 2 < b->next_ticket) return bfail(GVH_ERR_INVALID, "round %lld: its snapshot was overwritten", ticket);
  BCUDA(cudaSetDevice(b->device));
  const int r = (int)(ticket & 1);
  BCUDA(cudaEventSynchronize(b->round_end[r]));
  if (b->ticket_h[r] != ticket) return bfail(GVH_ERR_INTERNAL, "round %lld: snapshot not written", ticket);
  if (round_ms) {
    float ms = 0;
    BCUDA(cudaEventElapsedTime(&ms, b->round_start[r], b->round_end[r]));
    *round_ms = ms;
  }
  // the events of the round that are still admitted (a slot emptied or refilled since the
  // round was queued reports nothing: its snapshot row belongs to the old event)
  int n = 0;
  for (const auto &se : b->round_events[r]) {
    const int slot = se.first;
    if (slot >= (int)b->ev.size() || !b->ev[slot].used || b->ev[slot].serial != se.second) continue;
    if (n < max_events) {
      event_ids[n] = slot;
      infos[n] = b->snap_h[r][slot];
    }
    ++n;
  }
  *n_events = n;
  if (n > max_events) return bfail(GVH_ERR_INVALID, "%d events do not fit in %d", n, max_events);
  return GVH_OK;
}

}  // extern "C"
