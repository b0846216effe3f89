// gvh_stage.cuh -- the fused KT stage kernel (plain FP64 path).
//
// One launch is one RK substep of twoStepRungeKutta (FullyDiscreteKurganovTadmorScheme.cu
// :109-139) over every interior cell. Per cell it does what the reference spreads over
// eulerStepKernelSource_1D + X_1D + Y_1D + Z_1D (EulerStep.cu:946-1277), the convex
// combination (FullyDiscreteKurganovTadmorScheme.cu:60-104, stage 2 only),
// setInferredVariablesKernel (EnergyMomentumTensor.cu:110-154) and
// regulateDissipativeCurrents (RegulateDissipativeCurrents.cu:15-134), keeping everything
// in registers and writing each output once. setGhostCells (GhostCells.cu:15-144) is
// replaced by clamped neighbour indices: a zero-gradient ghost always equals the nearest
// interior cell, and every stencil is axis-aligned, so clamping reads the same values.
//
// Each cell evaluates both faces of each axis with its own energy density as the Newton
// guess, as the reference does (EulerStep.cu:1054-1062): for the QCD equation of state the
// face solution depends on that guess through the solver's stop test, so sharing a face
// between two cells would change the answer.
//
// Per axis the flux is done in two phases to keep few values live: (A) the half-cell states
// of the components the root find needs (T^{tau mu}, pi^{tau mu}, Pi) go to a shared-memory
// cache, and the four face recoveries (one Newton solve at a time) give u^axis/u^tau on both
// sides of both faces; (B) the cached components, then pi^{ij} (5 loads, 3 limited slopes),
// go through the two KT fluxes into the running update.
//
// Layout in HBM (interior only, no ghosts): component-major SoA, cell index
// s = i + sy*j + sz*k, component c at c*cs + s.
#pragma once

#include <stdint.h>

#include <type_traits>

#include "gvh_physics.cuh"
#include "gvh_sources.cuh"

namespace gvh {

struct StageArgs {
  int nx, ny, nz;
  long long sy, sz, cs;   // strides: row, plane, component
  long long ncells;       // nx*ny*nz
  double dx, dy, dz;      // lattice spacings
  double dt;              // lattice time step (d_dt) used in the Euler update
  double inv_dx, inv_dy, inv_dz, inv_dt;  // 1/dx, 1/dy, 1/dz, 1/dt (set_inverse_spacings)
  double etabar, theta;
  double t_euler;         // time passed to the Euler step
  double t_after;         // time passed to primitive recovery and regulation
  double e_reg;           // e(T_reg): cells with e <= e_reg are regulated
  const double *qin;      // conserved input (stencil)
  const double *qn;       // stage 2: q^n for the convex combination (may alias qout)
  double *qout;
  double *e;              // read (guess, source) and overwritten, centre only
  const double *pin;      // pressure (stencil)
  double *pout;
  const double *uin;      // u^mu (stencil)
  const double *uprev;    // u^mu of the previous time level, centre only (may alias uout)
  double *uout;
  unsigned *status;       // or-ed STATUS_* bits
  double *diag;           // stage 2, optional: regulation factor (component 0) and the centre's
                          // q^n pi^{mu nu}, Pi (components 13..23) for the validity diagnostics
  unsigned long long *speed_max;  // stage 1, optional: running max of a / dx_axis over cells, as
                                  // the bit pattern of a non-negative double (see kt_stage_kernel)
  int cartesian;          // GVH_COORDINATES_CARTESIAN: no Milne geometric sources (stage_source)
};

// Components of the validity block (VALIDITY_DOMAIN, DynamicalVariables.cuh:82-98, in that
// order), then the saved q^n dissipative currents the diagnostics read.
constexpr int kValidityFields = 13;
constexpr int kValiditySaved = 11;

#ifndef GVH_BLOCK
#define GVH_BLOCK 128
#endif
constexpr int kBlock = GVH_BLOCK;  // threads per block of the stage kernel

// The reciprocal spacings, computed once by whoever fills the arguments.
__host__ __device__ inline void set_inverse_spacings(StageArgs &a) {
  a.inv_dx = 1.0 / a.dx;
  a.inv_dy = 1.0 / a.dy;
  a.inv_dz = 1.0 / a.dz;
  a.inv_dt = 1.0 / a.dt;
}

template <bool SHEAR, bool BULK>
struct NComp {
  static constexpr int value = 4 + (SHEAR ? 10 : 0) + (BULK ? 1 : 0);
};

// u^axis/u^tau on the left and right of the faces i+1/2 (fwd) and i-1/2 (bwd), and the
// local propagation speed of each face (LocalPropagationSpeed.cu:15-24, SpectralRadius.cu).
template <class R>
struct FaceSpeeds {
  R wLf, wRf, af, wLb, wRb, ab;
};

// Phase A. Half-cell states (HalfSiteExtrapolation.cu:15-30) of the root-find components
// at both faces, then primitive recovery of all four (SemiDiscreteKurganovTadmorScheme.cu
// :41-44) with the cell's own energy density as guess.
// The half-cell states go to this thread's column of the shared-memory cache
// (cache[(4 r + f) * kBlock]), from which phase B takes them instead of recomputing them.
template <int EOS, bool SHEAR, bool BULK, bool MIXED>
__device__ __forceinline__ FaceSpeeds<double> face_speeds(const StageArgs &a, int s, int axis, const int (&o)[5],
                                                       const GuessEos &g0, double *cache, unsigned &status) {
  // index f: 0 fwd R, 1 fwd L, 2 bwd R, 3 bwd L. The states go to the cache first; the four
  // recoveries then read them back one at a time (runtime loops keep the code small:
  // instruction fetch, not arithmetic, is what the long straight-line variant waited on).
  constexpr int NR = 4 + (SHEAR ? 4 : 0) + (BULK ? 1 : 0);
  // three components per pass: their 15 stencil loads are in flight together (one at a time
  // the loop waited on each component's loads; 3 measured 4% faster than 1, 2 and 9 slower)
#pragma unroll 3
  for (int r = 0; r < NR; ++r) {
    const int c = (r < 8) ? r : 14;
    const double *q = a.qin + (size_t)c * a.cs + s;
    const double q0 = __ldg(q + o[0]), q1 = __ldg(q + o[1]), q2 = __ldg(q), q3 = __ldg(q + o[3]), q4 = __ldg(q + o[4]);
    const double theta2 = 2 * a.theta;  // the slopes come doubled: q -+ D/2 = q -+ D2/4
    double Dm, D0, Dp;
    if (MIXED) {
      // mixed: the limiter in FP32 on the FP64 differences (rounded), the states in FP64
      const float t2f = (float)theta2;
      const float d10 = (float)(q1 - q0), d21 = (float)(q2 - q1), d32 = (float)(q3 - q2), d43 = (float)(q4 - q3);
      Dm = slope2_from_differences(t2f, d10, (float)(q2 - q0), d21);
      D0 = slope2_from_differences(t2f, d21, (float)(q3 - q1), d32);
      Dp = slope2_from_differences(t2f, d32, (float)(q4 - q2), d43);
    } else {
      Dm = limited_slope2(theta2, q0, q1, q2);
      D0 = limited_slope2(theta2, q1, q2, q3);
      Dp = limited_slope2(theta2, q2, q3, q4);
    }
    double *cr = cache + 4 * r * kBlock;
    cr[0] = q3 - Dp * 0.25;           // fwd qR
    cr[kBlock] = q2 + D0 * 0.25;      // fwd qL
    cr[2 * kBlock] = q2 - D0 * 0.25;  // bwd qR
    cr[3 * kBlock] = q1 + Dm * 0.25;  // bwd qL
  }
  double w[4] = {0, 0, 0, 0};
#pragma unroll 1
  for (int h = 0; h < 4; ++h) {
    double st[9][1];
#pragma unroll
    for (int r = 0; r < 9; ++r) st[r][0] = r < NR ? cache[(4 * r + h) * kBlock] : 0.0;
    double w1[1];
    inferred_face_n<EOS, 1>(a.t_euler, axis, st[0], st[1], st[2], st[3], st[4], st[5], st[6], st[7], st[8], g0, w1,
                            status);
    w[0] = h == 0 ? w1[0] : w[0];
    w[1] = h == 1 ? w1[0] : w[1];
    w[2] = h == 2 ? w1[0] : w[2];
    w[3] = h == 3 ? w1[0] : w[3];
  }
  FaceSpeeds<double> f;
  f.wRf = w[0]; f.wLf = w[1]; f.wRb = w[2]; f.wLb = w[3];
  f.af = fmax(fabs(f.wLf), fabs(f.wRf));
  f.ab = fmax(fabs(f.wLb), fabs(f.wRb));
  return f;
}

// Phase B for one component: the KT fluxes H(i+1/2), H(i-1/2)
// (SemiDiscreteKurganovTadmorScheme.cu:48-56, F = q u^axis/u^tau, FluxFunctions.cu:18-31)
// and their difference (EulerStep.cu:1054-1062).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// 2 (-H(i+1/2) + H(i-1/2)) from the four half-cell states (fwd qR, fwd qL, bwd qR, bwd qL).
template <class R>
__device__ __forceinline__ R flux_from_states(R fR, R fL, R bR, R bL, const FaceSpeeds<R> &f) {
  // F(qR) and F(qL) are rounded separately (no fused multiply-add across the pair), which
  // keeps the scheme exactly mirror-symmetric.
  // Returned doubled: the halving of both fluxes is folded into the caller's 1/(2 d), a
  // power-of-two scaling that commutes with rounding, so the value is the same.
  const R Hf = mul_rn(fR, f.wRf) + mul_rn(fL, f.wLf) - f.af * (fR - fL);
  const R Hb = mul_rn(bR, f.wRb) + mul_rn(bL, f.wLb) - f.ab * (bR - bL);
  return -Hf + Hb;
}

template <class R>
__device__ __forceinline__ R flux_difference(R theta, const double *q, const int (&o)[5], const FaceSpeeds<R> &f) {
  const R q0 = (R)__ldg(q + o[0]), q1 = (R)__ldg(q + o[1]), q2 = (R)__ldg(q), q3 = (R)__ldg(q + o[3]);
  const R q4 = (R)__ldg(q + o[4]);
  const R theta2 = R(2) * theta;  // doubled slopes: q -+ D/2 = q -+ D2/4
  const R Dm = limited_slope2(theta2, q0, q1, q2);
  const R D0 = limited_slope2(theta2, q1, q2, q3);
  const R Dp = limited_slope2(theta2, q2, q3, q4);
  const R qu = R(0.25);
  return flux_from_states<R>(q3 - Dp * qu, q2 + D0 * qu, q2 - D0 * qu, q1 + Dm * qu, f);
}

// pi^{m a} component index for spatial m, a in {x, y, eta}.
__device__ __forceinline__ int pi_spatial(int m, int a) {
  // xx=8 xy=9 xn=10 yy=11 yn=12 nn=13
  return (m == 0) ? 8 + a : (m == 1) ? (a == 0 ? 9 : 10 + a) : (a == 0 ? 10 : 11 + a);
}

// One axis of the Euler update (EulerStep.cu:1011-1277, one of X/Y/Z, the axis chosen at
// run time so the code exists once): out += dt * ( (H(i-1/2) - H(i+1/2)) / d + S_axis ),
// with S_axis of SourceTerms.cu:443-567:
//   S_0     = d(pi^{tt}) v - d(pi^{t a}) [- v d(Pi)]
//   S_{m+1} = d(pi^{t m}) v - d(pi^{m a}) [- d(Pi), divided by tau^2 along eta, when m = a]
// Sa: the axis's pi and Pi derivative sources of T^{tau mu} (SourceTerms.cu:443-567), in the
// working precision; zero without shear.
template <bool SHEAR, bool BULK, class R>
__device__ __forceinline__ void axis_pi_sources(const StageArgs &a, int s, int axis, const int (&o)[5], R inv_d,
                                                const double *uc, R (&Sa)[4]) {
  Sa[0] = Sa[1] = Sa[2] = Sa[3] = R(0);
  if (SHEAR) {
    const R fac = inv_d / R(2);
    auto der = [&](int c) {
      const double *q = a.qin + (size_t)c * a.cs + s;
      return ((R)__ldg(q + o[3]) - (R)__ldg(q + o[1])) * fac;
    };
    const R v = dv((R)uc[1 + axis], (R)uc[0]);
    const R dPi = BULK ? der(14) : R(0);
    const R dPi_aa = (axis == 2) ? dv(dPi, (R)(a.t_euler * a.t_euler)) : dPi;
    R s0 = der(4) * v - der(5 + axis);
    if (BULK) s0 = s0 - v * dPi;
    Sa[0] = s0;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      R sm = der(5 + m) * v - der(pi_spatial(m, axis));
      if (BULK && m == axis) sm = sm - dPi_aa;
      Sa[1 + m] = sm;
    }
  }
}

// Returns the axis's local propagation speed, max(a(i+1/2), a(i-1/2)) (SpectralRadius.cu:17-30).
// INCREMENT: store each component's increment before the factor dt in out instead of adding
// dt times it (the split kernel, whose source warp adds them in axis order).
template <int EOS, bool SHEAR, bool BULK, bool MIXED, bool INCREMENT = false>
__device__ __forceinline__ double axis_update(const StageArgs &a, int s, int axis, int idx, int n_axis, int stride,
                                              double inv_spacing, const GuessEos &g0, const double *uc, double *out,
                                              double *cache, unsigned &status) {
  using R = typename std::conditional<MIXED, float, double>::type;
  constexpr int NQ = NComp<SHEAR, BULK>::value;
  const int o[5] = {(max(idx - 2, 0) - idx) * stride, (max(idx - 1, 0) - idx) * stride, 0,
                    (min(idx + 1, n_axis - 1) - idx) * stride, (min(idx + 2, n_axis - 1) - idx) * stride};
  const R inv_d = R(inv_spacing);
  const R half_inv_d = R(0.5) * inv_d;  // the fluxes come doubled from flux_from_states
  // Face states are recovered in FP64 on both paths (the mixed path rounds only the
  // resulting speeds): an FP32 recovery was tried and let a 2+1D hotspot event run away
  // to NaN that the FP64 recovery keeps finite.
  const FaceSpeeds<double> fd = face_speeds<EOS, SHEAR, BULK, MIXED>(a, s, axis, o, g0, cache, status);
  FaceSpeeds<R> f;
  f.wRf = (R)fd.wRf; f.wLf = (R)fd.wLf; f.wRb = (R)fd.wRb; f.wLb = (R)fd.wLb;
  f.af = (R)fd.af; f.ab = (R)fd.ab;

  R Sa[4];
  axis_pi_sources<SHEAR, BULK, R>(a, s, axis, o, inv_d, uc, Sa);
  const R th = (R)a.theta;
  // the root-find components from the cache
  constexpr int NRC = 4 + (SHEAR ? 4 : 0) + (BULK ? 1 : 0);
#pragma unroll 1
  for (int rc = 0; rc < NRC; ++rc) {
    const int n = rc < 8 ? rc : NQ - 1;
    const double *c = cache + 4 * rc * kBlock;
    R r = flux_from_states<R>((R)c[0], (R)c[kBlock], (R)c[2 * kBlock], (R)c[3 * kBlock], f);
    r = r * half_inv_d;
    if (SHEAR && n < 4) r += Sa[n];
    if (INCREMENT) out[n * kBlock] = (double)r;
    else out[n * kBlock] += (double)r * a.dt;
  }
  // pi^{ij} from the lattice, two components' stencil loads in flight at once (2 measured
  // faster than 1, 3 and 6)
  if (SHEAR) {
#pragma unroll 2
    for (int n = 8; n < 14; ++n) {
      R r = flux_difference<R>(th, a.qin + (size_t)n * a.cs + s, o, f);
      if (INCREMENT) out[n * kBlock] = (double)(r * half_inv_d);
      else out[n * kBlock] += (double)(r * half_inv_d) * a.dt;
    }
  }
  return fmax(fd.af, fd.ab);
}

// Shared memory of one stage block: the running update (NQ per thread) and the half-cell
// state cache (4 per root-find component per thread), in doubles.
template <bool SHEAR, bool BULK>
constexpr size_t stage_smem_bytes() {
  return (size_t)(NComp<SHEAR, BULK>::value + 4 * (4 + (SHEAR ? 4 : 0) + (BULK ? 1 : 0))) * kBlock * sizeof(double);
}

#ifndef GVH_MIN_BLOCKS
#define GVH_MIN_BLOCKS 4
#endif
// MIXED = false: plain FP64. MIXED = true: limiter, KT fluxes and source-term algebra in
// FP32; the state, every primitive-variable recovery (face states and cell centre), the
// differences feeding the source terms, the running update, the Heun combination and the
// regulation in FP64.
//
// stage_cell does one cell (interior index id < a.ncells); it returns the cell's new energy
// density so callers can reduce it (the batched engine tracks max e per event).
// The source-term Euler step of one cell: out[n * OSTRIDE] = q_n + dt * S_n
// (EulerStep.cu:946-1009, SourceTerms.cu:569-755).
template <int EOS, bool SHEAR, bool BULK, bool MIXED, int OSTRIDE>
__device__ __forceinline__ void stage_source(const StageArgs &a, long long s, int i, int j, int k, double ePrev,
                                             const double (&uc)[4], double *out) {
  using R = typename std::conditional<MIXED, float, double>::type;
  constexpr int NQ = NComp<SHEAR, BULK>::value;
  R q[NQ];
#pragma unroll
  for (int n = 0; n < NQ; ++n) q[n] = (R)__ldg(a.qin + n * a.cs + s);
  const R pc = (R)__ldg(a.pin + s);
  const long long xm = (i > 0) ? -1 : 0, xp = (i < a.nx - 1) ? 1 : 0;
  const long long ym = (j > 0) ? -a.sy : 0, yp = (j < a.ny - 1) ? a.sy : 0;
  const long long zm = (k > 0) ? -a.sz : 0, zp = (k < a.nz - 1) ? a.sz : 0;
  // Derivatives of u and p: differences of nearly equal values, so they are formed in
  // FP64 on both paths and only the results are rounded to the working precision.
  CellFlowT<R> f;
  R ucr[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) ucr[m] = (R)uc[m];
  f.ut = ucr[0]; f.ux = ucr[1]; f.uy = ucr[2]; f.un = ucr[3];
  // d u^mu / d tau = (u - u^{n-1}) / dt (SourceTerms.cu:68-71)
  const double inv_dt = a.inv_dt;
  f.dtut = (R)((uc[0] - a.uprev[s]) * inv_dt);
  f.dtux = (R)((uc[1] - a.uprev[a.cs + s]) * inv_dt);
  f.dtuy = (R)((uc[2] - a.uprev[2 * a.cs + s]) * inv_dt);
  f.dtun = (R)((uc[3] - a.uprev[3 * a.cs + s]) * inv_dt);
  // doubled slopes (limited_slope2) times 1/(2 dx): the limited derivatives of
  // SourceTerms.cu:659-720
  const double thd = 2 * a.theta;
  const double idxd = 0.5 * a.inv_dx, idyd = 0.5 * a.inv_dy, idzd = 0.5 * a.inv_dz;
  R du[3][4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const double *u = a.uin + m * a.cs + s;
    du[0][m] = (R)(limited_slope2(thd, __ldg(u + xm), uc[m], __ldg(u + xp)) * idxd);
    du[1][m] = (R)(limited_slope2(thd, __ldg(u + ym), uc[m], __ldg(u + yp)) * idyd);
    du[2][m] = (R)(limited_slope2(thd, __ldg(u + zm), uc[m], __ldg(u + zp)) * idzd);
  }
  f.dxut = du[0][0]; f.dyut = du[1][0]; f.dnut = du[2][0];
  f.dxux = du[0][1]; f.dyux = du[1][1]; f.dnux = du[2][1];
  f.dxuy = du[0][2]; f.dyuy = du[1][2]; f.dnuy = du[2][2];
  f.dxun = du[0][3]; f.dyun = du[1][3]; f.dnun = du[2][3];
  const double *p = a.pin + s;
  const double pcd = __ldg(p);
  const R dxp = (R)(limited_slope2(thd, __ldg(p + xm), pcd, __ldg(p + xp)) * idxd);
  const R dyp = (R)(limited_slope2(thd, __ldg(p + ym), pcd, __ldg(p + yp)) * idyd);
  const R dnp = (R)(limited_slope2(thd, __ldg(p + zm), pcd, __ldg(p + zp)) * idzd);

  const R t = (R)a.t_euler;
  const R Pi = BULK ? q[NQ - 1] : R(0);
  const R pitt = SHEAR ? q[4] : R(0), pitx = SHEAR ? q[5] : R(0), pity = SHEAR ? q[6] : R(0);
  const R pitn = SHEAR ? q[7] : R(0), pinn = SHEAR ? q[13] : R(0);
  const R ut = ucr[0], ux = ucr[1], uy = ucr[2], un = ucr[3];
  const R iut = dv(R(1), ut), it = dv(R(1), t);
  // Tnn (EnergyMomentumTensor.cu:205-207) with p + Pi
  const R pP = pc + Pi;
  const R er = (R)ePrev;
  const R tnn = (er + pP) * un * un + pP * it * it + pinn;
  const R vx = ux * iut, vy = uy * iut, vn = un * iut;
  const R dxvx = (f.dxux - vx * f.dxut) * iut;
  const R dyvy = (f.dyuy - vy * f.dyut) * iut;
  const R dnvn = (f.dnun - vn * f.dnut) * iut;
  const R dkvk = dxvx + dyvy + dnvn;
  // The Milne geometry enters through gi = 1/tau and gt = tau (the geometric sources) and
  // gn = 1/tau (the eta derivative's metric factor, taken twice). Cartesian coordinates
  // (USE_CARTESIAN_COORDINATES, SourceTerms.cu:738-743) drop the geometric sources and the
  // factor: gi = gt = 0 and gn = 1 give exactly the reference's Cartesian terms (the dropped
  // products are zeros that adding leaves out), and the Milne expressions keep their form.
  // The pi^{mu nu} sources below keep their Milne terms in both, as in the reference.
  const R gi = a.cartesian ? R(0) : it, gt = a.cartesian ? R(0) : t, gn = a.cartesian ? R(1) : it;
  R S[NQ];
  S[0] = -(q[0] * gi + gt * tnn) + dkvk * (pitt - pc - Pi) - vx * dxp - vy * dyp - vn * dnp;
  S[1] = -q[1] * gi - dxp + dkvk * pitx;
  S[2] = -q[2] * gi - dyp + dkvk * pity;
  S[3] = R(-3) * q[3] * gi - dnp * gn * gn + dkvk * pitn;
  if (SHEAR) {
    ShearT<R> pi{q[4], q[5], q[6], q[7], q[8], q[9], q[10], q[11], q[12], q[13]};
    R rhs[11];
    pimunu_rhs<EOS, BULK, R>(rhs, t, (R)a.etabar, er, pc, f, pi, Pi, dkvk);
#pragma unroll
    for (int n = 4; n < NQ; ++n) S[n] = rhs[n - 4];
  }
#pragma unroll
  for (int n = 0; n < NQ; ++n) {
    // the FP64 value of q is re-read for the accumulation (a no-op reload on the FP64 path)
    const double qd = MIXED ? __ldg(a.qin + n * a.cs + s) : (double)q[n];
    out[n * OSTRIDE] = qd + a.dt * (double)S[n];
  }
}

// The rest of a stage for one cell once out holds its Euler update: the Heun combination
// (stage 2), primitive recovery at the new time, regulation, and the writes. Returns e.
template <int EOS, bool SHEAR, bool BULK, bool STAGE2, int OSTRIDE>
__device__ __forceinline__ double stage_finish(const StageArgs &a, long long s, const double *out, const GuessEos &g0,
                                               unsigned status) {
  constexpr int NQ = NComp<SHEAR, BULK>::value;
  // ---- Heun combination Q = (Q + q^n)/2 (FullyDiscreteKurganovTadmorScheme.cu:60-104) ---
  double o[NQ];
#pragma unroll
  for (int n = 0; n < NQ; ++n) o[n] = out[n * OSTRIDE];
  if (STAGE2) {
#pragma unroll
    for (int n = 0; n < NQ; ++n) o[n] = (o[n] + a.qn[n * a.cs + s]) * 0.5;
  }

  // ---- primitive recovery at the new time (EnergyMomentumTensor.cu:110-154) ---------------
  const double tn = a.t_after;
  Prim pr = inferred<EOS>(tn, o[0], o[1], o[2], o[3], SHEAR ? o[4] : 0.0, SHEAR ? o[5] : 0.0,
                          SHEAR ? o[6] : 0.0, SHEAR ? o[7] : 0.0, BULK ? o[NQ - 1] : 0.0, g0, status);

  // ---- regulation (RegulateDissipativeCurrents.cu:15-134) ----------------------------------
  double fac_reg = 1.0;
  if (SHEAR && pr.e <= a.e_reg) {
    const double pitt = o[4], pitx = o[5], pity = o[6], pitn = o[7], pixx = o[8], pixy = o[9];
    const double pixn = o[10], piyy = o[11], piyn = o[12], pinn = o[13];
    const double t2 = tn * tn;
    const double xi0 = 0.1, rhomax = 1.0;
    double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy + piyy * piyy
                  - 2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 + pinn * pinn * t2 * t2;
    double spipi = sqrt(fabs(pipi));
    double pimumu = pitt - pixx - piyy - pinn * tn * tn;
    double piu0 = -pitn * t2 * pr.un + pitt * pr.ut - pitx * pr.ux - pity * pr.uy;
    double piu1 = -pixn * t2 * pr.un + pitx * pr.ut - pixx * pr.ux - pixy * pr.uy;
    double piu2 = -piyn * t2 * pr.un + pity * pr.ut - pixy * pr.ux - piyy * pr.uy;
    double piu3 = -pinn * t2 * pr.un + pitn * pr.ut - pixn * pr.ux - piyn * pr.uy;
    double a1 = (spipi / rhomax) * (1.0 / sqrt(pr.e * pr.e + 3 * pr.p * pr.p));
    double inv_den = 1.0 / (xi0 * rhomax * spipi);  // one reciprocal for the five quotients
    double rho = fmax(a1, fmax(pimumu * inv_den,
                               fmax(piu0 * inv_den, fmax(piu1 * inv_den, fmax(piu2 * inv_den, piu3 * inv_den)))));
    double facShear = tanh(rho) / rho;
    if (fabs(rho) < 1.e-7) facShear = 1.0;
    // The reference reads Pi as 0 here (its `#ifdef Pi` is never true), so rho_bulk = 0
    // and the bulk factor is always 1 (RegulateDissipativeCurrents.cu:54-58, 106-109).
#pragma unroll
    for (int n = 4; n < 14; ++n) o[n] *= facShear;
    fac_reg = facShear;
  }

  // ---- validity diagnostics inputs (stage 2, when asked for) ------------------------------
  // The reference's regulateDissipativeCurrents stores facShear (RegulateDissipativeCurrents
  // .cu:132; the last of its calls in a step is on the corrected state), and its checkValidity
  // reads pi^{mu nu} and Pi of d_q, the state before the step (FullyDiscreteKurganovTadmorScheme
  // .cu:137); q^n is overwritten below, so its centre values are kept here.
  if (STAGE2 && a.diag) {
    a.diag[s] = fac_reg;
#pragma unroll
    for (int m = 0; m < kValiditySaved; ++m) {
      const int c = 4 + m;
      a.diag[(kValidityFields + m) * a.cs + s] =
          (c < 14 ? SHEAR : BULK) ? a.qn[(c < 14 ? c : NQ - 1) * a.cs + s] : 0.0;
    }
  }

  // ---- write ----------------------------------------------------------------------------
#pragma unroll
  for (int n = 0; n < NQ; ++n) a.qout[n * a.cs + s] = o[n];
  a.e[s] = pr.e;
  a.pout[s] = pr.p;
  a.uout[s] = pr.ut;
  a.uout[a.cs + s] = pr.ux;
  a.uout[2 * a.cs + s] = pr.uy;
  a.uout[3 * a.cs + s] = pr.un;
  if (status) atomicOr(a.status, status);
  return pr.e;
}

// Whether every index a stage uses for cell (i, j, k) lies inside a component array
// [0, cs): the cell itself, its clamped stencil along each axis (axis_update's o[]) and its
// clamped neighbours (stage_source). The bounds-checked build (GVH_BOUNDS_CHECK) runs it before
// any load of the cell and skips a cell that fails, raising STATUS_BOUNDS; host-callable, so the
// same function is tested on the CPU.
__host__ __device__ inline bool cell_stencil_ok(const StageArgs &a, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= a.nx || j >= a.ny || k >= a.nz) return false;
  const long long s = i + a.sy * j + a.sz * k;
  if (s < 0 || s >= a.cs) return false;
  for (int axis = 0; axis < 3; ++axis) {
    const int idx = axis == 0 ? i : axis == 1 ? j : k;
    const int n = axis == 0 ? a.nx : axis == 1 ? a.ny : a.nz;
    const long long stride = axis == 0 ? 1 : axis == 1 ? a.sy : a.sz;
    for (int d = -2; d <= 2; ++d) {
      const int c = d < 0 ? (idx + d > 0 ? idx + d : 0) : (idx + d < n - 1 ? idx + d : n - 1);
      const long long t = s + (long long)(c - idx) * stride;
      if (t < 0 || t >= a.cs) return false;
    }
  }
  return true;
}

// speed: max over the axes with more than one cell of the local propagation speed over the lattice spacing,
// a / dx_axis (the CFL bound of the step is dt times its maximum over cells).
template <int EOS, bool SHEAR, bool BULK, bool STAGE2, bool MIXED>
__device__ __forceinline__ double stage_cell_ijk(const StageArgs &a, int i, int j, int k, double &speed) {
  using R = typename std::conditional<MIXED, float, double>::type;
  constexpr int NQ = NComp<SHEAR, BULK>::value;
  const long long s = i + a.sy * j + a.sz * k;
  unsigned status = 0;
#ifdef GVH_BOUNDS_CHECK
  if (!cell_stencil_ok(a, i, j, k)) {
    atomicOr(a.status, STATUS_BOUNDS);
    speed = 0.0;
    return 0.0;
  }
#endif

  const double ePrev = a.e[s];
  double uc[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) uc[m] = __ldg(a.uin + m * a.cs + s);

  // The running update of each component lives in shared memory (this thread's column): it
  // is read-modified-written once per axis, and keeping it out of registers leaves them to
  // the Newton solves and the source algebra. The half-cell state cache follows it.
  extern __shared__ double gvh_stage_smem[];
  double *out = gvh_stage_smem + threadIdx.x;
  double *cache = gvh_stage_smem + NQ * kBlock + threadIdx.x;

  stage_source<EOS, SHEAR, BULK, MIXED, kBlock>(a, s, i, j, k, ePrev, uc, out);

  // ---- flux divergence along x, y, eta (EulerStep.cu:1011-1277) -------------------------
  const GuessEos g0 = guess_eos<EOS>(ePrev);
  speed = 0.0;
#pragma unroll 1
  for (int axis = 0; axis < 3; ++axis) {
    const int idx = axis == 0 ? i : axis == 1 ? j : k;
    const int n_axis = axis == 0 ? a.nx : axis == 1 ? a.ny : a.nz;
    // An axis with one cell (eta of a 2+1D lattice) adds nothing: its clamped stencil is the
    // cell five times, so both faces carry the cell's own state, their two KT fluxes are the
    // same number and their difference is exactly 0, as are the centred pi, Pi derivatives.
    // The reference computes it anyway (EulerStep.cu:1011-1277); skipping its four face
    // recoveries changes at most the sign of a zero. The FP64 kernel skips it (2+1D steps
    // 23% faster, 3+1D unchanged); in the mixed kernel the test cost 0.26% on 3+1D events,
    // which carry nearly all of a serving mix's cell-updates, so it computes the axis. Such an
    // axis has no faces for the CFL bound either.
    if (!MIXED && n_axis == 1) continue;
    const int stride = axis == 0 ? 1 : axis == 1 ? (int)a.sy : (int)a.sz;
    const double inv_spacing = axis == 0 ? a.inv_dx : axis == 1 ? a.inv_dy : a.inv_dz;
    const double as = axis_update<EOS, SHEAR, BULK, MIXED>(a, (int)s, axis, idx, n_axis, stride, inv_spacing, g0,
                                                           uc, out, cache, status);
    speed = fmax(speed, n_axis > 1 ? as * inv_spacing : 0.0);
  }

  return stage_finish<EOS, SHEAR, BULK, STAGE2, kBlock>(a, s, out, g0, status);
}

// The cell with interior index id (i fastest).
template <int EOS, bool SHEAR, bool BULK, bool STAGE2, bool MIXED>
__device__ __forceinline__ double stage_cell(const StageArgs &a, long long id, double &speed) {
  const int i = (int)(id % a.nx);
  const int j = (int)((id / a.nx) % a.ny);
  const int k = (int)(id / ((long long)a.nx * a.ny));
  return stage_cell_ijk<EOS, SHEAR, BULK, STAGE2, MIXED>(a, i, j, k, speed);
}

// The grid of a stage launch: one block per kBlock consecutive cells (interior index order).
// (Blocks of 16x8 and 32x4 cells of one eta plane were measured too: the same time per step
// on the 131x131x61 event, so the stencil's y and eta neighbours do not limit the kernel.)
inline dim3 stage_grid(long long ncells) { return dim3((unsigned)((ncells + kBlock - 1) / kBlock)); }

// One RK substep over one lattice: one thread per interior cell. Launch with
// stage_smem_bytes<SHEAR, BULK>() of dynamic shared memory (above the 48 KB default: the
// launcher raises the kernel's cudaFuncAttributeMaxDynamicSharedMemorySize first).
//
// Stage 1 with a.speed_max set also reduces the cells' speed (a / dx_axis, stage_cell) to one
// maximum: a warp-shuffle max over the warp's cells, then one atomic max per warp on the
// value's bit pattern (for non-negative doubles the integer order of the bits is the numeric
// order). It is a by-product of the face recoveries the step does anyway: the step keeps the
// caller's dt.
template <int EOS, bool SHEAR, bool BULK, bool STAGE2, bool MIXED>
__global__ void __launch_bounds__(kBlock, GVH_MIN_BLOCKS) kt_stage_kernel(const StageArgs a) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double speed = 0.0;
  if (id < a.ncells) stage_cell<EOS, SHEAR, BULK, STAGE2, MIXED>(a, id, speed);
  if (!STAGE2 && a.speed_max) {
    unsigned long long b = (unsigned long long)__double_as_longlong(fmax(speed, 0.0));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if ((threadIdx.x & 31) == 0) atomicMax(a.speed_max, b);
  }
}

// ---- lattices too small to fill the GPU: one cell's stage on four warps -----------------
// With fewer cells than the GPU has thread slots (148 SMs x 4 blocks x kBlock) SMs sit idle
// and the time is one thread's dependency chain: the source term, then the three axes one
// after another. Here a block takes kSplitCells cells and each of its four warps does one part
// of every cell: warp 0 the source term, warps 1-3 the x, y and eta fluxes. An axis warp
// leaves its components' increments (before the factor dt) in its own shared-memory column;
// after a barrier warp 0 adds them to its Euler update in axis order, in the same expression
// as the one-thread-per-cell kernel's running update, and finishes the cell. The same
// functions in the same order of operations: the state is the same bit for bit.
constexpr int kSplitCells = kBlock / 4;
static_assert(kSplitCells == 32, "one warp per part of a cell's stage");

inline dim3 split_grid(long long ncells) { return dim3((unsigned)((ncells + kSplitCells - 1) / kSplitCells)); }

template <int EOS, bool SHEAR, bool BULK, bool STAGE2, bool MIXED>
__global__ void __launch_bounds__(kBlock, GVH_MIN_BLOCKS) kt_stage_split_kernel(const StageArgs a) {
  constexpr int NQ = NComp<SHEAR, BULK>::value;
  const int lane = threadIdx.x % kSplitCells;
  const int part = threadIdx.x / kSplitCells;  // 0: source and finish; 1..3: axis part - 1
  const long long id = (long long)blockIdx.x * kSplitCells + lane;
  extern __shared__ double gvh_stage_smem[];
  double *out = gvh_stage_smem + threadIdx.x;
  double *cache = gvh_stage_smem + NQ * kBlock + threadIdx.x;
  double speed = 0.0;
  bool live = id < a.ncells;
  int i = 0, j = 0, k = 0;
  long long s = 0;
  if (live) {
    i = (int)(id % a.nx);
    j = (int)((id / a.nx) % a.ny);
    k = (int)(id / ((long long)a.nx * a.ny));
    s = i + a.sy * j + a.sz * k;
#ifdef GVH_BOUNDS_CHECK
    if (!cell_stencil_ok(a, i, j, k)) {
      if (part == 0) atomicOr(a.status, STATUS_BOUNDS);
      live = false;
    }
#endif
  }
  unsigned status = 0;
  double ePrev = 0.0;
  if (live) {
    ePrev = a.e[s];
    double uc[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) uc[m] = __ldg(a.uin + m * a.cs + s);
    if (part == 0) {
      stage_source<EOS, SHEAR, BULK, MIXED, kBlock>(a, s, i, j, k, ePrev, uc, out);
    } else {
      const int axis = part - 1;
      const int idx = axis == 0 ? i : axis == 1 ? j : k;
      const int n_axis = axis == 0 ? a.nx : axis == 1 ? a.ny : a.nz;
      // the FP64 kernel's one-cell axes are skipped, as in kt_stage_kernel
      if (MIXED || n_axis > 1) {
        const int stride = axis == 0 ? 1 : axis == 1 ? (int)a.sy : (int)a.sz;
        const double inv_spacing = axis == 0 ? a.inv_dx : axis == 1 ? a.inv_dy : a.inv_dz;
        const GuessEos g0 = guess_eos<EOS>(ePrev);
        const double as = axis_update<EOS, SHEAR, BULK, MIXED, true>(a, (int)s, axis, idx, n_axis, stride,
                                                                     inv_spacing, g0, uc, out, cache, status);
        speed = n_axis > 1 ? as * inv_spacing : 0.0;
        if (status) atomicOr(a.status, status);
      }
    }
  }
  __syncthreads();
  if (live && part == 0) {
#pragma unroll 1
    for (int axis = 0; axis < 3; ++axis) {
      const int n_axis = axis == 0 ? a.nx : axis == 1 ? a.ny : a.nz;
      if (!MIXED && n_axis == 1) continue;
      const double *inc = gvh_stage_smem + (axis + 1) * kSplitCells + lane;
#pragma unroll
      for (int n = 0; n < NQ; ++n) out[n * kBlock] += inc[n * kBlock] * a.dt;
    }
    stage_finish<EOS, SHEAR, BULK, STAGE2, kBlock>(a, s, out, guess_eos<EOS>(ePrev), status);
  }
  if (!STAGE2 && a.speed_max) {
    unsigned long long b = (unsigned long long)__double_as_longlong(fmax(speed, 0.0));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if ((threadIdx.x & 31) == 0) atomicMax(a.speed_max, b);
  }
}

// Raises a stage kernel's dynamic shared-memory limit to what it is launched with. A kernel
// template instantiated in several translation units has one copy in each, so each file that
// launches one calls this for its own copies (host only; done once per device, before any
// stream capture).
template <class Kernel>
inline cudaError_t allow_stage_smem(Kernel *kernel, size_t bytes) {
  return cudaFuncSetAttribute(reinterpret_cast<const void *>(kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

// All 24 kt_stage_kernel instantiations of the calling translation unit.
inline cudaError_t allow_all_stage_kernels() {
  cudaError_t e = cudaSuccess;
#define GVH_ALLOW(EOS_, SH, BU)                                                                                \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_kernel<EOS_, SH, BU, false, false>, stage_smem_bytes<SH, BU>()); \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_kernel<EOS_, SH, BU, true, false>, stage_smem_bytes<SH, BU>());  \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_kernel<EOS_, SH, BU, false, true>, stage_smem_bytes<SH, BU>());  \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_kernel<EOS_, SH, BU, true, true>, stage_smem_bytes<SH, BU>());
  GVH_ALLOW(EOS_QCD, false, false) GVH_ALLOW(EOS_QCD, true, false) GVH_ALLOW(EOS_QCD, true, true)
  GVH_ALLOW(EOS_CONFORMAL, false, false) GVH_ALLOW(EOS_CONFORMAL, true, false) GVH_ALLOW(EOS_CONFORMAL, true, true)
#undef GVH_ALLOW
  return e;
}

// All 24 kt_stage_split_kernel instantiations of the calling translation unit, as
// allow_all_stage_kernels (only the single-lattice handle launches them).
inline cudaError_t allow_all_split_kernels() {
  cudaError_t e = cudaSuccess;
#define GVH_ALLOW(EOS_, SH, BU)                                                                                      \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_split_kernel<EOS_, SH, BU, false, false>, stage_smem_bytes<SH, BU>()); \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_split_kernel<EOS_, SH, BU, true, false>, stage_smem_bytes<SH, BU>());  \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_split_kernel<EOS_, SH, BU, false, true>, stage_smem_bytes<SH, BU>());  \
  if (e == cudaSuccess) e = allow_stage_smem(kt_stage_split_kernel<EOS_, SH, BU, true, true>, stage_smem_bytes<SH, BU>());
  GVH_ALLOW(EOS_QCD, false, false) GVH_ALLOW(EOS_QCD, true, false) GVH_ALLOW(EOS_QCD, true, true)
  GVH_ALLOW(EOS_CONFORMAL, false, false) GVH_ALLOW(EOS_CONFORMAL, true, false) GVH_ALLOW(EOS_CONFORMAL, true, true)
#undef GVH_ALLOW
  return e;
}

}  // namespace gvh
