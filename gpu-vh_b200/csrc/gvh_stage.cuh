// gvh_stage.cuh -- the fused KT stage kernel.
//
// One launch is one RK substep of twoStepRungeKutta (FullyDiscreteKurganovTadmorScheme.cu
// :109-139) over every interior cell. Per cell it does what the reference spreads over
// eulerStepKernelSource_1D + X_1D + Y_1D + Z_1D (EulerStep.cu:946-1277), the convex
// combination (FullyDiscreteKurganovTadmorScheme.cu:60-104, stage 2 only),
// setInferredVariablesKernel (EnergyMomentumTensor.cu:110-154) and
// regulateDissipativeCurrents (RegulateDissipativeCurrents.cu:15-134), keeping everything
// in registers and writing each output once. setGhostCells (GhostCells.cu:15-144) is
// replaced by clamped neighbour indices: a zero-gradient ghost always equals the nearest
// interior cell, and the stencils are axis-aligned, so clamping reads the same values.
//
// Layout in HBM (interior only, no ghosts): component-major SoA, cell index
// s = i + sy*j + sz*k, component c at c*cs + s.
#pragma once

#include <stdint.h>

#include "gvh_physics.cuh"
#include "gvh_sources.cuh"

namespace gvh {

struct StageArgs {
  int nx, ny, nz;
  long long sy, sz, cs;   // strides: row, plane, component
  long long ncells;       // nx*ny*nz
  double dx, dy, dz;      // lattice spacings
  double dt;              // lattice time step (d_dt) used in the Euler update
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
};

template <bool SHEAR, bool BULK>
struct NComp {
  static constexpr int value = 4 + (SHEAR ? 10 : 0) + (BULK ? 1 : 0);
};

// Half-cell states of one face from the 4 cells around it (HalfSiteExtrapolation.cu:15-30):
// qL = q0 + D(q-1,q0,q1)/2, qR = q1 - D(q0,q1,q2)/2.
__device__ __forceinline__ void face_states(double theta, double qa, double qb, double qc, double qd, double &qL,
                                            double &qR) {
  qL = qb + limited_slope(theta, qa, qb, qc) / 2;
  qR = qc - limited_slope(theta, qb, qc, qd) / 2;
}

// KT numerical flux at one face (SemiDiscreteKurganovTadmorScheme.cu:15-57):
// H = (F(qR) + F(qL) - a (qR - qL)) / 2, F = q v^axis, a = max |v^axis| over both sides.
// off[0..3] are the (clamped) offsets of the 4 cells around the face; H is combined into
// acc with sign `sgn` (-1 for the face at i+1/2, +1 for i-1/2).
template <int EOS, int NQ, int AXIS>
__device__ __forceinline__ void face_flux(const StageArgs &a, long long s, const long long off[4], double ePrev,
                                          double t, double sgn, double acc[NQ], unsigned &status) {
  double qL[NQ], qR[NQ];
#pragma unroll
  for (int n = 0; n < NQ; ++n) {
    const double *c = a.qin + n * a.cs + s;
    face_states(a.theta, __ldg(c + off[0]), __ldg(c + off[1]), __ldg(c + off[2]), __ldg(c + off[3]), qL[n], qR[n]);
  }
  const bool shear = NQ >= 14;
  const bool bulk = NQ == 15;
  Prim R = inferred<EOS>(t, qR[0], qR[1], qR[2], qR[3], shear ? qR[4] : 0.0, shear ? qR[5] : 0.0,
                         shear ? qR[6] : 0.0, shear ? qR[7] : 0.0, bulk ? qR[NQ - 1] : 0.0, ePrev, status);
  Prim L = inferred<EOS>(t, qL[0], qL[1], qL[2], qL[3], shear ? qL[4] : 0.0, shear ? qL[5] : 0.0,
                         shear ? qL[6] : 0.0, shear ? qL[7] : 0.0, bulk ? qL[NQ - 1] : 0.0, ePrev, status);
  const double vR = AXIS == 0 ? R.ux : AXIS == 1 ? R.uy : R.un;
  const double vL = AXIS == 0 ? L.ux : AXIS == 1 ? L.uy : L.un;
  const double sp = fmax(fabs(vL / L.ut), fabs(vR / R.ut));
#pragma unroll
  for (int n = 0; n < NQ; ++n) {
    double FqR = vR * qR[n] / R.ut;
    double FqL = vL * qL[n] / L.ut;
    double h = (FqR + FqL - sp * (qR[n] - qL[n])) / 2;
    acc[n] = (sgn < 0) ? -h : acc[n] + h;
  }
}

// One axis of the Euler update (EulerStep.cu:1011-1277, one of X/Y/Z):
// out += dt * ( (H(i-1/2) - H(i+1/2)) / d + S_axis ), S_axis from SourceTerms.cu:443-567.
template <int EOS, bool SHEAR, bool BULK, int AXIS>
__device__ __forceinline__ void axis_update(const StageArgs &a, long long s, int idx, int n_axis, long long stride,
                                            double ePrev, const double *uc, double out[NComp<SHEAR, BULK>::value],
                                            unsigned &status) {
  constexpr int NQ = NComp<SHEAR, BULK>::value;
  const long long m2 = (long long)(max(idx - 2, 0) - idx) * stride;
  const long long m1 = (long long)(max(idx - 1, 0) - idx) * stride;
  const long long p1 = (long long)(min(idx + 1, n_axis - 1) - idx) * stride;
  const long long p2 = (long long)(min(idx + 2, n_axis - 1) - idx) * stride;
  const double d = AXIS == 0 ? a.dx : AXIS == 1 ? a.dy : a.dz;
  double res[NQ];
  {
    const long long off[4] = {m1, 0, p1, p2};
    face_flux<EOS, NQ, AXIS>(a, s, off, ePrev, a.t_euler, -1.0, res, status);
  }
  {
    const long long off[4] = {m2, m1, 0, p1};
    face_flux<EOS, NQ, AXIS>(a, s, off, ePrev, a.t_euler, +1.0, res, status);
  }
#pragma unroll
  for (int n = 0; n < NQ; ++n) res[n] /= d;
  if (SHEAR) {
    // centred differences of pi^{mu nu} (and Pi) along this axis
    const double fac = 1 / d / 2;
    auto der = [&](int c) {
      const double *q = a.qin + c * a.cs + s;
      return (__ldg(q + p1) - __ldg(q + m1)) * fac;
    };
    const double ut = uc[0];
    double S0, S1, S2, S3;
    if (AXIS == 0) {
      double vx = uc[1] / ut;
      double dpitt = der(4), dpitx = der(5), dpity = der(6), dpitn = der(7), dpixx = der(8), dpixy = der(9),
             dpixn = der(10);
      if (!BULK) {
        S0 = dpitt * vx - dpitx;
        S1 = dpitx * vx - dpixx;
      } else {
        double dPi = der(14);
        S0 = dpitt * vx - dpitx - vx * dPi;
        S1 = dpitx * vx - dpixx - dPi;
      }
      S2 = dpity * vx - dpixy;
      S3 = dpitn * vx - dpixn;
    } else if (AXIS == 1) {
      double vy = uc[2] / ut;
      double dpitt = der(4), dpitx = der(5), dpity = der(6), dpitn = der(7), dpixy = der(9), dpiyy = der(11),
             dpiyn = der(12);
      if (!BULK) {
        S0 = dpitt * vy - dpity;
        S2 = dpity * vy - dpiyy;
      } else {
        double dPi = der(14);
        S0 = dpitt * vy - dpity - vy * dPi;
        S2 = dpity * vy - dpiyy - dPi;
      }
      S1 = dpitx * vy - dpixy;
      S3 = dpitn * vy - dpiyn;
    } else {
      double vn = uc[3] / ut;
      double dpitt = der(4), dpitx = der(5), dpity = der(6), dpitn = der(7), dpixn = der(10), dpiyn = der(12),
             dpinn = der(13);
      if (!BULK) {
        S0 = dpitt * vn - dpitn;
        S3 = dpitn * vn - dpinn;
      } else {
        double dPi = der(14);
        S0 = dpitt * vn - dpitn - vn * dPi;
        S3 = dpitn * vn - dpinn - dPi / (a.t_euler * a.t_euler);
      }
      S1 = dpitx * vn - dpixn;
      S2 = dpity * vn - dpiyn;
    }
    res[0] += S0;
    res[1] += S1;
    res[2] += S2;
    res[3] += S3;
  }
#pragma unroll
  for (int n = 0; n < NQ; ++n) out[n] += res[n] * a.dt;
}

template <int EOS, bool SHEAR, bool BULK, bool STAGE2>
__global__ void __launch_bounds__(128) kt_stage_kernel(const StageArgs a) {
  constexpr int NQ = NComp<SHEAR, BULK>::value;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= a.ncells) return;
  const int i = (int)(id % a.nx);
  const int j = (int)((id / a.nx) % a.ny);
  const int k = (int)(id / ((long long)a.nx * a.ny));
  const long long s = i + a.sy * j + a.sz * k;
  unsigned status = 0;

  // ---- centre state -------------------------------------------------------------------
  double q[NQ];
#pragma unroll
  for (int n = 0; n < NQ; ++n) q[n] = __ldg(a.qin + n * a.cs + s);
  const double ePrev = a.e[s];
  const double pc = __ldg(a.pin + s);
  double uc[4], up[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    uc[m] = __ldg(a.uin + m * a.cs + s);
    up[m] = a.uprev[m * a.cs + s];
  }

  // ---- source term: out = q + dt * S (EulerStep.cu:946-1009, SourceTerms.cu:569-755) ---
  double out[NQ];
  {
    const double th = a.theta;
    const long long xm = (i > 0) ? -1 : 0, xp = (i < a.nx - 1) ? 1 : 0;
    const long long ym = (j > 0) ? -a.sy : 0, yp = (j < a.ny - 1) ? a.sy : 0;
    const long long zm = (k > 0) ? -a.sz : 0, zp = (k < a.nz - 1) ? a.sz : 0;
    CellFlow f;
    f.ut = uc[0]; f.ux = uc[1]; f.uy = uc[2]; f.un = uc[3];
    f.utp = up[0]; f.uxp = up[1]; f.uyp = up[2]; f.unp = up[3];
    double du[3][4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const double *u = a.uin + m * a.cs + s;
      du[0][m] = limited_slope(th, __ldg(u + xm), uc[m], __ldg(u + xp)) / a.dx;
      du[1][m] = limited_slope(th, __ldg(u + ym), uc[m], __ldg(u + yp)) / a.dy;
      du[2][m] = limited_slope(th, __ldg(u + zm), uc[m], __ldg(u + zp)) / a.dz;
    }
    f.dxut = du[0][0]; f.dyut = du[1][0]; f.dnut = du[2][0];
    f.dxux = du[0][1]; f.dyux = du[1][1]; f.dnux = du[2][1];
    f.dxuy = du[0][2]; f.dyuy = du[1][2]; f.dnuy = du[2][2];
    f.dxun = du[0][3]; f.dyun = du[1][3]; f.dnun = du[2][3];
    const double *p = a.pin + s;
    const double dxp = limited_slope(th, __ldg(p + xm), pc, __ldg(p + xp)) / a.dx;
    const double dyp = limited_slope(th, __ldg(p + ym), pc, __ldg(p + yp)) / a.dy;
    const double dnp = limited_slope(th, __ldg(p + zm), pc, __ldg(p + zp)) / a.dz;

    const double t = a.t_euler;
    const double Pi = BULK ? q[NQ - 1] : 0.0;
    const double pitt = SHEAR ? q[4] : 0.0, pitx = SHEAR ? q[5] : 0.0, pity = SHEAR ? q[6] : 0.0;
    const double pitn = SHEAR ? q[7] : 0.0, pinn = SHEAR ? q[13] : 0.0;
    const double ut = uc[0], ux = uc[1], uy = uc[2], un = uc[3];
    // Tnn (EnergyMomentumTensor.cu:205-207) with p + Pi
    const double pP = pc + Pi;
    const double tnn = (ePrev + pP) * un * un + pP / t / t + pinn;
    const double vx = ux / ut, vy = uy / ut, vn = un / ut;
    const double dxvx = (f.dxux - vx * f.dxut) / ut;
    const double dyvy = (f.dyuy - vy * f.dyut) / ut;
    const double dnvn = (f.dnun - vn * f.dnut) / ut;
    const double dkvk = dxvx + dyvy + dnvn;
    double S[NQ];
    S[0] = -(q[0] / t + t * tnn) + dkvk * (pitt - pc - Pi) - vx * dxp - vy * dyp - vn * dnp;
    S[1] = -q[1] / t - dxp + dkvk * pitx;
    S[2] = -q[2] / t - dyp + dkvk * pity;
    S[3] = -3 * q[3] / t - dnp / (t * t) + dkvk * pitn;
    if (SHEAR) {
      Shear pi{q[4], q[5], q[6], q[7], q[8], q[9], q[10], q[11], q[12], q[13]};
      double rhs[11];
      pimunu_rhs<EOS, BULK>(rhs, t, a.dt, a.etabar, ePrev, pc, f, pi, Pi, dkvk);
#pragma unroll
      for (int n = 4; n < NQ; ++n) S[n] = rhs[n - 4];
    }
#pragma unroll
    for (int n = 0; n < NQ; ++n) out[n] = q[n] + a.dt * S[n];
  }

  // ---- flux divergence along x, y, eta (EulerStep.cu:1011-1277) -------------------------
  axis_update<EOS, SHEAR, BULK, 0>(a, s, i, a.nx, 1, ePrev, uc, out, status);
  axis_update<EOS, SHEAR, BULK, 1>(a, s, j, a.ny, a.sy, ePrev, uc, out, status);
  axis_update<EOS, SHEAR, BULK, 2>(a, s, k, a.nz, a.sz, ePrev, uc, out, status);

  // ---- Heun combination Q = (Q + q^n)/2 (FullyDiscreteKurganovTadmorScheme.cu:60-104) ---
  if (STAGE2) {
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
      out[n] += a.qn[n * a.cs + s];
      out[n] /= 2;
    }
  }

  // ---- primitive recovery at the new time (EnergyMomentumTensor.cu:110-154) ---------------
  const double tn = a.t_after;
  Prim pr = inferred<EOS>(tn, out[0], out[1], out[2], out[3], SHEAR ? out[4] : 0.0, SHEAR ? out[5] : 0.0,
                          SHEAR ? out[6] : 0.0, SHEAR ? out[7] : 0.0, BULK ? out[NQ - 1] : 0.0, ePrev, status);

  // ---- regulation (RegulateDissipativeCurrents.cu:15-134) ----------------------------------
  if (SHEAR) {
    const double pitt = out[4], pitx = out[5], pity = out[6], pitn = out[7], pixx = out[8], pixy = out[9];
    const double pixn = out[10], piyy = out[11], piyn = out[12], pinn = out[13];
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
    double den = xi0 * rhomax * spipi;
    double rho = fmax(a1, fmax(pimumu / den, fmax(piu0 / den, fmax(piu1 / den, fmax(piu2 / den, piu3 / den)))));
    double facShear = tanh(rho) / rho;
    if (fabs(rho) < 1.e-7) facShear = 1.0;
    // The reference reads Pi as 0 here (its `#ifdef Pi` is never true), so rho_bulk = 0
    // and the bulk factor is always 1 (RegulateDissipativeCurrents.cu:54-58, 106-109).
    if (pr.e > a.e_reg) facShear = 1.0;
#pragma unroll
    for (int n = 4; n < 14; ++n) out[n] *= facShear;
  }

  // ---- write ----------------------------------------------------------------------------
#pragma unroll
  for (int n = 0; n < NQ; ++n) a.qout[n * a.cs + s] = out[n];
  a.e[s] = pr.e;
  a.pout[s] = pr.p;
  a.uout[s] = pr.ut;
  a.uout[a.cs + s] = pr.ux;
  a.uout[2 * a.cs + s] = pr.uy;
  a.uout[3 * a.cs + s] = pr.un;
  if (status) atomicOr(a.status, status);
}

}  // namespace gvh
