// gvh_validity.cuh -- the validity diagnostics of the fluid-dynamic description
// (checkValidityKernel, HydrodynamicValidity.cu:18-226): inverse Reynolds and Knudsen
// numbers from the velocity shear, vorticity and the second-order terms of the pi^{mu nu}
// and Pi equations. Diagnostics only: nothing in the step reads them. The reference launches
// the kernel at the end of every twoStepRungeKutta (FullyDiscreteKurganovTadmorScheme.cu:137);
// here it runs after stage 2 only when the caller asked for the diagnostics.
#pragma once

#include "gvh_physics.cuh"
#include "gvh_stage.cuh"

namespace gvh {

struct ValidityArgs {
  int nx, ny, nz;
  long long sy, sz, cs, ncells;
  double dx, dy, dz, dt, etabar;
  double t;               // t + dt, the time of the new level
  const double *e, *p;    // new level
  const double *u;        // new u^mu (4 components)
  const double *up;       // u^mu one step earlier
  double *diag;           // kValidityFields outputs, then the saved q^n pi^{mu nu}, Pi
};

template <int EOS, bool SHEAR, bool BULK>
__global__ void validity_kernel(const ValidityArgs v) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= v.ncells) return;
  const int i = (int)(id % v.nx), j = (int)((id / v.nx) % v.ny), k = (int)(id / ((long long)v.nx * v.ny));
  const long long s = id;
  // zero-gradient ghosts: the neighbour across the lattice edge is the cell itself
  const long long xm = i > 0 ? -1 : 0, xp = i < v.nx - 1 ? 1 : 0;
  const long long ym = j > 0 ? -v.sy : 0, yp = j < v.ny - 1 ? v.sy : 0;
  const long long zm = k > 0 ? -v.sz : 0, zp = k < v.nz - 1 ? v.sz : 0;
  const double *utv = v.u, *uxv = v.u + v.cs, *uyv = v.u + 2 * v.cs, *unv = v.u + 3 * v.cs;
  const double e_s = v.e[s], p_s = v.p[s];
  const double ut = utv[s], ux = uxv[s], uy = uyv[s], un = unv[s];
  const double utp = v.up[s], uxp = v.up[v.cs + s], uyp = v.up[2 * v.cs + s], unp = v.up[3 * v.cs + s];
  const double t = v.t;

  // central differences of u^mu (HydrodynamicValidity.cu:46-67)
  const double facX = 1 / v.dx / 2, facY = 1 / v.dy / 2, facZ = 1 / v.dz / 2;
  const double dxut = (utv[s + xp] - utv[s + xm]) * facX, dxux = (uxv[s + xp] - uxv[s + xm]) * facX;
  const double dxuy = (uyv[s + xp] - uyv[s + xm]) * facX, dxun = (unv[s + xp] - unv[s + xm]) * facX;
  const double dyut = (utv[s + yp] - utv[s + ym]) * facY, dyux = (uxv[s + yp] - uxv[s + ym]) * facY;
  const double dyuy = (uyv[s + yp] - uyv[s + ym]) * facY, dyun = (unv[s + yp] - unv[s + ym]) * facY;
  const double dnut = (utv[s + zp] - utv[s + zm]) * facZ, dnux = (uxv[s + zp] - uxv[s + zm]) * facZ;
  const double dnuy = (uyv[s + zp] - uyv[s + zm]) * facZ, dnun = (unv[s + zp] - unv[s + zm]) * facZ;

  const double ut2 = ut * ut, un2 = un * un, t2 = t * t, t3 = t * t2;
  // transport coefficients (HydrodynamicValidity.cu:74-81)
  const double T = temperature<EOS>(e_s);
  const double cs2 = sound_speed2<EOS>(e_s);
  const double a = kF033 - cs2;
  const double a2 = a * a;
  const double lambda_Pipi = kF16 * a;
  const double zetabar = bulk_zeta_over_s(T);
  const double tauPiInv = 15 * a2 * (T / zetabar);

  const double dtut = (ut - utp) / v.dt, dtux = (ux - uxp) / v.dt, dtuy = (uy - uyp) / v.dt, dtun = (un - unp) / v.dt;
  // covariant derivatives, expansion rate (HydrodynamicValidity.cu:89-100)
  const double Dut = ut * dtut + ux * dxut + uy * dyut + un * dnut + t * un * un;
  const double dut = Dut - t * un * un;
  const double dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
  const double duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
  const double dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
  const double Dun = -t2 * dun - 2 * t * ut * un;
  const double theta = ut / t + dtut + dxux + dyuy + dnun;

  double *out = v.diag;
  const long long cs = v.cs;
  if (SHEAR) {
    // velocity shear sigma^{mu nu} (HydrodynamicValidity.cu:102-113)
    const double theta3 = theta / 3;
    const double stt = -t * ut * un2 + (dtut - ut * dut) + (ut2 - 1) * theta3;
    const double stx = -(t * un2 * ux) / 2 + (dtux - dxut) / 2 - (ux * dut + ut * dux) / 2 + ut * ux * theta3;
    const double sty = -(t * un2 * uy) / 2 + (dtuy - dyut) / 2 - (uy * dut + ut * duy) / 2 + ut * uy * theta3;
    const double stn = -un * (2 * ut2 + t2 * un2) / (2 * t) + (dtun - dnut / t2) / 2 - (un * dut + ut * dun) / 2 +
                       ut * un * theta3;
    const double sxx = -(dxux + ux * dux) + (1 + ux * ux) * theta3;
    const double sxy = -(dxuy + dyux) / 2 - (uy * dux + ux * duy) / 2 + ux * uy * theta3;
    const double sxn = -ut * ux * un / t - (dxun + dnux / t2) / 2 - (un * dux + ux * dun) / 2 + ux * un * theta3;
    const double syy = -(dyuy + uy * duy) + (1 + uy * uy) * theta3;
    const double syn = -ut * uy * un / t - (dyun + dnuy / t2) / 2 - (un * duy + uy * dun) / 2 + uy * un * theta3;
    const double snn = -ut * (1 + 2 * t2 * un2) / t3 - dnun / t2 - un * dun + (1 / t2 + un2) * theta3;
    // vorticity omega^{mu nu} (HydrodynamicValidity.cu:115-129)
    const double wtx = (dtux + dxut) / 2 + (ux * dut - ut * dux) / 2 + t * un2 * ux / 2;
    const double wty = (dtuy + dyut) / 2 + (uy * dut - ut * duy) / 2 + t * un2 * uy / 2;
    const double wtn = (t2 * dtun + 2 * t * un + dnut) / 2 + (t2 * un * dut - ut * Dun) + t3 * un * un2 / 2;
    const double wxy = (dyux - dxuy) / 2 + (uy * dux - ux * duy) / 2;
    const double wxn = (dnux - t2 * dxun) / 2 + (t2 * un * dux - ux * Dun) / 2;
    const double wyn = (dnuy - t2 * dyun) / 2 + (t2 * un * duy - uy * Dun) / 2;
    const double wxt = wtx, wyt = wty, wnt = wtn / t2, wyx = -wxy, wnx = -wxn / t2, wny = -wyn / t2;
    // pi^{mu nu} and Pi of the state before the step, saved by stage 2
    const double *sv = out + kValidityFields * cs + s;
    const double pitt = sv[0], pitx = sv[cs], pity = sv[2 * cs], pitn = sv[3 * cs], pixx = sv[4 * cs];
    const double pixy = sv[5 * cs], pixn = sv[6 * cs], piyy = sv[7 * cs], piyn = sv[8 * cs], pinn = sv[9 * cs];
    const double Pi = BULK ? sv[10 * cs] : 0.0;
    // I2 = theta pi, I3 (vorticity), I4 (shear) terms (HydrodynamicValidity.cu:149-195)
    const double I2tt = theta * pitt, I2tx = theta * pitx, I2ty = theta * pity, I2tn = theta * pitn;
    const double I2xx = theta * pixx, I2xy = theta * pixy, I2xn = theta * pixn, I2yy = theta * piyy;
    const double I2yn = theta * piyn, I2nn = theta * pinn;
    const double I3tt = 2 * (pitx * wtx + pity * wty + pitn * wtn);
    const double I3tx = pitt * wxt + pity * wxy + pitn * wxn + pixx * wtx + pixy * wty + pixn * wtn;
    const double I3ty = pitt * wyt + pitx * wyx + pitn * wyn + pixy * wtx + piyy * wty + piyn * wtn;
    const double I3tn = pitt * wnt + pitx * wnx + pity * wny + pixn * wtx + piyn * wty + pinn * wtn;
    const double I3xx = 2 * (pitx * wxt + pixy * wxy + pixn * wxn);
    const double I3xy = pitx * wyt + pity * wxt + pixx * wyx + piyy * wxy + pixn * wyn + piyn * wxn;
    const double I3xn = pitx * wnt + pitn * wxt + pixx * wnx + pixy * wny + piyn * wxy + pinn * wxn;
    const double I3yy = 2 * (pity * wyt + pixy * wyx + piyn * wyn);
    const double I3yn = pity * wnt + pitn * wyt + pixy * wnx + pixn * wyx + piyy * wny + pinn * wyn;
    const double I3nn = 2 * (pitn * wnt + pixn * wnx + piyn * wny);
    const double ux2 = ux * ux, uy2 = uy * uy;
    const double ps = pitt * stt - 2 * pitx * stx - 2 * pity * sty + pixx * sxx + 2 * pixy * sxy + piyy * syy -
                      2 * pitn * stn * t2 + 2 * pixn * sxn * t2 + 2 * piyn * syn * t2 + pinn * snn * t2 * t2;
    const double ps3 = ps / 3;
    const double I4tt = (pitt * stt - pitx * stx - pity * sty - t2 * pitn * stn) - (1 - ut2) * ps3;
    const double I4tx = (pitt * stx + pitx * stt) / 2 - (pitx * sxx + pixx * stx) / 2 - (pity * sxy + pixy * sty) / 2 -
                        t2 * (pitn * sxn + pixn * stn) / 2 + (ut * ux) * ps3;
    const double I4ty = (pitt * sty + pity * stt) / 2 - (pitx * sxy + pixy * stx) / 2 - (pity * syy + piyy * sty) / 2 -
                        t2 * (pitn * syn + piyn * stn) / 2 + (ut * uy) * ps3;
    const double I4tn = (pitt * stn + pitn * stt) / 2 - (pitx * sxn + pixn * stx) / 2 - (pity * syn + piyn * sty) / 2 -
                        t2 * (pitn * snn + pinn * stn) / 2 + (ut * un) * ps3;
    const double I4xx = (pitx * stx - pixx * sxx - pixy * sxy - t2 * pixn * sxn) + (1 + ux2) * ps3;
    const double I4xy = (pitx * sty + pity * stx) / 2 - (pixx * sxy + pixy * sxx) / 2 - (pixy * syy + piyy * sxy) / 2 -
                        t2 * (pixn * syn + piyn * sxn) / 2 + (ux * uy) * ps3;
    const double I4xn = (pitx * stn + pitn * stx) / 2 - (pixx * sxn + pixn * sxx) / 2 - (pixy * syn + piyn * sxy) / 2 -
                        t2 * (pixn * snn + pinn * sxn) / 2 + (ux * un) * ps3;
    const double I4yy = (pity * sty - pixy * sxy - piyy * syy - t2 * piyn * syn) + (1 + uy2) * ps3;
    const double I4yn = (pity * stn + pitn * sty) / 2 - (pixy * sxn + pixn * sxy) / 2 - (piyy * syn + piyn * syy) / 2 -
                        t2 * (piyn * snn + pinn * syn) / 2 + (uy * un) * ps3;
    const double I4nn = (pitn * stn - pixn * sxn - piyn * syn - t2 * pinn * snn) + (1 / t2 + un2) * ps3;
    const double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy +
                        piyy * piyy - 2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 +
                        pinn * pinn * t2 * t2;
    const double ss = stt * stt - 2 * stx * stx - 2 * sty * sty + sxx * sxx + 2 * sxy * sxy + syy * syy -
                      2 * stn * stn * t2 + 2 * sxn * sxn * t2 + 2 * syn * syn * t2 + snn * snn * t2 * t2;
    // second-order terms J^{mu nu}, J (HydrodynamicValidity.cu:202-214)
    const double Jtt = kDeltaPiPi * I2tt - I3tt + kTauPiPi * I4tt - kLambdaPiBulk * Pi * stt;
    const double Jtx = kDeltaPiPi * I2tx - I3tx + kTauPiPi * I4tx - kLambdaPiBulk * Pi * stx;
    const double Jty = kDeltaPiPi * I2ty - I3ty + kTauPiPi * I4ty - kLambdaPiBulk * Pi * sty;
    const double Jtn = kDeltaPiPi * I2tn - I3tn + kTauPiPi * I4tn - kLambdaPiBulk * Pi * stn;
    const double Jxx = kDeltaPiPi * I2xx - I3xx + kTauPiPi * I4xx - kLambdaPiBulk * Pi * sxx;
    const double Jxy = kDeltaPiPi * I2xy - I3xy + kTauPiPi * I4xy - kLambdaPiBulk * Pi * sxy;
    const double Jxn = kDeltaPiPi * I2xn - I3xn + kTauPiPi * I4xn - kLambdaPiBulk * Pi * sxn;
    const double Jyy = kDeltaPiPi * I2yy - I3yy + kTauPiPi * I4yy - kLambdaPiBulk * Pi * syy;
    const double Jyn = kDeltaPiPi * I2yn - I3yn + kTauPiPi * I4yn - kLambdaPiBulk * Pi * syn;
    const double Jnn = kDeltaPiPi * I2nn - I3nn + kTauPiPi * I4nn - kLambdaPiBulk * Pi * snn;
    const double J = -kDeltaBulk * Pi * theta + lambda_Pipi * ps;
    const double JJ = Jtt * Jtt - 2 * Jtx * Jtx - 2 * Jty * Jty + Jxx * Jxx + 2 * Jxy * Jxy + Jyy * Jyy -
                      2 * Jtn * Jtn * t2 + 2 * Jxn * Jxn * t2 + 2 * Jyn * Jyn * t2 + Jnn * Jnn * t2 * t2;
    // VALIDITY_DOMAIN: 1 knudsenNumberTaupi, 2 knudsenNumberTauPi, 3 inverseReynoldsNumberPimunu,
    // 5 inverseReynoldsNumberTilde2Pimunu, 6 inverseReynoldsNumberPi, 8 inverseReynoldsNumberTilde2Pi
    // (HydrodynamicValidity.cu:216-221; 4 and 7 are never written by the reference)
    out[3 * cs + s] = sqrt(fabs(pipi)) / p_s;
    out[5 * cs + s] = T / 2 / v.etabar / (e_s + p_s) * sqrt(fabs(JJ / ss));
    out[6 * cs + s] = fabs(Pi) / p_s;
    out[8 * cs + s] = fabs(J / zetabar / theta) * T / (e_s + p_s);
    out[1 * cs + s] = 5 * v.etabar * theta / T;
    out[2 * cs + s] = theta / tauPiInv;
  }
  // 9 taupi, 10 dxux, 11 dyuy, 12 theta (HydrodynamicValidity.cu:225-228)
  out[9 * cs + s] = 5 * v.etabar / T;
  out[10 * cs + s] = dxux;
  out[11 * cs + s] = dyuy;
  out[12 * cs + s] = theta;
}

}  // namespace gvh
