// gvh_sources.cuh -- right-hand sides of the KT step at one cell: the Milne geometric
// source of T^{tau mu} and the relaxation equations of pi^{mu nu} and Pi.
// Reproduces SourceTerms.cu:29-256 (setPimunuSourceTerms) and :569-755 (loadSourceTerms2,
// with USE_APPROX_DERIVATIVE). Operation order follows the reference.
#pragma once

#include "gvh_physics.cuh"

namespace gvh {

// Flow state and limited first derivatives at a cell.
struct CellFlow {
  double ut, ux, uy, un;      // u^mu (current)
  double utp, uxp, uyp, unp;  // u^mu one time step earlier (for d/dtau)
  double dxut, dyut, dnut, dxux, dyux, dnux, dxuy, dyuy, dnuy, dxun, dyun, dnun;
};

struct Shear {
  double tt, tx, ty, tn, xx, xy, xn, yy, yn, nn;
};

// SourceTerms.cu:29-256. rhs[0..9] = d pi^{mu nu}/dtau (pitt..pinn), rhs[10] = dPi/dtau.
template <int EOS, bool BULK>
__device__ __forceinline__ void pimunu_rhs(double *rhs, double t, double dt, double etabar, double e, double p,
                                           const CellFlow &f, const Shear &pi, double Pi, double dkvk) {
  const double ut = f.ut, ux = f.ux, uy = f.uy, un = f.un;
  const double pitt = pi.tt, pitx = pi.tx, pity = pi.ty, pitn = pi.tn, pixx = pi.xx, pixy = pi.xy, pixn = pi.xn;
  const double piyy = pi.yy, piyn = pi.yn, pinn = pi.nn;
  const double dxut = f.dxut, dyut = f.dyut, dnut = f.dnut, dxux = f.dxux, dyux = f.dyux, dnux = f.dnux;
  const double dxuy = f.dxuy, dyuy = f.dyuy, dnuy = f.dnuy, dxun = f.dxun, dyun = f.dyun, dnun = f.dnun;

  double T = temperature<EOS>(e);
  double taupiInv = kF02 * (T / etabar);
  double beta_pi = kF02 * (e + p);

  double ut2 = ut * ut, un2 = un * un, t2 = t * t, t3 = t * t2;
  double dtut = (ut - f.utp) / dt;
  double dtux = (ux - f.uxp) / dt;
  double dtuy = (uy - f.uyp) / dt;
  double dtun = (un - f.unp) / dt;

  double Dut = ut * dtut + ux * dxut + uy * dyut + un * dnut + t * un * un;
  double dut = Dut - t * un * un;
  double dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
  double Dux = -dux;
  double duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
  double Duy = -duy;
  double dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
  double Dun = -t2 * dun - 2.0 * t * ut * un;

  double theta = ut / t + dtut + dxux + dyuy + dnun;
  double theta3 = theta / 3.0;

  // shear tensor sigma^{mu nu}
  double stt = -t * ut * un2 + (dtut - ut * dut) + (ut2 - 1.0) * theta3;
  double stx = -(t * un2 * ux) / 2.0 + (dtux - dxut) / 2.0 - (ux * dut + ut * dux) / 2.0 + ut * ux * theta3;
  double sty = -(t * un2 * uy) / 2.0 + (dtuy - dyut) / 2.0 - (uy * dut + ut * duy) / 2.0 + ut * uy * theta3;
  double stn = -un * (2.0 * ut2 + t2 * un2) / (2.0 * t) + (dtun - dnut / t2) / 2.0 - (un * dut + ut * dun) / 2.0
               + ut * un * theta3;
  double sxx = -(dxux + ux * dux) + (1.0 + ux * ux) * theta3;
  double sxy = -(dxuy + dyux) / 2.0 - (uy * dux + ux * duy) / 2.0 + ux * uy * theta3;
  double sxn = -ut * ux * un / t - (dxun + dnux / t2) / 2.0 - (un * dux + ux * dun) / 2.0 + ux * un * theta3;
  double syy = -(dyuy + uy * duy) + (1.0 + uy * uy) * theta3;
  double syn = -ut * uy * un / t - (dyun + dnuy / t2) / 2.0 - (un * duy + uy * dun) / 2.0 + uy * un * theta3;
  double snn = -ut * (1.0 + 2.0 * t2 * un2) / t3 - dnun / t2 - un * dun + (1.0 / t2 + un2) * theta3;

  // vorticity (SourceTerms.cu:122-136)
  double wtx = (-dtux - dxut + ut * dux - ux * dut - t * un2 * ux) / 2.0;
  double wty = (-dtuy - dyut + ut * duy - uy * dut - t * un2 * uy) / 2.0;
  double wtn = (-t2 * dtun - 2.0 * t * un - dnut - ut * Dun - t2 * un * dut - t3 * un * un2) / 2.0;
  double wxy = (dxuy - dyux + ux * duy - uy * dux) / 2.0;
  double wxn = (t2 * dxun - dnux - ux * Dun - t2 * un * dux) / 2.0;
  double wyn = (t2 * dyun - dnuy - uy * Dun - t2 * un * duy) / 2.0;
  double wxt = wtx, wyt = wty, wnt = wtn / t2, wyx = -wxy, wnx = -wxn / t2, wny = -wyn / t2;

  // I1 (SourceTerms.cu:141-150)
  double I1tt = 2.0 * ut * (pitt * Dut + pitx * Dux + pity * Duy + pitn * Dun);
  double I1tx = (pitt * ux + pitx * ut) * Dut + (pitx * ux + pixx * ut) * Dux + (pity * ux + pixy * ut) * Duy
                + (pitn * ux + pixn * ut) * Dun;
  double I1ty = (pitt * uy + pity * ut) * Dut + (pitx * uy + pixy * ut) * Dux + (pity * uy + piyy * ut) * Duy
                + (pitn * uy + piyn * ut) * Dun;
  double I1tn = (pitt * un + pitn * ut) * Dut + (pitx * un + pixn * ut) * Dux + (pity * un + piyn * ut) * Duy
                + (pitn * un + pinn * ut) * Dun;
  double I1xx = 2.0 * ux * (pitx * Dut + pixx * Dux + pixy * Duy + pixn * Dun);
  double I1xy = (pitx * uy + pity * ux) * Dut + (pixx * uy + pixy * ux) * Dux + (pixy * uy + piyy * ux) * Duy
                + (pixn * uy + piyn * ux) * Dun;
  double I1xn = (pitx * un + pitn * ux) * Dut + (pixx * un + pixn * ux) * Dux + (pixy * un + piyn * ux) * Duy
                + (pixn * un + pinn * ux) * Dun;
  double I1yy = 2.0 * uy * (pity * Dut + pixy * Dux + piyy * Duy + piyn * Dun);
  double I1yn = (pity * un + pitn * uy) * Dut + (pixy * un + pixn * uy) * Dux + (piyy * un + piyn * uy) * Duy
                + (piyn * un + pinn * uy) * Dun;
  double I1nn = 2.0 * un * (pitn * Dut + pixn * Dux + piyn * Duy + pinn * Dun);

  // I3 (SourceTerms.cu:169-178)
  double I3tt = 2.0 * (pitx * wtx + pity * wty + pitn * wtn);
  double I3tx = pitt * wxt + pity * wxy + pitn * wxn + pixx * wtx + pixy * wty + pixn * wtn;
  double I3ty = pitt * wyt + pitx * wyx + pitn * wyn + pixy * wtx + piyy * wty + piyn * wtn;
  double I3tn = pitt * wnt + pitx * wnx + pity * wny + pixn * wtx + piyn * wty + pinn * wtn;
  double I3xx = 2.0 * (pitx * wxt + pixy * wxy + pixn * wxn);
  double I3xy = pitx * wyt + pity * wxt + pixx * wyx + piyy * wxy + pixn * wyn + piyn * wxn;
  double I3xn = pitx * wnt + pitn * wxt + pixx * wnx + pixy * wny + piyn * wxy + pinn * wxn;
  double I3yy = 2.0 * (pity * wyt + pixy * wyx + piyn * wyn);
  double I3yn = pity * wnt + pitn * wyt + pixy * wnx + pixn * wyx + piyy * wny + pinn * wyn;
  double I3nn = 2.0 * (pitn * wnt + pixn * wnx + piyn * wny);

  // I4 (SourceTerms.cu:183-203)
  double ux2 = ux * ux, uy2 = uy * uy;
  double ps = pitt * stt - 2.0 * pitx * stx - 2.0 * pity * sty + pixx * sxx + 2.0 * pixy * sxy + piyy * syy
              - 2.0 * pitn * stn * t2 + 2.0 * pixn * sxn * t2 + 2.0 * piyn * syn * t2 + pinn * snn * t2 * t2;
  double ps3 = ps / 3.0;
  double I4tt = (pitt * stt - pitx * stx - pity * sty - t2 * pitn * stn) - (1 - ut2) * ps3;
  double I4tx = (pitt * stx + pitx * stt) / 2.0 - (pitx * sxx + pixx * stx) / 2.0 - (pity * sxy + pixy * sty) / 2.0
                - t2 * (pitn * sxn + pixn * stn) / 2.0 + (ut * ux) * ps3;
  double I4ty = (pitt * sty + pity * stt) / 2.0 - (pitx * sxy + pixy * stx) / 2.0 - (pity * syy + piyy * sty) / 2.0
                - t2 * (pitn * syn + piyn * stn) / 2.0 + (ut * uy) * ps3;
  double I4tn = (pitt * stn + pitn * stt) / 2.0 - (pitx * sxn + pixn * stx) / 2.0 - (pity * syn + piyn * sty) / 2.0
                - t2 * (pitn * snn + pinn * stn) / 2.0 + (ut * un) * ps3;
  double I4xx = (pitx * stx - pixx * sxx - pixy * sxy - t2 * pixn * sxn) + (1.0 + ux2) * ps3;
  double I4xy = (pitx * sty + pity * stx) / 2.0 - (pixx * sxy + pixy * sxx) / 2.0 - (pixy * syy + piyy * sxy) / 2.0
                - t2 * (pixn * syn + piyn * sxn) / 2.0 + (ux * uy) * ps3;
  double I4xn = (pitx * stn + pitn * stx) / 2.0 - (pixx * sxn + pixn * sxx) / 2.0 - (pixy * syn + piyn * sxy) / 2.0
                - t2 * (pixn * snn + pinn * sxn) / 2.0 + (ux * un) * ps3;
  double I4yy = (pity * sty - pixy * sxy - piyy * syy - t2 * piyn * syn) + (1.0 + uy2) * ps3;
  double I4yn = (pity * stn + pitn * sty) / 2.0 - (pixy * sxn + pixn * sxy) / 2.0 - (piyy * syn + piyn * syy) / 2.0
                - t2 * (piyn * snn + pinn * syn) / 2.0 + (uy * un) * ps3;
  double I4nn = (pitn * stn - pixn * sxn - piyn * syn - t2 * pinn * snn) + (1.0 / t2 + un2) * ps3;

  // I = I1 + delta I2 - I3 + tau I4 - lambda Pi sigma (SourceTerms.cu:209-218); I2 = theta pi
  double Itt = I1tt + kDeltaPiPi * (theta * pitt) - I3tt + kTauPiPi * I4tt - kLambdaPiBulk * Pi * stt;
  double Itx = I1tx + kDeltaPiPi * (theta * pitx) - I3tx + kTauPiPi * I4tx - kLambdaPiBulk * Pi * stx;
  double Ity = I1ty + kDeltaPiPi * (theta * pity) - I3ty + kTauPiPi * I4ty - kLambdaPiBulk * Pi * sty;
  double Itn = I1tn + kDeltaPiPi * (theta * pitn) - I3tn + kTauPiPi * I4tn - kLambdaPiBulk * Pi * stn;
  double Ixx = I1xx + kDeltaPiPi * (theta * pixx) - I3xx + kTauPiPi * I4xx - kLambdaPiBulk * Pi * sxx;
  double Ixy = I1xy + kDeltaPiPi * (theta * pixy) - I3xy + kTauPiPi * I4xy - kLambdaPiBulk * Pi * sxy;
  double Ixn = I1xn + kDeltaPiPi * (theta * pixn) - I3xn + kTauPiPi * I4xn - kLambdaPiBulk * Pi * sxn;
  double Iyy = I1yy + kDeltaPiPi * (theta * piyy) - I3yy + kTauPiPi * I4yy - kLambdaPiBulk * Pi * syy;
  double Iyn = I1yn + kDeltaPiPi * (theta * piyn) - I3yn + kTauPiPi * I4yn - kLambdaPiBulk * Pi * syn;
  double Inn = I1nn + kDeltaPiPi * (theta * pinn) - I3nn + kTauPiPi * I4nn - kLambdaPiBulk * Pi * snn;

  // SourceTerms.cu:224-233
  double dpitt = 2.0 * beta_pi * stt - pitt * taupiInv - Itt - 2.0 * un * t * pitn;
  double dpitx = 2.0 * beta_pi * stx - pitx * taupiInv - Itx - un * t * pixn;
  double dpity = 2.0 * beta_pi * sty - pity * taupiInv - Ity - un * t * piyn;
  double dpitn = 2.0 * beta_pi * stn - pitn * taupiInv - Itn - un * t * pinn - (ut * pitn + un * pitt) / t;
  double dpixx = 2.0 * beta_pi * sxx - pixx * taupiInv - Ixx;
  double dpixy = 2.0 * beta_pi * sxy - pixy * taupiInv - Ixy;
  double dpixn = 2.0 * beta_pi * sxn - pixn * taupiInv - Ixn - (ut * pixn + un * pitx) / t;
  double dpiyy = 2.0 * beta_pi * syy - piyy * taupiInv - Iyy;
  double dpiyn = 2.0 * beta_pi * syn - piyn * taupiInv - Iyn - (ut * piyn + un * pity) / t;
  double dpinn = 2.0 * beta_pi * snn - pinn * taupiInv - Inn - 2.0 * (ut * pinn + un * pitn) / t;

  rhs[0] = dpitt / ut + pitt * dkvk;
  rhs[1] = dpitx / ut + pitx * dkvk;
  rhs[2] = dpity / ut + pity * dkvk;
  rhs[3] = dpitn / ut + pitn * dkvk;
  rhs[4] = dpixx / ut + pixx * dkvk;
  rhs[5] = dpixy / ut + pixy * dkvk;
  rhs[6] = dpixn / ut + pixn * dkvk;
  rhs[7] = dpiyy / ut + piyy * dkvk;
  rhs[8] = dpiyn / ut + piyn * dkvk;
  rhs[9] = dpinn / ut + pinn * dkvk;
  if (BULK) {
    // bulk coefficients (SourceTerms.cu:53-60, 238, 254)
    double cs2 = sound_speed2<EOS>(e);
    double a = kF033 - cs2;
    double a2 = a * a;
    double beta_Pi = 15.0 * a2 * (e + p);
    double lambda_Pipi = kF16 * a;
    double zetabar = bulk_zeta_over_s(T);
    double tauPiInv = 15 * a2 * (T / zetabar);
    double dPi = -beta_Pi * theta - Pi * tauPiInv - kDeltaBulk * Pi * theta + lambda_Pipi * ps;
    rhs[10] = dPi / ut + Pi * dkvk;
  }
}

}  // namespace gvh
