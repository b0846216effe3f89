// gvh_sources.cuh -- right-hand sides of the KT step at one cell: the Milne geometric
// source of T^{tau mu} and the relaxation equations of pi^{mu nu} and Pi.
// Reproduces SourceTerms.cu:29-256 (setPimunuSourceTerms) and :569-755 (loadSourceTerms2,
// with USE_APPROX_DERIVATIVE). Operation order follows the reference.
#pragma once

#include "gvh_physics.cuh"

namespace gvh {

// Division in the working precision: IEEE division in FP64 (the plain path follows the
// reference to rounding), the fast reciprocal-based division in FP32 (mixed path).
__device__ __forceinline__ double dv(double a, double b) { return a / b; }
__device__ __forceinline__ float dv(float a, float b) { return __fdividef(a, b); }

// Flow state and limited first derivatives at a cell.
template <class R>
struct CellFlowT {
  R ut, ux, uy, un;          // u^mu (current)
  R dtut, dtux, dtuy, dtun;  // (u^mu - u^mu one step earlier) / dt (SourceTerms.cu:68-71)
  R dxut, dyut, dnut, dxux, dyux, dnux, dxuy, dyuy, dnuy, dxun, dyun, dnun;
};

template <class R>
struct ShearT {
  R tt, tx, ty, tn, xx, xy, xn, yy, yn, nn;
};

// SourceTerms.cu:29-256. rhs[0..9] = d pi^{mu nu}/dtau (pitt..pinn), rhs[10] = dPi/dtau.
// R = double reproduces the reference's FP64 arithmetic; R = float is the mixed path.
template <int EOS, bool BULK, class R>
__device__ __forceinline__ void pimunu_rhs(R *rhs, R t, R etabar, R e, R p, const CellFlowT<R> &f,
                                           const ShearT<R> &pi, R Pi, R dkvk) {
  const R ut = f.ut, ux = f.ux, uy = f.uy, un = f.un;
  const R pitt = pi.tt, pitx = pi.tx, pity = pi.ty, pitn = pi.tn, pixx = pi.xx, pixy = pi.xy, pixn = pi.xn;
  const R piyy = pi.yy, piyn = pi.yn, pinn = pi.nn;
  const R dxut = f.dxut, dyut = f.dyut, dnut = f.dnut, dxux = f.dxux, dyux = f.dyux, dnux = f.dnux;
  const R dxuy = f.dxuy, dyuy = f.dyuy, dnuy = f.dnuy, dxun = f.dxun, dyun = f.dyun, dnun = f.dnun;

  R T = temperature<EOS>(e);
  R taupiInv = R(kF02) * dv(T, etabar);
  R beta_pi = R(kF02) * (e + p);

  R ut2 = ut * ut, un2 = un * un, t2 = t * t, t3 = t * t2;
  // reciprocals of the divisors used below (the reference divides each time; equal to rounding)
  const R it = dv(R(1), t), iut = dv(R(1), ut);
  const R it2 = it * it, it3 = it2 * it;
  const R dtut = f.dtut, dtux = f.dtux, dtuy = f.dtuy, dtun = f.dtun;

  R Dut = ut * dtut + ux * dxut + uy * dyut + un * dnut + t * un * un;
  R dut = Dut - t * un * un;
  R dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
  R Dux = -dux;
  R duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
  R Duy = -duy;
  R dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
  R Dun = -t2 * dun - R(2.0) * t * ut * un;

  R theta = (ut) * it + dtut + dxux + dyuy + dnun;
  R theta3 = theta * R(1.0 / 3.0);

  // shear tensor sigma^{mu nu}
  R stt = -t * ut * un2 + (dtut - ut * dut) + (ut2 - R(1.0)) * theta3;
  R stx = -(t * un2 * ux) / R(2.0) + (dtux - dxut) / R(2.0) - (ux * dut + ut * dux) / R(2.0) + ut * ux * theta3;
  R sty = -(t * un2 * uy) / R(2.0) + (dtuy - dyut) / R(2.0) - (uy * dut + ut * duy) / R(2.0) + ut * uy * theta3;
  R stn = (-un * (R(2.0) * ut2 + t2 * un2)) * (R(0.5) * it) + (dtun - dnut * it2) / R(2.0) - (un * dut + ut * dun) / R(2.0)
               + ut * un * theta3;
  R sxx = -(dxux + ux * dux) + (R(1.0) + ux * ux) * theta3;
  R sxy = -(dxuy + dyux) / R(2.0) - (uy * dux + ux * duy) / R(2.0) + ux * uy * theta3;
  R sxn = (-ut * ux * un) * it - (dxun + dnux * it2) / R(2.0) - (un * dux + ux * dun) / R(2.0) + ux * un * theta3;
  R syy = -(dyuy + uy * duy) + (R(1.0) + uy * uy) * theta3;
  R syn = (-ut * uy * un) * it - (dyun + dnuy * it2) / R(2.0) - (un * duy + uy * dun) / R(2.0) + uy * un * theta3;
  R snn = (-ut * (R(1.0) + R(2.0) * t2 * un2)) * it3 - dnun * it2 - un * dun + (it2 + un2) * theta3;

  // vorticity (SourceTerms.cu:122-136)
  R wtx = (-dtux - dxut + ut * dux - ux * dut - t * un2 * ux) / R(2.0);
  R wty = (-dtuy - dyut + ut * duy - uy * dut - t * un2 * uy) / R(2.0);
  R wtn = (-t2 * dtun - R(2.0) * t * un - dnut - ut * Dun - t2 * un * dut - t3 * un * un2) / R(2.0);
  R wxy = (dxuy - dyux + ux * duy - uy * dux) / R(2.0);
  R wxn = (t2 * dxun - dnux - ux * Dun - t2 * un * dux) / R(2.0);
  R wyn = (t2 * dyun - dnuy - uy * Dun - t2 * un * duy) / R(2.0);
  R wxt = wtx, wyt = wty, wnt = wtn * it2, wyx = -wxy, wnx = -wxn * it2, wny = -wyn * it2;

  // I1 (SourceTerms.cu:141-150)
  R I1tt = R(2.0) * ut * (pitt * Dut + pitx * Dux + pity * Duy + pitn * Dun);
  R I1tx = (pitt * ux + pitx * ut) * Dut + (pitx * ux + pixx * ut) * Dux + (pity * ux + pixy * ut) * Duy
                + (pitn * ux + pixn * ut) * Dun;
  R I1ty = (pitt * uy + pity * ut) * Dut + (pitx * uy + pixy * ut) * Dux + (pity * uy + piyy * ut) * Duy
                + (pitn * uy + piyn * ut) * Dun;
  R I1tn = (pitt * un + pitn * ut) * Dut + (pitx * un + pixn * ut) * Dux + (pity * un + piyn * ut) * Duy
                + (pitn * un + pinn * ut) * Dun;
  R I1xx = R(2.0) * ux * (pitx * Dut + pixx * Dux + pixy * Duy + pixn * Dun);
  R I1xy = (pitx * uy + pity * ux) * Dut + (pixx * uy + pixy * ux) * Dux + (pixy * uy + piyy * ux) * Duy
                + (pixn * uy + piyn * ux) * Dun;
  R I1xn = (pitx * un + pitn * ux) * Dut + (pixx * un + pixn * ux) * Dux + (pixy * un + piyn * ux) * Duy
                + (pixn * un + pinn * ux) * Dun;
  R I1yy = R(2.0) * uy * (pity * Dut + pixy * Dux + piyy * Duy + piyn * Dun);
  R I1yn = (pity * un + pitn * uy) * Dut + (pixy * un + pixn * uy) * Dux + (piyy * un + piyn * uy) * Duy
                + (piyn * un + pinn * uy) * Dun;
  R I1nn = R(2.0) * un * (pitn * Dut + pixn * Dux + piyn * Duy + pinn * Dun);

  // I3 (SourceTerms.cu:169-178)
  R I3tt = R(2.0) * (pitx * wtx + pity * wty + pitn * wtn);
  R I3tx = pitt * wxt + pity * wxy + pitn * wxn + pixx * wtx + pixy * wty + pixn * wtn;
  R I3ty = pitt * wyt + pitx * wyx + pitn * wyn + pixy * wtx + piyy * wty + piyn * wtn;
  R I3tn = pitt * wnt + pitx * wnx + pity * wny + pixn * wtx + piyn * wty + pinn * wtn;
  R I3xx = R(2.0) * (pitx * wxt + pixy * wxy + pixn * wxn);
  R I3xy = pitx * wyt + pity * wxt + pixx * wyx + piyy * wxy + pixn * wyn + piyn * wxn;
  R I3xn = pitx * wnt + pitn * wxt + pixx * wnx + pixy * wny + piyn * wxy + pinn * wxn;
  R I3yy = R(2.0) * (pity * wyt + pixy * wyx + piyn * wyn);
  R I3yn = pity * wnt + pitn * wyt + pixy * wnx + pixn * wyx + piyy * wny + pinn * wyn;
  R I3nn = R(2.0) * (pitn * wnt + pixn * wnx + piyn * wny);

  // I4 (SourceTerms.cu:183-203)
  R ux2 = ux * ux, uy2 = uy * uy;
  R ps = pitt * stt - R(2.0) * pitx * stx - R(2.0) * pity * sty + pixx * sxx + R(2.0) * pixy * sxy + piyy * syy
              - R(2.0) * pitn * stn * t2 + R(2.0) * pixn * sxn * t2 + R(2.0) * piyn * syn * t2 + pinn * snn * t2 * t2;
  R ps3 = ps * R(1.0 / 3.0);
  R I4tt = (pitt * stt - pitx * stx - pity * sty - t2 * pitn * stn) - (1 - ut2) * ps3;
  R I4tx = (pitt * stx + pitx * stt) / R(2.0) - (pitx * sxx + pixx * stx) / R(2.0) - (pity * sxy + pixy * sty) / R(2.0)
                - t2 * (pitn * sxn + pixn * stn) / R(2.0) + (ut * ux) * ps3;
  R I4ty = (pitt * sty + pity * stt) / R(2.0) - (pitx * sxy + pixy * stx) / R(2.0) - (pity * syy + piyy * sty) / R(2.0)
                - t2 * (pitn * syn + piyn * stn) / R(2.0) + (ut * uy) * ps3;
  R I4tn = (pitt * stn + pitn * stt) / R(2.0) - (pitx * sxn + pixn * stx) / R(2.0) - (pity * syn + piyn * sty) / R(2.0)
                - t2 * (pitn * snn + pinn * stn) / R(2.0) + (ut * un) * ps3;
  R I4xx = (pitx * stx - pixx * sxx - pixy * sxy - t2 * pixn * sxn) + (R(1.0) + ux2) * ps3;
  R I4xy = (pitx * sty + pity * stx) / R(2.0) - (pixx * sxy + pixy * sxx) / R(2.0) - (pixy * syy + piyy * sxy) / R(2.0)
                - t2 * (pixn * syn + piyn * sxn) / R(2.0) + (ux * uy) * ps3;
  R I4xn = (pitx * stn + pitn * stx) / R(2.0) - (pixx * sxn + pixn * sxx) / R(2.0) - (pixy * syn + piyn * sxy) / R(2.0)
                - t2 * (pixn * snn + pinn * sxn) / R(2.0) + (ux * un) * ps3;
  R I4yy = (pity * sty - pixy * sxy - piyy * syy - t2 * piyn * syn) + (R(1.0) + uy2) * ps3;
  R I4yn = (pity * stn + pitn * sty) / R(2.0) - (pixy * sxn + pixn * sxy) / R(2.0) - (piyy * syn + piyn * syy) / R(2.0)
                - t2 * (piyn * snn + pinn * syn) / R(2.0) + (uy * un) * ps3;
  R I4nn = (pitn * stn - pixn * sxn - piyn * syn - t2 * pinn * snn) + (it2 + un2) * ps3;

  // I = I1 + delta I2 - I3 + tau I4 - lambda Pi sigma (SourceTerms.cu:209-218); I2 = theta pi
  R Itt = I1tt + R(kDeltaPiPi) * (theta * pitt) - I3tt + R(kTauPiPi) * I4tt - R(kLambdaPiBulk) * Pi * stt;
  R Itx = I1tx + R(kDeltaPiPi) * (theta * pitx) - I3tx + R(kTauPiPi) * I4tx - R(kLambdaPiBulk) * Pi * stx;
  R Ity = I1ty + R(kDeltaPiPi) * (theta * pity) - I3ty + R(kTauPiPi) * I4ty - R(kLambdaPiBulk) * Pi * sty;
  R Itn = I1tn + R(kDeltaPiPi) * (theta * pitn) - I3tn + R(kTauPiPi) * I4tn - R(kLambdaPiBulk) * Pi * stn;
  R Ixx = I1xx + R(kDeltaPiPi) * (theta * pixx) - I3xx + R(kTauPiPi) * I4xx - R(kLambdaPiBulk) * Pi * sxx;
  R Ixy = I1xy + R(kDeltaPiPi) * (theta * pixy) - I3xy + R(kTauPiPi) * I4xy - R(kLambdaPiBulk) * Pi * sxy;
  R Ixn = I1xn + R(kDeltaPiPi) * (theta * pixn) - I3xn + R(kTauPiPi) * I4xn - R(kLambdaPiBulk) * Pi * sxn;
  R Iyy = I1yy + R(kDeltaPiPi) * (theta * piyy) - I3yy + R(kTauPiPi) * I4yy - R(kLambdaPiBulk) * Pi * syy;
  R Iyn = I1yn + R(kDeltaPiPi) * (theta * piyn) - I3yn + R(kTauPiPi) * I4yn - R(kLambdaPiBulk) * Pi * syn;
  R Inn = I1nn + R(kDeltaPiPi) * (theta * pinn) - I3nn + R(kTauPiPi) * I4nn - R(kLambdaPiBulk) * Pi * snn;

  // SourceTerms.cu:224-233
  R dpitt = R(2.0) * beta_pi * stt - pitt * taupiInv - Itt - R(2.0) * un * t * pitn;
  R dpitx = R(2.0) * beta_pi * stx - pitx * taupiInv - Itx - un * t * pixn;
  R dpity = R(2.0) * beta_pi * sty - pity * taupiInv - Ity - un * t * piyn;
  R dpitn = R(2.0) * beta_pi * stn - pitn * taupiInv - Itn - un * t * pinn - (ut * pitn + un * pitt) * it;
  R dpixx = R(2.0) * beta_pi * sxx - pixx * taupiInv - Ixx;
  R dpixy = R(2.0) * beta_pi * sxy - pixy * taupiInv - Ixy;
  R dpixn = R(2.0) * beta_pi * sxn - pixn * taupiInv - Ixn - (ut * pixn + un * pitx) * it;
  R dpiyy = R(2.0) * beta_pi * syy - piyy * taupiInv - Iyy;
  R dpiyn = R(2.0) * beta_pi * syn - piyn * taupiInv - Iyn - (ut * piyn + un * pity) * it;
  R dpinn = R(2.0) * beta_pi * snn - pinn * taupiInv - Inn - (R(2.0) * (ut * pinn + un * pitn)) * it;

  rhs[0] = dpitt * iut + pitt * dkvk;
  rhs[1] = dpitx * iut + pitx * dkvk;
  rhs[2] = dpity * iut + pity * dkvk;
  rhs[3] = dpitn * iut + pitn * dkvk;
  rhs[4] = dpixx * iut + pixx * dkvk;
  rhs[5] = dpixy * iut + pixy * dkvk;
  rhs[6] = dpixn * iut + pixn * dkvk;
  rhs[7] = dpiyy * iut + piyy * dkvk;
  rhs[8] = dpiyn * iut + piyn * dkvk;
  rhs[9] = dpinn * iut + pinn * dkvk;
  if (BULK) {
    // bulk coefficients (SourceTerms.cu:53-60, 238, 254)
    R cs2 = sound_speed2<EOS>(e);
    R a = R(kF033) - cs2;
    R a2 = a * a;
    R beta_Pi = R(15.0) * a2 * (e + p);
    R lambda_Pipi = R(kF16) * a;
    R zetabar = bulk_zeta_over_s(T);
    R tauPiInv = R(15) * a2 * dv(T, zetabar);
    R dPi = -beta_Pi * theta - Pi * tauPiInv - R(kDeltaBulk) * Pi * theta + lambda_Pipi * ps;
    rhs[10] = dPi * iut + Pi * dkvk;
  }
}

}  // namespace gvh
