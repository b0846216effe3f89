// gvh_physics.cuh -- device physics of the KT RK2 step: equation of state, primitive
// recovery, minmod limiter, KT face flux, Milne geometric sources and the
// Israel-Stewart/DNMR right-hand sides of pi^{mu nu} and Pi.
//
// Each routine states the reference routine it reproduces (gpu-vh rhic/src, file:line).
// The plain FP64 path keeps the reference's operation order and its single-precision
// literals (0.2f, 0.333333f, 1.6f) so it follows the reference's FP64 build to rounding;
// everything is inlined into the fused stage kernel (the reference passes these as
// function pointers across translation units, which blocks inlining).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace gvh {

enum : int { EOS_QCD = 0, EOS_CONFORMAL = 1 };

// Transport constants (TransportCoefficients.cuh:14-18).
constexpr double kDeltaPiPi = 1.33333;     // delta_pipi
constexpr double kTauPiPi = 1.42857;       // tau_pipi
constexpr double kLambdaPiBulk = 1.2;      // lambda_piPi
constexpr double kDeltaBulk = 0.666667;    // delta_PiPi
constexpr double kEosFactor = 13.8997;     // EquationOfState.cuh:20
constexpr double kF02 = (double)0.2f;      // SourceTerms.cu:47-48 float literal
constexpr double kF033 = (double)0.333333f;  // SourceTerms.cu:54
constexpr double kF16 = (double)1.6f;      // SourceTerms.cu:57

// ------------------------------------------------------------------------------------
// Equation of state (EquationOfState.cu)
// ------------------------------------------------------------------------------------

// The QCD fits of EquationOfState.cu are rational functions of e; they are evaluated here
// in Horner form (the reference builds explicit powers e^2..e^13 first). The two agree to
// rounding.

// The QCD fit's coefficients in Horner order (highest power first), one table per
// polynomial; every evaluation below runs the same multiply-adds in the same order.
__constant__ double kQcdPa[13] = {
    1.9531729608963267e-11, 3.1188455176941583e-7, 0.0009417586777847889,
    0.7158279081255019, 141.5073484468774, 6340.448389300905,
    41913.439282708554, 334334.4309240126, 1.6357487344679043e6,
    3.1729694865420084e6, 1.077580993288114e6, 9737.845799644809,
    -0.25181736420168666};
__constant__ double kQcdPb[13] = {
    3.2581066229887368e-18, 5.928138360995685e-11, 9.601103399348206e-7,
    0.002962497695527404, 2.3405487982094204, 499.04919730607065,
    26452.34905933697, 278581.2989342773, 1.7851642641834426e6,
    1.3512402226067686e7, 2.0931169138134286e7, 4.0574329080826794e6,
    45829.44617893836};
__constant__ double kQcdCa[14] = {
    8.189430244031285e-6, 0.03009027913262399, 6.504847576502024,
    58.60283714484669, 275.0492627924299, 1612.4245252438795,
    460.6487249985994, 15.382615282179595, 0.02969737949090831,
    6.087136671592452e-6, 1.4170364808063119e-10, 3.1955868410879504e-16,
    4.123605749683891e-23, 5.191934309650155e-32};
__constant__ double kQcdCb[14] = {
    0.000024810902623582917, 0.09301685073435291, 21.461303090563028,
    293.99144775704605, 590.2572000057821, 15190.225535036281,
    1800.5461219450308, 60.85769171450653, 0.13653226327408863,
    0.00003551782901018317, 1.1225580509306008e-9, 3.5477700458515908e-15,
    6.716598285341542e-22, 1.4637868900982493e-30};
__constant__ double kQcdTa[12] = {
    1.5780479034557783e-6, 0.015421252394182246, 14.055788949565482,
    1471.6180520527757, 14109.766109389702, 6686.07424325115,
    207.48582344326206, 0.4873490574161924, 0.000063810382643387,
    2.4954778310451065e-10, 8.014062800678687e-18, 1.510073201405604e-29};
__constant__ double kQcdTb[12] = {
    1.8472801679382593e-7, 0.003778342768228011, 5.916312075925817,
    1051.0730543534657, 17965.67607192861, 11179.193315394154,
    578.0778724946719, 2.316902328874072, 0.0005036835870305458,
    2.998130743142826e-9, 1.3686372302041508e-16, 7.558667139355393e-28};

// Horner evaluation of a constant-bank polynomial (coefficients highest power first).
template <int N>
__device__ __forceinline__ double horner(const double (&c)[N], double e) {
  double a = c[0];
#pragma unroll
  for (int k = 1; k < N; ++k) a = fma(a, e, c[k]);
  return a;
}

// p(e): EquationOfState.cu:30-80; conformal p = e/3.
template <int EOS>
__device__ __forceinline__ double eq_pressure(double e) {
  if (EOS == EOS_CONFORMAL) return e / 3;
  return horner(kQcdPa, e) / horner(kQcdPb, e);
}

// c_s^2(e): EquationOfState.cu:82-116. The conformal branch of the reference returns the
// integer quotient 1/3 == 0 (EquationOfState.cu:114) and that value is kept.
template <int EOS>
__device__ __forceinline__ double sound_speed2(double e) {
  if (EOS == EOS_CONFORMAL) return 0.0;
  return horner(kQcdCa, e) / horner(kQcdCb, e);
}

// T(e): EquationOfState.cu:118-148; conformal T = (e/13.8997)^(1/4).
template <int EOS>
__device__ __forceinline__ double temperature(double e) {
  if (EOS == EOS_CONFORMAL) return pow(e / kEosFactor, 0.25);
  return horner(kQcdTa, e) / horner(kQcdTb, e);
}

// e(T): EquationOfState.cu:150-204; conformal e = 13.8997 T^4. Host-callable: the host
// computes e(T_reg) and e(T_fo) once per call.
template <int EOS>
__host__ __device__ inline double energy_density_of_T(double T) {
  if (EOS == EOS_CONFORMAL) return kEosFactor * pow(T, 4.0);
  double T2 = T * T, T3 = T2 * T, T4 = T3 * T, T5 = T4 * T, T6 = T5 * T, T7 = T6 * T, T8 = T7 * T;
  double T9 = T8 * T, T10 = T9 * T, T11 = T10 * T, T12 = T11 * T, T13 = T12 * T, T14 = T13 * T;
  double T15 = T14 * T, T16 = T15 * T, T17 = T16 * T, T18 = T17 * T, T19 = T18 * T, T20 = T19 * T;
  double T21 = T20 * T, T22 = T21 * T, T23 = T22 * T;
  return (-0.011958188410851651 + 119.89423098138208 * T - 3156.9475699248055 * T2 + 32732.86844374939 * T3
          - 187899.8994764422 * T4 + 712537.3610845465 * T5 - 1.557049803609345e6 * T6
          + 1.4852519861308339e6 * T7 + 532132.6079941876 * T8 - 1.963099445042592e6 * T9
          - 4484.44579242679 * T10 + 1.7984228830058286e6 * T11 + 119345.25619517374 * T12
          - 1.3499773937058165e6 * T13 - 207838.4995663606 * T14 + 654970.2138652403 * T15
          - 78643.00334616247 * T16 + 40274.00078068926 * T17 + 422619.58977657766 * T18
          - 409688.07836393174 * T19 - 62005.75915066359 * T20 + 46788.14270090656 * T21
          + 40784.330477857235 * T22 - 12589.47744840392 * T23)
       / (31630.074365558292 - 127100.88940643385 * T + 173528.1225422275 * T2 - 39403.297956865215 * T3
          - 85582.57873541754 * T4 + 9320.560804233442 * T5 + 50882.74198960172 * T6
          + 20335.926473421183 * T7 - 14897.725710713818 * T8 - 23836.484117457 * T9
          - 13726.013896090335 * T10 + 4517.908673107615 * T11 + 18056.19917986404 * T12
          + 14954.82860467155 * T13 + 2569.623976952738 * T14 - 9304.046211514986 * T15
          - 15606.429173842751 * T16 + 8383.710735812094 * T17 + 1591.3177623932843 * T18
          - 678.748230997762 * T19 - 33.58687934953277 * T20 + 3.2520554133126285 * T21
          - 0.19647288043440464 * T22 + 0.005443394551264717 * T23);
}

// zeta/s(T): TransportCoefficients.cu:27-36.
__device__ __forceinline__ double bulk_zeta_over_s(double T) {
  double x = T / 1.01355;
  if (x > 1.05) return 0.9 * exp(-(x - 1) / 0.025) + 0.25 * exp(-(x - 1) / 0.13) + 0.001;
  else if (x < 0.995) return 0.9 * exp((x - 1) / 0.0025) + 0.22 * exp((x - 1) / 0.022) + 0.03;
  return -13.77 * x * x + 27.55 * x - 13.45;
}

// ------------------------------------------------------------------------------------
// Primitive recovery (EnergyMomentumTensor.cu)
// ------------------------------------------------------------------------------------

// Status bits a stage kernel may raise (or-ed into the per-lattice status word).
//   STATUS_NAN     an energy density came out NaN
//   STATUS_NEWTON  a Newton solve failed to converge even with damping
//   STATUS_DAMPED  informational: a Newton solve needed the damped phase (see below)
//   STATUS_BOUNDS  the bounds-checked build (GVH_BOUNDS_CHECK) found a stencil index outside
//                  the arrays; the cell was skipped
enum : unsigned { STATUS_NAN = 1u, STATUS_NEWTON = 2u, STATUS_DAMPED = 4u, STATUS_BOUNDS = 8u };

// Newton iteration budget. The reference iterates e <- e - f/f' up to 5x10^5 times and
// then switches to the damped update e <- e - 0.9 f/f' for up to another 5x10^5
// (EnergyMomentumTensor.cu:15, 22-41). Converging solves take a handful of iterations.
// The ones that do not converge undamped wander chaotically (the iterates of such a solve,
// recorded from the reference's algorithm, neither settle nor repeat exactly), so the
// state the reference reaches after 5x10^5 undamped iterations depends on every rounding
// on the way and no implementation reproduces it; what the reference does next -- damp --
// is what decides the answer. Here the undamped phase is kNewtonUndamped iterations, then
// the same damped update runs up to kNewtonMaxIters in total.
constexpr int kNewtonUndamped = 200;
constexpr int kNewtonMaxIters = 2000;

// p(e) and c_s^2(e) of the QCD fit together, both rational functions evaluated in Horner
// form (the reference evaluates the same polynomials from explicit powers,
// EquationOfState.cu:30-116; the two agree to rounding).
__device__ __forceinline__ void qcd_p_cs2(double e, double &p, double &cs2) {
  const double a = horner(kQcdPa, e), b = horner(kQcdPb, e), c = horner(kQcdCa, e), d = horner(kQcdCb, e);
  p = a / b;
  cs2 = c / d;
}

// The four polynomials of the QCD fit, p = pa/pb and c_s^2 = ca/cb, without the divisions (the
// Newton update below shares one reciprocal between them).
__device__ __forceinline__ void qcd_poly(double e, double &pa, double &pb, double &ca, double &cb) {
  pa = horner(kQcdPa, e);
  pb = horner(kQcdPb, e);
  ca = horner(kQcdCa, e);
  cb = horner(kQcdCb, e);
}

// The two polynomials of p = pa/pb alone.
__device__ __forceinline__ void qcd_poly_p(double e, double &pa, double &pb) {
  pa = horner(kQcdPa, e);
  pb = horner(kQcdPb, e);
}

// The Newton update of EnergyMomentumTensor.cu:22-40 at an iterate e0 where the fit's
// polynomials are pa, pb (p = pa/pb) and ca, cb (c_s^2 = ca/cb). The reference's six
// divisions (p, c_s^2, p/e0, D, f', f/f') become two: one reciprocal R = 1/(pa cb pb e0)
// gives 1/pa, 1/cb and 1/(pb e0) by multiplication, and f/f' = f H / (H - X) with
// X = g (...) pb / pa folds the division by p H into the last one. Equal to rounding.
__device__ __forceinline__ double newton_update_poly(double e0, double pa, double pb, double ca, double cb, double M0,
                                                     double M, double Pi, bool damped) {
  const double be = pb * e0;
  const double R = 1.0 / (pa * cb * be);
  const double inv_pa = cb * be * R;
  const double inv_be = pa * cb * R;
  const double cst2 = pa * inv_be;        // p / e0
  const double cs2 = ca * (pa * be * R);  // ca / cb
  const double inv_e0 = pb * inv_be;
  const double A = fma(M0, 1 - cst2, Pi);
  const double B = fma(M0, M0 + Pi, -M);
  const double H = sqrt(fabs(A * A + 4 * cst2 * B));
  const double D = (A - H) * (0.5 * be * inv_pa);  // (A - H) / (2 cst2)
  const double f = e0 + D;
  const double g = cs2 - cst2;
  const double X = (g * (B + D * H - (g * cst2 * D * M0) * inv_e0)) * (pb * inv_pa);  // f' = 1 - X / H
  return e0 - ((damped ? 0.9 * f : f) * H) / (H - X);
}

// The QCD fit at the Newton guess. Every solve of one cell starts from the same guess (the
// cell's energy density), so the first iteration's p and c_s^2 are computed once per cell.
struct GuessEos {
  double e, inv_e, p, cs2;
  double inv_p, half_inv_cst2;  // 1/p and 1/(2 p/e): the first update's divisions, per cell
};
template <int EOS>
__device__ __forceinline__ GuessEos guess_eos(double ePrev) {
  GuessEos g;
  g.e = ePrev;
  g.inv_e = 1.0 / ePrev;
  if (EOS == EOS_CONFORMAL) {
    g.p = 0.0;
    g.cs2 = 0.0;
    g.inv_p = 0.0;
    g.half_inv_cst2 = 0.0;
  } else {
    qcd_p_cs2(ePrev, g.p, g.cs2);
    g.inv_p = 1.0 / g.p;
    g.half_inv_cst2 = 0.5 * ePrev * g.inv_p;
  }
  return g;
}

// The first Newton update, at the guess (every solve of a cell starts there): the same
// update as newton_update with the guess's reciprocals taken from GuessEos, leaving one
// division (f/f' = f H / (H - X / p)).
__device__ __forceinline__ double newton_update_guess(const GuessEos &g, double M0, double M, double Pi) {
  const double e0 = g.e;
  const double cst2 = g.p * g.inv_e;
  const double A = fma(M0, 1 - cst2, Pi);
  const double B = fma(M0, M0 + Pi, -M);
  const double H = sqrt(fabs(A * A + 4 * cst2 * B));
  const double D = (A - H) * g.half_inv_cst2;
  const double f = e0 + D;
  const double gg = g.cs2 - cst2;
  const double X = (gg * (B + D * H - (gg * cst2 * D * M0) * g.inv_e)) * g.inv_p;
  return e0 - (f * H) / (H - X);
}

// The reference's Newton update (EnergyMomentumTensor.cu:22-40) at an iterate e0 with
// cst2 = p/e0, A = M0 (1 - cst2) + Pi, B = M0 (M0 + Pi) - M, H = sqrt|A^2 + 4 cst2 B|,
// D = (A - H) / (2 cst2), f = e0 + D, g = c_s^2 - cst2,
// f' = 1 - g (B + D H - g cst2 D M0 / e0) / (p H), e <- e0 - f/f' (or - 0.9 f/f' damped),
// is computed by newton_update_guess (first update) and newton_update_poly (the others).

// N independent Newton solves (EnergyMomentumTensor.cu:18-48) iterated together: each
// follows its own sequence of iterates and stops at its own iteration (|de| <= 1e-3 |e|),
// while the independent chains give the FP64 pipe instruction-level parallelism.
template <int EOS, int N>
__device__ __forceinline__ void energy_from_conserved_n(const GuessEos &g0, const double (&M0)[N],
                                                        const double (&M)[N], const double (&Pi)[N],
                                                        double (&out)[N], unsigned &status) {
  if (EOS == EOS_CONFORMAL) {
#pragma unroll
    for (int n = 0; n < N; ++n) out[n] = fabs(sqrt(fabs(4 * M0[n] * M0[n] - 3 * M[n])) - M0[n]);
    return;
  }
  double e0[N];
  bool done[N];
  bool all = true;
#pragma unroll
  for (int n = 0; n < N; ++n) {
    double e = newton_update_guess(g0, M0[n], M[n], Pi[n]);
    done[n] = fabs(e - g0.e) <= 0.001 * fabs(e);
    e0[n] = e;
    out[n] = e;
    all = all && done[n];
  }
  for (int j = 1; j < kNewtonMaxIters && !all; ++j) {
    const bool damped = j >= kNewtonUndamped;
    if (j == kNewtonUndamped) status |= STATUS_DAMPED;
    all = true;
#pragma unroll
    for (int n = 0; n < N; ++n) {
      if (done[n]) continue;
      double pa, pb, ca, cb;
      qcd_poly(e0[n], pa, pb, ca, cb);
      double e = newton_update_poly(e0[n], pa, pb, ca, cb, M0[n], M[n], Pi[n], damped);
      done[n] = fabs(e - e0[n]) <= 0.001 * fabs(e);
      e0[n] = e;
      out[n] = e;
      all = all && done[n];
    }
  }
  if (!all) status |= STATUS_NEWTON;
}

struct Prim {
  double e, p, ut, ux, uy, un;
};

// getInferredVariables: EnergyMomentumTensor.cu:50-108, guess g0.e. The Pi clamp guarded
// by the never-defined `Pi` macro (lines 82-85) is not part of the reference's behaviour.
template <int EOS>
__device__ __forceinline__ Prim inferred(double t, double ttt, double ttx, double tty, double ttn, double pitt,
                                         double pitx, double pity, double pitn, double Pi, const GuessEos &g0,
                                         unsigned &status) {
  Prim r;
  double M0 = ttt - pitt;
  double M1 = ttx - pitx;
  double M2 = tty - pity;
  double M3 = ttn - pitn;
  double M = M1 * M1 + M2 * M2 + t * t * M3 * M3;
  if (g0.e <= 0.1) {
    r.e = M0 - M / M0;
  } else {
    double m0[1] = {M0}, mm[1] = {M}, pi[1] = {Pi}, e[1];
    energy_from_conserved_n<EOS, 1>(g0, m0, mm, pi, e, status);
    r.e = e[0];
  }
  if (isnan(r.e)) status |= STATUS_NAN;
  r.p = eq_pressure<EOS>(r.e);
  if (r.e < 1.e-7) { r.e = 1.e-7; r.p = 1.e-7; }
  double P = r.p + Pi;
  double E = 1 / (r.e + P);
  r.ut = sqrt(fabs((M0 + P) * E));
  double E2 = E / r.ut;
  r.ux = M1 * E2;
  r.uy = M2 * E2;
  r.un = M3 * E2;
  return r;
}

// N primitive recoveries sharing one guess-independent formulation (EnergyMomentumTensor.cu
// :50-108), the Newton solves iterated together. Outputs e, p, u^tau and w = u^axis/u^tau
// for the axis the KT face flux needs (the only velocity the flux uses).
template <int EOS, int N>
__device__ __forceinline__ void inferred_face_n(double t, int axis, const double (&ttt)[N], const double (&ttx)[N],
                                                const double (&tty)[N], const double (&ttn)[N],
                                                const double (&pitt)[N], const double (&pitx)[N],
                                                const double (&pity)[N], const double (&pitn)[N],
                                                const double (&Pi)[N], const GuessEos &g0, double (&w)[N],
                                                unsigned &status) {
  const double ePrev = g0.e;
  double M0[N], M[N], Mi[N], e[N];
#pragma unroll
  for (int n = 0; n < N; ++n) {
    M0[n] = ttt[n] - pitt[n];
    double M1 = ttx[n] - pitx[n];
    double M2 = tty[n] - pity[n];
    double M3 = ttn[n] - pitn[n];
    M[n] = M1 * M1 + M2 * M2 + t * t * M3 * M3;
    Mi[n] = axis == 0 ? M1 : axis == 1 ? M2 : M3;
  }
  if (ePrev <= 0.1) {
#pragma unroll
    for (int n = 0; n < N; ++n) e[n] = M0[n] - M[n] / M0[n];
  } else {
    energy_from_conserved_n<EOS, N>(g0, M0, M, Pi, e, status);
  }
#pragma unroll
  for (int n = 0; n < N; ++n) {
    if (isnan(e[n])) status |= STATUS_NAN;
    // u^axis/u^tau = M_axis E / ut^2 with E = 1/(e + P) and ut^2 = |(M0 + P) E|
    // (EnergyMomentumTensor.cu:95-104), i.e. M_axis sign(e + P) / |M0 + P|: with the QCD fit
    // p = pa/pb (pb > 0) that is one division, M_axis pb sign(...) / |pb (M0 + Pi) + pa|.
    double en = e[n];
    double num, den, side;
    if (en < 1.e-7) {
      const double P = 1.e-7 + Pi[n];
      num = Mi[n]; den = M0[n] + P; side = 1.e-7 + P;
    } else if (EOS == EOS_CONFORMAL) {
      const double P = en / 3 + Pi[n];
      num = Mi[n]; den = M0[n] + P; side = en + P;
    } else {
      double pa, pb;
      qcd_poly_p(en, pa, pb);
      num = Mi[n] * pb; den = fma(pb, M0[n] + Pi[n], pa); side = fma(pb, en + Pi[n], pa);
    }
    w[n] = (side < 0 ? -num : num) / fabs(den);
  }
}

// ------------------------------------------------------------------------------------
// Limiter (FluxLimiter.cu:17-39): generalised minmod, sign(0) = +1.
// ------------------------------------------------------------------------------------
// minmod(left, minmod(ctr, right)) of FluxLimiter.cu:33-38 in closed form: 0 unless the
// three slopes have the same sign, else that sign times the smallest magnitude. The sign
// test is done on the sign bits (integer pipe) and the magnitude is two min operations, so
// the FP64 pipe -- the stage kernel's bottleneck -- sees two min operations instead of four
// min/max, two compares and two selects. The values are the reference's, except that where
// all three are negative and one of them is -0 the result is -0 instead of +0 (the same
// number in every sum and product it enters).
__device__ __forceinline__ unsigned sign_bit(double x) { return (unsigned)__double2hiint(x) >> 31; }
__device__ __forceinline__ unsigned sign_bit(float x) { return (unsigned)__float_as_int(x) >> 31; }
__device__ __forceinline__ double with_sign_of(double m, double s) {
  return __hiloint2double(__double2hiint(m) | (__double2hiint(s) & (int)0x80000000), __double2loint(m));
}
__device__ __forceinline__ float with_sign_of(float m, float s) {
  return __int_as_float(__float_as_int(m) | (__float_as_int(s) & (int)0x80000000));
}
// With theta > 0 (the C ABI rejects anything else) the slopes theta (y - x) and theta (z - y)
// have the signs of the differences, and rounding is monotonic, so
// min(|theta a|, |theta b|) = theta min(|a|, |b|) exactly: one multiplication by theta.
// limited_slope2 returns twice the slope, from theta2 = 2 theta: the centred slope (z - x)/2
// then needs no halving, and callers fold the 1/2 into a factor they apply anyway (the
// half-cell states q +- D/2 become q +- D2/4, a derivative D/dx becomes D2 (1/(2 dx))).
// Power-of-two scalings commute with rounding, so every value is the same.
template <class R>
__device__ __forceinline__ R slope2_from_differences(R theta2, R dl, R dc, R dr) {
  const unsigned sl = sign_bit(dl);
  const R m = fmin(theta2 * fmin(fabs(dl), fabs(dr)), fabs(dc));
  return ((sl ^ sign_bit(dc)) | (sl ^ sign_bit(dr))) ? R(0) : with_sign_of(m, dl);
}
template <class R>
__device__ __forceinline__ R limited_slope2(R theta2, R x, R y, R z) {
  return slope2_from_differences(theta2, y - x, z - x, z - y);
}

}  // namespace gvh

// ====================================================================================
// Single-precision equation of state used by the mixed-precision path's source-term
// algebra (temperature, c_s^2 and zeta/s of the cell).
// ====================================================================================
namespace gvh {

// Coefficients of the QCD fits (EquationOfState.cu), index k = power of e, as floats.
__constant__ float kPa_f[13] = {-0.25181736420168666f, 9737.845799644809f, 1.077580993288114e6f,
                                3.1729694865420084e6f, 1.6357487344679043e6f, 334334.4309240126f,
                                41913.439282708554f, 6340.448389300905f, 141.5073484468774f,
                                0.7158279081255019f, 0.0009417586777847889f, 3.1188455176941583e-7f,
                                1.9531729608963267e-11f};
__constant__ float kPb_f[13] = {45829.44617893836f, 4.0574329080826794e6f, 2.0931169138134286e7f,
                                1.3512402226067686e7f, 1.7851642641834426e6f, 278581.2989342773f,
                                26452.34905933697f, 499.04919730607065f, 2.3405487982094204f,
                                0.002962497695527404f, 9.601103399348206e-7f, 5.928138360995685e-11f,
                                3.2581066229887368e-18f};
__constant__ float kCn_f[14] = {5.191934309650155e-32f, 4.123605749683891e-23f, 3.1955868410879504e-16f,
                                1.4170364808063119e-10f, 6.087136671592452e-6f, 0.02969737949090831f,
                                15.382615282179595f, 460.6487249985994f, 1612.4245252438795f,
                                275.0492627924299f, 58.60283714484669f, 6.504847576502024f,
                                0.03009027913262399f, 8.189430244031285e-6f};
__constant__ float kCd_f[14] = {1.4637868900982493e-30f, 6.716598285341542e-22f, 3.5477700458515908e-15f,
                                1.1225580509306008e-9f, 0.00003551782901018317f, 0.13653226327408863f,
                                60.85769171450653f, 1800.5461219450308f, 15190.225535036281f,
                                590.2572000057821f, 293.99144775704605f, 21.461303090563028f,
                                0.09301685073435291f, 0.000024810902623582917f};
__constant__ float kTn_f[12] = {1.510073201405604e-29f, 8.014062800678687e-18f, 2.4954778310451065e-10f,
                                0.000063810382643387f, 0.4873490574161924f, 207.48582344326206f,
                                6686.07424325115f, 14109.766109389702f, 1471.6180520527757f,
                                14.055788949565482f, 0.015421252394182246f, 1.5780479034557783e-6f};
__constant__ float kTd_f[12] = {7.558667139355393e-28f, 1.3686372302041508e-16f, 2.998130743142826e-9f,
                                0.0005036835870305458f, 2.316902328874072f, 578.0778724946719f,
                                11179.193315394154f, 17965.67607192861f, 1051.0730543534657f,
                                5.916312075925817f, 0.003778342768228011f, 1.8472801679382593e-7f};

// num(e)/den(e) for polynomials of degree N-1 in float. Above e = 1 both are divided by
// e^(N-1) and evaluated in y = 1/e, which keeps every partial sum inside float range (the
// degree-13 sums alone reach ~1e38 near e ~ 2000 fm^-4).
template <int N>
__device__ __forceinline__ void poly_pair_f(const float *num, const float *den, float e, float &pn, float &pd) {
  if (e <= 1.f) {
    pn = num[N - 1];
    pd = den[N - 1];
#pragma unroll
    for (int k = N - 2; k >= 0; --k) {
      pn = fmaf(pn, e, num[k]);
      pd = fmaf(pd, e, den[k]);
    }
  } else {
    const float y = __fdividef(1.f, e);
    pn = num[0];
    pd = den[0];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      pn = fmaf(pn, y, num[k]);
      pd = fmaf(pd, y, den[k]);
    }
  }
}

template <int EOS>
__device__ __forceinline__ float eq_pressure(float e) {
  if (EOS == EOS_CONFORMAL) return e / 3.f;
  float a, b;
  poly_pair_f<13>(kPa_f, kPb_f, e, a, b);
  return __fdividef(a, b);
}

template <int EOS>
__device__ __forceinline__ float sound_speed2(float e) {
  if (EOS == EOS_CONFORMAL) return 0.f;
  float c, d;
  poly_pair_f<14>(kCn_f, kCd_f, e, c, d);
  return __fdividef(c, d);
}

template <int EOS>
__device__ __forceinline__ float temperature(float e) {
  if (EOS == EOS_CONFORMAL) return sqrtf(sqrtf(e * (float)(1.0 / kEosFactor)));
  float a, b;
  poly_pair_f<12>(kTn_f, kTd_f, e, a, b);
  return __fdividef(a, b);
}

__device__ __forceinline__ float bulk_zeta_over_s(float T) {
  float x = T * (float)(1.0 / 1.01355);
  if (x > 1.05f) return 0.9f * __expf(-(x - 1) * 40.f) + 0.25f * __expf(-(x - 1) * (float)(1.0 / 0.13)) + 0.001f;
  else if (x < 0.995f) return 0.9f * __expf((x - 1) * 400.f) + 0.22f * __expf((x - 1) * (float)(1.0 / 0.022)) + 0.03f;
  return -13.77f * x * x + 27.55f * x - 13.45f;
}

}  // namespace gvh
