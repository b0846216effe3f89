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

// p(e): EquationOfState.cu:30-80 (Wuppertal-Budapest rational fit, nested fma in double);
// conformal p = e/3.
template <int EOS>
__device__ __forceinline__ double eq_pressure(double e) {
  if (EOS == EOS_CONFORMAL) return e / 3;
  double e1 = e, e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e;
  double e7 = e6 * e, e8 = e7 * e, e9 = e8 * e, e10 = e9 * e, e11 = e10 * e, e12 = e11 * e;
  double a = fma(1.9531729608963267e-11, e12, fma(3.1188455176941583e-7, e11, fma(0.0009417586777847889, e10,
             fma(0.7158279081255019, e9, fma(141.5073484468774, e8, fma(6340.448389300905, e7,
             fma(41913.439282708554, e6, fma(334334.4309240126, e5, fma(1.6357487344679043e6, e4,
             fma(3.1729694865420084e6, e3, fma(1.077580993288114e6, e2, fma(9737.845799644809, e1,
             -0.25181736420168666))))))))))));
  double b = fma(3.2581066229887368e-18, e12, fma(5.928138360995685e-11, e11, fma(9.601103399348206e-7, e10,
             fma(0.002962497695527404, e9, fma(2.3405487982094204, e8, fma(499.04919730607065, e7,
             fma(26452.34905933697, e6, fma(278581.2989342773, e5, fma(1.7851642641834426e6, e4,
             fma(1.3512402226067686e7, e3, fma(2.0931169138134286e7, e2, fma(4.0574329080826794e6, e1,
             45829.44617893836))))))))))));
  return a / b;
}

// c_s^2(e): EquationOfState.cu:82-116. The conformal branch of the reference returns the
// integer quotient 1/3 == 0 (EquationOfState.cu:114) and that value is kept.
template <int EOS>
__device__ __forceinline__ double sound_speed2(double e) {
  if (EOS == EOS_CONFORMAL) return 0.0;
  double e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e, e7 = e6 * e;
  double e8 = e7 * e, e9 = e8 * e, e10 = e9 * e, e11 = e10 * e, e12 = e11 * e, e13 = e12 * e;
  return (5.191934309650155e-32 + 4.123605749683891e-23 * e + 3.1955868410879504e-16 * e2
          + 1.4170364808063119e-10 * e3 + 6.087136671592452e-6 * e4 + 0.02969737949090831 * e5
          + 15.382615282179595 * e6 + 460.6487249985994 * e7 + 1612.4245252438795 * e8
          + 275.0492627924299 * e9 + 58.60283714484669 * e10 + 6.504847576502024 * e11
          + 0.03009027913262399 * e12 + 8.189430244031285e-6 * e13)
       / (1.4637868900982493e-30 + 6.716598285341542e-22 * e + 3.5477700458515908e-15 * e2
          + 1.1225580509306008e-9 * e3 + 0.00003551782901018317 * e4 + 0.13653226327408863 * e5
          + 60.85769171450653 * e6 + 1800.5461219450308 * e7 + 15190.225535036281 * e8
          + 590.2572000057821 * e9 + 293.99144775704605 * e10 + 21.461303090563028 * e11
          + 0.09301685073435291 * e12 + 0.000024810902623582917 * e13);
}

// T(e): EquationOfState.cu:118-148; conformal T = (e/13.8997)^(1/4).
template <int EOS>
__device__ __forceinline__ double temperature(double e) {
  if (EOS == EOS_CONFORMAL) return pow(e / kEosFactor, 0.25);
  double e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e, e7 = e6 * e;
  double e8 = e7 * e, e9 = e8 * e, e10 = e9 * e, e11 = e10 * e;
  return (1.510073201405604e-29 + 8.014062800678687e-18 * e + 2.4954778310451065e-10 * e2
          + 0.000063810382643387 * e3 + 0.4873490574161924 * e4 + 207.48582344326206 * e5
          + 6686.07424325115 * e6 + 14109.766109389702 * e7 + 1471.6180520527757 * e8
          + 14.055788949565482 * e9 + 0.015421252394182246 * e10 + 1.5780479034557783e-6 * e11)
       / (7.558667139355393e-28 + 1.3686372302041508e-16 * e + 2.998130743142826e-9 * e2
          + 0.0005036835870305458 * e3 + 2.316902328874072 * e4 + 578.0778724946719 * e5
          + 11179.193315394154 * e6 + 17965.67607192861 * e7 + 1051.0730543534657 * e8
          + 5.916312075925817 * e9 + 0.003778342768228011 * e10 + 1.8472801679382593e-7 * e11);
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
enum : unsigned { STATUS_NAN = 1u, STATUS_NEWTON = 2u };

// Newton iteration cap. The reference allows 10^6 iterations and damps after 5x10^5
// (EnergyMomentumTensor.cu:15,37-38); converged cells take a handful. Hitting the cap
// returns the last iterate (as the reference does at its cap) and raises STATUS_NEWTON.
constexpr int kNewtonMaxIters = 500;

// e from (M0, M, Pi): EnergyMomentumTensor.cu:18-48.
template <int EOS>
__device__ __forceinline__ double energy_from_conserved(double ePrev, double M0, double M, double Pi,
                                                        unsigned &status) {
  if (EOS == EOS_CONFORMAL) return fabs(sqrt(fabs(4 * M0 * M0 - 3 * M)) - M0);
  double e0 = ePrev;
  for (int j = 0; j < kNewtonMaxIters; ++j) {
    double p = eq_pressure<EOS>(e0);
    double cs2 = sound_speed2<EOS>(e0);
    double cst2 = p / e0;
    double A = fma(M0, 1 - cst2, Pi);
    double B = fma(M0, M0 + Pi, -M);
    double H = sqrt(fabs(A * A + 4 * cst2 * B));
    double D = (A - H) / (2 * cst2);
    double f = e0 + D;
    double fp = 1 - ((cs2 - cst2) * (B + D * H - ((cs2 - cst2) * cst2 * D * M0) / e0)) / (cst2 * e0 * H);
    double e = e0 - f / fp;
    if (fabs(e - e0) <= 0.001 * fabs(e)) return e;
    e0 = e;
  }
  status |= STATUS_NEWTON;
  return e0;
}

struct Prim {
  double e, p, ut, ux, uy, un;
};

// getInferredVariables: EnergyMomentumTensor.cu:50-108. The Pi clamp guarded by the
// never-defined `Pi` macro (lines 82-85) is not part of the reference's behaviour.
template <int EOS>
__device__ __forceinline__ Prim inferred(double t, double ttt, double ttx, double tty, double ttn, double pitt,
                                         double pitx, double pity, double pitn, double Pi, double ePrev,
                                         unsigned &status) {
  Prim r;
  double M0 = ttt - pitt;
  double M1 = ttx - pitx;
  double M2 = tty - pity;
  double M3 = ttn - pitn;
  double M = M1 * M1 + M2 * M2 + t * t * M3 * M3;
  if (ePrev <= 0.1) r.e = M0 - M / M0;
  else r.e = energy_from_conserved<EOS>(ePrev, M0, M, Pi, status);
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

// ------------------------------------------------------------------------------------
// Limiter (FluxLimiter.cu:17-39): generalised minmod, sign(0) = +1.
// ------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R sgn1(R x) { return x < R(0) ? R(-1) : R(1); }
template <class R>
__device__ __forceinline__ R minmod2(R x, R y) { return (sgn1(x) + sgn1(y)) * fmin(fabs(x), fabs(y)) / R(2); }
template <class R>
__device__ __forceinline__ R limited_slope(R theta, R x, R y, R z) {
  R left = theta * (y - x);
  R ctr = (z - x) / R(2);
  R right = theta * (z - y);
  return minmod2(left, minmod2(ctr, right));
}

}  // namespace gvh
