/*
 * kt_oracle.c -- CPU restatement of gpu-vh's 3+1D Milne Kurganov-Tadmor RK2 step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the oracle: the parity tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it to check (or time beside) the CUDA
 * path. Nothing in the product links it, and the product never falls back to it.
 *
 * It restates, in plain C and in double precision, the reference's FP64 semantics of
 * the hot path: the reference compiled with PRECISION double and its float intrinsics
 * mapped to their double versions (fminf -> fmin, sqrtf -> sqrt, powf -> pow, ...).
 * Every expression keeps the reference's operation order and its float literals
 * (0.2f, 0.333333f, 1.6f, ...) so that, compiled without FMA contraction, it agrees bit
 * for bit with the reference's own sources built for the CPU (oracle/_ref). It is
 * pinned against that build by tests/test_oracle_pin.py and tests/golden/.
 *
 * Layout: the reference's ghosted SoA lattice, ncx = nx+4, index i + ncx*(j + ncy*k)
 * (DynamicalVariables.cu:32-35, LatticeParameters.h:13-15). Conserved components in
 * CONSERVED_VARIABLES order (DynamicalVariables.cuh:50-71): ttt ttx tty ttn, then
 * pitt pitx pity pitn pixx pixy pixn piyy piyn pinn when shear is evolved, then Pi when
 * bulk is evolved (index 14; the reference hard-codes that slot,
 * EnergyMomentumTensor.cu:72).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#include "kt_oracle.h"

#define NG_M 2 /* LatticeParameters.h:13 */

/* TransportCoefficients.cuh:14-18 */
static const double DELTA_PIPI = 1.33333;
static const double TAU_PIPI = 1.42857;
static const double LAMBDA_PIPI_BULK = 1.2; /* lambda_piPi */
static const double DELTA_PIPI_BULK = 0.666667; /* delta_PiPi */

/* EquationOfState.cuh:20 */
#define EOS_FACTOR 13.8997

/* ---------------------------------------------------------------------------------- */
/* Equation of state (EquationOfState.cu)                                               */
/* ---------------------------------------------------------------------------------- */

/* EquationOfState.cu:30-80 -- Wuppertal-Budapest rational fit p(e) evaluated as nested
 * fma in double; conformal p = e/3. */
double kt_equilibrium_pressure(const kt_params *P, double e) {
	if (P->conformal) return e / 3;
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

/* EquationOfState.cu:82-116. The conformal branch returns the C++ integer quotient 1/3,
 * i.e. 0 (EquationOfState.cu:114); that value feeds the bulk coefficients below. */
double kt_speed_of_sound_squared(const kt_params *P, double e) {
	if (P->conformal) return 0.0;
	double e1 = e, e2 = e * e1, e3 = e2 * e1, e4 = e3 * e1, e5 = e4 * e1, e6 = e5 * e1, e7 = e6 * e1;
	double e8 = e7 * e1, e9 = e8 * e1, e10 = e9 * e1, e11 = e10 * e1, e12 = e11 * e1, e13 = e12 * e1;
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

/* EquationOfState.cu:118-148; conformal T = (e/13.8997)^(1/4). */
double kt_effective_temperature(const kt_params *P, double e) {
	if (P->conformal) return pow(e / EOS_FACTOR, 0.25);
	double e1 = e, e2 = e * e1, e3 = e2 * e1, e4 = e3 * e1, e5 = e4 * e1, e6 = e5 * e1;
	double e7 = e6 * e1, e8 = e7 * e1, e9 = e8 * e1, e10 = e9 * e1, e11 = e10 * e1;
	return (1.510073201405604e-29 + 8.014062800678687e-18 * e + 2.4954778310451065e-10 * e2
	        + 0.000063810382643387 * e3 + 0.4873490574161924 * e4 + 207.48582344326206 * e5
	        + 6686.07424325115 * e6 + 14109.766109389702 * e7 + 1471.6180520527757 * e8
	        + 14.055788949565482 * e9 + 0.015421252394182246 * e10 + 1.5780479034557783e-6 * e11)
	     / (7.558667139355393e-28 + 1.3686372302041508e-16 * e + 2.998130743142826e-9 * e2
	        + 0.0005036835870305458 * e3 + 2.316902328874072 * e4 + 578.0778724946719 * e5
	        + 11179.193315394154 * e6 + 17965.67607192861 * e7 + 1051.0730543534657 * e8
	        + 5.916312075925817 * e9 + 0.003778342768228011 * e10 + 1.8472801679382593e-7 * e11);
}

/* EquationOfState.cu:150-204; conformal e = 13.8997 T^4. */
double kt_equilibrium_energy_density(const kt_params *P, double T) {
	if (P->conformal) return EOS_FACTOR * pow(T, 4.0);
	double T1 = T, T2 = T1 * T1, T3 = T2 * T1, T4 = T3 * T1, T5 = T4 * T1, T6 = T5 * T1, T7 = T6 * T1;
	double T8 = T7 * T1, T9 = T8 * T1, T10 = T9 * T1, T11 = T10 * T1, T12 = T11 * T1, T13 = T12 * T1;
	double T14 = T13 * T1, T15 = T14 * T1, T16 = T15 * T1, T17 = T16 * T1, T18 = T17 * T1, T19 = T18 * T1;
	double T20 = T19 * T1, T21 = T20 * T1, T22 = T21 * T1, T23 = T22 * T1;
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

/* TransportCoefficients.cu:27-36 -- zeta/s(T), piecewise in x = T/1.01355. */
double kt_bulk_zeta_over_s(double T) {
	double x = T / 1.01355;
	if (x > 1.05) return 0.9 * exp(-(x - 1) / 0.025) + 0.25 * exp(-(x - 1) / 0.13) + 0.001;
	else if (x < 0.995) return 0.9 * exp((x - 1) / 0.0025) + 0.22 * exp((x - 1) / 0.022) + 0.03;
	else return -13.77 * x * x + 27.55 * x - 13.45;
}

/* ---------------------------------------------------------------------------------- */
/* Primitive recovery (EnergyMomentumTensor.cu)                                         */
/* ---------------------------------------------------------------------------------- */

/* EnergyMomentumTensor.cu:18-48. Newton iteration for e with |de| <= 1e-3 |e| as the stop
 * test, damped by 0.9 after MAX_ITERS/2; conformal closed form. */
double kt_energy_density_from_conserved(const kt_params *P, double ePrev, double M0, double M, double Pi) {
	if (P->conformal) return fabs(sqrt(fabs(4 * M0 * M0 - 3 * M)) - M0);
	const int MAX_ITERS = 1000000;
	double e0 = ePrev;
	for (int j = 0; j < MAX_ITERS; ++j) {
		double p = kt_equilibrium_pressure(P, e0);
		double cs2 = kt_speed_of_sound_squared(P, e0);
		double cst2 = p / e0;
		double A = fma(M0, 1 - cst2, Pi);
		double B = fma(M0, M0 + Pi, -M);
		double H = sqrt(fabs(A * A + 4 * cst2 * B));
		double D = (A - H) / (2 * cst2);
		double f = e0 + D;
		double fp = 1 - ((cs2 - cst2) * (B + D * H - ((cs2 - cst2) * cst2 * D * M0) / e0)) / (cst2 * e0 * H);
		double e;
		if (j < MAX_ITERS / 2) e = e0 - f / fp;
		else e = e0 - 0.9 * f / fp;
		if (fabs(e - e0) <= 0.001 * fabs(e)) return e;
		e0 = e;
	}
	return e0;
}

/* EnergyMomentumTensor.cu:50-108. The bulk clamp guarded by `#ifdef Pi` (lower case,
 * lines 82-85) is never compiled in the reference and is omitted here too. */
void kt_get_inferred_variables(const kt_params *P, double t, const double *q, double ePrev, double *e, double *p,
                               double *ut, double *ux, double *uy, double *un) {
	double ttt = q[0], ttx = q[1], tty = q[2], ttn = q[3];
	double pitt = 0, pitx = 0, pity = 0, pitn = 0;
	if (P->shear) { pitt = q[4]; pitx = q[5]; pity = q[6]; pitn = q[7]; }
	double Pi = P->bulk ? q[14] : 0;
	double M0 = ttt - pitt;
	double M1 = ttx - pitx;
	double M2 = tty - pity;
	double M3 = ttn - pitn;
	double M = M1 * M1 + M2 * M2 + t * t * M3 * M3;
	if (ePrev <= 0.1) *e = M0 - M / M0;
	else *e = kt_energy_density_from_conserved(P, ePrev, M0, M, Pi);
	*p = kt_equilibrium_pressure(P, *e);
	if (*e < 1.e-7) { *e = 1.e-7; *p = 1.e-7; }
	double Pt = *p + Pi;
	double E = 1 / (*e + Pt);
	*ut = sqrt(fabs((M0 + Pt) * E));
	double E2 = E / (*ut);
	*ux = M1 * E2;
	*uy = M2 * E2;
	*un = M3 * E2;
}

/* EnergyMomentumTensor.cu:159-207 (the components the path uses). */
static double Ttt(double e, double p, double ut, double pitt) { return (e + p) * ut * ut - p + pitt; }
static double Ttx(double e, double p, double ut, double ux, double pitx) { return (e + p) * ut * ux + pitx; }
static double Tty(double e, double p, double ut, double uy, double pity) { return (e + p) * ut * uy + pity; }
static double Ttn(double e, double p, double ut, double un, double pitn) { return (e + p) * ut * un + pitn; }
static double Tnn(double e, double p, double un, double pinn, double t) { return (e + p) * un * un + p / t / t + pinn; }

/* ---------------------------------------------------------------------------------- */
/* Limiter and KT flux                                                                   */
/* ---------------------------------------------------------------------------------- */

/* FluxLimiter.cu:17-39: generalised minmod with sign(0) = +1. */
static double sgn(double x) { return x < 0 ? -1 : 1; }
static double minmod(double x, double y) { return (sgn(x) + sgn(y)) * fmin(fabs(x), fabs(y)) / 2; }
static double approximate_derivative(double theta, double x, double y, double z) {
	double left = theta * (y - x);
	double ctr = (z - x) / 2;
	double right = theta * (z - y);
	return minmod(left, minmod(ctr, right));
}

/* SemiDiscreteKurganovTadmorScheme.cu:15-57 with HalfSiteExtrapolation.cu:15-30,
 * LocalPropagationSpeed.cu:15-24, SpectralRadius.cu:17-30, FluxFunctions.cu:18-31.
 * `stencil` holds the 5 points (i-2..i+2) of each component; `forward` selects the face
 * i+1/2 (else i-1/2); `axis` 1,2,3 = x,y,eta. */
static void kt_flux(const kt_params *P, int nq, const double *stencil, double *H, int forward, int axis, double t,
                    double ePrev, double *a_out) {
	double qR[KT_MAX_NQ], qL[KT_MAX_NQ];
	const double th = P->theta;
	for (int n = 0; n < nq; ++n) {
		const double *d = stencil + 5 * n;
		double qmm = d[0], qm = d[1], q = d[2], qp = d[3], qpp = d[4];
		if (forward) {
			qR[n] = qp - approximate_derivative(th, q, qp, qpp) / 2;
			qL[n] = q + approximate_derivative(th, qm, q, qp) / 2;
		} else {
			qR[n] = q - approximate_derivative(th, qm, q, qp) / 2;
			qL[n] = qm + approximate_derivative(th, qmm, qm, q) / 2;
		}
	}
	double eR, pR, utR, uR[3], eL, pL, utL, uL[3];
	kt_get_inferred_variables(P, t, qR, ePrev, &eR, &pR, &utR, &uR[0], &uR[1], &uR[2]);
	kt_get_inferred_variables(P, t, qL, ePrev, &eL, &pL, &utL, &uL[0], &uL[1], &uL[2]);
	double vR = uR[axis - 1], vL = uL[axis - 1];
	double a = fmax(fabs(vL / utL), fabs(vR / utR));
	*a_out = a;
	for (int n = 0; n < nq; ++n) {
		double FqR = vR * qR[n] / utR;
		double FqL = vL * qL[n] / utL;
		double res = FqR + FqL - a * (qR[n] - qL[n]);
		res /= 2;
		H[n] = res;
	}
}

/* ---------------------------------------------------------------------------------- */
/* Source terms (SourceTerms.cu)                                                        */
/* ---------------------------------------------------------------------------------- */

/* SourceTerms.cu:29-256 -- right-hand side of the pi^{mu nu} (10) and Pi equations. */
static void pimunu_source(const kt_params *P, double *rhs, double t, double e, double p, double ut, double ux,
                          double uy, double un, double utp, double uxp, double uyp, double unp, double pitt,
                          double pitx, double pity, double pitn, double pixx, double pixy, double pixn, double piyy,
                          double piyn, double pinn, double Pi, double dxut, double dyut, double dnut, double dxux,
                          double dyux, double dnux, double dxuy, double dyuy, double dnuy, double dxun, double dyun,
                          double dnun, double dkvk) {
	const double dt = P->dt;
	double T = kt_effective_temperature(P, e);
	double taupiInv = (double)0.2f * (T / P->etabar);
	double beta_pi = (double)0.2f * (e + p);

	double cs2 = kt_speed_of_sound_squared(P, e);
	double a = (double)0.333333f - cs2;
	double a2 = a * a;
	double beta_Pi = 15.0 * a2 * (e + p);
	double lambda_Pipi = (double)1.6f * a;
	double zetabar = kt_bulk_zeta_over_s(T);
	double tauPiInv = 15 * a2 * (T / zetabar);

	double ut2 = ut * ut, un2 = un * un, t2 = t * t, t3 = t * t2;

	double dtut = (ut - utp) / dt;
	double dtux = (ux - uxp) / dt;
	double dtuy = (uy - uyp) / dt;
	double dtun = (un - unp) / dt;

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

	double wtx = (-dtux - dxut + ut * dux - ux * dut - t * un2 * ux) / 2.0;
	double wty = (-dtuy - dyut + ut * duy - uy * dut - t * un2 * uy) / 2.0;
	double wtn = (-t2 * dtun - 2.0 * t * un - dnut - ut * Dun - t2 * un * dut - t3 * un * un2) / 2.0;
	double wxy = (dxuy - dyux + ux * duy - uy * dux) / 2.0;
	double wxn = (t2 * dxun - dnux - ux * Dun - t2 * un * dux) / 2.0;
	double wyn = (t2 * dyun - dnuy - uy * Dun - t2 * un * duy) / 2.0;
	double wxt = wtx, wyt = wty, wnt = wtn / t2, wyx = -wxy, wnx = -wxn / t2, wny = -wyn / t2;

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

	double I2tt = theta * pitt, I2tx = theta * pitx, I2ty = theta * pity, I2tn = theta * pitn;
	double I2xx = theta * pixx, I2xy = theta * pixy, I2xn = theta * pixn, I2yy = theta * piyy;
	double I2yn = theta * piyn, I2nn = theta * pinn;

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

	double Itt = I1tt + DELTA_PIPI * I2tt - I3tt + TAU_PIPI * I4tt - LAMBDA_PIPI_BULK * Pi * stt;
	double Itx = I1tx + DELTA_PIPI * I2tx - I3tx + TAU_PIPI * I4tx - LAMBDA_PIPI_BULK * Pi * stx;
	double Ity = I1ty + DELTA_PIPI * I2ty - I3ty + TAU_PIPI * I4ty - LAMBDA_PIPI_BULK * Pi * sty;
	double Itn = I1tn + DELTA_PIPI * I2tn - I3tn + TAU_PIPI * I4tn - LAMBDA_PIPI_BULK * Pi * stn;
	double Ixx = I1xx + DELTA_PIPI * I2xx - I3xx + TAU_PIPI * I4xx - LAMBDA_PIPI_BULK * Pi * sxx;
	double Ixy = I1xy + DELTA_PIPI * I2xy - I3xy + TAU_PIPI * I4xy - LAMBDA_PIPI_BULK * Pi * sxy;
	double Ixn = I1xn + DELTA_PIPI * I2xn - I3xn + TAU_PIPI * I4xn - LAMBDA_PIPI_BULK * Pi * sxn;
	double Iyy = I1yy + DELTA_PIPI * I2yy - I3yy + TAU_PIPI * I4yy - LAMBDA_PIPI_BULK * Pi * syy;
	double Iyn = I1yn + DELTA_PIPI * I2yn - I3yn + TAU_PIPI * I4yn - LAMBDA_PIPI_BULK * Pi * syn;
	double Inn = I1nn + DELTA_PIPI * I2nn - I3nn + TAU_PIPI * I4nn - LAMBDA_PIPI_BULK * Pi * snn;

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

	double dPi = -beta_Pi * theta - Pi * tauPiInv - DELTA_PIPI_BULK * Pi * theta + lambda_Pipi * ps;

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
	if (P->bulk) rhs[10] = dPi / ut + Pi * dkvk;
}

/* ---------------------------------------------------------------------------------- */
/* Lattice state                                                                         */
/* ---------------------------------------------------------------------------------- */

struct kt_lattice {
	kt_params P;
	int nq, ncx, ncy, ncz;
	size_t ng;
	double *q[KT_MAX_NQ], *Q[KT_MAX_NQ], *qS[KT_MAX_NQ];
	double *e, *p, *u[4], *up[4], *uS[4];
	double *block;
	/* max over the axes of a / dx_axis per cell in the predictor stage (the CFL bound,
	 * SpectralRadius.cu:17-30), and its running maximum over cells and steps */
	double *speed;
	double speed_max;
};

static int idx(const kt_lattice *L, int i, int j, int k) { return i + L->ncx * (j + L->ncy * k); }

int kt_nq(const kt_params *P) { return 4 + (P->shear ? 10 : 0) + (P->bulk ? 1 : 0); }

kt_lattice *kt_create(const kt_params *P) {
	if (P->nx < 1 || P->ny < 1 || P->nz < 1) return NULL;
	if (P->bulk && !P->shear) return NULL; /* the reference's slot 14 for Pi needs the shear block */
	kt_lattice *L = (kt_lattice *)calloc(1, sizeof(kt_lattice));
	L->P = *P;
	L->nq = kt_nq(P);
	L->ncx = P->nx + 4; L->ncy = P->ny + 4; L->ncz = P->nz + 4;
	L->ng = (size_t)L->ncx * L->ncy * L->ncz;
	size_t nbuf = 3 * (size_t)L->nq + 2 + 12;
	L->block = (double *)calloc(nbuf * L->ng, sizeof(double));
	double *b = L->block;
	for (int n = 0; n < L->nq; ++n) { L->q[n] = b; b += L->ng; }
	for (int n = 0; n < L->nq; ++n) { L->Q[n] = b; b += L->ng; }
	for (int n = 0; n < L->nq; ++n) { L->qS[n] = b; b += L->ng; }
	L->e = b; b += L->ng;
	L->p = b; b += L->ng;
	for (int m = 0; m < 4; ++m) { L->u[m] = b; b += L->ng; }
	for (int m = 0; m < 4; ++m) { L->up[m] = b; b += L->ng; }
	for (int m = 0; m < 4; ++m) { L->uS[m] = b; b += L->ng; }
	L->speed = (double *)calloc(L->ng, sizeof(double));
	return L;
}

void kt_destroy(kt_lattice *L) {
	if (!L) return;
	free(L->block);
	free(L->speed);
	free(L);
}

size_t kt_num_cells(const kt_lattice *L) { return L->ng; }

/* GhostCells.cu:15-144 -- zero-gradient copies of every field into the two ghost layers
 * of each face (edges and corners untouched). */
static void ghost_copy(kt_lattice *L, double **q, double *e, double *p, double **u, int s, int sb) {
	e[s] = e[sb]; p[s] = p[sb];
	for (int m = 0; m < 4; ++m) u[m][s] = u[m][sb];
	for (int n = 0; n < L->nq; ++n) q[n][s] = q[n][sb];
}
static void set_ghost_cells(kt_lattice *L, double **q, double *e, double *p, double **u) {
	const int nx = L->P.nx, ny = L->P.ny, nz = L->P.nz;
	for (int k = 2; k < nz + 2; ++k)
		for (int j = 2; j < ny + 2; ++j) {
			for (int i = 0; i <= 1; ++i) ghost_copy(L, q, e, p, u, idx(L, i, j, k), idx(L, 2, j, k));
			for (int i = nx + 2; i <= nx + 3; ++i) ghost_copy(L, q, e, p, u, idx(L, i, j, k), idx(L, nx + 1, j, k));
		}
	for (int k = 2; k < nz + 2; ++k)
		for (int i = 2; i < nx + 2; ++i) {
			for (int j = 0; j <= 1; ++j) ghost_copy(L, q, e, p, u, idx(L, i, j, k), idx(L, i, 2, k));
			for (int j = ny + 2; j <= ny + 3; ++j) ghost_copy(L, q, e, p, u, idx(L, i, j, k), idx(L, i, ny + 1, k));
		}
	for (int j = 2; j < ny + 2; ++j)
		for (int i = 2; i < nx + 2; ++i) {
			for (int k = 0; k <= 1; ++k) ghost_copy(L, q, e, p, u, idx(L, i, j, k), idx(L, i, j, 2));
			for (int k = nz + 2; k <= nz + 3; ++k) ghost_copy(L, q, e, p, u, idx(L, i, j, k), idx(L, i, j, nz + 1));
		}
}

/* SourceTerms.cu:569-755 (loadSourceTerms2) + EulerStep.cu:946-1009
 * (eulerStepKernelSource_1D): out = q + dt * S at one interior cell. */
static void euler_source_cell(kt_lattice *L, int s, double t, double **cur, double **upd, const double *e,
                              const double *p, double **u, double **up) {
	const kt_params *P = &L->P;
	const int nq = L->nq;
	double Q[KT_MAX_NQ], S[KT_MAX_NQ];
	for (int n = 0; n < nq; ++n) Q[n] = cur[n][s];
	double ttt = Q[0], ttx = Q[1], tty = Q[2], ttn = Q[3];
	double pitt = 0, pitx = 0, pity = 0, pitn = 0, pixx = 0, pixy = 0, pixn = 0, piyy = 0, piyn = 0, pinn = 0;
	if (P->shear) {
		pitt = Q[4]; pitx = Q[5]; pity = Q[6]; pitn = Q[7]; pixx = Q[8];
		pixy = Q[9]; pixn = Q[10]; piyy = Q[11]; piyn = Q[12]; pinn = Q[13];
	}
	double Pi = P->bulk ? Q[14] : 0;
	double pc = p[s], ut = u[0][s], ux = u[1][s], uy = u[2][s], un = u[3][s];
	const int sx = 1, sy = L->ncx, sz = L->ncx * L->ncy;
	const double th = P->theta;
	/* USE_APPROX_DERIVATIVE (SourceTerms.cu:27, 659-720): limited one-cell derivatives */
	double dxut = approximate_derivative(th, u[0][s - sx], ut, u[0][s + sx]) / P->dx;
	double dxux = approximate_derivative(th, u[1][s - sx], ux, u[1][s + sx]) / P->dx;
	double dxuy = approximate_derivative(th, u[2][s - sx], uy, u[2][s + sx]) / P->dx;
	double dxun = approximate_derivative(th, u[3][s - sx], un, u[3][s + sx]) / P->dx;
	double dyut = approximate_derivative(th, u[0][s - sy], ut, u[0][s + sy]) / P->dy;
	double dyux = approximate_derivative(th, u[1][s - sy], ux, u[1][s + sy]) / P->dy;
	double dyuy = approximate_derivative(th, u[2][s - sy], uy, u[2][s + sy]) / P->dy;
	double dyun = approximate_derivative(th, u[3][s - sy], un, u[3][s + sy]) / P->dy;
	double dnut = approximate_derivative(th, u[0][s - sz], ut, u[0][s + sz]) / P->dz;
	double dnux = approximate_derivative(th, u[1][s - sz], ux, u[1][s + sz]) / P->dz;
	double dnuy = approximate_derivative(th, u[2][s - sz], uy, u[2][s + sz]) / P->dz;
	double dnun = approximate_derivative(th, u[3][s - sz], un, u[3][s + sz]) / P->dz;
	double dxp = approximate_derivative(th, p[s - sx], pc, p[s + sx]) / P->dx;
	double dyp = approximate_derivative(th, p[s - sy], pc, p[s + sy]) / P->dy;
	double dnp = approximate_derivative(th, p[s - sz], pc, p[s + sz]) / P->dz;

	double tnn = Tnn(e[s], pc + Pi, un, pinn, t);
	double vx = ux / ut, vy = uy / ut, vn = un / ut;
	double dxvx = (dxux - vx * dxut) / ut;
	double dyvy = (dyuy - vy * dyut) / ut;
	double dnvn = (dnun - vn * dnut) / ut;
	double dkvk = dxvx + dyvy + dnvn;
	S[0] = -(ttt / t + t * tnn) + dkvk * (pitt - pc - Pi) - vx * dxp - vy * dyp - vn * dnp;
	S[1] = -ttx / t - dxp + dkvk * pitx;
	S[2] = -tty / t - dyp + dkvk * pity;
	S[3] = -3 * ttn / t - dnp / pow(t, 2) + dkvk * pitn;
	if (P->cartesian) { /* SourceTerms.cu:738-743 replaces the four Milne terms */
		S[0] = dkvk * (pitt - pc - Pi) - vx * dxp - vy * dyp - vn * dnp;
		S[1] = -dxp + dkvk * pitx;
		S[2] = -dyp + dkvk * pity;
		S[3] = -dnp + dkvk * pitn;
	}
	if (P->shear) {
		double rhs[11];
		pimunu_source(P, rhs, t, e[s], pc, ut, ux, uy, un, up[0][s], up[1][s], up[2][s], up[3][s], pitt, pitx, pity,
		              pitn, pixx, pixy, pixn, piyy, piyn, pinn, Pi, dxut, dyut, dnut, dxux, dyux, dnux, dxuy, dyuy,
		              dnuy, dxun, dyun, dnun, dkvk);
		for (int n = 4; n < nq; ++n) S[n] = rhs[n - 4];
	}
	for (int n = 0; n < nq; ++n) upd[n][s] = Q[n] + P->dt * S[n];
}

/* EulerStep.cu:1011-1277 (eulerStepKernelX_1D / Y_1D / Z_1D) with SourceTerms.cu:443-567
 * (loadSourceTermsX/Y/Z): out += dt * ( -(H(i+1/2) - H(i-1/2))/d + S_axis ). */
static void euler_axis_cell(kt_lattice *L, int s, int axis, double t, double **cur, double **upd, const double *e,
                            double **u) {
	const kt_params *P = &L->P;
	const int nq = L->nq;
	const int stride = axis == 1 ? 1 : axis == 2 ? L->ncx : L->ncx * L->ncy;
	const double d = axis == 1 ? P->dx : axis == 2 ? P->dy : P->dz;
	double I[5 * KT_MAX_NQ], H[KT_MAX_NQ], result[KT_MAX_NQ];
	for (int n = 0; n < nq; ++n)
		for (int o = 0; o < 5; ++o) I[5 * n + o] = cur[n][s + (o - 2) * stride];
	double af, ab;
	kt_flux(P, nq, I, H, 1, axis, t, e[s], &af);
	for (int n = 0; n < nq; ++n) result[n] = -H[n];
	kt_flux(P, nq, I, H, 0, axis, t, e[s], &ab);
	/* the CFL bound counts the axes with more than one cell (a one-cell axis has no faces) */
	const int n_axis = axis == 1 ? P->nx : axis == 2 ? P->ny : P->nz;
	if (n_axis > 1) L->speed[s] = fmax(L->speed[s], fmax(af, ab) * (1.0 / d));
	for (int n = 0; n < nq; ++n) {
		result[n] += H[n];
		result[n] /= d;
	}
	if (P->shear) {
		double fac = 1 / d / 2;
#define DER(c) ((I[5 * (c) + 3] - I[5 * (c) + 1]) * fac)
		double Sa[4];
		double ut = u[0][s];
		if (axis == 1) {
			double vx = u[1][s] / ut;
			double dxpitt = DER(4), dxpitx = DER(5), dxpity = DER(6), dxpitn = DER(7);
			double dxpixx = DER(8), dxpixy = DER(9), dxpixn = DER(10);
			if (!P->bulk) {
				Sa[0] = dxpitt * vx - dxpitx;
				Sa[1] = dxpitx * vx - dxpixx;
			} else {
				double dxPi = DER(14);
				Sa[0] = dxpitt * vx - dxpitx - vx * dxPi;
				Sa[1] = dxpitx * vx - dxpixx - dxPi;
			}
			Sa[2] = dxpity * vx - dxpixy;
			Sa[3] = dxpitn * vx - dxpixn;
		} else if (axis == 2) {
			double vy = u[2][s] / ut;
			double dypitt = DER(4), dypitx = DER(5), dypity = DER(6), dypitn = DER(7);
			double dypixy = DER(9), dypiyy = DER(11), dypiyn = DER(12);
			if (!P->bulk) {
				Sa[0] = dypitt * vy - dypity;
				Sa[2] = dypity * vy - dypiyy;
			} else {
				double dyPi = DER(14);
				Sa[0] = dypitt * vy - dypity - vy * dyPi;
				Sa[2] = dypity * vy - dypiyy - dyPi;
			}
			Sa[1] = dypitx * vy - dypixy;
			Sa[3] = dypitn * vy - dypiyn;
		} else {
			double vn = u[3][s] / ut;
			double dnpitt = DER(4), dnpitx = DER(5), dnpity = DER(6), dnpitn = DER(7);
			double dnpixn = DER(10), dnpiyn = DER(12), dnpinn = DER(13);
			if (!P->bulk) {
				Sa[0] = dnpitt * vn - dnpitn;
				Sa[3] = dnpitn * vn - dnpinn;
			} else {
				double dnPi = DER(14);
				Sa[0] = dnpitt * vn - dnpitn - vn * dnPi;
				Sa[3] = dnpitn * vn - dnpinn - dnPi / pow(t, 2);
			}
			Sa[1] = dnpitx * vn - dnpixn;
			Sa[2] = dnpity * vn - dnpiyn;
		}
#undef DER
		for (int n = 0; n < 4; ++n) {
			result[n] += Sa[n];
			result[n] *= P->dt;
		}
	} else {
		for (int n = 0; n < 4; ++n) result[n] *= P->dt;
	}
	for (int n = 4; n < nq; ++n) result[n] *= P->dt;
	for (int n = 0; n < nq; ++n) upd[n][s] += result[n];
}

/* Every loop body below touches its own cell only (the reference's kernels read one
 * buffer set and write another), so the planes run in parallel when built with OpenMP. */
#define FOR_INTERIOR(L, s)                                                              \
	_Pragma("omp parallel for schedule(static)")                                        \
	for (int k_ = 2; k_ < (L)->P.nz + 2; ++k_)                                          \
		for (int j_ = 2; j_ < (L)->P.ny + 2; ++j_)                                      \
			for (int i_ = 2, s = idx((L), 2, j_, k_); i_ < (L)->P.nx + 2; ++i_, ++s)

static void euler_step(kt_lattice *L, double t, double **cur, double **upd, double *e, double *p, double **u,
                       double **up) {
	FOR_INTERIOR(L, s) euler_source_cell(L, s, t, cur, upd, e, p, u, up);
	for (int axis = 1; axis <= 3; ++axis) FOR_INTERIOR(L, s) euler_axis_cell(L, s, axis, t, cur, upd, e, u);
}

/* EnergyMomentumTensor.cu:110-154 */
static void set_inferred(kt_lattice *L, double **q, double *e, double *p, double **u, double t) {
	FOR_INTERIOR(L, s) {
		double qs[KT_MAX_NQ];
		for (int n = 0; n < L->nq; ++n) qs[n] = q[n][s];
		double ee, pp, ut, ux, uy, un;
		kt_get_inferred_variables(&L->P, t, qs, e[s], &ee, &pp, &ut, &ux, &uy, &un);
		e[s] = ee; p[s] = pp;
		u[0][s] = ut; u[1][s] = ux; u[2][s] = uy; u[3][s] = un;
	}
}

/* RegulateDissipativeCurrents.cu:15-134. Pi is read as 0 (the `#ifdef Pi` guard at line
 * 54 is never true), so the bulk factor is always 1. */
static void regulate(kt_lattice *L, double t, double **q, const double *e, const double *p, double **u,
                     double T_reg) {
	const kt_params *P = &L->P;
	if (!P->shear) return;
	double e_reg = kt_equilibrium_energy_density(P, T_reg);
	FOR_INTERIOR(L, s) {
		double pitt = q[4][s], pitx = q[5][s], pity = q[6][s], pitn = q[7][s], pixx = q[8][s];
		double pixy = q[9][s], pixn = q[10][s], piyy = q[11][s], piyn = q[12][s], pinn = q[13][s];
		double Pi = 0;
		double ut = u[0][s], ux = u[1][s], uy = u[2][s], un = u[3][s];
		double e_s = e[s], p_s = p[s];
		double xi0 = 0.1, rhomax = 1.0;
		double t2 = t * t;
		double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy + piyy * piyy
		              - 2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 + pinn * pinn * t2 * t2;
		double spipi = sqrt(fabs(pipi));
		double pimumu = pitt - pixx - piyy - pinn * t * t;
		double piu0 = -pitn * t2 * un + pitt * ut - pitx * ux - pity * uy;
		double piu1 = -pixn * t2 * un + pitx * ut - pixx * ux - pixy * uy;
		double piu2 = -piyn * t2 * un + pity * ut - pixy * ux - piyy * uy;
		double piu3 = -pinn * t2 * un + pitn * ut - pixn * ux - piyn * uy;
		double a1 = (spipi / rhomax) * (1.0 / sqrt(e_s * e_s + 3 * p_s * p_s));
		double den = xi0 * rhomax * spipi;
		double a2 = pimumu / den, a3 = piu0 / den, a4 = piu1 / den, a5 = piu2 / den, a6 = piu3 / den;
		double rho = fmax(a1, fmax(a2, fmax(a3, fmax(a4, fmax(a5, a6)))));
		double facShear = tanh(rho) / rho;
		if (fabs(rho) < 1.e-7) facShear = 1.0;
		double rhoBulk = fabs(Pi) / p[s];
		double facBulk = tanh(rhoBulk) / rhoBulk;
		if (fabs(rhoBulk) < 1.e-7) facBulk = 1.0;
		if (e[s] > e_reg) { facShear = 1.0; facBulk = 1.0; }
		for (int n = 4; n < 14; ++n) q[n][s] *= facShear;
		if (P->bulk) q[14][s] *= facBulk;
	}
}

/* FullyDiscreteKurganovTadmorScheme.cu:60-104 */
static void convex_combination(kt_lattice *L, double **q, double **Q) {
	FOR_INTERIOR(L, s) for (int n = 0; n < L->nq; ++n) {
		Q[n][s] += q[n][s];
		Q[n][s] /= 2;
	}
}

/* FullyDiscreteKurganovTadmorScheme.cu:109-139 followed by the host swap d_q <-> d_Q
 * (HydroPlugin.cpp:422). The leading regulation of qS (line 112) is dead work for the
 * state (the predictor overwrites every interior qS) and is skipped; checkValidity
 * (line 137) writes diagnostics only. */
void kt_rk2_step(kt_lattice *L, double t, double dt, double T_reg) {
	double *tmp[KT_MAX_NQ];
	memset(L->speed, 0, L->ng * sizeof(double));
	euler_step(L, t, L->q, L->qS, L->e, L->p, L->u, L->up);
	for (size_t s = 0; s < L->ng; ++s) L->speed_max = fmax(L->speed_max, L->speed[s]);
	t += dt;
	set_inferred(L, L->qS, L->e, L->p, L->uS, t);
	regulate(L, t, L->qS, L->e, L->p, L->uS, T_reg);
	set_ghost_cells(L, L->qS, L->e, L->p, L->uS);

	euler_step(L, t, L->qS, L->Q, L->e, L->p, L->uS, L->u);
	convex_combination(L, L->q, L->Q);
	for (int m = 0; m < 4; ++m) { double *x = L->up[m]; L->up[m] = L->u[m]; L->u[m] = x; }
	set_inferred(L, L->Q, L->e, L->p, L->u, t);
	regulate(L, t, L->Q, L->e, L->p, L->u, T_reg);
	set_ghost_cells(L, L->Q, L->e, L->p, L->u);

	memcpy(tmp, L->q, sizeof(tmp));
	memcpy(L->q, L->Q, sizeof(tmp));
	memcpy(L->Q, tmp, sizeof(tmp));
}

/* The running maximum of a / dx_axis over cells, faces, axes and the predictor stages of the
 * steps since the last call; it starts again at 0. */
double kt_max_propagation_speed(kt_lattice *L) {
	double v = L->speed_max;
	L->speed_max = 0;
	return v;
}

/* Full state: nq conserved components, e, p, u(4), up(4); a null up pointer means up = u. */
int kt_set_state(kt_lattice *L, const double *const *f) {
	size_t bytes = L->ng * sizeof(double);
	for (int n = 0; n < L->nq; ++n) memcpy(L->q[n], f[n], bytes);
	memcpy(L->e, f[L->nq], bytes);
	memcpy(L->p, f[L->nq + 1], bytes);
	for (int m = 0; m < 4; ++m) memcpy(L->u[m], f[L->nq + 2 + m], bytes);
	for (int m = 0; m < 4; ++m) memcpy(L->up[m], f[L->nq + 6 + m] ? f[L->nq + 6 + m] : f[L->nq + 2 + m], bytes);
	return 0;
}

int kt_get_state(const kt_lattice *L, double *const *f) {
	size_t bytes = L->ng * sizeof(double);
	for (int n = 0; n < L->nq; ++n) if (f[n]) memcpy(f[n], L->q[n], bytes);
	if (f[L->nq]) memcpy(f[L->nq], L->e, bytes);
	if (f[L->nq + 1]) memcpy(f[L->nq + 1], L->p, bytes);
	for (int m = 0; m < 4; ++m) if (f[L->nq + 2 + m]) memcpy(f[L->nq + 2 + m], L->u[m], bytes);
	for (int m = 0; m < 4; ++m) if (f[L->nq + 6 + m]) memcpy(f[L->nq + 6 + m], L->up[m], bytes);
	return 0;
}

/* Initial state from primitives (HydroPlugin.cpp:214-220): p = p(e) as the type-10 reader
 * sets it (InitialConditions.cpp:124-127), T^{tau mu} from setConservedVariables
 * (DynamicalVariables.cu:349-392), up = u, ghost cells. prim: e, ut, ux, uy, un, then the
 * evolved dissipative components (pitt..pinn, Pi). Every array is ghosted; only the
 * interior is read. */
int kt_set_primitive_state(kt_lattice *L, const double *const *prim) {
	const kt_params *P = &L->P;
	memset(L->block, 0, (3 * (size_t)L->nq + 14) * L->ng * sizeof(double));
	FOR_INTERIOR(L, s) {
		L->e[s] = prim[0][s];
		L->p[s] = kt_equilibrium_pressure(P, L->e[s]);
		for (int m = 0; m < 4; ++m) L->u[m][s] = prim[1 + m][s];
		for (int n = 4; n < L->nq; ++n) L->q[n][s] = prim[5 + (n - 4)][s];
	}
	FOR_INTERIOR(L, s) {
		double pitt = 0, pitx = 0, pity = 0, pitn = 0, Pi = 0;
		if (P->shear) { pitt = L->q[4][s]; pitx = L->q[5][s]; pity = L->q[6][s]; pitn = L->q[7][s]; }
		if (P->bulk) Pi = L->q[14][s];
		double e = L->e[s], p = L->p[s], ut = L->u[0][s];
		L->q[0][s] = Ttt(e, p + Pi, ut, pitt);
		L->q[1][s] = Ttx(e, p + Pi, ut, L->u[1][s], pitx);
		L->q[2][s] = Tty(e, p + Pi, ut, L->u[2][s], pity);
		L->q[3][s] = Ttn(e, p + Pi, ut, L->u[3][s], pitn);
	}
	FOR_INTERIOR(L, s) for (int m = 0; m < 4; ++m) L->up[m][s] = L->u[m][s];
	set_ghost_cells(L, L->q, L->e, L->p, L->u);
	return 0;
}
