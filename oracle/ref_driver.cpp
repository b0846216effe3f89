/*
 * CPU driver for the reference's OWN hot-path sources (gpu-vh rhic/src), compiled with g++
 * through oracle/ref_shim. Test infrastructure only: it is the pinning oracle and the
 * reference arm of the benchmark, never the product.
 *
 * The reference's __global__ kernels (eulerStepKernelSource_1D / X_1D / Y_1D / Z_1D,
 * setInferredVariablesKernel, regulateDissipativeCurrents) are compiled unmodified from
 * rhic/src and called here once per thread id, in parallel over OpenMP threads. Their GPU
 * semantics carry over exactly: every kernel reads one buffer set and writes another, or
 * updates only its own cell.
 *
 * Three pieces of the reference cannot compile as host C++ because they contain <<<>>>
 * launches, so their (tiny) bodies are restated here and cited:
 *   - the launch sequence of twoStepRungeKutta      FullyDiscreteKurganovTadmorScheme.cu:109-139
 *   - convexCombinationEulerStepKernel               FullyDiscreteKurganovTadmorScheme.cu:60-104
 *   - setGhostCells (kernels I/J/K, faces only)      GhostCells.cu:15-144
 * plus the __constant__ set-up of CudaConfiguration.cu:209-248 and the host-side
 * setConservedVariables of DynamicalVariables.cu:349-392.
 *
 * C API (doubles in, doubles out; the build's PRECISION is used inside):
 *   field order = the CONSERVED_VARIABLES members (DynamicalVariables.cuh:50-71), then
 *   e, p, ut, ux, uy, un, utp, uxp, uyp, unp; every array is the full ghosted lattice
 *   (nx+4)(ny+4)(nz+4), index i + ncx*(j + ncy*k) (DynamicalVariables.cu:32-35).
 */
#include <cuda.h>
#include <cuda_runtime.h>
#include <omp.h>
#include <vector>

#include "DynamicalVariables.cuh"
#include "LatticeParameters.h"
#include "EulerStep.cuh"
#include "EnergyMomentumTensor.cuh"
#include "EquationOfState.cuh"
#ifndef IDEAL
#include "RegulateDissipativeCurrents.cuh"
#endif
#include "HydrodynamicValidity.cuh"

thread_local dim3 threadIdx;
thread_local dim3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

/* __constant__ scalars of CudaConfiguration.cuh:12-13 (defined there as device symbols). */
int d_nx, d_ny, d_nz, d_ncx, d_ncy, d_ncz, d_nElements, d_nCompElements;
PRECISION d_dt, d_dx, d_dy, d_dz, d_etabar;

/* Runtime limiter slope; FluxLimiter.cu's `#define THETA 2.0` is replaced by this name in
 * the generated overlay copy of that file (see oracle/Makefile). */
double gvh_ref_theta = 2.0;

/* DynamicalVariables.cu:32-35 */
int columnMajorLinearIndex(int i, int j, int k, int nx, int ny) { return i + nx * (j + ny * k); }

namespace {

const int NQ = NUMBER_CONSERVED_VARIABLES;

struct Buffers {
	std::vector<PRECISION> comp[NQ];
	CONSERVED_VARIABLES view;
	void alloc(size_t n) {
		for (int c = 0; c < NQ; ++c) comp[c].assign(n, (PRECISION)0);
		PRECISION **slots = reinterpret_cast<PRECISION **>(&view);
		for (int c = 0; c < NQ; ++c) slots[c] = comp[c].data();
	}
};
struct Velocity {
	std::vector<PRECISION> c[4];
	FLUID_VELOCITY view;
	void alloc(size_t n) {
		for (int m = 0; m < 4; ++m) c[m].assign(n, (PRECISION)0);
		view.ut = c[0].data(); view.ux = c[1].data(); view.uy = c[2].data(); view.un = c[3].data();
	}
};

Buffers g_q, g_Q, g_qS;
Velocity g_u0, g_u1, g_uS;
FLUID_VELOCITY *g_u = nullptr, *g_up = nullptr;
CONSERVED_VARIABLES *g_cur = nullptr, *g_next = nullptr;
std::vector<PRECISION> g_e, g_p, g_reg;
std::vector<PRECISION> g_vd[13];  /* the VALIDITY_DOMAIN arrays (regulations is g_vd[0]) */
VALIDITY_DOMAIN g_validity;
size_t g_ng = 0;
int g_nx = 0, g_ny = 0, g_nz = 0;

template <class F>
void launch(int nthreads, F &&kernel) {
#pragma omp parallel for schedule(static)
	for (int id = 0; id < nthreads; ++id) {
		blockDim = dim3(1, 1, 1);
		threadIdx = dim3(0, 0, 0);
		blockIdx = dim3((unsigned)id, 0, 0);
		kernel();
	}
}

PRECISION **slots(CONSERVED_VARIABLES *q) { return reinterpret_cast<PRECISION **>(q); }

/* GhostCells.cu:31-63 (setGhostCellVars) */
void ghostCopy(CONSERVED_VARIABLES *q, PRECISION *e, PRECISION *p, FLUID_VELOCITY *u, int s, int sBC) {
	e[s] = e[sBC];
	p[s] = p[sBC];
	u->ut[s] = u->ut[sBC];
	u->ux[s] = u->ux[sBC];
	u->uy[s] = u->uy[sBC];
	u->un[s] = u->un[sBC];
	PRECISION **c = slots(q);
	for (int n = 0; n < NQ; ++n) c[n][s] = c[n][sBC];
}

/* GhostCells.cu:65-144: zero-gradient copy into two ghost layers on each face; edges and
 * corners are not touched. The three kernels write disjoint cells and read interior cells
 * only, so their order does not matter. */
void setGhostCells(CONSERVED_VARIABLES *q, PRECISION *e, PRECISION *p, FLUID_VELOCITY *u) {
	const int nx = d_nx, ny = d_ny, nz = d_nz, ncx = d_ncx, ncy = d_ncy;
#pragma omp parallel for schedule(static)
	for (int id = 0; id < ny * nz; ++id) {
		int j = id % ny + 2, k = id / ny + 2;
		for (int i = 0; i <= 1; ++i) ghostCopy(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy), columnMajorLinearIndex(2, j, k, ncx, ncy));
		for (int i = nx + 2; i <= nx + 3; ++i) ghostCopy(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy), columnMajorLinearIndex(nx + 1, j, k, ncx, ncy));
	}
#pragma omp parallel for schedule(static)
	for (int id = 0; id < nx * nz; ++id) {
		int i = id % nx + 2, k = id / nx + 2;
		for (int j = 0; j <= 1; ++j) ghostCopy(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy), columnMajorLinearIndex(i, 2, k, ncx, ncy));
		for (int j = ny + 2; j <= ny + 3; ++j) ghostCopy(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy), columnMajorLinearIndex(i, ny + 1, k, ncx, ncy));
	}
#pragma omp parallel for schedule(static)
	for (int id = 0; id < nx * ny; ++id) {
		int i = id % nx + 2, j = id / nx + 2;
		for (int k = 0; k <= 1; ++k) ghostCopy(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy), columnMajorLinearIndex(i, j, 2, ncx, ncy));
		for (int k = nz + 2; k <= nz + 3; ++k) ghostCopy(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy), columnMajorLinearIndex(i, j, nz + 1, ncx, ncy));
	}
}

/* FullyDiscreteKurganovTadmorScheme.cu:35-58 with EULER_STEP_SPLIT_1D (line 33). */
void eulerStep(PRECISION t, CONSERVED_VARIABLES *cur, CONSERVED_VARIABLES *upd, PRECISION *e, PRECISION *p,
               FLUID_VELOCITY *u, FLUID_VELOCITY *up) {
	const int n = d_nElements;
	launch(n, [&] { eulerStepKernelSource_1D(t, cur, upd, e, p, u, up); });
	launch(n, [&] { eulerStepKernelX_1D(t, cur, upd, u, e); });
	launch(n, [&] { eulerStepKernelY_1D(t, cur, upd, u, e); });
	launch(n, [&] { eulerStepKernelZ_1D(t, cur, upd, u, e); });
}

/* FullyDiscreteKurganovTadmorScheme.cu:60-104 */
void convexCombination(CONSERVED_VARIABLES *q, CONSERVED_VARIABLES *Q) {
	PRECISION **a = slots(q), **b = slots(Q);
	const int nx = d_nx, ny = d_ny, ncx = d_ncx, ncy = d_ncy;
#pragma omp parallel for schedule(static)
	for (int id = 0; id < d_nElements; ++id) {
		int k = id / (nx * ny) + 2, j = (id % (nx * ny)) / nx + 2, i = id % nx + 2;
		int s = columnMajorLinearIndex(i, j, k, ncx, ncy);
		for (int c = 0; c < NQ; ++c) {
			b[c][s] += a[c][s];
			b[c][s] /= 2;
		}
	}
}

void regulate(PRECISION t, CONSERVED_VARIABLES *q, PRECISION *e, PRECISION *p, FLUID_VELOCITY *u, PRECISION T_reg) {
#ifndef IDEAL
	launch(d_nElements, [&] { regulateDissipativeCurrents(t, q, e, p, u, &g_validity, T_reg); });
#else
	(void)t; (void)q; (void)e; (void)p; (void)u; (void)T_reg;
#endif
}

} // namespace

/* The current level's host state, for the freeze-out replay in ref_surface.cpp. */
void gvh_ref_current(CONSERVED_VARIABLES **q, PRECISION **e, FLUID_VELOCITY **u) {
	*q = g_cur;
	*e = g_e.data();
	*u = g_u;
}

extern "C" {

int gvh_ref_nq(void) { return NQ; }
int gvh_ref_precision_bytes(void) { return (int)sizeof(PRECISION); }
int gvh_ref_conformal(void) {
#ifdef CONFORMAL_EOS
	return 1;
#else
	return 0;
#endif
}
void gvh_ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int gvh_ref_max_threads(void) { return omp_get_max_threads(); }

/* CudaConfiguration.cu:209-248 (constants) and DynamicalVariables.cu:147-269 (buffers). */
int gvh_ref_init(int nx, int ny, int nz, double dx, double dy, double dz, double dt, double etabar, double theta) {
	if (nx < 1 || ny < 1 || nz < 1) return -1;
	d_nx = nx; d_ny = ny; d_nz = nz;
	d_ncx = nx + N_GHOST_CELLS; d_ncy = ny + N_GHOST_CELLS; d_ncz = nz + N_GHOST_CELLS;
	d_nElements = nx * ny * nz;
	d_nCompElements = d_ncx * d_ncy * d_ncz;
	d_dt = (PRECISION)dt; d_dx = (PRECISION)dx; d_dy = (PRECISION)dy; d_dz = (PRECISION)dz;
	d_etabar = (PRECISION)etabar;
	gvh_ref_theta = theta;
	g_nx = nx; g_ny = ny; g_nz = nz;
	g_ng = (size_t)d_nCompElements;
	g_q.alloc(g_ng); g_Q.alloc(g_ng); g_qS.alloc(g_ng);
	g_u0.alloc(g_ng); g_u1.alloc(g_ng); g_uS.alloc(g_ng);
	g_e.assign(g_ng, 0); g_p.assign(g_ng, 0); g_reg.assign(g_ng, 1);
	memset(&g_validity, 0, sizeof(g_validity));
	for (int f = 1; f < 13; ++f) g_vd[f].assign(g_ng, 0);
	{
		PRECISION **vs = reinterpret_cast<PRECISION **>(&g_validity);
		vs[0] = g_reg.data();
		for (int f = 1; f < 13; ++f) vs[f] = g_vd[f].data();
	}
	g_cur = &g_q.view; g_next = &g_Q.view;
	g_u = &g_u0.view; g_up = &g_u1.view;
	return 0;
}

static void put(PRECISION *dst, const double *src) { for (size_t s = 0; s < g_ng; ++s) dst[s] = (PRECISION)src[s]; }
static void get(double *dst, const PRECISION *src) { for (size_t s = 0; s < g_ng; ++s) dst[s] = (double)src[s]; }

/* Full state in: NQ conserved components, e, p, u(4), up(4); up may be null (then up = u,
 * as copyHostToDeviceMemory seeds it, DynamicalVariables.cu:280-284). */
int gvh_ref_set_state(const double *const *fields) {
	if (!g_ng) return -1;
	PRECISION **c = slots(g_cur);
	for (int n = 0; n < NQ; ++n) put(c[n], fields[n]);
	put(g_e.data(), fields[NQ]);
	put(g_p.data(), fields[NQ + 1]);
	PRECISION *u[4] = {g_u->ut, g_u->ux, g_u->uy, g_u->un};
	PRECISION *up[4] = {g_up->ut, g_up->ux, g_up->uy, g_up->un};
	for (int m = 0; m < 4; ++m) put(u[m], fields[NQ + 2 + m]);
	for (int m = 0; m < 4; ++m) put(up[m], fields[NQ + 6 + m] ? fields[NQ + 6 + m] : fields[NQ + 2 + m]);
	return 0;
}

int gvh_ref_get_state(double *const *fields) {
	if (!g_ng) return -1;
	PRECISION **c = slots(g_cur);
	for (int n = 0; n < NQ; ++n) if (fields[n]) get(fields[n], c[n]);
	if (fields[NQ]) get(fields[NQ], g_e.data());
	if (fields[NQ + 1]) get(fields[NQ + 1], g_p.data());
	const PRECISION *u[4] = {g_u->ut, g_u->ux, g_u->uy, g_u->un};
	const PRECISION *up[4] = {g_up->ut, g_up->ux, g_up->uy, g_up->un};
	for (int m = 0; m < 4; ++m) if (fields[NQ + 2 + m]) get(fields[NQ + 2 + m], u[m]);
	for (int m = 0; m < 4; ++m) if (fields[NQ + 6 + m]) get(fields[NQ + 6 + m], up[m]);
	return 0;
}

/* Initial state from primitives on the interior, as HydroPlugin.cpp:214-220 builds it:
 * p = equilibriumPressure(e) (InitialConditions.cpp type-10 reader), conserved T^{tau mu}
 * from setConservedVariables (DynamicalVariables.cu:349-392), up = u, then setGhostCells.
 * prim order: e, ut, ux, uy, un, then (if evolved) pitt..pinn, then (if evolved) Pi. */
static int set_primitive(const double *const *prim, const double *p_in);

int gvh_ref_set_primitive_state(const double *const *prim) { return set_primitive(prim, nullptr); }

/* Type 11 (setInitialTmunuFromFile, InitialConditions.cpp:29-97): p is read, not p(e). */
int gvh_ref_set_primitive_state_p(const double *const *prim, const double *p_in) { return set_primitive(prim, p_in); }

static int set_primitive(const double *const *prim, const double *p_in) {
	if (!g_ng) return -1;
	const int ncx = d_ncx, ncy = d_ncy;
	PRECISION **c = slots(g_cur);
	for (size_t s = 0; s < g_ng; ++s) {
		for (int n = 0; n < NQ; ++n) c[n][s] = 0;
		g_e[s] = 0; g_p[s] = 0;
		g_u->ut[s] = 0; g_u->ux[s] = 0; g_u->uy[s] = 0; g_u->un[s] = 0;
	}
	for (int k = 2; k < g_nz + 2; ++k)
		for (int j = 2; j < g_ny + 2; ++j)
			for (int i = 2; i < g_nx + 2; ++i) {
				int s = columnMajorLinearIndex(i, j, k, ncx, ncy);
				g_e[s] = (PRECISION)prim[0][s];
				g_p[s] = p_in ? (PRECISION)p_in[s] : equilibriumPressure(g_e[s]);
				g_u->ut[s] = (PRECISION)prim[1][s];
				g_u->ux[s] = (PRECISION)prim[2][s];
				g_u->uy[s] = (PRECISION)prim[3][s];
				g_u->un[s] = (PRECISION)prim[4][s];
				for (int n = 4; n < NQ; ++n) c[n][s] = (PRECISION)prim[5 + (n - 4)][s];
			}
	for (int k = 2; k < g_nz + 2; ++k)
		for (int j = 2; j < g_ny + 2; ++j)
			for (int i = 2; i < g_nx + 2; ++i) {
				int s = columnMajorLinearIndex(i, j, k, ncx, ncy);
				PRECISION ux_s = g_u->ux[s], uy_s = g_u->uy[s], un_s = g_u->un[s], ut_s = g_u->ut[s];
				PRECISION e_s = g_e[s], p_s = g_p[s];
				PRECISION pitt_s = 0, pitx_s = 0, pity_s = 0, pitn_s = 0;
#ifdef PIMUNU
				pitt_s = c[4][s]; pitx_s = c[5][s]; pity_s = c[6][s]; pitn_s = c[7][s];
#endif
				PRECISION Pi_s = 0;
#ifdef PI
				Pi_s = c[14][s];
#endif
				c[0][s] = Ttt(e_s, p_s + Pi_s, ut_s, pitt_s);
				c[1][s] = Ttx(e_s, p_s + Pi_s, ut_s, ux_s, pitx_s);
				c[2][s] = Tty(e_s, p_s + Pi_s, ut_s, uy_s, pity_s);
				c[3][s] = Ttn(e_s, p_s + Pi_s, ut_s, un_s, pitn_s);
			}
	for (size_t s = 0; s < g_ng; ++s) {
		g_up->ut[s] = g_u->ut[s]; g_up->ux[s] = g_u->ux[s]; g_up->uy[s] = g_u->uy[s]; g_up->un[s] = g_u->un[s];
	}
	setGhostCells(g_cur, g_e.data(), g_p.data(), g_u);
	/* the up ghosts follow u's (copyHostToDeviceMemory copies the host u, ghosts included,
	 * into up BEFORE setGhostCells runs on the device: DynamicalVariables.cu:280-284 and
	 * HydroPlugin.cpp:218-220), so up ghosts keep the host values (zero here) */
	return 0;
}

/* One call of twoStepRungeKutta (FullyDiscreteKurganovTadmorScheme.cu:109-139) followed by
 * the host swap d_q <-> d_Q (HydroPlugin.cpp:422, DynamicalVariables.cu:400-402). The
 * diagnostic checkValidity launch (line 137) writes only validity arrays and is omitted. */
int gvh_ref_rk2_step(double t_in, double dt_in, double T_reg_in) {
	if (!g_ng) return -1;
	PRECISION t = (PRECISION)t_in, dt = (PRECISION)dt_in, T_reg = (PRECISION)T_reg_in;
	PRECISION *e = g_e.data(), *p = g_p.data();
	CONSERVED_VARIABLES *q = g_cur, *Q = g_next, *qS = &g_qS.view;
	FLUID_VELOCITY *uS = &g_uS.view;

	regulate(t, qS, e, p, uS, T_reg);
	eulerStep(t, q, qS, e, p, g_u, g_up);
	t += dt;
	launch(d_nElements, [&] { setInferredVariablesKernel(qS, e, p, uS, t); });
	regulate(t, qS, e, p, uS, T_reg);
	setGhostCells(qS, e, p, uS);

	eulerStep(t, qS, Q, e, p, uS, g_u);
	convexCombination(q, Q);
	FLUID_VELOCITY *tmp = g_up; g_up = g_u; g_u = tmp;
	launch(d_nElements, [&] { setInferredVariablesKernel(Q, e, p, g_u, t); });
	regulate(t, Q, e, p, g_u, T_reg);
	setGhostCells(Q, e, p, g_u);
	/* checkValidity(t, d_validityDomain, d_q, d_e, d_p, d_u, d_up): the 3-D launch of
	 * HydrodynamicValidity.cu:18-23 over the interior (line 137) */
	{
		const int nx = g_nx, ny = g_ny, nz = g_nz;
#pragma omp parallel for collapse(2) schedule(static)
		for (int kk = 0; kk < nz; ++kk)
			for (int jj = 0; jj < ny; ++jj)
				for (int ii = 0; ii < nx; ++ii) {
					blockDim = dim3(1, 1, 1);
					threadIdx = dim3(0, 0, 0);
					blockIdx = dim3((unsigned)ii, (unsigned)jj, (unsigned)kk);
					checkValidityKernel(t, &g_validity, q, e, p, g_u, g_up);
				}
	}

	g_cur = Q; g_next = q;
	return 0;
}

/* The VALIDITY_DOMAIN arrays after the last step (13 ghosted arrays, NULL entries skipped). */
int gvh_ref_get_validity(double *const *fields) {
	if (!g_ng) return -1;
	PRECISION **vs = reinterpret_cast<PRECISION **>(&g_validity);
	for (int f = 0; f < 13; ++f)
		if (fields[f]) get(fields[f], vs[f]);
	return 0;
}

double gvh_ref_equilibrium_pressure(double e) { return (double)equilibriumPressure((PRECISION)e); }
double gvh_ref_effective_temperature(double e) { return (double)effectiveTemperature((PRECISION)e); }
double gvh_ref_equilibrium_energy_density(double T) { return (double)equilibriumEnergyDensity((PRECISION)T); }
double gvh_ref_speed_of_sound_squared(double e) { return (double)speedOfSoundSquared((PRECISION)e); }

/* getInferredVariables (EnergyMomentumTensor.cu:50-108) on one conserved vector. */
void gvh_ref_inferred(double t, const double *q_in, double ePrev, double *out6) {
	PRECISION q[NQ];
	for (int n = 0; n < NQ; ++n) q[n] = (PRECISION)q_in[n];
	PRECISION e, p, ut, ux, uy, un;
	getInferredVariables((PRECISION)t, q, (PRECISION)ePrev, &e, &p, &ut, &ux, &uy, &un);
	out6[0] = e; out6[1] = p; out6[2] = ut; out6[3] = ux; out6[4] = uy; out6[5] = un;
}

} // extern "C"
