/*
 * GPU driver for the reference's OWN hot path (gpu-vh rhic/src) compiled with nvcc for
 * sm_100a: the as-shipped FP32 build and its FP64 overlay. Test and measurement
 * infrastructure only: it is the reference timed beside the product on the same GPU, and
 * the reference's own FP64 CUDA build used as an oracle, never the product.
 *
 * Everything that runs on the device is the reference's own code: its allocation
 * (allocateHostMemory / allocateDeviceMemory, DynamicalVariables.cu:37-269), its launch
 * set-up (initializeCUDALaunchParameters / initializeCUDAConstantParameters,
 * CudaConfiguration.cu:61-248), its initial-state path (setConservedVariables,
 * copyHostToDeviceMemory, setGhostCells: HydroPlugin.cpp:214-220) and its step
 * (twoStepRungeKutta, FullyDiscreteKurganovTadmorScheme.cu:109-139, followed by the host
 * swap setCurrentConservedVariables, HydroPlugin.cpp:422). This file only moves arrays in
 * and out and times the calls.
 *
 * C API: the same names and field order as the CPU driver (ref_driver.cpp), plus
 * gvh_ref_time_steps. Field order = the CONSERVED_VARIABLES members, then e, p, ut, ux,
 * uy, un, utp, uxp, uyp, unp; every array is the full ghosted lattice.
 */
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>
#include <vector>

#include "DynamicalVariables.cuh"
#include "LatticeParameters.h"
#include "HydroParameters.h"
#include "InitialConditionParameters.h"
#include "CudaConfiguration.cuh"
#include "FullyDiscreteKurganovTadmorScheme.cuh"
#include "GhostCells.cuh"
#include "EquationOfState.cuh"

/* DynamicalVariables.cu:271-408 (host functions; not all declared in its header) */
void setCurrentConservedVariables();
void swapFluidVelocity(FLUID_VELOCITY **arr1, FLUID_VELOCITY **arr2);
void setConservedVariables(double t, void *latticeParams);
void copyHostToDeviceMemory(size_t bytes);

namespace {

const int NQ = NUMBER_CONSERVED_VARIABLES;

LatticeParameters g_lattice;
HydroParameters g_hydro;
InitialConditionParameters g_ic;
size_t g_ng = 0;
int g_nx = 0, g_ny = 0, g_nz = 0;
long long g_steps = 0;  /* parity of the d_q/d_Q and d_u/d_up swaps */
bool g_ready = false;

/* Runs f with stdout sent to /dev/null (the reference's launch set-up prints its block
 * sizes; the benchmark's stdout carries one JSON line). */
template <class F>
void quiet(F &&f) {
	fflush(stdout);
	int saved = dup(1);
	FILE *null = fopen("/dev/null", "w");
	if (saved >= 0 && null) dup2(fileno(null), 1);
	f();
	fflush(stdout);
	if (saved >= 0) {
		dup2(saved, 1);
		close(saved);
	}
	if (null) fclose(null);
}

int check(const char *what) {
	cudaError_t err = cudaGetLastError();
	if (err != cudaSuccess) {
		fprintf(stderr, "[ref gpu] %s: %s\n", what, cudaGetErrorString(err));
		return -2;
	}
	return 0;
}

/* The device pointers behind the current state structs (the structs live in device memory,
 * DynamicalVariables.cu:88-145). */
void current_pointers(PRECISION **dq, PRECISION **du, PRECISION **dup) {
	CONSERVED_VARIABLES hq;
	FLUID_VELOCITY hu, hup;
	cudaMemcpy(&hq, d_q, sizeof hq, cudaMemcpyDeviceToHost);
	cudaMemcpy(&hu, d_u, sizeof hu, cudaMemcpyDeviceToHost);
	cudaMemcpy(&hup, d_up, sizeof hup, cudaMemcpyDeviceToHost);
	memcpy(dq, &hq, NQ * sizeof(PRECISION *));
	du[0] = hu.ut; du[1] = hu.ux; du[2] = hu.uy; du[3] = hu.un;
	dup[0] = hup.ut; dup[1] = hup.ux; dup[2] = hup.uy; dup[3] = hup.un;
}

void put(PRECISION *dst, const double *src, std::vector<PRECISION> &tmp) {
	for (size_t s = 0; s < g_ng; ++s) tmp[s] = (PRECISION)src[s];
	cudaMemcpy(dst, tmp.data(), g_ng * sizeof(PRECISION), cudaMemcpyHostToDevice);
}

void get(double *dst, const PRECISION *src, std::vector<PRECISION> &tmp) {
	cudaMemcpy(tmp.data(), src, g_ng * sizeof(PRECISION), cudaMemcpyDeviceToHost);
	for (size_t s = 0; s < g_ng; ++s) dst[s] = (double)tmp[s];
}

/* Undo an odd number of step swaps, so that d_q / d_u are the first-allocated sets that
 * copyHostToDeviceMemory writes (DynamicalVariables.cu:271-308). */
void restore_initial_sets() {
	if (g_steps & 1) {
		setCurrentConservedVariables();
		swapFluidVelocity(&d_up, &d_u);
	}
	g_steps = 0;
}

} // namespace

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
/* limiter slope compiled into this build (FluxLimiter.cu:15, or the overlay copy's value) */
double gvh_ref_theta(void) { return GVH_REF_THETA; }
int gvh_ref_gpu(void) { return 1; }
void gvh_ref_set_threads(int) {}
int gvh_ref_max_threads(void) { return 1; }

/* HydroPlugin.cpp:117-153: parameters, launch set-up, constants, host and device buffers.
 * The reference keeps one lattice per process (globals); a second call must use the same
 * sizes. */
int gvh_ref_init(int nx, int ny, int nz, double dx, double dy, double dz, double dt, double etabar, double theta) {
	if (nx < 1 || ny < 1 || nz < 1) return -1;
	if (theta != GVH_REF_THETA) {
		fprintf(stderr, "[ref gpu] this build's limiter slope is %g, not %g\n", (double)GVH_REF_THETA, theta);
		return -1;
	}
	if (g_ready && (nx != g_nx || ny != g_ny || nz != g_nz)) return -1;
	memset(&g_lattice, 0, sizeof g_lattice);
	g_lattice.numLatticePointsX = nx;
	g_lattice.numLatticePointsY = ny;
	g_lattice.numLatticePointsRapidity = nz;
	g_lattice.numComputationalLatticePointsX = nx + N_GHOST_CELLS;
	g_lattice.numComputationalLatticePointsY = ny + N_GHOST_CELLS;
	g_lattice.numComputationalLatticePointsRapidity = nz + N_GHOST_CELLS;
	g_lattice.latticeSpacingX = dx;
	g_lattice.latticeSpacingY = dy;
	g_lattice.latticeSpacingRapidity = dz;
	g_lattice.latticeSpacingProperTime = dt;
	memset(&g_hydro, 0, sizeof g_hydro);
	g_hydro.shearViscosityToEntropyDensity = etabar;
	memset(&g_ic, 0, sizeof g_ic);
	g_nx = nx; g_ny = ny; g_nz = nz;
	g_ng = (size_t)(nx + N_GHOST_CELLS) * (ny + N_GHOST_CELLS) * (nz + N_GHOST_CELLS);
	quiet([] { initializeCUDALaunchParameters(&g_lattice); });
	initializeCUDAConstantParameters(&g_lattice, &g_ic, &g_hydro);
	if (!g_ready) {
		allocateHostMemory((int)g_ng);
		allocateDeviceMemory(g_ng * sizeof(PRECISION));
		g_ready = true;
	}
	return check("init");
}

/* Initial state from primitives on the interior, as HydroPlugin.cpp:214-220 builds it: the
 * type-10 reader's p = equilibriumPressure(e) (InitialConditions.cpp:124-127), or p as
 * given (type 11), then setConservedVariables, copyHostToDeviceMemory (which also seeds
 * up = u, ghosts included) and setGhostCells. prim order: e, ut, ux, uy, un, then (if
 * evolved) pitt..pinn, then (if evolved) Pi. */
static int set_primitive(const double *const *prim, const double *p_in) {
	if (!g_ready) return -1;
	restore_initial_sets();
	const int ncx = g_nx + N_GHOST_CELLS, ncy = g_ny + N_GHOST_CELLS;
	PRECISION **c = reinterpret_cast<PRECISION **>(q);
	for (size_t s = 0; s < g_ng; ++s) {
		for (int n = 0; n < NQ; ++n) c[n][s] = 0;
		e[s] = 0; p[s] = 0;
		u->ut[s] = 0; u->ux[s] = 0; u->uy[s] = 0; u->un[s] = 0;
	}
	for (int k = 2; k < g_nz + 2; ++k)
		for (int j = 2; j < g_ny + 2; ++j)
			for (int i = 2; i < g_nx + 2; ++i) {
				int s = columnMajorLinearIndex(i, j, k, ncx, ncy);
				e[s] = (PRECISION)prim[0][s];
				p[s] = p_in ? (PRECISION)p_in[s] : equilibriumPressure(e[s]);
				u->ut[s] = (PRECISION)prim[1][s];
				u->ux[s] = (PRECISION)prim[2][s];
				u->uy[s] = (PRECISION)prim[3][s];
				u->un[s] = (PRECISION)prim[4][s];
				for (int n = 4; n < NQ; ++n) c[n][s] = (PRECISION)prim[5 + (n - 4)][s];
			}
	setConservedVariables(0.0, &g_lattice);
	copyHostToDeviceMemory(g_ng * sizeof(PRECISION));
	setGhostCells(d_q, d_e, d_p, d_u);
	cudaDeviceSynchronize();
	return check("set_primitive_state");
}

int gvh_ref_set_primitive_state(const double *const *prim) { return set_primitive(prim, nullptr); }
int gvh_ref_set_primitive_state_p(const double *const *prim, const double *p_in) { return set_primitive(prim, p_in); }

/* Full state in: NQ conserved components, e, p, u(4), up(4); up may be null (then up = u,
 * as copyHostToDeviceMemory seeds it). */
int gvh_ref_set_state(const double *const *fields) {
	if (!g_ready) return -1;
	std::vector<PRECISION> tmp(g_ng);
	PRECISION *dq[NQ], *du[4], *dup[4];
	current_pointers(dq, du, dup);
	for (int n = 0; n < NQ; ++n) put(dq[n], fields[n], tmp);
	put(d_e, fields[NQ], tmp);
	put(d_p, fields[NQ + 1], tmp);
	for (int m = 0; m < 4; ++m) put(du[m], fields[NQ + 2 + m], tmp);
	for (int m = 0; m < 4; ++m) put(dup[m], fields[NQ + 6 + m] ? fields[NQ + 6 + m] : fields[NQ + 2 + m], tmp);
	return check("set_state");
}

int gvh_ref_get_state(double *const *fields) {
	if (!g_ready) return -1;
	cudaDeviceSynchronize();
	std::vector<PRECISION> tmp(g_ng);
	PRECISION *dq[NQ], *du[4], *dup[4];
	current_pointers(dq, du, dup);
	for (int n = 0; n < NQ; ++n) if (fields[n]) get(fields[n], dq[n], tmp);
	if (fields[NQ]) get(fields[NQ], d_e, tmp);
	if (fields[NQ + 1]) get(fields[NQ + 1], d_p, tmp);
	for (int m = 0; m < 4; ++m) if (fields[NQ + 2 + m]) get(fields[NQ + 2 + m], du[m], tmp);
	for (int m = 0; m < 4; ++m) if (fields[NQ + 6 + m]) get(fields[NQ + 6 + m], dup[m], tmp);
	return check("get_state");
}

/* One iteration of HydroPlugin.cpp's loop body (lines 418-422): twoStepRungeKutta, then
 * the host swap d_q <-> d_Q. */
int gvh_ref_rk2_step(double t, double dt, double T_reg) {
	if (!g_ready) return -1;
	twoStepRungeKutta((PRECISION)t, (PRECISION)dt, d_q, d_Q, (PRECISION)T_reg);
	setCurrentConservedVariables();
	++g_steps;
	return check("rk2_step");
}

/* n steps of HydroPlugin.cpp's loop (t = t0 + (k-1) dt for step k), timed with CUDA events
 * on the legacy stream the reference launches on; *ms = the whole loop's time. */
int gvh_ref_time_steps(int n, double t0, double dt, double T_reg, double *ms) {
	if (!g_ready || n < 1) return -1;
	cudaEvent_t a, b;
	cudaEventCreate(&a);
	cudaEventCreate(&b);
	cudaDeviceSynchronize();
	cudaEventRecord(a, 0);
	for (int k = 1; k <= n; ++k) {
		twoStepRungeKutta((PRECISION)(t0 + (k - 1) * dt), (PRECISION)dt, d_q, d_Q, (PRECISION)T_reg);
		setCurrentConservedVariables();
		++g_steps;
	}
	cudaEventRecord(b, 0);
	cudaEventSynchronize(b);
	float f = 0;
	cudaEventElapsedTime(&f, a, b);
	cudaEventDestroy(a);
	cudaEventDestroy(b);
	*ms = f;
	return check("time_steps");
}

double gvh_ref_equilibrium_pressure(double x) { return (double)equilibriumPressure((PRECISION)x); }

} // extern "C"
