/* kt_oracle.h -- CPU restatement (oracle) of gpu-vh's KT RK2 step. Test infrastructure
 * only; see kt_oracle.c for what it follows and how it is pinned. */
#ifndef KT_ORACLE_H_
#define KT_ORACLE_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KT_MAX_NQ 15

typedef struct {
	int nx, ny, nz;       /* interior cells (LatticeParameters.h:19-21) */
	double dx, dy, dz;    /* lattice spacings (fm, fm, 1) */
	double dt;            /* d_dt: the lattice time step used inside the Euler steps */
	double etabar;        /* eta/s */
	double theta;         /* minmod limiter slope (FluxLimiter.cu:15) */
	int conformal;        /* CONFORMAL_EOS */
	int shear;            /* PIMUNU: evolve pi^{mu nu} */
	int bulk;             /* PI: evolve the bulk pressure (requires shear) */
	int cartesian;        /* USE_CARTESIAN_COORDINATES (SourceTerms.cu:25, 738-743) */
} kt_params;

typedef struct kt_lattice kt_lattice;

int kt_nq(const kt_params *P);
kt_lattice *kt_create(const kt_params *P);
void kt_destroy(kt_lattice *L);
size_t kt_num_cells(const kt_lattice *L);
int kt_set_state(kt_lattice *L, const double *const *fields);
int kt_get_state(const kt_lattice *L, double *const *fields);
int kt_set_primitive_state(kt_lattice *L, const double *const *prim);
void kt_rk2_step(kt_lattice *L, double t, double dt, double T_reg);
double kt_max_propagation_speed(kt_lattice *L);

double kt_equilibrium_pressure(const kt_params *P, double e);
double kt_speed_of_sound_squared(const kt_params *P, double e);
double kt_effective_temperature(const kt_params *P, double e);
double kt_equilibrium_energy_density(const kt_params *P, double T);
double kt_bulk_zeta_over_s(double T);
double kt_energy_density_from_conserved(const kt_params *P, double ePrev, double M0, double M, double Pi);
void kt_get_inferred_variables(const kt_params *P, double t, const double *q, double ePrev, double *e, double *p,
                               double *ut, double *ux, double *uy, double *un);

#ifdef __cplusplus
}
#endif
#endif
