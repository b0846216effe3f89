/*
 * gvh.h -- C ABI of the B200 KT RK2 step (gpu-vh's hot path), libgvh.so.
 *
 * Plain C types only (no CUDA or torch types), so any FFI can bind it. Every function
 * returns an int status: GVH_OK (0) or a negative GVH_ERR_* code; gvh_last_error() gives
 * a one-line reason for the calling thread's last failure.
 *
 * What it replaces in the reference (gpu-vh, paths within its tree):
 *   gvh_create / gvh_destroy     allocateDeviceMemory / freeDeviceMemory
 *                                (DynamicalVariables.cu:147-269, 443-485) and the
 *                                constant set-up initializeCUDAConstantParameters
 *                                (CudaConfiguration.cu:209-248)
 *   gvh_set_primitive_state      setConservedVariables + copyHostToDeviceMemory +
 *                                setGhostCells (HydroPlugin.cpp:214-220,
 *                                DynamicalVariables.cu:271-308, 349-392)
 *   gvh_set_state / gvh_get_state
 *                                copyHostToDeviceMemory / copyDeviceToHostMemory
 *                                (DynamicalVariables.cu:271-347), full state
 *   gvh_rk2_step                 twoStepRungeKutta (FullyDiscreteKurganovTadmorScheme.cuh:18,
 *                                FullyDiscreteKurganovTadmorScheme.cu:109-139) followed by
 *                                the host swap setCurrentConservedVariables
 *                                (HydroPlugin.cpp:422)
 *   gvh_status                   (none: the reference printf()s NaN and Newton failures,
 *                                EnergyMomentumTensor.cu:43, 92-94)
 *
 * State arrays use the reference's layout: one array per field over the ghosted lattice
 * (nx+4)(ny+4)(nz+4), index i + (nx+4)*(j + (ny+4)*k) (DynamicalVariables.cu:32-35), interior
 * at i,j,k in [2, n+2) (LatticeParameters.h:13-15). Host or device pointers are accepted
 * (unified addressing). Field order (gvh_set_state / gvh_get_state): the evolved conserved
 * components in CONSERVED_VARIABLES order (DynamicalVariables.cuh:50-71) -- ttt ttx tty ttn,
 * then pitt pitx pity pitn pixx pixy pixn piyy piyn pinn if shear is evolved, then Pi if bulk
 * is evolved -- followed by e, p, ut, ux, uy, un, utp, uxp, uyp, unp (u one step earlier).
 */
#ifndef GVH_H_
#define GVH_H_

#ifdef __cplusplus
extern "C" {
#endif

#define GVH_OK 0
#define GVH_ERR_INVALID -1   /* bad argument or configuration */
#define GVH_ERR_CUDA -2      /* a CUDA call failed (message in gvh_last_error) */
#define GVH_ERR_NUMERIC -3   /* the step raised a status bit (see gvh_status) */
#define GVH_ERR_NOMEM -4     /* device allocation failed */
#define GVH_ERR_INTERNAL -5  /* an internal consistency check failed; the object that
                                reported it refuses further work */

/* status bits (gvh_status) */
#define GVH_STATUS_NAN 1u          /* an energy density came out NaN */
#define GVH_STATUS_NEWTON 2u       /* warning: a QCD-EoS Newton solve did not converge, even
                                      damped; like the reference (EnergyMomentumTensor.cu:42-44)
                                      the last iterate is used and the run goes on */
#define GVH_STATUS_DAMPED 4u       /* informational: a Newton solve needed the damped update
                                      (the reference switches to it after 5e5 undamped
                                      iterations, EnergyMomentumTensor.cu:37-38; here after 200) */
#define GVH_STATUS_BOUNDS 8u       /* the bounds-checked build (libgvh_bounds.so, compiled with
                                      GVH_BOUNDS_CHECK) found a stencil index outside the
                                      lattice's arrays and skipped that cell */
#define GVH_STATUS_ERRORS 9u       /* the bits that mean the state is not trustworthy */

#define GVH_EOS_QCD 0              /* Wuppertal-Budapest fit (the reference default) */
#define GVH_EOS_CONFORMAL 1        /* p = e/3 (CONFORMAL_EOS, EquationOfState.cuh:16) */

#define GVH_COORDINATES_MILNE 0     /* (tau, x, y, eta): the reference's default */
#define GVH_COORDINATES_CARTESIAN 1 /* (t, x, y, z): USE_CARTESIAN_COORDINATES, SourceTerms.cu:25 */

#define GVH_PRECISION_FP64 0       /* plain FP64 path */
#define GVH_PRECISION_MIXED 1      /* FP32 fluxes/limiter/sources, FP64 state and root find */

/* Same members, order and types as the reference's struct LatticeParameters
 * (LatticeParameters.h:17-31), so a pointer to one can be passed as the other. */
typedef struct gvh_lattice_params {
	int numLatticePointsX;
	int numLatticePointsY;
	int numLatticePointsRapidity;
	int numComputationalLatticePointsX;
	int numComputationalLatticePointsY;
	int numComputationalLatticePointsRapidity;
	int numProperTimePoints;
	double latticeSpacingX;
	double latticeSpacingY;
	double latticeSpacingRapidity;
	double latticeSpacingProperTime;
} gvh_lattice_params;

/* Same layout as the reference's struct HydroParameters (HydroParameters.h:15-22). */
typedef struct gvh_hydro_params {
	double initialProperTimePoint;
	double shearViscosityToEntropyDensity;
	double freezeoutTemperatureGeV;
	int initializePimunuNavierStokes;
	double regulationTemperatureGeV;
} gvh_hydro_params;

/* The reference's compile-time switches, chosen at run time here. */
typedef struct gvh_options {
	int eos;        /* GVH_EOS_* (reference: CONFORMAL_EOS macro) */
	int shear;      /* evolve pi^{mu nu} (reference: PIMUNU macro, DynamicalVariables.cuh:13) */
	int bulk;       /* evolve Pi, needs shear (reference: PI macro, DynamicalVariables.cuh:14) */
	int precision;  /* GVH_PRECISION_* (reference: PRECISION macro, DynamicalVariables.cuh:44) */
	double theta;   /* minmod limiter slope, > 0 (reference: THETA 2.0, FluxLimiter.cu:15) */
	int device;     /* CUDA device ordinal; -1 = current device */
	int coordinates; /* GVH_COORDINATES_* (reference: USE_CARTESIAN_COORDINATES, off as shipped:
	                    SourceTerms.cu:25). Cartesian replaces only the geometric sources of
	                    T^{tau mu} (SourceTerms.cu:738-743), as the reference's switch does; the
	                    rest of the step keeps its Milne form there too */
} gvh_options;

typedef struct gvh_handle gvh_handle;

/* Fills opts with the reference's shipped configuration: QCD EoS, shear + bulk, theta 2.0,
 * FP64, current device, Milne coordinates. */
void gvh_default_options(gvh_options *opts);

int gvh_create(const gvh_lattice_params *lattice, const gvh_hydro_params *hydro, const gvh_options *opts,
               gvh_handle **out);
int gvh_destroy(gvh_handle *h);

/* Number of evolved conserved components (4, 14 or 15) and of state fields (+10). */
int gvh_num_conserved(const gvh_handle *h);
int gvh_num_fields(const gvh_handle *h);
/* Ghosted lattice size (nx+4)(ny+4)(nz+4): the length of every state array. */
long long gvh_num_lattice_cells(const gvh_handle *h);

/* Initial state from primitive fields on the interior of ghosted arrays: prim[0]=e,
 * prim[1..4]=ut,ux,uy,un, then the evolved dissipative components (pitt..pinn, Pi).
 * Sets p = p(e), T^{tau mu} from (e, p, u, pi, Pi), u one step earlier = u. */
int gvh_set_primitive_state(gvh_handle *h, const double *const *prim, int n_prim);
/* The same with the pressure given (a ghosted array) instead of p(e) of the EoS, as the type-11
 * reader sets it from its file (InitialConditions.cpp:60); T^{tau mu} is built with it
 * (setConservedVariables, DynamicalVariables.cu:349-392). */
int gvh_set_primitive_state_p(gvh_handle *h, const double *const *prim, int n_prim, const double *p_ghosted);
int gvh_set_state(gvh_handle *h, const double *const *fields, int n_fields);

/* A Glauber-hotspot initial state, generated on the device (the seeded event generator of
 * the benchmark's events; the reference builds its initial states on the host, e.g. its
 * Monte-Carlo Glauber model, MonteCarloGlauberModel.cpp:19-110 with InitialConditions.cpp
 * :1168-1245). The caller draws the sources (nucleon participants and weights); the lattice
 * fill runs on the device:
 *   e(x, y, eta) = fz(eta) * scale * sum_p w_p exp(-((x - x_p)^2 + (y - y_p)^2) / (2 sigma^2))
 *                  + background,   fz = exp(-max(|eta| - eta_flat, 0)^2 / (2 sigma_eta^2)),
 * on the cell centres x_i = (i - (nx - 1)/2) dx (likewise y, eta), each value rounded to float
 * and + 1e-3 as the type-10 reader stores a value written to its files
 * (InitialConditions.cpp:106, 122-124); u = (1, 0, 0, 0), pi^{mu nu} = Pi = 0, p = p(e). Only
 * the 3n source values cross to the device. */
typedef struct gvh_hotspots {
	int n;               /* sources */
	const double *x;     /* source positions (fm) and weights: host arrays of n values */
	const double *y;
	const double *w;
	double sigma;        /* Gaussian width of a source (fm) */
	double scale;        /* multiplies the weighted sum (fm^-4) */
	double eta_flat;     /* |eta| up to which the longitudinal profile is flat */
	double sigma_eta;    /* width of its Gaussian tails */
	double background;   /* added everywhere (fm^-4) */
} gvh_hotspots;
int gvh_set_hotspot_state(gvh_handle *h, const gvh_hotspots *hs);

/* Null entries are skipped. Ghost layers come back zero-gradient filled, edges and
 * corners included. Synchronises the handle's stream. */
int gvh_get_state(gvh_handle *h, double *const *fields, int n_fields);
/* The seam of the drop-in twoStepRungeKutta (gpu-vh_b200/dropin/twoStepRungeKutta_gvh.cu),
 * which replaces FullyDiscreteKurganovTadmorScheme.cu:109-139 inside the reference's own
 * program: the reference's device state arrays -- the components behind d_q / d_Q, d_e, d_p,
 * and the components behind d_u, d_up (DynamicalVariables.cuh:101-117) -- go into and out of
 * the handle with one gather launch and one scatter launch for all fields, converted from and
 * to the reference's PRECISION (elem_bytes 4: float, as shipped; 8: its double build). Device
 * pointers only, in gvh_set_state's field order, ghosted layout. Both calls are queued on the
 * handle's stream and return without waiting. gather: a null up entry takes u.
 * scatter: null entries are skipped; every ghost cell of a written field is filled with its
 * nearest interior cell (the reference's zero-gradient faces, setGhostCells, GhostCells.cu
 * :15-144; edges and corners alike). */
int gvh_gather_state_device(gvh_handle *h, const void *const *fields, int n_fields, int elem_bytes);
int gvh_scatter_state_device(gvh_handle *h, void *const *fields, int n_fields, int elem_bytes);
/* Pipelined set/get for a caller that streams states through the handle (a new state in,
 * one or more steps, the result out, again and again): the copies go on the handle's own
 * copy streams, one each way, through two device staging areas each way used in turn (four
 * copies of the ghosted state, allocated on the first call), and are ordered with the
 * handle's stream by events, so the next state's copy in, the step and the last result's
 * copy out overlap, and neither direction's copies wait for the layout conversion of the
 * call before. The calls return without waiting. Host arrays should be
 * pinned (pageable memory still works but the copies then serialise) and must not be
 * touched until gvh_synchronize(h) returns. gvh_join_async(h) joins the handle's stream
 * and its copy streams both ways: work queued on the handle's stream afterwards waits for
 * every copy queued so far, and copies queued afterwards wait for the work queued on the
 * handle's stream so far (so that events recorded on the handle's stream on either side of
 * a join bracket the copies too). */
int gvh_set_state_async(gvh_handle *h, const double *const *fields, int n_fields);
int gvh_get_state_async(gvh_handle *h, double *const *fields, int n_fields);
int gvh_join_async(gvh_handle *h);

/* One Heun RK2 step from time t (t and dt as twoStepRungeKutta takes them). Cells with
 * e <= e(T_reg) have pi^{mu nu} regulated; T_reg is in fm^-1 and 0 (the reference's default
 * configuration) regulates nothing, since e(0) lies below every energy density.
 * Asynchronous on the handle's stream. */
int gvh_rk2_step(gvh_handle *h, double t, double dt, double T_reg);

/* Waits for the handle's stream and reports the status bits raised since the last
 * gvh_clear_status in *flags (may be null). Returns GVH_ERR_NUMERIC when an error bit
 * (GVH_STATUS_ERRORS) is set, else GVH_OK. */
int gvh_status(gvh_handle *h, unsigned *flags);
int gvh_clear_status(gvh_handle *h);
int gvh_synchronize(gvh_handle *h);

/* One RK2 step on caller-owned device arrays that allocates nothing (no counterpart in the
 * reference). For callers that own all their device memory and cannot allocate at step
 * time -- a run loop with a fixed memory plan, a framework pool allocator that forbids
 * foreign cudaMalloc, a region where an allocation would synchronise the device. The
 * intermediate RK stage lives in a 32 MiB array compiled into the library (held on every
 * GPU that loads it until exit), so the interior lattice is limited to
 * (gvh_rk2_step_noalloc_max_bytes() - 256) / ((nq + 5) * 8) cells (about 200k cells with
 * shear + bulk); larger lattices are rejected with GVH_ERR_INVALID.
 * Arrays are interior-only (no ghosts), cell s = i + nx*(j + ny*k), components stacked with
 * stride nx*ny*nz: q (nq components; in q^n, out q^{n+1}), e and p (in/out), u_prev (u one
 * step earlier) and u (current u^mu, 4 components each; read only), u_next (out u^{n+1};
 * must not alias u or u_prev). The step is queued on `stream` (a cudaStream_t, NULL = the
 * legacy default stream); if status_out is not null the call waits and stores the
 * GVH_STATUS_* bits. With opts->device >= 0 the work runs on that device and the caller's
 * current device is current again when the call returns. The first call on a device looks
 * up the scratch address (do it before any stream capture). All calls share the scratch and
 * its status word, which each call clears: calls whose work overlaps on the GPU race, so
 * order them. */
int gvh_rk2_step_noalloc(const gvh_lattice_params *lattice, const gvh_hydro_params *hydro, const gvh_options *opts,
                         double t, double dt, double T_reg, double *q, double *e, double *p, const double *u_prev,
                         const double *u, double *u_next, unsigned *status_out, void *stream);
long long gvh_rk2_step_noalloc_max_bytes(void);
const char *gvh_noalloc_last_error(void);

/* Maximum interior energy density of the current state (fm^-4), reduced on the device;
 * with e(T_fo) it gives the reference's stop test (HydroPlugin.cpp:396-413) without copying
 * the lattice to the host. Synchronises the handle's stream. */
int gvh_max_energy_density(gvh_handle *h, double *out);

/* The CFL bound of the step: the largest local propagation speed over the lattice spacing,
 * max over interior cells, both faces and the axes with more than one cell of a / dx_axis
 * (a one-cell axis, eta of a 2+1D lattice, has no faces), where a is the KT
 * spectral radius max(|u^i/u^tau| left, |u^i/u^tau| right) of the face
 * (SpectralRadius.cu:17-30, LocalPropagationSpeed.cu:15-24), in fm^-1 (dtau times it is the
 * CFL number). The first stage of every gvh_rk2_step keeps a running maximum of it, reduced on
 * the device by warp shuffles from the face recoveries the step does anyway; the step itself
 * keeps the caller's dt, as the reference does. Returns the maximum over the steps since the
 * previous call (or since gvh_create) and starts a new one; 0 before any step. Synchronises
 * the handle's stream. (The reference computes these speeds inside its flux and keeps no
 * maximum.) */
int gvh_max_propagation_speed(gvh_handle *h, double *out);

/* Validity diagnostics of the fluid-dynamic description (checkValidityKernel,
 * HydrodynamicValidity.cu:18-226, and the regulation factor of RegulateDissipativeCurrents.cu:132):
 * when enabled, every gvh_rk2_step also computes them for the new level, one extra kernel
 * after the second stage (the reference runs them in every step). They are read back as the
 * 13 members of the reference's VALIDITY_DOMAIN (DynamicalVariables.cuh:82-98), in its order:
 * regulations, knudsenNumberTaupi, knudsenNumberTauPi, inverseReynoldsNumberPimunu,
 * inverseReynoldsNumber2Pimunu (never written, 0), inverseReynoldsNumberTilde2Pimunu,
 * inverseReynoldsNumberPi, inverseReynoldsNumber2Pi (never written, 0),
 * inverseReynoldsNumberTilde2Pi, taupi, dxux, dyuy, theta; ghosted arrays like
 * gvh_get_state's (a NULL entry skips a field). */
#define GVH_VALIDITY_FIELDS 13
int gvh_enable_validity(gvh_handle *h, int on);
int gvh_get_validity(gvh_handle *h, double *const *fields, int n_fields);

/* e(T) of the equation of state (equilibriumEnergyDensity, EquationOfState.cu:150-204) at
 * T = T_GeV / hbarc, in fm^-4: the freeze-out threshold of HydroPlugin.cpp:131-135. */
double gvh_energy_density_of_temperature(int eos, double T_GeV);

/* Checkpoint and resume (the reference has none: its field dumps are text in another order
 * than its readers expect, FileIO.cpp:47-56 against InitialConditions.cpp:119-121). A binary
 * snapshot of the handle's state -- the interior lattice's nq + 10 fields, with the lattice
 * sizes, options, spacings, the caller's time tau and step count, and a checksum -- is written
 * after the work queued so far; gvh_load_state restores it into a handle of the same lattice
 * and physics (else GVH_ERR_INVALID), checking the file before changing anything, and returns
 * tau and step (may be null). Steps from a restored state give the values the original run
 * gives. */
int gvh_save_state(gvh_handle *h, const char *path, double tau, long long step);
int gvh_load_state(gvh_handle *h, const char *path, double *tau, long long *step);

/* Runs the handle's work on a caller-owned stream (a cudaStream_t passed as void*); NULL
 * returns to the handle's own stream. Waits for work already queued on the old stream. */
int gvh_set_stream(gvh_handle *h, void *stream);

/* Number of stage-kernel launches one gvh_rk2_step issues. */
int gvh_launches_per_step(const gvh_handle *h);

const char *gvh_last_error(void);

/* ------------------------------------------------------------------------------------
 * Batched events (no counterpart in the reference, which runs one event per process:
 * HydroPlugin.cpp:107-434). A batch owns one HBM arena and advances every admitted event
 * together: the stage kernel walks a packed queue of 128-cell tiles of all events, and one
 * RK2 step (stage 1, stage 2, per-event bookkeeping) is a CUDA graph replayed per step. All
 * events of a batch share the options (EoS, shear/bulk, precision, theta); each has its own
 * lattice, spacings, dtau, tau0, eta/s, T_fo and T_reg (from its parameters). Each event
 * advances exactly as a gvh_handle with the same inputs would, until it has frozen out by
 * the reference's stop rule; from then on it stays at that state (the reference's loop ends
 * there). Admission, removal and serving rounds are queued on the batch's stream without
 * waiting for the device.
 * ---------------------------------------------------------------------------------- */
typedef struct gvh_batch gvh_batch;

typedef struct gvh_event_info {
	long long step;                   /* RK2 steps completed */
	double tau;                       /* proper time reached: tau0 + step * dtau */
	double max_energy_density;        /* max interior e after the last step (fm^-4) */
	double freezeout_energy_density;  /* e(T_fo) */
	int frozen_checks;                /* steps (initial state included) with max e <= e(T_fo) */
	int frozen_out;                   /* frozen_checks >= 11, the reference's stop rule
	                                     (FOFREQ+1 all-frozen checks, HydroPlugin.cpp:396-413) */
	unsigned status;                  /* GVH_STATUS_* bits raised by this event */
	long long cells;                  /* interior cells */
} gvh_event_info;

/* HBM bytes one event of this lattice takes in a batch arena. */
long long gvh_batch_event_bytes(const gvh_lattice_params *lattice, const gvh_options *opts);
int gvh_batch_create(const gvh_options *opts, long long arena_bytes, gvh_batch **out);
int gvh_batch_destroy(gvh_batch *b);
int gvh_batch_set_stream(gvh_batch *b, void *stream);
/* Admits an event from primitive fields (same arrays as gvh_set_primitive_state; host or
 * device pointers). Returns GVH_ERR_NOMEM without side effects when the arena cannot hold it.
 * The arrays are copied before the call returns (host arrays into pinned staging); the
 * event's set-up is queued behind the work in flight. */
int gvh_batch_add_event(gvh_batch *b, const gvh_lattice_params *lattice, const gvh_hydro_params *hydro,
                        const double *const *prim, int n_prim, int *event_id);
/* The same with the initial state generated on the device from hotspot sources (as
 * gvh_set_hotspot_state): only the sources cross to the device. */
int gvh_batch_add_event_hotspots(gvh_batch *b, const gvh_lattice_params *lattice, const gvh_hydro_params *hydro,
                                 const gvh_hotspots *hotspots, int *event_id);
int gvh_batch_remove_event(gvh_batch *b, int event_id);
int gvh_batch_num_events(const gvh_batch *b);
long long gvh_batch_free_bytes(const gvh_batch *b);
long long gvh_batch_active_cells(const gvh_batch *b);
/* Queues nsteps RK2 steps of every admitted event (asynchronous). */
int gvh_batch_step(gvh_batch *b, int nsteps);
int gvh_batch_synchronize(gvh_batch *b);
int gvh_batch_event_info(gvh_batch *b, int event_id, gvh_event_info *info);
int gvh_batch_get_state(gvh_batch *b, int event_id, double *const *fields, int n_fields);
/* Stage-kernel grid: 0 = one 128-thread block per 128-cell tile (the default), n > 0 = a
 * persistent grid of n blocks walking the tile queue. */
int gvh_batch_launch_config(const gvh_batch *b, int *grid_blocks, int *block_threads);
int gvh_batch_set_grid(gvh_batch *b, int grid_blocks);
/* Tile shape: tile_x = 0 (the default), 128 consecutive cells of an event; tile_x > 0 (a
 * divisor of 128), blocks of tile_x x (128 / tile_x) cells of one eta plane. */
int gvh_batch_set_tile_shape(gvh_batch *b, int tile_x);
int gvh_batch_tile_shape(const gvh_batch *b, int *tile_x, int *tile_y);
/* Chooses the schedule by timing `steps` real steps per candidate -- tile shapes 128
 * consecutive cells, 32 x 4 and 16 x 8, each with one block per tile and persistent grids of
 * 1..4 blocks per SM (the events advance; every candidate computes the same values). The
 * chosen grid is returned, the chosen shape is read with gvh_batch_tile_shape. */
int gvh_batch_autotune(gvh_batch *b, int steps, int *chosen_grid);
/* Serving rounds. gvh_batch_round queues nsteps RK2 steps of every admitted event and then a
 * copy of every event's bookkeeping into mapped host memory, and returns the round's ticket
 * without waiting. gvh_batch_poll waits for that round only (not for work queued after it)
 * and gives, for each event admitted when the round was queued and still admitted now, its
 * id and its gvh_event_info at the end of the round (up to max_events; *n_events is the
 * count), and the round's device time in ms (round_ms may be null). Two rounds can be in
 * flight: a round's snapshot is overwritten two rounds later, so poll ticket k before
 * queueing round k + 2 (gvh_batch_round waits for round k - 2 to finish). */
int gvh_batch_round(gvh_batch *b, int nsteps, long long *ticket);
int gvh_batch_poll(gvh_batch *b, long long ticket, int max_events, int *event_ids, gvh_event_info *infos,
                   int *n_events, double *round_ms);
const char *gvh_batch_last_error(void);

/* ------------------------------------------------------------------------------------
 * Host side of a run: the reference's run-time inputs and run loop (libgvh.so).
 * ---------------------------------------------------------------------------------- */

/* Same layout as the reference's struct InitialConditionParameters
 * (InitialConditionParameters.h:13-26). */
typedef struct gvh_ic_params {
	int initialConditionType;
	int numberOfNucleonsPerNuclei;
	int numberOfSourceFiles;
	double initialEnergyDensity;
	double scatteringCrossSectionNN;
	double impactParameter;
	double fractionOfBinaryCollisions;
	double rapidityVariance;
	double rapidityMean;
	int sourceType;
} gvh_ic_params;

typedef struct gvh_run_report {
	long long steps;                  /* RK2 steps taken */
	double tau_end;                   /* proper time reached */
	double average_ms_per_step;       /* wall time per step ("Average time/step",
	                                     HydroPlugin.cpp:426) */
	int frozen_out;                   /* stopped by the freeze-out rule (else by numProperTimePoints) */
	unsigned status;                  /* GVH_STATUS_* bits */
	double freezeout_energy_density;  /* e(T_fo) in fm^-4 */
	long long surface_elements;       /* rows written to surface.dat */
	double surface_seconds;           /* wall time of the freeze-out surface finder */
	long long surface_hypercubes;     /* crossed hypercubes over all slabs */
	double surface_bytes_to_host;     /* bytes the finder copied from the device */
	double surface_host_seconds;      /* of surface_seconds: host cornelius and formatting */
} gvh_run_report;

/* gvh_run outputs (bit flags) */
#define GVH_RUN_FIELDS 1  /* field dumps every 10 steps (FileIO.cpp:15-60) */
#define GVH_RUN_SURFACE 2 /* <output_dir>/surface.dat, the reference's freeze-out surface */

/* Positional .properties readers: readLatticeParameters (LatticeParameters.cpp:65-138),
 * readHydroParameters (HydroParameters.cpp:49-98), readInitialConditionParameters
 * (InitialConditionParameters.cpp:65-149). Line n is field n; lines a file lacks leave 0
 * (the shipped hydro.properties has no regulation temperature: T_reg = 0). */
int gvh_read_lattice_parameters(const char *config_dir, gvh_lattice_params *out);
int gvh_read_hydro_parameters(const char *config_dir, gvh_hydro_params *out);
int gvh_read_ic_parameters(const char *config_dir, gvh_ic_params *out);

/* Initial-condition type 10 (setInitialTmunuFromFiles, InitialConditions.cpp:98-489): reads
 * <root>/input/{e,ut,ux,uy,un}.dat, then pitt..pinn if shear and bulk.dat if bulk, into
 * ghosted arrays ordered as gvh_set_primitive_state takes them; e gets +1e-3. */
int gvh_read_ic_files(const char *root_dir, const gvh_lattice_params *lattice, int shear, int bulk,
                      double *const *prim, int n_prim);

/* Initial-condition type 11 (setInitialTmunuFromFile, InitialConditions.cpp:29-97): reads
 * <root>/input/Tmunu.dat (20 columns: x y z e p ut ux uy un pitt..pinn Pi) into ghosted arrays
 * ordered as gvh_set_primitive_state takes them (e gets +1e-3) and the pressure into p_out;
 * pass both to gvh_set_primitive_state_p. */
int gvh_read_ic_tmunu(const char *root_dir, const gvh_lattice_params *lattice, int shear, int bulk,
                      double *const *prim, int n_prim, double *p_out);

/* One field dump in the reference's output format (output(), FileIO.cpp:15-60). */
int gvh_write_field(const char *output_dir, const char *name, double tau, const gvh_lattice_params *lattice,
                    const double *field_ghosted);

/* The run loop of run() (HydroPlugin.cpp:107-434) for initial-condition types 10 and 11: read the
 * input files, then for n = 1 .. numProperTimePoints+1: dump fields every 10 steps
 * (GVH_RUN_FIELDS), find the freeze-out surface of the last slab and write it to
 * <output_dir>/surface.dat in chunks of 10 steps as the reference does (GVH_RUN_SURFACE;
 * the reference writes output/surface.dat relative to its working directory), stop after 11
 * checks with every cell at or below e(T_fo), take one RK2 step. Other initial-condition
 * types (generated by the reference's own code) return GVH_ERR_INVALID. */
int gvh_run(const gvh_lattice_params *lattice, const gvh_ic_params *ic, const gvh_hydro_params *hydro,
            const char *root_dir, const char *output_dir, const gvh_options *opts, int outputs,
            gvh_run_report *report);

/* The same loop on a handle whose initial state the caller has set (gvh_set_primitive_state or
 * gvh_set_state; an in-memory initial condition instead of input files): output_dir may be
 * NULL for no output. The handle is left at the last level reached. */
int gvh_run_loop(gvh_handle *h, const gvh_lattice_params *lattice, const gvh_hydro_params *hydro,
                 const char *output_dir, int outputs, gvh_run_report *report);

/* The reference's labels for the slab between time levels k and k+1 (HydroPlugin.cpp:262-314,
 * FOFREQ = 10): its rows go to the file at loop iteration *flush_iteration (state = level
 * flush_iteration - 1), with tau_label added to the centroid's tau and the normal multiplied by
 * tau_scale. Slabs of a chunk whose flush iteration the loop does not reach are not written. */
void gvh_surface_slab_labels(long long k, double tau0, double dtau, double *tau_label, double *tau_scale,
                             long long *flush_iteration);
const char *gvh_plugin_last_error(void);

/* ---- Freeze-out hypersurface (surface.dat) ------------------------------------------------
 *
 * Replaces the reference's host freeze-out finder: the FOFREQ+1 host copies of ten fields
 * (FreezeOut.cpp:45-160, filled from a full device-to-host copy every step,
 * HydroPlugin.cpp:264-281), the scan of every hypercube with cornelius
 * (HydroPlugin.cpp:283-305, freezeout/cornelius-c++-1.3/cornelius.cpp) and the
 * interpolated surface.dat row of each element (HydroPlugin.cpp:306-372, FreezeOut.cpp:1-43,
 * 242-280). A gvh_surface keeps one time level of u^x, u^y, u^eta, e, pi^{xx,xy,x eta,yy,y eta}
 * and Pi of its handle on the device; gvh_surface_find marks on the device the hypercubes of
 * the slab (that level, the handle's current level) which the surface e = e_freezeout
 * crosses, copies only their corner data to the host, runs the cornelius algorithm there on
 * a pool of host threads and keeps the slab's rows in the reference's order (x outer, then
 * y, then eta). The 3+1D case (nz > 1) finds 4D elements, nz == 1 3D (tau, x, y) elements. */
typedef struct gvh_surface gvh_surface;

#define GVH_SURFACE_COLUMNS 20 /* tau x y eta, tau*dsigma_mu (4), u^x u^y u^eta, e, T, p,
                                  pi^{xx,xy,x eta,yy,y eta}, Pi */

typedef struct {
  long long slabs;               /* gvh_surface_find calls */
  long long hypercubes_last;     /* hypercubes crossed in the last slab */
  long long hypercubes_total;
  long long points_last;         /* lattice points copied to the host for the last slab */
  long long elements_last;       /* surface elements (rows) of the last slab */
  long long elements_total;
  long long errors_total;        /* hypercubes where the algorithm stops (the reference exits) */
  double bytes_to_host_total;
  double device_seconds_total;   /* marking, compaction and copies, host wall clock */
  double host_seconds_total;     /* cornelius, interpolation and formatting */
} gvh_surface_info;

/* e_freezeout: the surface's energy density (fm^-4), e(T_fo) in the reference
 * (HydroPlugin.cpp:131-135). Needs nx > 1 and ny > 1 (the reference's finder handles
 * nothing else, HydroPlugin.cpp:157-182). The handle must outlive the surface. */
int gvh_surface_create(gvh_handle *h, double e_freezeout, gvh_surface **out);
int gvh_surface_destroy(gvh_surface *s);
/* Host threads of the cornelius stage (default: the machine's hardware threads). */
int gvh_surface_set_threads(gvh_surface *s, int nthreads);
/* What gvh_surface_find keeps of each slab (default both): binary rows, text, or both. */
#define GVH_SURFACE_ROWS 1
#define GVH_SURFACE_TEXT 2
int gvh_surface_set_outputs(gvh_surface *s, int outputs);
/* Where a slab's elements and rows are made. 1 (the default for the QCD EoS): on the device,
 * one thread per crossed hypercube running the same cornelius and row code as the host pool,
 * without FMA contraction, so the rows are the same to the last bit; only the rows are
 * copied to the host, which formats them. 0: the corner values go to the host and the host
 * pool makes the rows (the only form for the conformal EoS, whose T(e) = (e/13.8997)^(1/4)
 * is a pow the device does not evaluate as the host's libm does; 1 is refused there). */
int gvh_surface_set_device_rows(gvh_surface *s, int on);
/* Takes the handle's current state as the lower time level of the next slab. */
int gvh_surface_set_lower(gvh_surface *s);
/* Elements of the slab (lower level, handle's current level); then the current level becomes
 * the lower one. tau_label is added to each element's centroid tau and tau_scale multiplies
 * its normal, as the reference labels its rows (HydroPlugin.cpp:298-314). */
int gvh_surface_find(gvh_surface *s, double tau_label, double tau_scale, long long *n_elements);
/* gvh_surface_find in two halves, so that the host half of one slab overlaps the device's
 * next steps: _begin marks and compacts the slab on the device and queues the copies to the
 * host on the handle's stream (later work the caller queues there, such as gvh_rk2_step,
 * runs after them); _end waits for those copies and runs the host half. One slab at a time:
 * _begin again before _end is an error. */
int gvh_surface_find_begin(gvh_surface *s, double tau_label, double tau_scale);
int gvh_surface_find_end(gvh_surface *s, long long *n_elements);
/* The last slab's rows: n_elements x GVH_SURFACE_COLUMNS doubles, or as the text the
 * reference writes (ostream default format, space separated, one row per line). The text
 * stays valid until the next gvh_surface_find. */
int gvh_surface_get_rows(gvh_surface *s, double *rows, long long max_rows);
int gvh_surface_get_text(gvh_surface *s, const char **text, long long *length);
int gvh_surface_get_info(const gvh_surface *s, gvh_surface_info *info);
const char *gvh_surface_last_error(void);

/* Iso-surface elements of one cube of dimension dim = 2, 3 or 4 (Cornelius::find_surface_2d,
 * _3d, _4d; cornelius.cpp:2115-2245). corners: 2^dim values, C order over the dim axes;
 * dx: dim edge lengths; iso: the surface value. Writes up to max_elements centroids and
 * normals (dim values each, relative to the cube's first corner; the normal is the
 * covariant surface vector pointing to lower values, without Jacobian factors) and their
 * count. Returns GVH_ERR_NUMERIC where the reference exits (cornelius.cpp:1287, 1552) and
 * GVH_ERR_INVALID for bad arguments or too small output arrays. Host only; no GPU needed. */
int gvh_cornelius(int dim, const double *corners, const double *dx, double iso, double *centroids, double *normals,
                  int max_elements, int *n_elements);

#ifdef __cplusplus
}
#endif
#endif /* GVH_H_ */
