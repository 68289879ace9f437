/*
 * vh_b200.h -- C ABI of the B200 implementation of the cpu-vh hot path
 * (Kurganov-Tadmor RK2 evolution of T^{tau mu}, pi^{mu nu}, Pi and the
 * Cornelius freezeout-surface search).
 *
 * Plain pointers and sizes only.  Every call returns an int status (VH_OK on
 * success).  An event handle owns its device buffers and one CUDA stream; calls
 * on different handles may run from different host threads.  Host arrays are
 * caller-owned.
 *
 * Lattice layout shared with the reference: SoA arrays over the padded grid
 * ncx*ncy*ncz = (nx+4)(ny+4)(nz+4), index i + ncx*(j + ncy*k), two ghost
 * cells per side (DynamicalVariables.cpp:35-41, LatticeParameters.h:13-15).
 * "Interior" arrays are nx*ny*nz with index i + nx*(j + ny*k).
 *
 * Units follow the reference: lengths in fm, energy densities in fm^-4,
 * temperatures in fm^-1, except where a name ends in _GeV.
 */
#ifndef VH_B200_H
#define VH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define VH_OK              0
#define VH_ERR_ARG         1   /* bad argument / size / null pointer                     */
#define VH_ERR_CUDA        2   /* a CUDA runtime call failed (message: vh_last_error)     */
#define VH_ERR_NOMEM       3   /* device allocation failed                                */
#define VH_ERR_NAN         4   /* NaN energy density, Newton f/fp or regulation factor:   */
                               /* the reference prints and exit(-1)s here                 */
                               /* (EnergyMomentumTensor.cpp:42, :197-203;                 */
                               /*  FullyDiscreteKurganovTadmorScheme.cpp:849, :854)       */
#define VH_ERR_CORNELIUS   5   /* Cornelius edge/polygon construction error (cornelius.cpp:1250-1252, :1589-1591) */
#define VH_ERR_CAPACITY    6   /* caller buffer too small (the count is still returned)   */
#define VH_ERR_NODEVICE    7   /* no CUDA device / the CUDA path is not available         */
#define VH_ERR_STATE       8   /* call out of order (e.g. step before set_initial)        */

/* EoS kinds (EquationOfState.h:13-15) */
#define VH_EOS_CONFORMAL   0   /* e = a T^4, p = e/3                                      */
#define VH_EOS_TABLE       1   /* uniform-in-e table, EquationOfState.cpp:292-360         */

/* bulk viscosity laws zeta/s(T) */
#define VH_ZETA_REFERENCE  0   /* SourceTerms.cpp:40-48                                   */
#define VH_ZETA_GAUSSIAN   1   /* zeta_norm * exp(-((T_GeV - zeta_T0_GeV)/zeta_width_GeV)^2) */

/* arithmetic modes */
#define VH_PREC_FP64       0   /* FP64 throughout, op-for-op with the reference (parity)  */
#define VH_PREC_MIXED      1   /* FP32 limiter, flux and source arithmetic; FP64 conserved */
                               /* variables, RK accumulation, root solve, EoS and storage  */

/* field ids for vh_event_get_field / vh_event_set_field */
#define VH_F_Q0            0   /* 0..14: ttt ttx tty ttn pitt pitx pity pitn pixx pixy pixn piyy piyn pinn Pi */
#define VH_F_UT          100   /* 100..103: u^tau u^x u^y u^eta  */
#define VH_F_UPT         110   /* 110..113: previous-step u (the reference's `up`) */
#define VH_F_E           200
#define VH_F_P           201
#define VH_F_W           300   /* 300..305: thermal vorticity w_tx w_ty w_tn w_xy w_xn w_yn (vh_event_vorticity) */
#define VH_F_BETA        310   /* 310..313: thermal velocity beta_t beta_x beta_y beta_n = u_mu / T */
#define VH_F_REGFAC      400   /* 400, 401: regulation factors regFacShear, regFacBulk (vh_event_keep_regulation) */

/* columns of one freezeout element, the 20 columns of surface.dat
 * (FreezeOut.cpp:265-270): tau x y eta  ds0 ds1 ds2 ds3  ux uy un  e T P
 * pixx pixy pixn piyy piyn  Pi */
#define VH_FO_COLUMNS     20

typedef struct vh_config {
    int nx, ny, nz;            /* interior lattice points (LatticeParameters.h:19-21)            */
    double dx, dy, dz;         /* lattice spacings [fm], [fm], [1] (LatticeParameters.h:28-30)   */
    double dt;                 /* time step [fm/c] (LatticeParameters.h:31)                      */
    double t0;                 /* initial proper time [fm/c] (HydroParameters.h:17)              */
    double etabar;             /* eta/s (HydroParameters.h:18)                                   */
    double T_freezeout_GeV;    /* HydroParameters.h:19                                           */
    double T_reg_GeV;          /* regulation temperature (HydroParameters.h:21)                  */
    int fo_factor;             /* coarseProperTimeFOFactor (LatticeParameters.h:26)              */
    double theta;              /* minmod limiter theta (FluxLimiter.h:13)                        */
    int eos_kind;              /* VH_EOS_*                                                       */
    double eos_factor;         /* a of the conformal EoS (EquationOfState.h:19)                  */
    int bulk;                  /* 1: evolve Pi (DynamicalVariables.h:14, `PI`)                   */
    int zeta_law;              /* VH_ZETA_*                                                      */
    double zeta_norm, zeta_T0_GeV, zeta_width_GeV;
    int precision;             /* VH_PREC_*                                                      */
} vh_config;

typedef struct vh_event vh_event;

/* ------------------------------------------------------------- library */
/* The reference's shipped settings: rhic-conf properties defaults plus the
 * compile-time macros THETA 1.1, CONFORMAL_EOS, EOS_FACTOR 13.8997, PIMUNU on,
 * PI off. */
int vh_config_default(vh_config *cfg);

/* Number of conserved components evolved for cfg (14 or 15). */
int vh_config_nq(const vh_config *cfg);

/* Last error message of the calling thread ("" if none). */
const char *vh_last_error(void);

/* 1 if a CUDA device is usable, else 0. */
int vh_device_available(void);

/* ---------------------------------------------------------- event API */
/* Create an event on the current CUDA device.  For VH_EOS_TABLE, eos_rows holds
 * eos_nrows rows of (e [GeV/fm^3], P [GeV/fm^3], s [fm^-3], T [GeV]) on a
 * uniform e grid -- the record layout of EoS/hrg_hotqcd_eos_binary.dat
 * (EquationOfState.cpp:308-324); nrows in [2, 100000]. */
int vh_event_create(const vh_config *cfg, const double *eos_rows, int eos_nrows, vh_event **out);
int vh_event_destroy(vh_event *ev);

/* Replaces the state with an initial condition given over the interior:
 * e, p [fm^-4]; u as 4 planes (ut, ux, uy, un); pi as 10 planes
 * (pitt pitx pity pitn pixx pixy pixn piyy piyn pinn) or NULL for zero; Pi or
 * NULL.  Builds T^{tau mu} (DynamicalVariables.cpp:169-218) and the ghost
 * cells (DynamicalVariables.cpp:220-378) on the device; the previous-step
 * velocity is set equal to u.  Resets the step counter to 0 and t to t0. */
int vh_event_set_initial(vh_event *ev, const double *e, const double *p, const double *u,
                         const double *pi, const double *Pi);

/* Same, from device pointers (already resident in HBM). */
int vh_event_set_initial_device(vh_event *ev, const double *d_e, const double *d_p, const double *d_u,
                                const double *d_pi, const double *d_Pi);

/* Advance nsteps RK2 steps (rungeKutta2 + q<->Q swap + t = t0 + n dt,
 * FullyDiscreteKurganovTadmorScheme.cpp:867-924, HydroPlugin.cpp:292-307).
 * Asynchronous on the event's stream; errors detected on the device are
 * reported by vh_event_status or by the next synchronising call. */
int vh_event_step(vh_event *ev, int nsteps);

/* Wait for the event's stream; returns VH_ERR_NAN etc. if the device flagged
 * an error, with the step and cell index in *err_step, *err_cell (nullable). */
int vh_event_status(vh_event *ev, int *err_step, long long *err_cell);

/* Completed steps and current proper time. */
int vh_event_progress(vh_event *ev, int *steps_done, double *t);

/* Copy one padded field (ncx*ncy*ncz doubles) to host memory. */
int vh_event_get_field(vh_event *ev, int field, double *host_out);

/* One freezeout block of the driver loop (HydroPlugin.cpp:242-266) at loop
 * index n = steps_done + 1: shift the coarse time slabs, find the surface
 * elements of every (hyper)cube between the previous and the current slab
 * (callFOFinder2p1D / callFOFinder3p1D, FreezeOut.cpp:200-361) and count the
 * interior cells above the freezeout energy density (FreezeOut.cpp:364-381).
 * The elements stay on the device; *n_elements (nullable) and *n_above
 * (nullable) are written.  Order of elements: ix, iy, iz, element index --
 * the order in which the reference writes them. */
int vh_event_freezeout(vh_event *ev, int *n_elements, int *n_above);

/* The same block in two halves, so that the host can queue the freezeout of
 * many events before waiting for any: _launch queues the block on the
 * event's stream and returns; _finish waits for it and returns what
 * vh_event_freezeout returns.  The event must not be stepped in between. */
int vh_event_freezeout_launch(vh_event *ev);
int vh_event_freezeout_finish(vh_event *ev, int *n_elements, int *n_above);

/* Copy the elements of the last freezeout block to host memory, VH_FO_COLUMNS
 * doubles per element.  Returns VH_ERR_CAPACITY if cap_elements is too small. */
int vh_event_fetch_surface(vh_event *ev, double *host_out, int cap_elements, int *n_elements);

/* Kernel launches one vh_event_step(ev, 1) issues (2 RK stages; a stage is
 * one fused kernel on small lattices, or the source, x, y, [eta] flux and
 * finalize phase kernels on large ones). */
int vh_event_kernel_launches(vh_event *ev, int *per_step);

/* Initial conditions generated on the device directly into the event (no
 * host arrays), the same fields as vh_ic_glauber / vh_ic_hotspots followed by
 * vh_event_set_initial (pi = 0, Pi = 0); the values may differ from the host
 * generators' in the last bits (device exp).  Optical Glauber: the
 * reference's thickness geometry (GlauberModel.cpp:26-108) and longitudinal
 * plateau (InitialConditions.cpp:1046-1063); hotspots: 2+1D events only. */
int vh_event_init_glauber(vh_event *ev, double R, double a, double sigma_nn, double b, double e0_GeV,
                          double eta_flat, double eta_sigma);
int vh_event_init_hotspots(vh_event *ev, unsigned long long seed, double mean_spots, double w, double k_gamma,
                           double amp_mean_GeV, double R, double a);

/* Dynamical sources J^mu of the energy-momentum equations (the reference's
 * Source arrays, SourceTerms.cpp:584-587, filled from HDF5 files by
 * DynamicalSources.cpp for jet sources): interior arrays of the t, x, y, eta
 * components, nx*ny*nz values each, used by every following step until
 * replaced; st == NULL removes them.  A batch picks up a member's sources at
 * its next vh_batch_step. */
int vh_event_set_sources(vh_event *ev, const double *st, const double *sx, const double *sy, const double *sn);

/* Keep the regulation factors (regFacShear, regFacBulk of
 * regulateDissipativeCurrents, FullyDiscreteKurganovTadmorScheme.cpp:835-855:
 * 1 where e > e_reg, tanh(rho)/rho below) of the last RK stage in the fields
 * VH_F_REGFAC, VH_F_REGFAC + 1 (0 before the first step, as the reference's
 * calloc'd arrays).  Off by default: it costs one plane write per stage. */
int vh_event_keep_regulation(vh_event *ev, int enable);

/* Thermal vorticity (calculateThermalVorticity, Vorticity.cpp:6-171, which
 * the reference runs after the initial condition and after every step,
 * HydroPlugin.cpp:197-199, :302-305).  Enabling computes it for the current
 * state and then after every vh_event_step; the fields VH_F_W.. and
 * VH_F_BETA.. hold it (interior cells; ghost cells are 0).  Batched steps do
 * not update it. */
int vh_event_vorticity(vh_event *ev, int enable);

/* Per-phase device timing of the RK stages (no counterpart in the reference,
 * which times the whole loop, HydroPlugin.cpp:284-297).  While enabled,
 * vh_event_step records CUDA events between the stage kernels on the event's
 * stream.  vh_event_phase_times waits for the stream, writes per phase the
 * summed milliseconds and launch count since enabling (or since the previous
 * read), and clears the record. */
#define VH_PHASE_SOURCE 0   /* eulerStepKernelSource */
#define VH_PHASE_FLUX_X 1   /* eulerStepKernelX */
#define VH_PHASE_FLUX_Y 2   /* eulerStepKernelY */
#define VH_PHASE_FLUX_ETA 3 /* eulerStepKernelZ */
#define VH_PHASE_FINAL 4    /* convex combination, inference, regulation, ghosts */
#define VH_PHASE_FUSED 5    /* all of one stage in one kernel (small lattices) */
#define VH_NPHASES 6
int vh_event_phase_timing(vh_event *ev, int enable);
int vh_event_phase_times(vh_event *ev, double ms[VH_NPHASES], long long launches[VH_NPHASES]);

/* The CUDA stream (cudaStream_t) the event's work is queued on. */
int vh_event_stream(vh_event *ev, void **stream);

/* ------------------------------------------------------------------ batches
 * Many resident events advanced together (no counterpart in the reference,
 * which evolves one event per process, HydroPlugin.cpp:226-307).  A batch
 * refers to existing events (it owns none of their memory): one launch per
 * RK phase covers every member, a CUDA graph of one whole RK2 step is
 * replayed, and the tile shape, grid form and fused/split choice come from
 * timing the batch's own members.  In FP64 each member's results are
 * bit-identical to vh_event_step on it alone, whatever the tuning.  A mixed-
 * precision batch evaluates each face once in its flux phases (as single
 * events of 2^15 cells and more do) and its tuner keeps the phase kernels, so
 * its results do not depend on timing.  Members must share the EoS kind, bulk
 * on/off, the precision and the device, must have an initial state, and must
 * outlive the batch.
 * Between batch steps every single-event call (freezeout, fields, status,
 * even vh_event_step) may be used on a member; its stream is ordered after
 * the batch's work and the batch after its stream.
 */
typedef struct vh_batch vh_batch;

typedef struct vh_batch_tuning {
    int fused;                   /* 1: one kernel per RK stage; 0: the phase kernels      */
    int tile_x[VH_NPHASES];      /* tile (= 128-thread block) shape per phase, indexed by  */
    int tile_y[VH_NPHASES];      /* VH_PHASE_*: 32x4, 64x2, 16x8, 128x1 or 8x16             */
    int persistent[VH_NPHASES];  /* 1: grid of resident blocks striding over the tiles;    */
                                 /* 0: one block per tile                                   */
    double stage_ms;             /* measured RK stage-1 time of this choice (autotuner)    */
} vh_batch_tuning;

int vh_batch_create(vh_event *const *events, int n_events, vh_batch **out);
int vh_batch_destroy(vh_batch *b);
int vh_batch_size(vh_batch *b, int *n_events);
/* nsteps RK2 steps of every active member (autotunes on the first call).
 * A member whose device has flagged an error (vh_event_status) is no longer
 * computed by later steps (its state is invalid, as the reference's would be
 * at its exit): its error stays, its energy density stays that of the
 * failing step, and its step count advances with the batch. */
int vh_batch_step(vh_batch *b, int nsteps);
/* An inactive member is skipped (its tiles do no work) until re-activated. */
int vh_batch_set_active(vh_batch *b, int member, int active);
/* Run the tuner now (members' state is untouched) and report its choice. */
int vh_batch_autotune(vh_batch *b, vh_batch_tuning *out);
int vh_batch_get_tuning(vh_batch *b, vh_batch_tuning *out);
/* Fix the launch configuration (tile shapes must be one of the five). */
int vh_batch_set_tuning(vh_batch *b, const vh_batch_tuning *t);
/* Kernel launches per batch step (the step-argument kernel + both stages). */
int vh_batch_kernel_launches(vh_batch *b, int *per_step);
/* Per-phase device timing, as for events; while enabled the steps are
 * launched one by one instead of through the CUDA graph. */
int vh_batch_phase_timing(vh_batch *b, int enable);
int vh_batch_phase_times(vh_batch *b, double ms[VH_NPHASES], long long launches[VH_NPHASES]);
int vh_batch_stream(vh_batch *b, void **stream);

/* ------------------------------------------------------------------- server
 * An event server (no counterpart in the reference, which evolves one event
 * per process): events are submitted with their host initial condition at
 * any time; a worker thread admits them while their estimated device
 * footprint fits hbm_fraction of the free device memory, keeps their state on
 * the device, advances the admitted events concurrently -- the small ones as
 * batches (one per kind: precision, bulk, EoS), events of at least solo_cells
 * interior cells alone with the single-event kernels -- runs each event's
 * freezeout blocks at its fo_factor cadence (HydroPlugin.cpp:249-266) and
 * streams the elements to host memory, and retires an event after three
 * blocks with no cell above e_F (HydroPlugin.cpp:267-281), at max_steps, or on
 * a device error.  Events of one server share its EoS rows.
 */
typedef struct vh_server vh_server;

typedef struct vh_server_config {
    double hbm_fraction;     /* share of the free device memory at creation the events may use */
    int max_events;          /* most events resident at once                                     */
    int max_steps;           /* RK2 steps after which an event is retired (0: no cap)            */
    int solo_cells;          /* events with at least this many interior cells are stepped alone,
                                on their own stream, beside the batches (0: every event batched) */
} vh_server_config;

typedef struct vh_server_done {
    unsigned long long tag;  /* the caller's tag from vh_server_submit */
    int status;              /* VH_OK or the event's error             */
    int steps;               /* RK2 steps the event took               */
    long long n_elements;    /* freezeout elements collected           */
    double t_submit, t_admit, t_done;   /* seconds since vh_server_create */
} vh_server_done;

typedef struct vh_server_stats {
    long long submitted, queued, active, done;
    long long steps;         /* steps run (each advances every active event) */
    long long fo_blocks;     /* freezeout blocks run     */
    long long batch_builds;  /* batches (re)built        */
    unsigned long long bytes_in_use, budget_bytes;
    double t_admit_s;        /* worker wall time: creating and initialising events */
    double t_build_s;        /*   (re)building and tuning batches                  */
    double t_step_s;         /*   steps of the batches and solo events, launch to completion */
    double t_fo_s;           /*   freezeout blocks and surface copies              */
    double t_fo_copy_s;      /*     of which surface copies to host memory          */
    long long fo_elements;   /* freezeout elements collected                         */
    double t_retire_s;       /*   retiring events (freeing their device memory)      */
    double t_wait_s;         /*   idle, waiting for submissions                      */
} vh_server_stats;

void vh_server_config_default(vh_server_config *c);
int vh_server_create(const vh_server_config *cfg, const double *eos_rows, int eos_nrows, vh_server **out);
/* Copies the initial condition (interior arrays as vh_event_set_initial) and
 * returns at once. */
int vh_server_submit(vh_server *s, const vh_config *cfg, const double *e, const double *p, const double *u,
                     const double *pi, const double *Pi, unsigned long long tag);
/* The same with the initial condition generated on the device when the event
 * is admitted (vh_event_init_glauber / vh_event_init_hotspots): nothing but
 * the parameters crosses from the host. */
int vh_server_submit_glauber(vh_server *s, const vh_config *cfg, double R, double a, double sigma_nn, double b,
                             double e0_GeV, double eta_flat, double eta_sigma, unsigned long long tag);
int vh_server_submit_hotspots(vh_server *s, const vh_config *cfg, unsigned long long seed, double mean_spots, double w,
                              double k_gamma, double amp_mean_GeV, double R, double a, unsigned long long tag);
/* Up to max finished events, oldest first. */
int vh_server_poll(vh_server *s, vh_server_done *out, int max, int *n);
/* The surface of a polled event (VH_FO_COLUMNS doubles per element); the
 * server drops it once taken. */
int vh_server_take_surface(vh_server *s, unsigned long long tag, double *out, long long cap_elements, long long *n);
/* Wait until every submitted event is finished (VH_ERR_STATE on timeout). */
int vh_server_wait(vh_server *s, double timeout_s);
int vh_server_stats_get(vh_server *s, vh_server_stats *out);
int vh_server_destroy(vh_server *s);

/* Device pointer of a padded field (for zero-copy inspection / timing).  A
 * 2+1D event keeps no eta ghost planes while it steps; for its state fields
 * this call writes them on the event's stream first, so read the plane in
 * that stream's order. */
int vh_event_device_field(vh_event *ev, int field, double **d_ptr);

/* Energy density [fm^-4] for temperature T [fm^-1] with the event's EoS
 * (EquationOfState.cpp:201-290); used for e_F and e_reg. */
int vh_event_energy_of_T(vh_event *ev, double T, double *e_out);

/* Cornelius surface elements of arbitrary cubes on the device, the routine
 * the freezeout block applies to every lattice cube (freezeout/
 * cornelius-c++-1.3/cornelius.cpp: Cornelius::find_surface_3d :2161-2237 and
 * find_surface_4d :2248-2287).  dim 3: 8 corner values per cube in [t][x][y]
 * order; dim 4: 16 values in [t][x][y][z] order; dx holds dim spacings.
 * Writes, per element and in cube order, 2*dim doubles (centroid then normal,
 * as get_centroid_elem/get_normal_elem return them), the element count of
 * every cube into counts[n_cubes], and the total into *n_elements. */
int vh_cornelius_surfaces(int dim, const double *cubes, int n_cubes, double value0, const double *dx,
                          double *elements, int cap_elements, int *counts, int *n_elements);

/* No counterpart in the reference.  The same surface elements as
 * vh_cornelius_surfaces for callers that cannot let a library allocate device
 * memory (a host framework whose pool owns the whole GPU, or a loop sharing
 * the GPU where cudaMalloc's device-wide synchronisation would stall other
 * streams).  Everything is caller-owned device memory: d_cubes (n_cubes cubes,
 * layout as above), d_elements (cap_elements x 2*dim doubles, compacted in cube
 * order), d_counts (n_cubes ints) and d_n_elements (one int: the total, or -1
 * after a Cornelius construction error); dx is a host array of dim spacings.
 * When the total exceeds cap_elements, only the first cap_elements elements
 * are written and *d_n_elements still holds the total: the output is then
 * truncated, which the caller detects by comparing the two (the allocating
 * entry point returns VH_ERR_CAPACITY instead).
 * Work is queued on `stream` (a cudaStream_t, 0 for the legacy stream) and the
 * call returns without waiting; read the outputs after synchronising.
 * The library's working memory is a fixed device array of about 1 MiB held by
 * every GPU that loads the library, so n_cubes is limited to
 * VH_NOALLOC_MAX_CUBES (larger batches are rejected with VH_ERR_ARG).  The
 * first call on each device looks up that array's address with that device
 * current; make it before any stream capture.  All calls on a device share
 * the array: calls that overlap on the GPU race. */
#define VH_NOALLOC_MAX_CUBES 262144
int vh_cornelius_surfaces_noalloc(int dim, const double *d_cubes, int n_cubes, double value0, const double *dx,
                                  double *d_elements, int cap_elements, int *d_counts, int *d_n_elements,
                                  void *stream);

/* Self-check of the device arithmetic that must equal the host libm bit for
 * bit: which = 0 out[i] = tanh(a[i]) (the regulation factor,
 * FullyDiscreteKurganovTadmorScheme.cpp:775), 1 = a[i]/b[i] through the
 * shared-reciprocal division, 2 = a[i]/b[i] IEEE, 3 = powf((float)a[i], 0.25f)
 * (EquationOfState.cpp:196).  Host arrays of n doubles. */
int vh_device_math_check(int which, const double *a, const double *b, int n, double *out);

/* Inputs seen outside the calibrated powf range since creation (diagnostic;
 * 0 means every temperature matched the host libm exactly). */
int vh_event_powf_misses(vh_event *ev, unsigned long long *misses);

/* ------------------------------------------------ host-side helpers */
/* Synthetic crossover EoS table in the binary record layout above:
 * cs^2(T) = 1/3 - dip * exp(-((T - Tc)/w)^2) integrated from T_lo_GeV,
 * tabulated on nrows points uniform in e from e(T_lo) to e_max_GeV. */
int vh_eos_synthetic_table(int nrows, double T_lo_GeV, double e_max_GeV, double a_conformal,
                           double dip, double Tc_GeV, double w_GeV, double *rows);

/* Host copy of the reference EoS functions for a given configuration and
 * table (EquationOfState.cpp:44-290). what: 0 p(e), 1 cs2(e), 2 T(e), 3 e(T);
 * 4: the energy density up to which the table's cs2 is exactly 1/3, so that
 * the kernels skip its evaluation there (-inf: no such bound; x unused). */
double vh_eos_eval(const vh_config *cfg, const double *eos_rows, int eos_nrows, int what, double x);

/* Viscous Gubser flow at proper time t0 (2+1D, nz = 1): e, p [fm^-4],
 * u (4 planes), pi (10 planes, Navier-Stokes value 2 eta sigma^{mu nu}).
 * T0_GeV is the temperature at the origin, q the Gubser scale [fm^-1]. */
int vh_ic_gubser(const vh_config *cfg, double q, double T0_GeV,
                 double *e, double *p, double *u, double *pi);

/* Optical-Glauber event: e = e0 * n_part(x,y)/max n_part * L(eta) + 1e-3
 * (the reference adds 1e-3 fm^-4, InitialConditions.cpp:1093), Woods-Saxon
 * (R, a, n0 = 0.17 fm^-3), sigma_NN [fm^2], impact parameter b [fm];
 * L(eta) = plateau |eta| < eta_flat/2 with Gaussian tails of width eta_sigma
 * (InitialConditions.cpp:1046-1063).  u at rest, pi = Pi = 0. */
int vh_ic_glauber(const vh_config *cfg, const double *eos_rows, int eos_nrows,
                  double R, double a, double sigma_nn, double b, double e0_GeV,
                  double eta_flat, double eta_sigma,
                  double *e, double *p, double *u);

/* Lumpy 2+1D event: sum of Gaussian hotspots (width w [fm]); the number is
 * Poisson(mean_spots), amplitudes Gamma(k_gamma) scaled so their mean is
 * amp_mean_GeV, centres drawn from the b = 0 Woods-Saxon overlap density;
 * all draws come from a counter-based generator keyed by `seed`. */
int vh_ic_hotspots(const vh_config *cfg, const double *eos_rows, int eos_nrows,
                   uint64_t seed, double mean_spots, double w, double k_gamma, double amp_mean_GeV,
                   double R, double a, double *e, double *p, double *u);

#ifdef __cplusplus
}
#endif

#endif /* VH_B200_H */
