/*
 * symmetry.h -- C ABI of the B200 lattice-update library (libsymmetry_b200.so).
 *
 * The reference (X-Sheen/Symmetry, Source1.f90) is one Fortran program whose
 * time loop (Source1.f90:215-252) calls a fixed sequence of implicit-interface
 * subroutines on FP64 arrays it owns.  This library keeps that boundary: every
 * subroutine on the per-timestep path has an entry point of the same name,
 * operating on device-resident state held by an opaque handle, so a Fortran
 * driver can bind them with ISO_C_BINDING and keep its loop unchanged.
 *
 * Conventions
 *   - Every function returns an int status (SYM_OK == 0) unless noted.
 *     sym_last_error() gives a message for the last failing call on a handle.
 *   - Host arrays use the reference's Fortran layout: scalars are
 *     (z,y,x) column-major with z fastest; populations are (0:18,z,y,x) with
 *     the velocity index fastest (Source1.f90:611,702,739).  The library
 *     transposes to its own device layout on upload and back on download.
 *   - Lattice coordinates: in SYM_MODE_REFERENCE node (x,y,z) sits at the
 *     1-based integer position of the Fortran arrays; in SYM_MODE_CONFIG at
 *     the 0-based position (x=0..nx-1).  Particle centres use the same frame.
 *   - One CUDA stream per handle; calls are synchronous with respect to the
 *     host buffers they take (the call returns after the copy completes).
 */
#ifndef SYMMETRY_B200_H
#define SYMMETRY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SYM_OK              0
#define SYM_ERR_PARAM       1  /* invalid parameter (NaN tau, tau<=0.5, bad dims...) */
#define SYM_ERR_OOM         2  /* device allocation failed / over budget             */
#define SYM_ERR_CUDA        3  /* CUDA runtime error                                 */
#define SYM_ERR_NAN         4  /* non-finite field detected                          */
#define SYM_ERR_TIMEOUT     5  /* a bounded device wait gave up                      */
#define SYM_ERR_STATE       6  /* call not valid in the current state                */
#define SYM_ERR_UNSUPPORTED 7  /* feature not available for this mode/storage        */
#define SYM_ERR_NOTFOUND    8  /* unknown field / job id                             */
#define SYM_ERR_DRIFT       9  /* a served job's conserved quantity drifted          */

/* ---- geometry modes ---------------------------------------------------- */
/* REFERENCE: the reference's own domain (Source1.f90:4, 1443-1592): updates on
 * interior nodes 2..n-1, mirror planes at x=nx, y=1, y=ny, z=nz, halfway
 * bounce-back wall node planes at x=1 and z=1, and every reference-geometry
 * special case (force skip z<3/x<3 at :624, mirror force doubling :1272-1319,
 * the pp==par/3+1 averaging :1321-1335, hard-coded repulsion planes :1607-1650,
 * the Lagrange domain test :1832).
 * CONFIG: periodic box (all nodes updated), optional solid wetting wall planes
 * at x=0 and x=nx-1, minimum-image particle geometry, none of the special cases. */
#define SYM_MODE_REFERENCE 0
#define SYM_MODE_CONFIG    1

/* ---- population storage of the fused fast path ------------------------- */
#define SYM_STORE_FP64 0   /* plain FP64 (parity path)                                  */
#define SYM_STORE_FP32 1   /* FP32 populations, FP32 arithmetic                         */
#define SYM_STORE_FP16 2   /* FP16 shifted storage (deviation from w_i*rho0), FP32 math */

#define SYM_MAX_PAR 32     /* particles per handle */

/* Solid wall ids used in the walls/pin/pout masks for CONFIG wall planes. */
#define SYM_WALL_ID_XLO(par) ((par) + 1)
#define SYM_WALL_ID_XHI(par) ((par) + 2)

/*
 * Runtime replacement for the reference's compile-time constants and the
 * hard-coded assignments in main (Source1.f90:7-26, 57-103).
 */
typedef struct sym_params {
  int32_t nx, ny, nz;   /* xl, yl, zl (Source1.f90:9-11)                          */
  int32_t mode;         /* SYM_MODE_*                                             */
  int32_t wall_x;       /* CONFIG only: 1 = solid wetting walls at x=0 and x=nx-1 */
  int32_t storage;      /* SYM_STORE_* used by sym_step in CONFIG mode            */
  int32_t par;          /* number of particles, 0..SYM_MAX_PAR (:24)              */
  int32_t la_m, la_n;   /* Lagrange grid La_m, La_n (:87-88); 0 = from alpha      */
  int32_t bounce;       /* moving-particle bounce-back: 0 halfway (curve, :990-1034),
                           1 interpolated with the link fraction (curve2, :1036-1101) */
  double rho0;          /* reference density (:67); solid-node rho (:788)         */
  double nu_r, nu_b;    /* kinematic viscosities of red/blue (:69-70)             */
  /* MRT rates. A value <= 0 selects the reference's node-local rate
   * (Source1.f90:682-684): s_e, s_eps, s_pi -> su = 1/(3nu+1/2);
   * s_q, s_m -> sq = 8(2-su)/(8-su). */
  double s_e, s_eps, s_q, s_pi, s_m;
  double sigma;         /* CSF surface tension (:66, :664)                        */
  double beta;          /* recolouring parameter (:17)                            */
  double cita;          /* contact angle in radians (:21)                         */
  double body[3];       /* CONFIG only: body acceleration on fluid and particles  */
  double rad;           /* particle radius Rad (:76)                              */
  double rho_p;         /* particle density (:79)                                 */
  double mass;          /* particle mass (:81); <= 0 -> 4/3 rho_p pi Rad^3        */
  double inertia;       /* moment of inertia (:82); <= 0 -> 2/5 mass Rad^2        */
  double fg;            /* repulsion scale Fg (:84)                               */
  double alpha;         /* Lagrange angular step (:22)                            */
  double evap_lim;      /* EVAP_LIM (:16); <= 0 -> 1e-8                           */
} sym_params;

/* Field ids for sym_set_field / sym_get_field. Populations are double
 * (0:18,z,y,x); scalars double (z,y,x); masks int32 (z,y,x); FLAG is int32 0/1
 * (the storage size of a default Fortran LOGICAL). */
enum {
  SYM_F_RI = 0, SYM_F_BI, SYM_F_FI, SYM_F_FFI,          /* 19*N doubles */
  SYM_F_RHO, SYM_F_UX, SYM_F_UY, SYM_F_UZ,              /* N doubles    */
  SYM_F_RHO_N, SYM_F_RHO_R, SYM_F_RHO_B,
  SYM_F_NX, SYM_F_NY, SYM_F_NZ, SYM_F_GRADX, SYM_F_GRADY, SYM_F_GRADZ,
  SYM_F_FLAG,                                           /* N int32      */
  SYM_F_WALLS, SYM_F_WALLS_OLD, SYM_F_WALLS_ALL, SYM_F_PIN, SYM_F_POUT,
  SYM_F_COUNT
};

/* Particle state block, all (par,3) column-major like the reference
 * (Source1.f90:46-53): index [k*par + pp] for component k of particle pp. */
typedef struct sym_particles {
  double center[3 * SYM_MAX_PAR];
  double center_old[3 * SYM_MAX_PAR];
  double center0[3 * SYM_MAX_PAR];
  double up[3 * SYM_MAX_PAR];        /* upx, upy, upz  */
  double rp[3 * SYM_MAX_PAR];        /* rpx, rpy, rpz  */
  double fp[3 * SYM_MAX_PAR];        /* Fpx, Fpy, Fpz  (momentum, :1178)        */
  double tp[3 * SYM_MAX_PAR];        /* Tpx, Tpy, Tpz                           */
  double fre[3 * SYM_MAX_PAR];       /* Frex.. (repulsive, :1594)               */
  double tension[3 * SYM_MAX_PAR];   /* capillary force (capillary_force2)      */
  double tension_t[3 * SYM_MAX_PAR]; /* capillary torque                        */
  double shb[SYM_MAX_PAR];           /* immersed area Shb (Lagrange_points)     */
} sym_particles;

typedef struct sym_handle sym_handle;

/* ---- lifetime ---------------------------------------------------------- */
/* Fill p with the reference's built-in constants (Source1.f90:9-26, 57-103)
 * for an nx*ny*nz reference-mode domain. */
int sym_params_reference(sym_params* p, int nx, int ny, int nz);
/* Validate p; returns SYM_ERR_PARAM with a message in `msg` (may be NULL). */
int sym_params_check(const sym_params* p, char* msg, size_t msg_len);
int sym_create(const sym_params* p, int device, sym_handle** out);
int sym_destroy(sym_handle* h);
const char* sym_last_error(const sym_handle* h);
/* The D3Q19 tables the kernels are compiled with: tables = cix, ciy, ciz, opc,
 * symx, symy, symz (7 rows of 19, Source1.f90:132-138), wi (:140-142) and the
 * moment matrix m[r*19+c] = M(r,c) of the data statement (:105-123).  Any
 * pointer may be NULL. */
int sym_lattice_tables(int32_t tables[7 * 19], double wi[19], double m[19 * 19]);
/* Device bytes the handle holds (state + fast-path buffers). */
int sym_footprint(const sym_params* p, size_t* bytes);

/* ---- state transfer (Fortran layout on the host) ------------------------ */
int sym_set_field(sym_handle* h, int field, const void* host);
int sym_get_field(sym_handle* h, int field, void* host);
/* Upload both colours' populations (0:18,z,y,x) in one call: the state a
 * Fortran driver holds after initialization (Source1.f90:883-894). */
int sym_set_populations(sym_handle* h, const double* ri, const double* bi);
/* The macroscopic fields calmacros (Source1.f90:770-831) computes from the
 * current populations -- rho, ux, uy, uz and rho_N, each (z,y,x) -- without
 * changing the stepping state (the fields an output step of the reference
 * driver writes, :218-234).  On a handle stepped by sym_step the fused state
 * stays authoritative, so reading does not re-encode reduced storage.  Any
 * pointer may be NULL. */
int sym_get_macros(sym_handle* h, double* rho, double* ux, double* uy, double* uz, double* rho_n);

/* Error flags the fused kernels recorded on the device since the fused state
 * was last built from the canonical one (no counterpart in the reference):
 *   SYM_DEV_NONFINITE  FP64 storage: a next-step colour density was not
 *                      finite or left the fixed-point accumulator's range
 *   SYM_DEV_TIMEOUT    a tile load did not complete within the bounded wait
 *                      (the kernel carried on instead of hanging)
 * In FP64 storage either flag also makes every later phase field NaN.  The
 * server reads the flags of a job at each of its checks and retires it as
 * failed (SYM_ERR_TIMEOUT, SYM_ERR_NAN).  0 when nothing was recorded or the
 * handle never ran the fused path. */
#define SYM_DEV_NONFINITE 1
#define SYM_DEV_TIMEOUT   2
int sym_device_status(sym_handle* h, int32_t* flags);

/* Runs the timeout path of the bounded mbarrier wait the fused kernels use
 * for their tile loads: one thread waits `polls` polls on a barrier that
 * nothing arrives on.  *status receives the flags the kernels would record
 * (SYM_DEV_TIMEOUT; bit 4 if a completed barrier was not seen), *ms the
 * event-timed duration of the launch.  Allocates 4 bytes of device memory. */
int sym_selftest_wait_timeout(int device, int polls, int32_t* status, double* ms, char* msg, size_t msg_len);
int sym_set_particles(sym_handle* h, const sym_particles* s);
int sym_get_particles(sym_handle* h, sym_particles* s);
/* Lagrange point arrays (par, La_num) column-major as in :1805; any pointer may be NULL. */
int sym_get_lagrange(sym_handle* h, double* lax, double* lay, double* laz, double* la_rhon,
                     double* la_nx, double* la_ny, double* la_nz, int32_t* la_flag, double* ds);

/* ---- checkpoint / restart --------------------------------------------------
 * No counterpart in the reference, whose OUT_t.dat files hold macroscopic
 * fields only (Source1.f90:898-924) and cannot restart a run.  save writes the
 * handle's complete stepping state to `path`; load restores it into a handle
 * created with the same sym_params, after which stepping continues bit for
 * bit as if the run had not stopped.  The fused state of a sym_step handle is
 * saved in its storage format (no re-encoding). */
int sym_checkpoint_save(sym_handle* h, const char* path);
int sym_checkpoint_load(sym_handle* h, const char* path);

/* ---- initial state --------------------------------------------------------
 * sym_initia_center     <- initia_center   Source1.f90:926-976 (REFERENCE only)
 * sym_initialization    <- initialization  Source1.f90:850-896 (REFERENCE only)
 * sym_init_phase        CONFIG: rho_N/rho from a host phase field, then the
 *                       same equilibrium fill as initialization (:883-894)
 * sym_init_thread       CONFIG: Rayleigh-Plateau thread along z, on device
 * sym_init_slab         CONFIG: red slab z0<=z<=z1, on device                   */
int sym_initia_center(sym_handle* h);
int sym_initialization(sym_handle* h);
int sym_init_phase(sym_handle* h, const double* rho_n, const double* rho);
int sym_init_thread(sym_handle* h, double radius, double amp, double wavelength,
                    double width, double noise, uint64_t seed);
int sym_init_slab(sym_handle* h, double z0, double z1, double width, double noise,
                  uint64_t seed);

/* ---- the reference's per-timestep subroutines (drop-in) ------------------ */
int sym_set_walls(sym_handle* h);         /* set_walls        Source1.f90:326-395   */
int sym_calmacros(sym_handle* h);         /* calmacros        Source1.f90:770-831   */
int sym_derivatives(sym_handle* h);       /* derivatives      Source1.f90:452-597   */
int sym_collision(sym_handle* h);         /* collision+equilf Source1.f90:599-695   */
int sym_recolor(sym_handle* h);           /* Recolor          Source1.f90:697-732   */
int sym_boundary(sym_handle* h);          /* boundary         Source1.f90:1544-1592 */
int sym_streaming(sym_handle* h, int which); /* streaming(ri|bi) Source1.f90:735-768; which 0=ri 1=bi */
int sym_curve(sym_handle* h);             /* curve            Source1.f90:990-1034  */
int sym_lagrange_points(sym_handle* h);   /* Lagrange_points  Source1.f90:1799-1978 */
int sym_capillary_force2(sym_handle* h);  /* capillary_force2 Source1.f90:1980-2028 */
int sym_momentum(sym_handle* h);          /* momentum         Source1.f90:1178-1261 */
int sym_repulsive(sym_handle* h);         /* repulsive        Source1.f90:1594-1671 */
int sym_movement(sym_handle* h);          /* movement         Source1.f90:1263-1349 */
int sym_refilling(sym_handle* h);         /* refilling        Source1.f90:1351-1418 */

/* One loop body of main (Source1.f90:216-251, output gate excluded), nsteps
 * times.  REFERENCE mode runs the subroutine kernels above in the reference
 * order; CONFIG mode runs the fused fast path in the handle's storage mode. */
int sym_step(sym_handle* h, int nsteps);
/* sym_step with CUDA events recorded on the handle's stream (CONFIG mode).
 * use_graph=0: eager launches, ms[0]=whole region, ms[1]=phase-field kernel,
 * ms[2]=particle coupling and pin fill, ms[3]=fused collide kernel (sums over
 * the steps).  use_graph=1: captured-graph replay, ms[0] only (others -1). */
int sym_step_timed(sym_handle* h, int nsteps, int use_graph, double ms[4]);

/* ---- batches: many independent CONFIG domains stepped together ----------
 * No counterpart in the reference (it runs one domain).  A batch references
 * existing handles (same device, CONFIG mode, same storage) and steps them in
 * lockstep: one CUDA graph per step containing one phase-field launch for all
 * domains, the particle and wall work of all domains (one launch per
 * subroutine over a (domain, particle, block) table), and one persistent
 * collide launch whose CTAs pull 32x8xX tiles of any domain from a work-tile
 * table (largest first).  Results per domain are identical to sym_step on that
 * domain alone with the same tile x extent.  Member handles stay usable on
 * their own; the batch rebuilds its graphs when a member was stepped or read
 * back outside it. */
typedef struct sym_batch sym_batch;
int sym_batch_create(sym_handle* const* handles, int n, sym_batch** out);
int sym_batch_destroy(sym_batch* b);
const char* sym_batch_last_error(const sym_batch* b);
int sym_batch_step(sym_batch* b, int nsteps);
/* nsteps graph steps bracketed by CUDA events on the batch stream; *ms = elapsed. */
int sym_batch_step_timed(sym_batch* b, int nsteps, double* ms);
int sym_batch_set_xchunk(sym_batch* b, int domain, int xchunk);
int sym_batch_get_xchunk(sym_batch* b, int domain, int* xchunk);
/* Resident collide CTAs per SM of the persistent launch (1 .. the most that
 * fit; default the most): grid = per_sm x SM count. */
int sym_batch_set_ctas_per_sm(sym_batch* b, int per_sm);
/* Picks the tile x extent per size class (nx <= 32, <= 48, larger) from
 * {8,12,16,24,32,64}, then the resident CTAs per SM, by timing; the trial steps
 * advance every domain (*steps_taken). */
int sym_batch_autotune(sym_batch* b, int trial_steps, int* steps_taken);
int sym_batch_info(sym_batch* b, int64_t* nodes, int* ntiles, int* grid);
/* nsteps eager batch steps (not the graph) with CUDA events on the batch
 * stream: ms[0] = whole region, ms[1] = phase-field launches, ms[2] = the
 * per-domain particle/wall chains (fork to join), ms[3] = collide launches. */
int sym_batch_step_kernels(sym_batch* b, int nsteps, double ms[4]);
/* Kernel launches in one captured batch step (kernel nodes of its graph). */
int sym_batch_kernels_per_step(sym_batch* b, int* kernels);

/* ---- serving: a continuous-batching job server -----------------------------
 * No counterpart in the reference (it runs one job per process).  Jobs are
 * CONFIG domains with their own geometry, viscosity, surface tension, contact
 * angle, particle and stop rule.  The server admits pending jobs first come
 * first served while their device footprint (sym_footprint) fits the byte
 * budget and a slot is free, keeps admitted jobs resident on the device, and
 * steps all running jobs of one storage mode as one batch (sym_batch_*),
 * rebuilt when a job joins or leaves; batches of different storage modes run
 * on their own streams and overlap.  Every `check_every` steps of a job the
 * server reduces its phase field to r_eq(z) = sqrt(sum_xy (1+phi)/2 / pi) and
 * retires the job when min_z r_eq falls below its stop radius (breakup, time
 * interpolated linearly between the last two checks), when it reaches its
 * step limit, or as failed when the field is no longer finite (SYM_ERR_NAN)
 * or the device recorded a timed-out tile load (SYM_ERR_TIMEOUT; see
 * sym_device_status).  Jobs are admitted only at multiples of `check_every` server steps, so a
 * job's checks fall on the same steps whatever else runs beside it: its
 * result is the one it gets alone.  One host thread drives a server through
 * sym_server_tick. */
#define SYM_JOB_THREAD 0   /* Rayleigh-Plateau thread along z (sym_init_thread) */
#define SYM_JOB_SLAB   1   /* red slab z0 <= z <= z1 (sym_init_slab)            */

#define SYM_JOB_PENDING 0
#define SYM_JOB_RUNNING 1
#define SYM_JOB_BREAKUP 2  /* done: min r_eq fell below stop_radius */
#define SYM_JOB_LIMIT   3  /* done: reached max_steps                */
#define SYM_JOB_FAILED  4  /* error (see sym_job_result.error)       */

typedef struct sym_job_spec {
  sym_params p;         /* CONFIG mode; p.storage selects the batch it joins     */
  int32_t kind;         /* SYM_JOB_THREAD or SYM_JOB_SLAB                        */
  int32_t max_steps;    /* step limit (> 0)                                      */
  double gen[5];        /* THREAD: radius, amp, wavelength, width, noise;
                           SLAB: z0, z1, width, noise, unused                     */
  uint64_t seed;        /* phase-field noise seed                                */
  double stop_radius;   /* breakup when min_z r_eq(z) < stop_radius (<= 0: 1.0)  */
  double center[3];     /* particle centre (p.par == 1)                          */
  double up[3];         /* particle velocity                                     */
  double t_arrival;     /* arrival on the server clock in seconds; < 0 = now     */
  /* failure detection (no counterpart in the reference, which only warns):
   * drift_tol     > 0: FAILED with SYM_ERR_DRIFT when the red-phase volume
   *               sum (1+phi)/2 moves by more than drift_tol (relative) from
   *               the admission reading (evaporation or a blow-up);
   * wall_budget_s > 0: FAILED with SYM_ERR_TIMEOUT when the job has been
   *               resident longer than this many seconds at a check.       */
  double drift_tol;
  double wall_budget_s;
} sym_job_spec;

typedef struct sym_job_result {
  int32_t status;       /* SYM_JOB_*                                             */
  int32_t error;        /* SYM_ERR_* when FAILED                                 */
  int32_t steps;        /* lattice steps run                                     */
  int32_t reserved;
  double breakup_step;  /* interpolated breakup step; -1 if none                 */
  double rmin;          /* min_z r_eq at the last check                          */
  double t_arrival, t_admit, t_done;   /* server clock, seconds (-1 = not yet)   */
  int64_t node_updates; /* nodes x steps                                         */
} sym_job_result;

typedef struct sym_server sym_server;
/* budget_bytes: device bytes the resident jobs may hold (sum of footprints);
 * slots: most jobs resident at once; check_every: stop-rule interval (<= 0: 10). */
int sym_server_create(int device, size_t budget_bytes, int slots, int check_every, sym_server** out);
int sym_server_destroy(sym_server* s);
const char* sym_server_last_error(const sym_server* s);
/* Queue a job; *id identifies it in sym_server_result. */
int sym_server_submit(sym_server* s, const sym_job_spec* spec, int64_t* id);
/* One round of the request loop: admit what fits, run every batch for up to
 * max_steps steps (to the next check; <= 0: no cap), check, retire.  Returns
 * after the device work of the round; *running and *pending may be NULL. */
int sym_server_tick(sym_server* s, int max_steps, int* running, int* pending);
int sym_server_result(sym_server* s, int64_t id, sym_job_result* out);
/* Tile x extent used for jobs of one size class (0: nx <= 32, 1: <= 48,
 * 2: larger) in the batches the server builds (default 32). */
int sym_server_set_xchunk(sym_server* s, int size_class, int xchunk);
/* out[0] node updates, [1] device milliseconds of the batch steps, [2] jobs
 * done, [3] jobs failed, [4] running, [5] pending, [6] resident footprint
 * bytes, [7] server clock in seconds. */
int sym_server_stats(sym_server* s, double out[8]);

/* ---- diagnostics ------------------------------------------------------- */
/* output3 (Source1.f90:1673-1717): neck height hmin on plane x=xl-1 and the y
 * where it occurs (REFERENCE geometry). */
int sym_output3(sym_handle* h, double* hmin, int32_t* y0);
/* CONFIG stop rule: min over z of r_eq(z) = sqrt(sum_xy (1+phi)/2 / pi) over
 * fluid nodes.  After sym_step in CONFIG mode it reduces the fused phase
 * field in place (the phase field of the last step, i.e. of the state the
 * last step started from) without exporting the populations. */
int sym_neck_radius(sym_handle* h, double* rmin);
/* FP64 sums over fluid nodes: out[0]=sum rho_R, [1]=sum rho_B, [2..4]=momentum. */
int sym_mass_momentum(sym_handle* h, double out[5]);
/* The energy budget of output4 (Source1.f90:1719-1797) before normalisation,
 * from calmacros of the current populations (the stepping state is kept):
 * out[0] pressure energy sum (rho-rho0)/3 and out[1] kinetic energy
 * sum rho|u|^2/2 over red fluid nodes, out[2] interface nodes (fluid nodes with
 * a fluid neighbour of the other colour), out[3] particle kinetic energy,
 * out[4] capillary power (tension.up + tension_t.rp), out[5] immersed area
 * sum Shb; particles that start on a mirror plane count half (:1765-1779).
 * The reference's walls_all(z,y,z), rho(z,y,z) and uz(z,y,z) (:1736, :1739)
 * read (z,y,x) here. */
int sym_energy(sym_handle* h, double out[6]);
/* Writers of the reference's output step (Source1.f90:218-234), Tecplot
 * ASCII with its variables and formats.  The logs get one record per call
 * appended (the header and a new file at t = 0; the reference re-opens them
 * on each call and keeps only the last record):
 *   sym_output_results  OUT file of output_results (:898-924): x,y,z (1-based),
 *                       walls_all, rho_N, u, v, w, rho of calmacros
 *   sym_output_result2  prefix + "P_<pp>.dat" of output_result2 (:1420-1441)
 *   sym_output3_write   the neck record of output3 (:1673-1717): t, t/tr,
 *                       hmin/rad_c, y0/lamda_d
 *   sym_output4         the Energy.dat record of output4 (:1751-1792): energies
 *                       over pi rad_c^2 sigma (times 8 in REFERENCE mode, the
 *                       reference's 1/8 domain); *wcap_acc carries Wcap_old */
int sym_output_results(sym_handle* h, const char* path);
int sym_output_result2(sym_handle* h, const char* prefix, int t, double tr);
int sym_output3_write(sym_handle* h, const char* path, int t, double tr, double rad_c, double lamda_d);
int sym_output4(sym_handle* h, const char* path, int t, double tr, double rad_c, double* wcap_acc);

/* The same five sums for callers that may not allocate device memory: no
 * counterpart in the reference.  It is meant for code that never creates a
 * handle and must not call cudaMalloc -- for example a serving loop that has
 * reserved its whole device budget up front, or a host program whose own
 * memory manager owns every device byte -- because an allocation there can
 * fail or stall the device.  It calls no cudaMalloc, cudaFree or allocating
 * library routine: its scratch is a fixed 2.6 MB array inside the library
 * (held on every GPU that loads the library until the process exits).
 *   ri, bi     device populations, structure of arrays [19][n_nodes] (FP64)
 *   walls_all  device int32 mask (nodes with walls_all > 0 are skipped), or NULL
 *   n_nodes    1 .. 16,777,216; larger sizes are rejected with SYM_ERR_PARAM
 *   out        device memory for 5 doubles, written on `stream`
 *   stream     cudaStream_t to enqueue on (NULL = legacy default stream)
 *   msg        optional buffer for an error message
 * The call is asynchronous on `stream`.  The first call on each device looks
 * up the scratch address (cudaGetSymbolAddress) and should come before any
 * stream capture; the address is kept for the life of the process, so a
 * process that resets a device (cudaDeviceReset) must not call this entry
 * point on that device afterwards.  Calls share the scratch: calls that
 * overlap on the GPU race, so serialise them (one stream, or events). */
int sym_mass_momentum_noalloc(const double* ri, const double* bi, const int32_t* walls_all, int64_t n_nodes,
                              double* out, void* stream, char* msg, size_t msg_len);

#ifdef __cplusplus
}
#endif
#endif /* SYMMETRY_B200_H */
