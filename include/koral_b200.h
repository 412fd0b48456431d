/*
 * koral_b200 — C-ABI boundary of the B200 (sm_100a) implementation of
 * KORAL's per-step hot path.
 *
 * The reference is a C code whose time loop (solve_the_problem, ko.c:259-914)
 * calls a small set of grid operators on global arrays, and whose per-cell
 * solvers take plain double arrays plus a struct geometry.  This header
 * exposes the same operators and solvers behind an opaque device context:
 * the host keeps KORAL's own loop and calls these entry points instead of the
 * CPU routines; state, metric tables and flags live in HBM between calls.
 *
 * Conventions
 *  - All arrays crossing this boundary are HOST pointers in KORAL's own
 *    layout: cell arrays are [SZ][SY][SX][NV] doubles with ghost cells
 *    (ko.h:505-508), metric tables hold gSIZE=20 doubles per point
 *    (g_{mu nu} in [i][j], d ln(gdet)/dx^i in [i][4], gdet in [3][4]; the
 *    inverse table holds g^{mu nu} and the g_tt perturbation in [3][4]),
 *    Christoffel tables hold 64 doubles per point (ko.h:113, misc.c:122-186).
 *  - Every function returns 0 on success and a negative KGPU_E* code on
 *    failure; no function aborts the process.
 *  - One context is used by one host thread; calls are ordered on the
 *    context's CUDA stream.  Functions that return data to the host
 *    synchronise that stream.
 */
#ifndef KORAL_B200_H
#define KORAL_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define KGPU_ABI_VERSION 1

/* error codes */
#define KGPU_OK 0
#define KGPU_EINVAL (-1)      /* bad argument or unsupported configuration   */
#define KGPU_ECUDA (-2)       /* a CUDA runtime call failed                   */
#define KGPU_ENOMEM (-3)      /* device allocation failed                     */
#define KGPU_ESTATE (-4)      /* call out of order (e.g. no metric uploaded)  */
#define KGPU_EIO (-5)         /* a restart file could not be read or written  */

/* reconstruction / Riemann solver / time integrator choices
 * (INT_ORDER, FLUXMETHOD, TIMESTEPPING; choices.h:150-160, mnemonics.h:117-124) */
#define KGPU_PPM 2
#define KGPU_MP5 4
#define KGPU_LAXF 0
#define KGPU_HLL 1

/* which state array an array-algebra call addresses (u, p, ut0, ut1) */
#define KGPU_ARR_U 0
#define KGPU_ARR_P 1
#define KGPU_ARR_UT0 2
#define KGPU_ARR_UT1 3
#define KGPU_ARR_UT2 4   /* RK2's k2 (ko.c:614-615: addi_u(1.,u,-1.,ut1,ut2)) */

/* boundary conditions per axis (set_bc_core finite.c:2673-2748 and the
 * problem plug-ins' calc_bc):
 *  PERIODIC       primitives copied from the periodic image, conserved from p2u
 *  OUTFLOW        primitives copied from the nearest domain cell, p2u
 *  REFLECT        mirror image with the normal velocity and normal magnetic
 *                 field reversed (polar axis), p2u
 *  PERIODIC_COPY  conserved and primitives both copied from the periodic image */
#define KGPU_BC_PERIODIC 0
#define KGPU_BC_OUTFLOW 1
#define KGPU_BC_REFLECT 2
#define KGPU_BC_PERIODIC_COPY 3

typedef struct kgpu_ctx kgpu_ctx;

/* Compile-time choices of a KORAL problem build (define.h/choices.h),
 * given at run time here. */
typedef struct {
  int nx, ny, nz;          /* TNX, TNY, TNZ (one subdomain)                  */
  int ng;                  /* ghost layers, NG (3 for PPM, 4 for MP5)        */
  int nv;                  /* variables per cell, NV (9: MHD; 13: MHD + M1)   */
  int int_order;           /* KGPU_PPM or KGPU_MP5                           */
  int fluxmethod;          /* KGPU_LAXF or KGPU_HLL                          */
  int axisym_metric;       /* METRICAXISYMMETRIC: one phi slice of metric     */
  int bc[3];               /* boundary kind per axis, KGPU_BC_* below         */
  double gamma;            /* GAMMA                                           */
  double tsteplim;         /* TSTEPLIM (Courant number)                       */
  double rhofloor;         /* RHOFLOOR                                        */
  double uurhoratiomin;    /* UURHORATIOMIN                                   */
  double uurhoratiomax;    /* UURHORATIOMAX                                   */
  double b2rhoratiomax;    /* B2RHORATIOMAX                                   */
  double gammamaxhd;       /* GAMMAMAXHD                                      */
  double u2pconv;          /* U2PCONV                                         */
} kgpu_config;

/* Fill a config with KORAL's defaults (choices.h) for an nx x ny x nz grid. */
int kgpu_default_config(kgpu_config *cfg, int nx, int ny, int nz);

/* Allocates the device state for one subdomain (initialize_arrays,
 * misc.c:98-289) on the current CUDA device. */
int kgpu_create(const kgpu_config *cfg, kgpu_ctx **out);
int kgpu_destroy(kgpu_ctx *ctx);

/* Cell-face coordinates per axis, KORAL layout xb[ic+NG], ic in [-NG, N+NG]
 * (set_grid, finite.c:1629-1699).  Also sets the minimum cell sizes used
 * for the first time step. */
int kgpu_upload_grid(kgpu_ctx *ctx, const double *xb_x, const double *xb_y, const double *xb_z);
/* Uniform grid in code coordinates, as calc_xb (problem.c:9-36) builds it. */
int kgpu_set_uniform_grid(kgpu_ctx *ctx, const double lo[3], const double hi[3]);

/* Metric tables as calc_metric (metric.c:3866-4075) leaves them: centres
 * (g, G, gKr) and the three face sets (gbx..gbz, Gbx..Gbz). */
int kgpu_upload_metric(kgpu_ctx *ctx, const double *g, const double *G, const double *gKr,
                       const double *gbx, const double *gby, const double *gbz,
                       const double *Gbx, const double *Gby, const double *Gbz);
/* The context's metric tables back in the same layout (KGPU_ESTATE before
 * any metric was uploaded or computed). */
int kgpu_download_metric(kgpu_ctx *ctx, double *g, double *G, double *gKr, double *gbx, double *gby,
                         double *gbz, double *Gbx, double *Gby, double *Gbz);
/* Radius-dependent density floor (RHOFLOOR_BH, u2p.c:546-557) tabulated per
 * x-index: at cell centres (SX values, ic in [-NG, NX+NG)) and at x-faces
 * (SX+1 values).  Pass null pointers to switch it off. */
int kgpu_set_density_floor(kgpu_ctx *ctx, const double *centres, const double *xfaces);
/* Flat spacetime (MINKCOORDS) tables generated on the device. */
int kgpu_set_minkowski_metric(kgpu_ctx *ctx);

/* Conserved (u) and primitive (p) arrays, whole padded grid, in the layout
 * of KORAL's global arrays u and p (ko.h:275-280, indexed by get_u,
 * ko.h:505: [SZ][SY][SX][NV], ghost cells included).  download_array reads
 * one of the context's arrays (KGPU_ARR_*) in the same layout. */
int kgpu_upload_state(kgpu_ctx *ctx, const double *u, const double *p);
int kgpu_download_state(kgpu_ctx *ctx, double *u, double *p);
int kgpu_download_array(kgpu_ctx *ctx, int which, double *out);

/* Restart files in the reference's serial format (fprint_restartfile_bin /
 * fread_restartfile_bin, fileop.c:910-1111): folder/resNNNN.head holds
 * "## nout1 nout2 t PROBLEM NX NY NZ", folder/resNNNN.dat the global indices
 * of the domain cells (x outer, z inner, three ints each) followed by their
 * primitives in the same order; reslast.* are made links to the newest.
 * Reading (nout1 < 0: reslast) puts the primitives into the domain cells and
 * recomputes their conserved variables (p2u), leaving the ghosts to set_bc;
 * it returns the time, the next file number and nout2.  A file of another
 * grid size is rejected. */
int kgpu_write_restart(kgpu_ctx *ctx, const char *folder, int nout1, int nout2, double t, int problem);
int kgpu_read_restart(kgpu_ctx *ctx, const char *folder, int nout1, double *t, int *nout1_next, int *nout2);

/* Grid operators of KORAL's time loop. ------------------------------------ */
/* op_explicit(t,dt), finite.c:646-1234 (set_bc, wavespeeds, reconstruction,
 * face fluxes, flux-CT, unsplit update with metric source terms). */
int kgpu_op_explicit(kgpu_ctx *ctx, double t, double dt);
/* op_implicit(t,dt), finite.c:1241-1292: the implicit radiation source step
 * over the domain and its fixup (kgpu_set_radiation); a no-op for MHD. */
int kgpu_op_implicit(kgpu_ctx *ctx, double t, double dt);
/* calc_u2p(), finite.c:501-561: inversion, floors, fixups, set_bc. */
int kgpu_calc_u2p(kgpu_ctx *ctx);
/* set_bc(t,ifinit), finite.c:2752-4463. */
int kgpu_set_bc(kgpu_ctx *ctx, double t, int ifinit);
/* save_timesteps(), finite.c:404-496 (no SELFTIMESTEP: nothing to store). */
int kgpu_save_timesteps(kgpu_ctx *ctx);
/* copyi_u(factor,src,dst), finite.c:2492; addi_u(f1,a,f2,b,c), finite.c:2545;
 * addi_u_3(f1,a,f2,b,f3,c,d), finite.c:2603: d = f1 a + f2 b + f3 c.  Domain
 * cells, all NV variables, arrays named by KGPU_ARR_*. */
int kgpu_copyi_u(kgpu_ctx *ctx, double factor, int src, int dst);
int kgpu_addi_u(kgpu_ctx *ctx, double f1, int a, double f2, int b, int c);
int kgpu_addi_u_3(kgpu_ctx *ctx, double f1, int a, double f2, int b, double f3, int c, int d);
/* do_correct(), finite.c:605-640: the polar-axis corrections switched on by
 * kgpu_set_polar_correction (none by default, when it returns at once); the
 * problem's my_finger hook stays host code.  The fused steps call it where
 * the reference's loop does (ko.c:444-626). */
int kgpu_do_correct(kgpu_ctx *ctx);
/* The polar-axis corrections of a problem build (spherical-like
 * coordinates, theta along y), NCCORRECTPOLAR = nc rows at each axis:
 *  KGPU_POLAR_CORRECT     CORRECT_POLARAXIS, correct_polaraxis
 *                         (finite.c:4923-5166): the nc most polar cells of a
 *                         column take density, energy, entropy, radial and
 *                         azimuthal velocities (and radiation) from the cell
 *                         nc rows from the axis, the theta velocities scaled
 *                         by the distance from the axis; flux-CT's EMFs 1 and
 *                         3 vanish on the polar edges (magn.c:343-376)
 *  KGPU_POLAR_CORRECT_3D  CORRECT_POLARAXIS_3D without POLARAXISAVGIN3D,
 *                         correct_polaraxis_3d (finite.c:5170-5474): those
 *                         cells take the whole state of that cell
 *  KGPU_POLAR_SMOOTH      SMOOTH_POLARAXIS, smooth_polaraxis
 *                         (finite.c:4832-4921): the nc most polar rows take
 *                         their phi average
 * Every corrected state is converted with p2u and the magnetic field is
 * left as it is.  With CORRECT or CORRECT_3D the corrected cells are not
 * evolved as the reference treats them (is_cell_corrected_polaraxis,
 * finite.c:5604-5625): their inversion recovers the field only
 * (u2p_solver_Bonly, u2p.c:49-101) and the implicit source step skips
 * them (finite.c:1270).  Needs NY >= 2 nc + 2.  Drops the captured step
 * graph. */
#define KGPU_POLAR_CORRECT 1
#define KGPU_POLAR_CORRECT_3D 2
#define KGPU_POLAR_SMOOTH 4
int kgpu_set_polar_correction(kgpu_ctx *ctx, int flags, int nc);
/* flux_ct(), magn.c:199-339: corner EMFs from the face fluxes of the last
 * op_explicit and the magnetic components of those fluxes rewritten from
 * them, as the reference leaves flbx/flby/flbz (kgpu_download_flux reads
 * them).  kgpu_op_explicit applies flux-CT inside its update without
 * storing the rewritten fluxes; this call stores them.  KGPU_ESTATE when
 * called twice for one op_explicit (the EMFs need the fluxes before the
 * rewrite). */
int kgpu_flux_ct(kgpu_ctx *ctx);

/* Time-step bookkeeping of solve_the_problem (ko.c:290-313, 399-425). ----- */
/* Initial 1/dt from max_ws = 10000 (ko.c:290-300). */
int kgpu_begin_run(kgpu_ctx *ctx);
/* dt = 1/tstepdenmax, then reset of the running maximum (ko.c:399-425). */
int kgpu_begin_step(kgpu_ctx *ctx, double *dt_out);
int kgpu_get_tstepdenmax(kgpu_ctx *ctx, double *out);
int kgpu_set_tstepdenmax(kgpu_ctx *ctx, double v);

/* Whole RK2 steps (ko.c:571-626) enqueued on the device without a host
 * round trip: dt stays in device memory.  nsteps >= 1. */
int kgpu_rk2_steps(kgpu_ctx *ctx, int nsteps);
/* Same, replayed from a CUDA graph captured on the first call. */
int kgpu_rk2_steps_graph(kgpu_ctx *ctx, int nsteps);

/* Counters of the last calc_u2p calls since kgpu_reset_counters:
 * out[0] cells flagged for fixup, out[1] entropy inversions,
 * out[2] failed inversions (old primitives kept), out[3] negative densities. */
int kgpu_get_counters(kgpu_ctx *ctx, unsigned long long out[4]);
/* All counters (up to n, 20 in all): the four above, then Newton steps of
 * the energy and of the entropy solves, energy solves paused after the first
 * pass, cells handed to the entropy equation; with radiation: [8] M1
 * inversions corrected (U2PRAD fixup requests), [9] implicit solves where
 * every attempt failed (RADIMP fixups), [10] their Newton iterations over
 * all attempts, [11] passes of the batched solver with work, [12] warm-start
 * fallbacks, [13] residual evaluations of the implicit solves, [14] Newton
 * steps of the MHD inversions nested in those evaluations, [15] their
 * W-function evaluations, [16] evaluations whose nested inversion went over
 * its per-lane cap and was handed to a whole warp, [17] implicit solves,
 * [18] cells where the radiation floors acted; [19] faces where a side's
 * reconstructed state needed the magnetic floor.  Returns how many were
 * written. */
int kgpu_get_counters_ex(kgpu_ctx *ctx, unsigned long long *out, int n);
/* Tuning: Newton steps a cell may take in the first inversion pass before
 * it is queued for the resumption pass (default 8; results do not depend
 * on it). */
int kgpu_set_u2p_pass_iters(kgpu_ctx *ctx, int n);
int kgpu_reset_counters(kgpu_ctx *ctx);

/* Problem set-up helpers (host-side, then uploaded). ---------------------- */
/* Relativistic Orszag-Tang vortex on the current grid (Minkowski metric). */
int kgpu_init_orszag_tang(kgpu_ctx *ctx);

/* Magnetised Kerr torus in modified Kerr-Schild coordinates (MKS2). ------ */
typedef struct {
  double spin;               /* black-hole spin a                              */
  double r0, h0;             /* MKS2 parameters: r = exp(x1)+r0, theta(x2; h0) */
  double r_lo, r_hi;         /* radial extent of the grid                      */
  double x2_lo, x2_hi;       /* extent in the theta code coordinate            */
  double rin, rmax;          /* torus inner edge and pressure maximum          */
  double kappa;              /* polytropic constant of the torus               */
  double noise;              /* relative amplitude of the pressure noise       */
  unsigned long long seed;   /* seed of the per-cell noise                     */
  double atm_rho0, atm_uu0;  /* atmosphere rho0 r^-1.5, u0 r^-2.5 (and floor)  */
  double maxbeta;            /* max pmag/pgas after normalisation (1/beta_min) */
} kgpu_torus_params;

/* The benchmark torus: a = 0.9, r in [1.8, 1000], r_in = 6, r_max = 12. */
int kgpu_default_torus_params(kgpu_torus_params *tp);
/* Metric tables of MKS2 Kerr on the given faces, KORAL layout (host-only,
 * no GPU needed); same argument order as kgpu_upload_metric. */
int kgpu_mks2_metric_tables(double a, double r0, double h0, int nx, int ny, int nz, int ng, int axisym,
                            const double *xbx, const double *xby, const double *xbz, double *g, double *G,
                            double *gKr, double *gbx, double *gby, double *gbz, double *Gbx, double *Gby,
                            double *Gbz);
/* Fishbone-Moncrief torus state (host-only), KORAL layout, ghosts zero. */
int kgpu_fm_torus_state(const kgpu_torus_params *tp, const kgpu_config *cfg, const double *xbx, const double *xby,
                        const double *xbz, const double *g, const double *G, double *u, double *p);
/* Density floor table of the torus (host-only), as kgpu_set_density_floor takes it. */
int kgpu_fm_torus_floor(const kgpu_torus_params *tp, int nx, int ng, const double *xbx, double *centres,
                        double *xfaces);
/* Whole set-up on a context: grid, metric, floor, state, boundaries, first dt.
 * The metric tables (calc_metric, metric.c:3866-4075) and the torus state
 * (the problem's init.c with calc_BfromA, magn.c:380-586) are computed by
 * kernels straight into device memory; only the grid faces and the floor
 * table cross from the host.  The _host form computes both with the
 * host-only functions above and uploads them (the same formulas; the
 * results differ in the last places of sin, cos, tan, exp, log and pow). */
int kgpu_init_fm_torus(kgpu_ctx *ctx, const kgpu_torus_params *tp);
int kgpu_init_fm_torus_host(kgpu_ctx *ctx, const kgpu_torus_params *tp);

/* Batched per-cell solvers (host arrays, n cells, one metric point each:
 * g and G hold 20 doubles per cell).  They replace per-cell calls of
 *   int u2p(ldouble *uu, ldouble *pp, void *geom, int corrected[3],
 *           int fixups[2], int type)                          u2p.c:176
 *   int p2u(ldouble *p, ldouble *u, void *geom)               p2u.c:40
 *   int check_floors_mhd(ldouble *pp, int whichvel, void *geom) u2p.c:492
 * pp is input (initial guess) and output; status[i] is u2p's return value. */
int kgpu_u2p_cells(int n, const kgpu_config *cfg, const double *uu, double *pp,
                   const double *g, const double *G, int *status, int *fixup);
int kgpu_p2u_cells(int n, const kgpu_config *cfg, const double *pp, double *uu,
                   const double *g, const double *G);

/* kgpu_u2p_cells without any memory allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate when they invert
 * cells (device memory owned by another allocator or pool, a region where
 * cudaMalloc's implicit device synchronisation would stall other streams, a
 * long-running service that must not grow the device heap).  Same arguments,
 * layout and results as kgpu_u2p_cells; staging goes through one file-scope
 * device array of KGPU_STATIC_MAX_CELLS cells (about 3.9 MB per device).
 *  - n > KGPU_STATIC_MAX_CELLS returns KGPU_EINVAL; split larger batches.
 *  - The first call on a device (that device current) looks up the array's
 *    address with cudaGetSymbolAddress; make it before any stream capture.
 *  - All calls share the array and it keeps the last call's contents; calls
 *    that overlap on the GPU race on it and must be serialised by the caller.
 *  - Copies and the kernel run on the legacy default stream and the call
 *    returns when the results are on the host.
 * Errors are described by kgpu_u2p_cells_static_error(). */
#define KGPU_STATIC_MAX_CELLS 8192
int kgpu_u2p_cells_static(int n, const kgpu_config *cfg, const double *uu, double *pp,
                          const double *g, const double *G, int *status, int *fixup);
const char *kgpu_u2p_cells_static_error(void);

/* Instrumentation. ------------------------------------------------------- */
/* The context's CUDA stream (cudaStream_t), for events and copies that must
 * be ordered with the operators. */
int kgpu_get_stream(kgpu_ctx *ctx, void **stream);
/* When enabled, every launch outside a CUDA graph is bracketed by CUDA
 * events; kgpu_profile_read returns the summed device time and launch count
 * of one kernel kind (0 <= kernel < kgpu_num_kernels()) and its name.  The
 * face flux of a direction (k_flux_x/y/z) is timed and counted together
 * with its magnetic-floor pass, as one. */
int kgpu_profile_enable(kgpu_ctx *ctx, int on);
int kgpu_profile_read(kgpu_ctx *ctx, int kernel, double *total_ms, long long *count, const char **name);
int kgpu_profile_reset(kgpu_ctx *ctx);
int kgpu_num_kernels(void);
/* Kernels launched by this context so far (graph replays included). */
int kgpu_launch_count(kgpu_ctx *ctx, long long *out);

/* Face fluxes of the last explicit operator along axis d (flbx/flby/flbz,
 * KORAL layout [face][NV]) and the corner EMFs of flux-CT (emf, KORAL layout
 * [(NZ+1)(NY+1)(NX+1)][3]).  The magnetic-field components of the face
 * fluxes are the Riemann fluxes before flux_ct rewrites them. */
int kgpu_download_flux(kgpu_ctx *ctx, int d, double *out);
int kgpu_download_emf(kgpu_ctx *ctx, double *out);

/* Radiation: per-cell implicit gas-radiation source solve. ----------------
 * A cell carries 13 doubles: the nine MHD variables followed by the M1
 * radiation variables (primitives: rest-frame energy density and the
 * relative four-velocity of the radiation frame; conserved: R^t_t, R^t_i),
 * KORAL's order with RADIATION and MAGNFIELD (mnemonics.h:29-55).  Metric
 * points are 20 + 20 doubles as elsewhere.  Opacities: Kramers-type
 * absorption kappa = kramers rho T^-3.5 cm^2/g plus electron scattering kes
 * cm^2/g, converted to code units with the black-hole mass. */
typedef struct {
  double gamma;                        /* adiabatic index                         */
  double kb, mp, sigma, mu;            /* K_BOLTZ, M_PROTON, SIGMA_RAD, MU_GAS    */
  double ggg, ccc, masscm;             /* G, c (cgs) and GM/c^2 (cm)              */
  double kramers, kes;                 /* opacity law coefficients (cgs)          */
  double kes_gu;                       /* kes in code units                       */
  double gammamaxrad, eradfloor;       /* GAMMAMAXRAD, ERADFLOOR                  */
  double gammasmalllimit, numepsilon;  /* GAMMASMALLLIMIT, NUMEPSILON             */
  double eps, conv, entrconv, maxiter; /* RADIMPEPS, RADIMPCONV, RADIMPENTRCONV,  */
                                       /* RADIMPMAXITER                           */
  double dampfac, maxdown, maxup;      /* RADIMPLICITDAMPINGFACTOR,               */
                                       /* RADIMPLICITMAXENCHANGEDOWN/UP           */
  double maxdamping, threshold;        /* MAXRADIMPDAMPING, RADIMPLICITTHRESHOLD  */
  double u2pconv;                      /* U2PCONV of the nested MHD inversion     */
  double eerhoratiomin, eerhoratiomax; /* EERHORATIOMIN/MAX: radiation floors     */
  double eeuuratiomin, eeuuratiomax;   /* EEUURATIOMIN/MAX                        */
} kgpu_rad_params;

/* KORAL's defaults (choices.h:320-597, ko.h:17-48) for a black hole of
 * `mass` solar masses, adiabatic index gamma and the given opacity law. */
int kgpu_rad_default_params(kgpu_rad_params *rp, double mass, double gamma, double kramers, double kes);

/* Solver variants of kgpu_rad_implicit_cells. */
#define KGPU_RAD_PLAIN 0       /* one thread runs a cell's whole cascade        */
#define KGPU_RAD_BATCHED 1     /* passes over a work queue of unfinished cells  */
#define KGPU_RAD_PERSISTENT 2  /* one resident kernel whose lanes take cells    */
                               /* from a work list as they finish, then a       */
                               /* warp-per-cell kernel for the cells left over  */

/* Tuning of the batched and persistent forms.  Results and statistics
 * (Newton iterations, evaluations) do not depend on any field except
 * warm_attempts, which chooses how long a warm-started cell trusts its
 * prediction.
 *  pass_iters     batched: Newton iterations a cell may take per pass (4)
 *  inner_cap      W-function evaluations the MHD inversion nested in one
 *                 residual evaluation may take in a single lane before that
 *                 evaluation is repeated by a whole warp with the damped
 *                 trials tried 32 at a time (64; 0: never)
 *  tail           batched: the size of the warp-per-cell tail, in blocks of
 *                 four warps per SM (0..32, default 8; 0: none): once the
 *                 cells left after a pass are no more than its warps, each is
 *                 run to its end by a whole warp
 *  warm_attempts  learned warm start: attempts of the cascade a warm-started
 *                 cell runs from the predicted iterate before the reference
 *                 cascade runs from the reference guess (1..6, default 6)
 *  thin           persistent: once the work list is empty, a warp hands the
 *                 cells it still holds to the warp-per-cell kernel when at
 *                 most this many of its 32 lanes hold one (0..32, default 8)
 *  blocks_per_sm  persistent: resident blocks of 128 threads per SM
 *                 (0: as many as the kernel's registers allow)
 *  skip           learned warm start: 1 (default): a warm-started cell
 *                 begins with the energy-equation attempt the network expects
 *                 to be the first that succeeds (outputs 5 and 6), skipping
 *                 those it expects to fail; 2: besides, only the cells the
 *                 network expects to fail their first attempt start from the
 *                 prediction, the others from their own guess; 0: every
 *                 warm-started cell begins with attempt 0.  Every cell still
 *                 converges to RADIMPCONV or runs the reference cascade
 *  hard           batched, in a context's implicit step: a cell whose
 *                 previous solve in that context took a later attempt,
 *                 failed, or took more than `hard` Newton iterations skips
 *                 the first pass and starts in the warp-per-cell tail, where
 *                 long cascades run fastest (default 16; -1: every cell
 *                 starts in the first pass; the context-free entry points
 *                 have no previous solve and ignore it) */
typedef struct {
  int pass_iters;
  int inner_cap;
  int tail;
  int warm_attempts;
  int thin;
  int blocks_per_sm;
  int skip;
  int hard;
} kgpu_rad_solver_opts;
int kgpu_rad_default_solver_opts(kgpu_rad_solver_opts *opts);

/* Batched solve_implicit_lab (rad.c:1225-1570): for each of n cells, the
 * conserved state uu after the explicit update, the primitive guess pp,
 * its metric point and time step dt; the cascade of 4D Newton solves
 * (energy equation on the dominant then the other component, lab then
 * fluid frame, then the entropy equation) runs until one converges to the
 * residual RADIMPCONV.  Outputs: primitives and conserved variables
 * (unchanged inputs where all attempts fail), status (0 or -1 as
 * solve_implicit_lab returns), the attempt that succeeded (0..5, -1) and
 * its Newton iterations.  Host pointers. */
int kgpu_rad_implicit_cells(int n, const kgpu_rad_params *rp, const double *uu, const double *pp, const double *g,
                            const double *G, const double *dt, double *pp_out, double *uu_out, int *status,
                            int *attempt, int *iters, int mode);
/* The same on device pointers, asynchronously on `stream` (a cudaStream_t,
 * or null for the default stream).  stats, when not null, receives after
 * completion: [0] Newton iterations over all attempts, [1] passes run.
 * Temporary device memory of the batched and persistent variants is taken
 * from `work`, which must hold kgpu_rad_work_bytes(n) bytes (null for the
 * plain one). */
size_t kgpu_rad_work_bytes(int n);
int kgpu_rad_implicit_cells_device(int n, const kgpu_rad_params *rp, const double *uu, const double *pp,
                                   const double *g, const double *G, const double *dt, double *pp_out,
                                   double *uu_out, int *status, int *attempt, int *iters, int mode, void *work,
                                   void *stream, unsigned long long *stats);
/* Learned warm start.  kgpu_rad_implicit_cells_warm_device is the batched
 * form whose first attempt starts from the iterate predicted by the warm-
 * start network (ypred, float [n][8], the output of kgpu_mlp_forward on
 * the cells' features); where that attempt fails it is repeated from the
 * cell's own guess and the reference cascade follows, so every cell still
 * converges to RADIMPCONV or fails as the reference would.  stats: [0]
 * Newton iterations over all attempts, [1] passes, [2] cells whose warm
 * attempt failed (fallbacks). */
int kgpu_rad_implicit_cells_warm_device(int n, const kgpu_rad_params *rp, const double *uu, const double *pp,
                                        const double *g, const double *G, const double *dt, const float *ypred,
                                        double *pp_out, double *uu_out, int *status, int *attempt, int *iters,
                                        void *work, void *stream, unsigned long long *stats);
/* The general device form: any solver variant, an optional prediction
 * ypred (null: the reference guess; not with KGPU_RAD_PLAIN), the solver
 * tuning opts (null: the process-wide values), and up to nstats (<= 8)
 * counters: [0] Newton iterations over all attempts, [1] launches that had
 * work, [2] warm-start fallbacks, [3] residual evaluations, [4] Newton steps
 * and [5] W-function evaluations of the nested MHD inversions, [6]
 * evaluations handed to a whole warp. */
int kgpu_rad_implicit_cells_device_ex(int n, const kgpu_rad_params *rp, const double *uu, const double *pp,
                                      const double *g, const double *G, const double *dt, const float *ypred,
                                      double *pp_out, double *uu_out, int *status, int *attempt, int *iters,
                                      int mode, const kgpu_rad_solver_opts *opts, void *work, void *stream,
                                      unsigned long long *stats, int nstats);
/* Network inputs (float [n][16]) of cells before a solve, and training
 * targets (float [n][7]: ln of the gas and radiation energy ratios, change
 * of the iterated velocity, then 1/0 for "the first attempt failed" and
 * "the first two attempts failed") from the states before and after and
 * the attempt that succeeded; the first five NaN where status is not 0.
 * Device pointers, asynchronous on stream. */
int kgpu_rad_features_device(int n, const kgpu_rad_params *rp, const double *pp, const double *g, const double *G,
                             const double *dt, float *X, void *stream);
int kgpu_rad_targets_device(int n, const kgpu_rad_params *rp, const double *pp, const double *pp1,
                            const double *g, const double *G, const int *status, const int *attempt, float *T,
                            void *stream);

/* Learned warm start of the MHD inversion.  Replaces, on independent cells,
 * the per-cell u2p(uu,pp,geom,corrected,fixups,0) of u2p.c:176, whose
 * Newton iteration starts from W = (rho + GAMMA u) gamma^2 of the guess pp
 * (u2p.c:2093-2112).  Cells are rows of nv >= 9 doubles (the nine MHD
 * variables first; 13 with radiation), metric points 20 doubles; device
 * pointers, the call waits for its stream when stats are asked for.
 * kgpu_u2p_cells_device: with ypred null, the reference's u2p (same results
 * as kgpu_u2p_cells); with ypred (float [n][8], kgpu_mlp_forward's output)
 * the solve starts from W_guess exp(ypred[0]) where |ypred[0]| >= wgate
 * (from W_guess elsewhere), with the entropy equation alone where
 * ypred[1] > sgate, and falls back to the reference's u2p from the guess
 * where it does not converge.  iters (optional) gets each cell's
 * Newton iterations over all its solves; stats: [0] Newton iterations,
 * [1] fallbacks, [2] W-function evaluations (bracketing and damped trials
 * included).  kgpu_u2p_features_device: network inputs (float [n][16]) of
 * the conserved state uu and the guess pp; kgpu_u2p_targets_device:
 * training targets (float [n][7]: ln(W/W_guess), 1/0 for an entropy
 * inversion, zeros) from the guess and the inverted primitives pp1, NaN
 * where status is neither 0 nor -1.  cfg supplies GAMMA, U2PCONV and
 * the density floor; its grid fields are not read. */
int kgpu_u2p_cells_device(int n, const kgpu_config *cfg, int nv, const double *uu, double *pp, const double *g,
                          const double *G, const float *ypred, float wgate, float sgate, int *status, int *fixup,
                          int *iters, void *stream, unsigned long long *stats, int nstats);
int kgpu_u2p_features_device(int n, const kgpu_config *cfg, int nv, const double *uu, const double *pp,
                             const double *g, const double *G, float *X, void *stream);
int kgpu_u2p_targets_device(int n, const kgpu_config *cfg, int nv, const double *pp, const double *pp1,
                            const double *g, const double *G, const int *status, float *T, void *stream);

/* The warm-start network: 16 -> 128 -> 128 -> 7, SiLU, BF16 weights and
 * activations with FP32 accumulation on the tensor cores; trained and run on
 * the device.  The parameter blob (kgpu_mlp_blob_size() floats) holds
 * W1[16][128], b1[128], W2[128][128], b2[128], W3[128][8], b3[8] (output 7
 * unused), then the output standardisation mean[8] and scale[8]. */
typedef struct kgpu_mlp kgpu_mlp;
int kgpu_mlp_blob_size(void);
int kgpu_mlp_create(kgpu_mlp **mlp, unsigned long long seed);
int kgpu_mlp_destroy(kgpu_mlp *mlp);
int kgpu_mlp_get(kgpu_mlp *mlp, float *blob);
int kgpu_mlp_set(kgpu_mlp *mlp, const float *blob);
/* Y[n][8] (unstandardised outputs) from X[n][16]; device pointers. */
int kgpu_mlp_forward(kgpu_mlp *mlp, const float *X, int n, float *Y, void *stream);
/* Gradient (the blob's first part) and mean loss of one batch of n samples
 * at the current weights, without an update; device X, T, host outputs. */
int kgpu_mlp_gradient(kgpu_mlp *mlp, const float *X, const float *T, int n, float *grad, double *loss);
/* One shuffled epoch of Adam over n samples in batches of `batch`. */
int kgpu_mlp_train_epoch(kgpu_mlp *mlp, const float *X, const float *T, int n, int batch, float lr,
                         unsigned long long seed, double *mean_loss);

/* Solver tuning of the context-free entry points (kgpu_rad_implicit_cells*):
 * process-wide values, one field of kgpu_rad_solver_opts each (see there).
 * A context does not read them: it holds its own options
 * (kgpu_set_implicit_options). */
int kgpu_rad_set_pass_iters(int k);
int kgpu_rad_set_inner_cap(int cap);
int kgpu_rad_set_tail(int on);
int kgpu_rad_set_warm_attempts(int k);
int kgpu_rad_set_solver_opts(const kgpu_rad_solver_opts *opts);
int kgpu_rad_get_solver_opts(kgpu_rad_solver_opts *opts);
/* M1 closure u2p_rad (u2prad.c:485) and p2u (p2u.c:40) of n cells, host
 * pointers; corrected[i] is u2p_rad's corrected flag. */
int kgpu_rad_u2p_cells(int n, const kgpu_rad_params *rp, const double *uu, double *pp, const double *g,
                       const double *G, int *status, int *corrected);
int kgpu_rad_p2u_cells(int n, const kgpu_rad_params *rp, const double *pp, double *uu, const double *g,
                       const double *G);
/* The per-cell u2p of the reference with all its outputs (u2p.c:176-485,
 * type 0): the MHD inversion with its entropy fallback and, when rp is
 * given (cfg->nv = 13), the M1 inversion u2p_rad.  n cells in KORAL's
 * cell-major layout with cfg->nv variables; per cell status (u2p's return
 * value), corrected[3] (hydro corrected, radiation corrected, entropy
 * balance not applied: always 0 here) and fixups[2] (hydro fixup requested,
 * radiation fixup requested: DORADFIXUPS).  rp must be null for nv = 9. */
int kgpu_u2p_cells_full(int n, const kgpu_config *cfg, const kgpu_rad_params *rp, const double *uu, double *pp,
                        const double *g, const double *G, int *status, int *corrected, int *fixups);
/* Kerr-Schild metric point (r, theta) of spin a in the 20 + 20 layout
 * (g_{mu nu}, d ln sqrt(-g)/dx^i, sqrt(-g); g^{mu nu}, g_tt + 1).  Host. */
int kgpu_ks_metric(double a, double r, double th, double *g20, double *G20);
int kgpu_ks_metric_batch(double a, int n, const double *r, const double *th, double *g20, double *G20);
/* Measured FP64 issue rate of this GPU (DMUL + DADD per second, no FMA
 * contraction, as the library's kernels are built): the denominator of the
 * FP64 roofline of the solver kernels. */
int kgpu_fp64_peak(double *ops_per_s);
/* The device's powers and logarithm of the hot path on n host values, for
 * checks against the host C library: kind 0 x^2, 1 x^4, 2 x^-3.5 (the
 * Planck and Kramers terms), 3 x^y with 4y an integer (the entropy),
 * 4 log(x), 5 the device library's pow(x, y).  Kinds 0-3 are products and
 * square roots carried to double-double accuracy and rounded once. */
int kgpu_eval_powers(int n, int kind, double y, const double *x, double *out);

/* Radiation in the grid step (nv = 13: the nine MHD variables, then E and
 * the radiation frame's relative four-velocity; conserved R^t_t, R^t_i).
 * kgpu_set_radiation switches a 13-variable context to the RADIATION build
 * of the time loop: M1 fluxes and characteristic speeds in op_explicit
 * (optionally with the optical-depth limiter of calc_rad_wavespeeds,
 * rad.c:2489-2502), u2p_rad and check_floors_rad in calc_u2p, and the
 * implicit lab-frame source solve in op_implicit (finite.c:1242-1292) with
 * the RADIMP fixup.  rp->gamma must equal the grid's adiabatic index.
 * Allocates the solver's buffers for the domain cells once. */
int kgpu_set_radiation(kgpu_ctx *ctx, const kgpu_rad_params *rp, int wavespeed_limiter);
/* Solver of op_implicit: KGPU_RAD_PLAIN, KGPU_RAD_BATCHED (default) or
 * KGPU_RAD_PERSISTENT, and the warm-start network (batched and
 * persistent only; null for the reference's guess).  The network is
 * borrowed: it must outlive its use by the context. */
int kgpu_set_implicit_solver(kgpu_ctx *ctx, int mode, kgpu_mlp *warm);
/* The context's own solver tuning (kgpu_rad_solver_opts; defaults from
 * kgpu_rad_default_solver_opts at kgpu_set_radiation).  Setting it drops the
 * context's captured step graph, so the next graph step runs with the new
 * values. */
int kgpu_set_implicit_options(kgpu_ctx *ctx, const kgpu_rad_solver_opts *opts);
int kgpu_get_implicit_options(kgpu_ctx *ctx, kgpu_rad_solver_opts *opts);
/* With a warm-start network: start from the prediction only the cells whose
 * previous implicit solve in this context needed a later attempt of the
 * cascade or more than `iters` Newton iterations (the others start from the
 * reference guess, which the time step's own evolution keeps close);
 * -1 (default): every cell. */
int kgpu_set_warm_gate(kgpu_ctx *ctx, int iters);
/* Launch shapes and solver settings of a context.  None changes results:
 * every choice performs the same arithmetic (the kernels' variants differ
 * in the registers they are compiled for, the solver settings in how work
 * is scheduled).
 *  flux_blocks     blocks of 128 threads per SM the face-flux kernels are
 *                  compiled for: 5..8 (default 7)
 *  flux_split      1: the face states are reconstructed by a kernel of
 *                  their own (one thread per face and variable) and read by
 *                  the flux kernel; 0 (default): reconstructed inside it
 *  update_blocks   the same for the update kernel: 3..5 (default 4)
 *  u2p_blocks      the same for the first inversion pass: 4..6 (default 5)
 *  u2p_pass_iters  Newton steps of the first inversion pass before a solve
 *                  is queued for resumption (default 8)
 *  implicit_mode   solver of op_implicit (KGPU_RAD_*; default batched)
 *  implicit        its tuning (kgpu_rad_solver_opts) */
typedef struct {
  int flux_blocks;
  int flux_split;
  int update_blocks;
  int u2p_blocks;
  int u2p_pass_iters;
  int implicit_mode;
  kgpu_rad_solver_opts implicit;
} kgpu_tuning;
int kgpu_get_tuning(kgpu_ctx *ctx, kgpu_tuning *t);
/* Applies a tuning (drops the captured step graph; the network of the
 * implicit solver is kept; a plain implicit mode with a network set is
 * KGPU_EINVAL). */
int kgpu_set_tuning(kgpu_ctx *ctx, const kgpu_tuning *t);
/* The autotuner.  Times candidate values of each field of kgpu_tuning, one
 * field after another (coordinate descent from the current tuning), on
 * this context's own state: each trial restores the state, runs `steps`
 * whole time steps (RK2, or RK2IMEX with radiation) from the stream and
 * times them with CUDA events; the state, the time step and the counters
 * are restored afterwards, and the choice is applied.  Candidates: the
 * fused or split face flux, flux 5..8, update 3..5, u2p 4..6 blocks; u2p_pass_iters 4, 8, 16; with
 * radiation the batched and the persistent solver, pass_iters 4, 8, 16,
 * inner_cap 32, 64, 128, tail 0, 4, 8, 16, hard -1, 8, 16, 32 or thin 4, 8,
 * 16.  A candidate
 * replaces the incumbent only when it is faster by min_gain (a fraction,
 * e.g. 0.02) in the same round of trials.  The choice is cached per device
 * and grid configuration for the process: with reuse = 1 a cached choice
 * is applied without trials.  Outputs (optional): the chosen tuning and
 * the time per step of the starting and of the chosen tuning (ms[2]). */
int kgpu_autotune(kgpu_ctx *ctx, int steps, double min_gain, int reuse, kgpu_tuning *chosen, double *ms);
/* The autotuner's selection rule on its own: index of the fastest of n
 * timings if it beats timings[incumbent] by the fraction min_gain, else
 * incumbent.  Negative or non-finite timings (failed trials) never win. */
int kgpu_tune_select(int n, const double *ms, int incumbent, double min_gain);

/* Whole RK2IMEX steps (ko.c:444-570), dt in device memory; and the same
 * replayed from a CUDA graph captured on the first call. */
int kgpu_rk2imex_steps(kgpu_ctx *ctx, int nsteps);
int kgpu_rk2imex_steps_graph(kgpu_ctx *ctx, int nsteps);
/* Device buffers of the most recent implicit source step (cell-major, the
 * domain cells with x fastest): its n cells' primitive guess and conserved
 * input, the primitives it produced (the input where every attempt failed),
 * metric points (20 + 20 doubles), time steps, status, the attempt that
 * succeeded (0..5, -1) and its Newton iterations.  Valid until the next
 * step; for diagnostics and for training the warm-start network on the
 * cells a run solves.  Null output pointers are skipped. */
int kgpu_get_implicit_buffers(kgpu_ctx *ctx, int *n, const double **pp_in, const double **uu_in,
                              const double **pp_out, const double **g20, const double **G20, const double **dt,
                              const int **status, const int **attempt, const int **iters);

/* The radiative torus (nv = 13): the pressure of the torus shared by gas and
 * M1 radiation in thermal equilibrium at one temperature (radiation frame
 * comoving with the gas), the atmosphere with a radiation energy of eradatm
 * times its gas energy at rest with it; host-only state, and the whole
 * set-up on a context with radiation switched on (kgpu_set_radiation),
 * computed on the device (or on the host by the _host form), as
 * kgpu_init_fm_torus. */
int kgpu_fm_radtorus_state(const kgpu_torus_params *tp, const kgpu_rad_params *rp, double eradatm,
                           const kgpu_config *cfg, const double *xbx, const double *xby, const double *xbz,
                           const double *g, const double *G, double *u, double *p);
int kgpu_init_fm_radtorus(kgpu_ctx *ctx, const kgpu_torus_params *tp, const kgpu_rad_params *rp, double eradatm,
                          int wavespeed_limiter);
int kgpu_init_fm_radtorus_host(kgpu_ctx *ctx, const kgpu_torus_params *tp, const kgpu_rad_params *rp,
                               double eradatm, int wavespeed_limiter);

/* ---------------------------------------------------------------------------
 * Scalar diagnostics of a black-hole disk, computed on the device.  Replaces
 *   int calc_scalars(ldouble *scalars, ldouble t)          postproc.c:996
 * for the Kerr tori (MKS2 coordinates written in their own coordinates,
 * OUTCOORDS = MYCOORDS), entry by entry:
 *   [0]  total mass (calc_totalmass)            [1] -accretion rate at the
 *   horizon (calc_mdot, type 0)                 [4] the same in Eddington units
 *   [3]  magnetic flux through the horizon, [7] MAD parameter, [9] its
 *        quadrupole form (calc_Bflux: phi-symmetric grids; 0 in 3D as there)
 *   [5]  MRI resolution Q_theta (calc_resmri; -1 unless bhdisk)
 *   [6]  rho-weighted temperature at r = 15 (calc_meantemp; -1 unless
 *        bhdisk and phi-symmetric)
 *   [8]  scale height: -1 unless bhdisk; 0 with it (CALCHRONTHEGO is not
 *        configured and r = 15 lies beyond every x1 of these grids)
 *   [11] local total luminosity (calc_local_lum at the radial index of
 *        r = 5e3 and theta index 3; R^r_t is 0 without radiation, where the
 *        reference adds an unset value)
 *   [2], [10], [12]: 0 (calc_lum leaves [2] and [10] unset on 3D grids and
 *        its phi-symmetric sum is not built; [12] is never written).
 * Radius searches, like the reference's for OUTCOORDS = MYCOORDS, compare
 * the x1 coordinate of cell centres with the radius.  Sums run on the
 * device in a fixed order: repeated calls give the same bits.
 * kgpu_calc_scalars copies the result to host memory and waits;
 * kgpu_calc_scalars_device writes it to device memory on the context's
 * stream without waiting (it may be captured into a graph after one call
 * outside capture, which allocates the work arrays). */
#define KGPU_NSCALARS 13
typedef struct kgpu_scalars_params {
  double spin;   /* BHSPIN                                             */
  double mass;   /* MASS in solar masses: units of the accretion rate  */
  int bhdisk;    /* BHDISK_PROBLEMTYPE: MRI resolution, mean temperature */
} kgpu_scalars_params;
int kgpu_calc_scalars(kgpu_ctx *ctx, const kgpu_scalars_params *sp, double t, double *scalars);
int kgpu_calc_scalars_device(kgpu_ctx *ctx, const kgpu_scalars_params *sp, double t, double *scalars_dev);

/* Time averages.  Replaces save_avg(dt) (fileop.c:10-70): every domain cell
 * adds the quantities of p2avg (p2u.c:313-541) times dt to the running sums
 * pavg, and dt is added to avgtime; the reference's loop calls it once per
 * time step with AVGOUTPUT=1 (ko.c:504-507, 606-610), after the second
 * stage's inversion and implicit step.  Per cell the sums hold NV + NAVGVARS
 * values (NAVGVARS = 112 + 3 NV, or 153 + 3 NV with radiation, choices.h:
 * 260-265) in the slots of mnemonics.h:170-199; kgpu_avg_count returns the
 * count.  The face fluxes of the last op_explicit are given flux_ct's
 * rewrite first, as the reference's flbx/flby/flbz hold it.  Two slots the
 * reference leaves as an uninitialised local value are zero here:
 * AVGEHAT without radiation and AVGGHATCOMPT (Comptonisation only).
 *  kgpu_set_avg      allocates and zeroes the sums on first use; with on = 1
 *                    the fused steps (kgpu_rk2_steps, kgpu_rk2imex_steps and
 *                    their graph forms) call save_avg once per step as the
 *                    reference's loop does.  mass (solar masses) sets the
 *                    unit constants of the averaged gas temperature
 *                    (K_BOLTZ, M_PROTON, ko.h:4-48) and is read on the
 *                    first call only; with radiation the context's radiation
 *                    constants are used.
 *  kgpu_save_avg     one save_avg(dt) now (after kgpu_set_avg).
 *  kgpu_download_avg the sums in KORAL's layout [SZ][SY][SX][NV+NAVGVARS]
 *                    (ghost cells zero) and avgtime; the reference divides by
 *                    avgtime when it writes an avg file (ko.c:785).
 *  kgpu_reset_avg    zeroes the sums and avgtime (ko.c:798-799). */
int kgpu_avg_count(kgpu_ctx *ctx);
int kgpu_set_avg(kgpu_ctx *ctx, int on, double mass);
int kgpu_save_avg(kgpu_ctx *ctx, double dt);
int kgpu_download_avg(kgpu_ctx *ctx, double *pavg, double *avgtime);
int kgpu_reset_avg(kgpu_ctx *ctx);

/* Last CUDA error string of this thread's most recent failing call. */
const char *kgpu_last_error(void);
int kgpu_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
