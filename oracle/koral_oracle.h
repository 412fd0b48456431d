/*
 * CPU restatement of KORAL's per-step hot path (TEST INFRASTRUCTURE).
 *
 * This is the parity oracle: a plain-C restatement of the reference
 * algorithm, written for this project, with the grid size, reconstruction
 * order, Riemann solver and adiabatic index chosen at run time instead of
 * at compile time.  Each function cites the reference routine it follows.
 * It keeps the reference's storage order (variable index fastest, ghost
 * cells included, ko.h:505-508) and its floating-point operation order, so
 * that it reproduces the reference bit for bit; it is itself pinned against
 * the reference built from its own sources (oracle/ref/build_ref.sh).
 *
 * Only tests/, the smoke check and the CPU-baseline leg of the benchmark may
 * load it.  The product path never calls it.
 */
#ifndef KORAL_ORACLE_H
#define KORAL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* primitive / conserved ordering, mnemonics.h:13-41 */
enum { KO_RHO = 0, KO_UU = 1, KO_VX = 2, KO_VY = 3, KO_VZ = 4, KO_ENTR = 5,
       KO_B1 = 6, KO_B2 = 7, KO_B3 = 8 };

/* cell flags, mnemonics.h:103-114 */
enum { KO_ENTROPYFLAG = 0, KO_RADIMPFIXUPFLAG = 1, KO_HDFIXUPFLAG = 2,
       KO_RADFIXUPFLAG = 3, KO_ENTROPYFLAG2 = 4, KO_ENTROPYFLAG3 = 5,
       KO_RADSOURCETYPEFLAG = 6, KO_NFLAGS = 7 };

enum { KO_LAXF = 0, KO_HLL = 1 };          /* mnemonics.h:118-119 */
enum { KO_U2P_HOT = 0, KO_U2P_ENTROPY = 1 };

typedef struct {
  double gg[4][5];   /* g_{mu nu}; [i][4] = dlog(gdet)/dx^i, [3][4] = gdet */
  double GG[4][5];   /* g^{mu nu}; [3][4] = perturbed part of g_tt        */
  double gdet, gttpert, alpha;
} ko_geom;

typedef struct {
  /* physics switches */
  double gamma;        /* adiabatic index                                  */
  double tsteplim;     /* Courant number                                   */
  int int_order;       /* 2 = PPM, 4 = MP5                                 */
  int fluxmethod;      /* KO_LAXF or KO_HLL                                */
  int periodic[3];     /* periodic boundary per axis                       */
  /* floors, choices.h:55-118 */
  double rhofloor, uurhoratiomin, uurhoratiomax, b2rhoratiomax, gammamaxhd;
  double u2pconv;      /* U2PCONV, choices.h:457                           */

  /* grid */
  int nx, ny, nz, ng, nv;
  int sx, sy, sz, ngcx, ngcy, ngcz;
  int axisym;          /* metric stored for a single phi slice             */
  int szmet, ngczmet;
  double *xb[3];       /* cell faces, index ic+ng, ic in [-ng, n+ng]        */
  double *xc[3];       /* cell centres, index ic+ng, ic in [-ng, n+ng)      */
  double min_dx, min_dy, min_dz;

  /* metric tables (KORAL layout, gSIZE=20 per point, 64 per Christoffel)  */
  double *g, *G, *gKr;           /* centres                                */
  double *gb[3], *Gb[3];         /* faces                                  */

  /* state and work arrays, [sz][sy][sx][nv] */
  double *u, *p, *ut0, *ut1, *ut2, *ubak, *pbak;
  double *flb[3];                /* face fluxes                            */
  double *emf;                   /* corner EMFs, (nx+1)(ny+1)(nz+1)*3      */
  double *ahd[3], *ahdl[3], *ahdr[3];  /* wavespeeds per cell              */
  double *cell_tstepden, *cell_dt;
  int *cellflag;

  double tstepdenmax, tstepdenmin, dt, t;
  int nstep;
  long long n_mhd_fixups, n_entropy_u2p, n_u2p_fail;
} ko_grid;

/* grid set-up */
ko_grid *ko_grid_create(int nx, int ny, int nz, int ng, int nv, int axisym);
void ko_grid_destroy(ko_grid *G);
void ko_set_uniform_grid(ko_grid *G, const double *lo, const double *hi);
void ko_set_minkowski_metric(ko_grid *G);

/* per-cell physics (restated reference routines) */
void ko_p2u_mhd(const ko_grid *G, const double *pp, double *uu, const ko_geom *geom);
int ko_u2p_solver_W(const ko_grid *G, const double *uu, double *pp, const ko_geom *geom, int Etype);
int ko_u2p(const ko_grid *G, const double *uu0, double *pp, const ko_geom *geom, int corrected[3], int fixups[2]);
int ko_check_floors_mhd(const ko_grid *G, double *pp, const ko_geom *geom);
void ko_flux_prime(const ko_grid *G, const double *pp, int idim, const ko_geom *geom, double *ff);
void ko_wavespeeds_lr_pure(const ko_grid *G, const double *pp, const ko_geom *geom, double *aaa);
void ko_avg2point(const ko_grid *G, const double *um2, const double *um1, double *u0, const double *up1,
                  const double *up2, double *ul, double *ur, double dxm2, double dxm1, double dx0,
                  double dxp1, double dxp2);
double ko_calc_Sfromu(double gamma, double rho, double u);

/* geometry lookups */
void ko_fill_geometry(const ko_grid *G, int ix, int iy, int iz, ko_geom *geom);
void ko_fill_geometry_face(const ko_grid *G, int ix, int iy, int iz, int idim, ko_geom *geom);

/* grid operators */
void ko_set_bc(ko_grid *G);
void ko_calc_wavespeeds(ko_grid *G);
void ko_op_explicit(ko_grid *G, double dt);
void ko_calc_u2p(ko_grid *G);
void ko_save_timesteps(ko_grid *G);
void ko_begin_run(ko_grid *G);
double ko_begin_step(ko_grid *G);
int ko_rk2_step(ko_grid *G);

/* initial data: relativistic Orszag-Tang vortex on the current grid */
void ko_init_orszag_tang(ko_grid *G);

/* batched per-cell calls (parameters taken from G) */
int ko_u2p_batch(const ko_grid *G, int n, const double *uu, double *pp, const double *g, const double *Gm,
                 int *status, int *fixup);
int ko_p2u_batch(const ko_grid *G, int n, const double *pp, double *uu, const double *g, const double *Gm);
int ko_floors_batch(const ko_grid *G, int n, double *pp, const double *g, const double *Gm, int *ret);

/* accessors for the ctypes wrapper */
double *ko_array(ko_grid *G, int which);
int ko_layout(const ko_grid *G, int *out);
double ko_scalar(const ko_grid *G, int which);
void ko_set_scalar(ko_grid *G, int which, double v);
void ko_set_physics(ko_grid *G, double gamma, double tsteplim, int int_order, int fluxmethod);
void ko_set_floors(ko_grid *G, double rhofloor, double uurhomin, double uurhomax, double b2rhomax, double gammamax);

#ifdef __cplusplus
}
#endif
#endif
