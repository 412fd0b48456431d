/*
 * Test harness around the reference KORAL build (the parity oracle's
 * "reference" leg).  Test infrastructure only: it is linked with the
 * unmodified reference translation units, compiled from their own sources
 * by oracle/ref/build_ref.sh, and loaded by the tests through ctypes.
 *
 * It reproduces, by calling the reference's own routines, the start-up that
 * main() performs (ko.c:8-216, without files or restarts) and one iteration
 * of the time loop of solve_the_problem() for the RK2 and RK2IMEX
 * integrators (ko.c:347-626, 714-722).  The operators themselves
 * (op_explicit, calc_u2p, op_implicit, set_bc, save_timesteps, ...) are
 * exported by the reference objects and may also be called directly.
 */
#include "ko.h"

static ldouble kref_time;

/* Grid and layout constants of this build. */
int kref_sizes(int *out)
{
  out[0] = NX; out[1] = NY; out[2] = NZ; out[3] = NG; out[4] = NV;
  out[5] = SX; out[6] = SY; out[7] = SZ; out[8] = SZMET;
  out[9] = INT_ORDER; out[10] = FLUXMETHOD; out[11] = TIMESTEPPING;
#ifdef MAGNFIELD
  out[12] = 1;
#else
  out[12] = 0;
#endif
#ifdef RADIATION
  out[13] = 1;
#else
  out[13] = 0;
#endif
  out[14] = MYCOORDS;
  return 15;
}

double kref_gamma(void) { return GAMMA; }
double kref_tsteplim(void) { return TSTEPLIM; }
double kref_time_now(void) { return kref_time; }

/* main(): ko.c:10-216 with output and restart logic left out. */
int kref_init(void)
{
  omp_myinit();
  mstep_init();
  doingavg = 0;
  doingpostproc = 0;
  global_time = 0.;
  gsl_set_error_handler_off();
  initialize_arrays();
  set_grid(&min_dx, &min_dy, &min_dz, &max_dt);
  alloc_loops(1, 0., 0.);
  calc_metric();

  set_initial_profile();
  mpi_exchangedata();
  calc_avgs_throughout();
  set_bc(0., 1);
#ifdef MAGNFIELD
#ifdef VECPOTGIVEN
  calc_BfromA(p, 1);
  mpi_exchangedata();
  calc_avgs_throughout();
  set_bc(0., 1);
#endif
#endif
#ifdef PR_POSTINIT
#include PR_POSTINIT
#endif
  copy_u(1., p, pinit);

  /* solve_the_problem() before its loop: ko.c:290-313 */
  int ii;
  dt = -1.;
  max_ws[0] = max_ws[1] = max_ws[2] = 10000.;
  if (NZ > 1)
    tstepdenmax = max_ws[0] / min_dx + max_ws[1] / min_dy + max_ws[2] / min_dz;
  else if (NY > 1)
    tstepdenmax = max_ws[0] / min_dx + max_ws[1] / min_dy;
  else
    tstepdenmax = max_ws[0] / min_dx;
  tstepdenmax /= TSTEPLIM;
  tstepdenmin = tstepdenmax;
  for (ii = 0; ii < Nloop_0; ii++) {
    int ix = loop_0[ii][0], iy = loop_0[ii][1], iz = loop_0[ii][2];
    set_u_scalar(cell_tstepden, ix, iy, iz, tstepdenmax);
    set_u_scalar(cell_dt, ix, iy, iz, 1. / tstepdenmax);
  }
  nstep = 0;
  kref_time = 0.;
  return 0;
}

/* Start of one loop iteration: ko.c:352-425 (dt from the previous
 * wavespeeds, reset of the running maxima). Returns dt. */
double kref_begin_step(void)
{
  global_int_slot[GLOBALINTSLOT_NTOTALRADIMPFIXUPS] = 0;
  global_int_slot[GLOBALINTSLOT_NTOTALMHDFIXUPS] = 0;
  global_int_slot[GLOBALINTSLOT_NTOTALRADFIXUPS] = 0;
  global_time = kref_time;
  nstep++;
  dt = 1. / tstepdenmax;
  global_dt = dt;
  max_ws[0] = -1.;
  max_ws[1] = -1.;
  max_ws[2] = -1.;
  max_ws_ph = -1.;
  tstepdenmax = -1.;
  tstepdenmin = BIG;
  return dt;
}

/* Failure accounting after a step: ko.c:697-722.  Returns 0, or -1 where the
 * reference would exit because more than 10% of the cells failed. */
int kref_end_step(void)
{
  int maxfailures = TNX * TNY * TNZ / 10;
  kref_time += dt;
  if (global_int_slot[GLOBALINTSLOT_NTOTALCRITFAILURES] > maxfailures ||
      global_int_slot[GLOBALINTSLOT_NTOTALMHDFIXUPS] > maxfailures ||
      global_int_slot[GLOBALINTSLOT_NTOTALRADFIXUPS] > maxfailures)
    return -1;
  return 0;
}

/* RK2 body of the loop: ko.c:571-626. */
static void kref_rk2_body(ldouble t)
{
  save_timesteps();
  copyi_u(1., u, ut0);
  do_correct();
  op_explicit(t, 0.5 * dt);
  calc_u2p();
  op_implicit(t, 0.5 * dt);
  copyi_u(1., u, ut1);
  op_explicit(t, dt);
  calc_u2p();
  op_implicit(t, dt);
  addi_u(1., u, -1., ut1, ut2);
  addi_u(1., ut0, 1., ut2, u);
}

/* RK2IMEX body of the loop: ko.c:444-570 (SELFTIMESTEP off). */
static void kref_rk2imex_body(ldouble t)
{
  int ii, iv, ix, iy, iz;
  ldouble gamma = 1. - 1. / sqrt(2.), dtcell;
  save_timesteps();
  dtcell = dt;

  copyi_u(1., u, ut0);
  op_implicit(t, dt * gamma);
  for (ii = 0; ii < Nloop_0; ii++) {
    ix = loop_0[ii][0]; iy = loop_0[ii][1]; iz = loop_0[ii][2];
    PLOOP(iv) set_u(drt1, iv, ix, iy, iz, (1. / (dtcell * gamma)) * get_u(u, iv, ix, iy, iz) + (-1. / (dtcell * gamma)) * get_u(ut0, iv, ix, iy, iz));
  }
  copyi_u(1., u, ut1);
  calc_u2p();
  do_correct();
  op_explicit(t, dt);
  for (ii = 0; ii < Nloop_0; ii++) {
    ix = loop_0[ii][0]; iy = loop_0[ii][1]; iz = loop_0[ii][2];
    PLOOP(iv) set_u(dut1, iv, ix, iy, iz, (1. / (dtcell)) * get_u(u, iv, ix, iy, iz) + (-1. / (dtcell)) * get_u(ut1, iv, ix, iy, iz));
  }
  for (ii = 0; ii < Nloop_0; ii++) {
    ix = loop_0[ii][0]; iy = loop_0[ii][1]; iz = loop_0[ii][2];
    PLOOP(iv) set_u(u, iv, ix, iy, iz, get_u(ut0, iv, ix, iy, iz) + (dtcell) * get_u(dut1, iv, ix, iy, iz) + (dtcell * (1. - 2. * gamma)) * get_u(drt1, iv, ix, iy, iz));
  }
  copyi_u(1., u, uforget);
  calc_u2p();
  do_correct();
  op_implicit(t, gamma * dt);
  for (ii = 0; ii < Nloop_0; ii++) {
    ix = loop_0[ii][0]; iy = loop_0[ii][1]; iz = loop_0[ii][2];
    PLOOP(iv) set_u(drt2, iv, ix, iy, iz, (1. / (dtcell * gamma)) * get_u(u, iv, ix, iy, iz) + (-1. / (dtcell * gamma)) * get_u(uforget, iv, ix, iy, iz));
  }
  copyi_u(1., u, ut2);
  calc_u2p();
  do_correct();
  op_explicit(t, dt);
  for (ii = 0; ii < Nloop_0; ii++) {
    ix = loop_0[ii][0]; iy = loop_0[ii][1]; iz = loop_0[ii][2];
    PLOOP(iv) set_u(dut2, iv, ix, iy, iz, (1. / (dtcell)) * get_u(u, iv, ix, iy, iz) + (-1. / (dtcell)) * get_u(ut2, iv, ix, iy, iz));
  }
  for (ii = 0; ii < Nloop_0; ii++) {
    ix = loop_0[ii][0]; iy = loop_0[ii][1]; iz = loop_0[ii][2];
    PLOOP(iv) set_u(u, iv, ix, iy, iz, get_u(ut0, iv, ix, iy, iz) + (dtcell / 2.) * get_u(dut1, iv, ix, iy, iz) + (dtcell / 2.) * get_u(dut2, iv, ix, iy, iz));
  }
  for (ii = 0; ii < Nloop_0; ii++) {
    ix = loop_0[ii][0]; iy = loop_0[ii][1]; iz = loop_0[ii][2];
    PLOOP(iv) set_u(u, iv, ix, iy, iz, get_u(u, iv, ix, iy, iz) + (dtcell / 2.) * get_u(drt1, iv, ix, iy, iz) + (dtcell / 2.) * get_u(drt2, iv, ix, iy, iz));
  }
  calc_u2p();
  do_correct();
}

/* One full time step.  Returns 0, or -1 on the reference's failure cap. */
int kref_step(void)
{
  kref_begin_step();
  if (TIMESTEPPING == RK2)
    kref_rk2_body(kref_time);
  else
    kref_rk2imex_body(kref_time);
  return kref_end_step();
}

int kref_nsteps(int n)
{
  int i, r = 0;
  for (i = 0; i < n && r == 0; i++)
    r = kref_step();
  return r;
}

/* The radius-dependent density floor of check_floors_mhd (u2p.c:546-557)
 * evaluated exactly as there, at cell centres (SX values) and x-faces
 * (SX+1 values) of the x axis.  Returns 0 when the build has no such floor. */
int kref_rhofloor_table(double *centres, double *xfaces)
{
#ifdef RHOFLOOR_BH
  int ix;
  for (ix = -NG; ix < NX + NG; ix++) {
    ldouble xx[4] = {0., get_x(ix, 0), get_x(0, 1), get_x(0, 2)}, xxBL[4];
    coco_N(xx, xxBL, MYCOORDS, BLCOORDS);
    ldouble rr = xxBL[1] / rhorizonBL;
    centres[ix + NG] = RHOFLOOR_BH_NORM / sqrt(rr * rr * rr);
  }
  for (ix = -NG; ix <= NX + NG; ix++) {
    ldouble xx[4] = {0., get_xb(ix, 0), get_x(0, 1), get_x(0, 2)}, xxBL[4];
    coco_N(xx, xxBL, MYCOORDS, BLCOORDS);
    ldouble rr = xxBL[1] / rhorizonBL;
    xfaces[ix + NG] = RHOFLOOR_BH_NORM / sqrt(rr * rr * rr);
  }
  return 1;
#else
  (void)centres; (void)xfaces;
  return 0;
#endif
}

/* Physics constants of this build needed to configure the GPU path. */
int kref_physics(double *out)
{
  out[0] = GAMMA;
  out[1] = TSTEPLIM;
  out[2] = RHOFLOOR;
  out[3] = UURHORATIOMIN;
  out[4] = UURHORATIOMAX;
  out[5] = B2RHORATIOMAX;
  out[6] = GAMMAMAXHD;
  out[7] = U2PCONV;
  out[8] = BHSPIN;
#ifdef METRICAXISYMMETRIC
  out[9] = 1.;
#else
  out[9] = 0.;
#endif
  return 10;
}

#ifdef RADIATION
/* ---------------------------------------------------------------------
 * Per-cell radiation entry points (RADCELLS build).  Independent cells are
 * stored in the domain (cell k at ix = k % NX, iy = k / NX, iz = 0), each
 * with its own metric written into the reference's metric tables, and the
 * reference's solve_implicit_lab (rad.c:1225-1570) is called on each.
 * --------------------------------------------------------------------- */

/* Unit constants and solver parameters of this build, in code units. */
int kref_rad_consts(double *out)
{
  out[0] = K_BOLTZ;
  out[1] = M_PROTON;
  out[2] = SIGMA_RAD;
  out[3] = MU_GAS;
  out[4] = GGG;
  out[5] = CCC;
  out[6] = MASSCM;
  out[7] = GAMMAMAXRAD;
  out[8] = ERADFLOOR;
  out[9] = RADIMPEPS;
  out[10] = RADIMPCONV;
  out[11] = RADIMPENTRCONV;
  out[12] = RADIMPMAXITER;
  out[13] = RADIMPLICITDAMPINGFACTOR;
  out[14] = RADIMPLICITMAXENCHANGEDOWN;
  out[15] = RADIMPLICIMAXENCHANGEUP;
  out[16] = MAXRADIMPDAMPING;
  out[17] = RADIMPLICITTHRESHOLD;
  out[18] = GAMMASMALLLIMIT;
  out[19] = NUMEPSILON;
  out[20] = EERHORATIOMIN;
  out[21] = EERHORATIOMAX;
  out[22] = EEUURATIOMIN;
  out[23] = EEUURATIOMAX;
  out[24] = NX * NY;
  return 25;
}

/* The metric of the build's coordinates at xx[4], laid out as one cell of
 * the metric tables (calc_metric, metric.c:3900-3920). */
int kref_metric_at(const double *xx, double *g20, double *G20)
{
  ldouble x[4] = {xx[0], xx[1], xx[2], xx[3]}, gl[4][5];
  int i, j;
  calc_g(x, gl);
  for (i = 0; i < 4; i++)
    for (j = 0; j < 4; j++) g20[i * 5 + j] = gl[i][j];
  for (j = 0; j < 3; j++) g20[j * 5 + 4] = calc_dlgdet(x, j);
  g20[3 * 5 + 4] = calc_gdet(x);
  calc_G(x, gl);
  for (i = 0; i < 4; i++)
    for (j = 0; j < 4; j++) G20[i * 5 + j] = gl[i][j];
  for (j = 0; j < 3; j++) G20[j * 5 + 4] = 0.;
  G20[3 * 5 + 4] = calc_gttpert(x);
  return 0;
}

static void kref_geom_from(const double *g20, const double *G20, struct geometry *geom)
{
  int i, j;
  memset(geom, 0, sizeof(*geom));
  for (i = 0; i < 4; i++)
    for (j = 0; j < 5; j++) {
      geom->gg[i][j] = g20[i * 5 + j];
      geom->GG[i][j] = G20[i * 5 + j];
    }
  geom->alpha = sqrt(-1. / geom->GG[0][0]);
  geom->gdet = geom->gg[3][4];
  geom->gttpert = geom->GG[3][4];
  geom->ifacedim = -1;
  geom->par = -1;
  geom->coords = MYCOORDS;
}

/* Entropy primitive from (rho, u) and the conserved variables (p2u.c:40),
 * n cells of NV primitives each; opacities (calc_kappa, calc_kappaes) of
 * each cell go to kap[2k], kap[2k+1]. */
int kref_rad_prepare(int n, double *pp, const double *g20, const double *G20, double *uu, double *kap)
{
  int k;
  for (k = 0; k < n; k++) {
    struct geometry geom;
    kref_geom_from(g20 + 20 * k, G20 + 20 * k, &geom);
    double *p1 = pp + (long)k * NV;
    p1[ENTR] = calc_Sfromu(p1[RHO], p1[UU]);
    p2u(p1, uu + (long)k * NV, &geom);
    ldouble k1, k2, k3, k4;
    kap[2 * k] = calc_kappa(p1, &geom, &k1, &k2, &k3, &k4);
    kap[2 * k + 1] = calc_kappaes(p1, &geom);
  }
  return 0;
}

static void kref_rad_load(int k, const double *uu, const double *pp, const double *g20, const double *G20)
{
  int ix = k % NX, iy = k / NX, i, j, iv;
  for (i = 0; i < 4; i++)
    for (j = 0; j < 5; j++) {
      set_g(g, i, j, ix, iy, 0, g20[20 * k + i * 5 + j]);
      set_g(G, i, j, ix, iy, 0, G20[20 * k + i * 5 + j]);
    }
  for (iv = 0; iv < NV; iv++) {
    set_u(u, iv, ix, iy, 0, uu[(long)k * NV + iv]);
    set_u(p, iv, ix, iy, 0, pp[(long)k * NV + iv]);
  }
}

/* solve_implicit_lab on n <= NX*NY cells, one after another.  Outputs per
 * cell: the primitives and conserved left in the reference's arrays, the
 * return value, which attempt succeeded (the index of the global counter
 * slot it incremented: 0 RAD energy lab, 13 RAD energy fluid frame, 2 MHD
 * energy lab, 14 MHD energy fluid frame, 4 RAD entropy, 6 MHD entropy; -1
 * when all failed) and the Newton iterations of the successful attempt. */
int kref_rad_implicit(int n, const double *uu, const double *pp, const double *g20, const double *G20,
                      const double *dtc, double *pp_out, double *uu_out, int *status, int *which, int *iters)
{
  int k, s, iv;
  if (n > NX * NY) return -1;
  for (k = 0; k < n; k++) {
    int ix = k % NX, iy = k / NX;
    int before[NGLOBALINTSLOT];
    ldouble deltas[5];
    kref_rad_load(k, uu, pp, g20, G20);
    for (s = 0; s < NGLOBALINTSLOT; s++) before[s] = global_int_slot[s];
    status[k] = solve_implicit_lab(ix, iy, 0, dtc[k], deltas, 0);
    which[k] = -1;
    iters[k] = 0;
    const int succ[6] = {GLOBALINTSLOT_NIMPENERRAD, GLOBALINTSLOT_NIMPENERRADFF, GLOBALINTSLOT_NIMPENERMHD,
                         GLOBALINTSLOT_NIMPENERMHDFF, GLOBALINTSLOT_NIMPENTRRAD, GLOBALINTSLOT_NIMPENTRMHD};
    for (s = 0; s < 6; s++)
      if (global_int_slot[succ[s]] != before[succ[s]]) which[k] = succ[s];
    const int its[4] = {GLOBALINTSLOT_ITERIMPENERRAD, GLOBALINTSLOT_ITERIMPENERMHD, GLOBALINTSLOT_ITERIMPENTRRAD,
                        GLOBALINTSLOT_ITERIMPENTRMHD};
    for (s = 0; s < 4; s++) iters[k] += global_int_slot[its[s]] - before[its[s]];
    for (iv = 0; iv < NV; iv++) {
      pp_out[(long)k * NV + iv] = get_u(p, iv, ix, iy, 0);
      uu_out[(long)k * NV + iv] = get_u(u, iv, ix, iy, 0);
    }
  }
  return 0;
}

/* u2p_rad (u2prad.c:485) on n cells with their own metric points. */
int kref_rad_u2p(int n, const double *uu, double *pp, const double *g20, const double *G20, int *status, int *corr)
{
  int k;
  for (k = 0; k < n; k++) {
    struct geometry geom;
    int c[3] = {0, 0, 0};
    kref_geom_from(g20 + 20 * k, G20 + 20 * k, &geom);
    status[k] = u2p_rad((double *)uu + (long)k * NV, pp + (long)k * NV, &geom, c);
    corr[k] = c[0];
  }
  return 0;
}

/* The reference's own u2p (u2p.c:176, type 0) on n cells with their own
 * metric points, with all its outputs: status, corrected[3], fixups[2] per
 * cell. */
int kref_u2p_full(int n, const double *uu, double *pp, const double *g20, const double *G20, int *status,
                  int *corrected, int *fixups)
{
  int k;
  for (k = 0; k < n; k++) {
    struct geometry geom;
    kref_geom_from(g20 + 20 * k, G20 + 20 * k, &geom);
    status[k] = u2p((double *)uu + (long)k * NV, pp + (long)k * NV, &geom, corrected + 3 * k, fixups + 2 * k, 0);
  }
  return 0;
}

/* The same solves for CPU timing: all cells loaded first, then solved in an
 * OpenMP loop when the build has OpenMP (the reference's counters are then
 * updated without synchronisation, as in its own parallel loops). */
int kref_rad_implicit_timed(int n, const double *uu, const double *pp, const double *g20, const double *G20,
                            const double *dtc, int *status)
{
  int k;
  if (n > NX * NY) return -1;
  for (k = 0; k < n; k++) kref_rad_load(k, uu, pp, g20, G20);
#pragma omp parallel for schedule(dynamic, 16)
  for (k = 0; k < n; k++) {
    ldouble deltas[5];
    status[k] = solve_implicit_lab(k % NX, k / NX, 0, dtc[k], deltas, 0);
  }
  return 0;
}
#endif
