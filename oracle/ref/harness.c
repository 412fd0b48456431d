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
