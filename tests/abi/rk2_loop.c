/* KORAL's RK2 time loop (ko.c:571-626) written against the C-ABI exactly
 * as a host code would call it, operator by operator, and compared bit for
 * bit with the same steps run by kgpu_rk2_steps (the fused device step).
 *
 * Two problems: the relativistic Orszag-Tang vortex (64x64, PPM + LLF,
 * periodic) and the magnetised Kerr torus with its device set-up (32x16x8,
 * MP5 + HLL, outflow / reflecting / periodic boundaries, density floor).
 * Prints one line per problem and returns 0 when every byte of u and p and
 * the next time step agree.
 *
 * Build: gcc -std=c99 -I include tests/abi/rk2_loop.c \
 *            -L koral_b200/_lib -lkoral_b200 -Wl,-rpath,<abs>/koral_b200/_lib */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "koral_b200.h"

#define CHECK(call)                                                              \
  do {                                                                           \
    int rc_ = (call);                                                            \
    if (rc_) {                                                                   \
      fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, kgpu_last_error());    \
      exit(2);                                                                   \
    }                                                                            \
  } while (0)

/* one time step: the body of ko.c:571-626 with KORAL's calls swapped for
 * the library's (count_entropy and the intensity updates are not on this
 * path) */
static void rk2_step(kgpu_ctx *kg, double *t) {
  double dt;
  CHECK(kgpu_begin_step(kg, &dt)); /* dt = 1/tstepdenmax, maxima reset (ko.c:399-425) */
  CHECK(kgpu_save_timesteps(kg));
  CHECK(kgpu_copyi_u(kg, 1., KGPU_ARR_U, KGPU_ARR_UT0));
  CHECK(kgpu_do_correct(kg));
  CHECK(kgpu_op_explicit(kg, *t, 0.5 * dt));
  CHECK(kgpu_calc_u2p(kg));
  CHECK(kgpu_op_implicit(kg, *t, 0.5 * dt));
  CHECK(kgpu_copyi_u(kg, 1., KGPU_ARR_U, KGPU_ARR_UT1));
  CHECK(kgpu_op_explicit(kg, *t, dt));
  CHECK(kgpu_calc_u2p(kg));
  CHECK(kgpu_op_implicit(kg, *t, dt));
  CHECK(kgpu_addi_u(kg, 1., KGPU_ARR_U, -1., KGPU_ARR_UT1, KGPU_ARR_UT2)); /* k2 in ut2 */
  CHECK(kgpu_addi_u(kg, 1., KGPU_ARR_UT0, 1., KGPU_ARR_UT2, KGPU_ARR_U));
  *t += dt;
}

static kgpu_ctx *make_ot(int n) {
  kgpu_config c;
  kgpu_ctx *kg;
  const double lo[3] = {0., 0., -1.}, hi[3] = {2. * 3.14159265358979323846, 2. * 3.14159265358979323846, 1.};
  CHECK(kgpu_default_config(&c, n, n, 1));
  c.ng = 3;
  c.int_order = KGPU_PPM;
  c.fluxmethod = KGPU_LAXF;
  c.gamma = 5. / 3.;
  c.tsteplim = 0.5;
  CHECK(kgpu_create(&c, &kg));
  CHECK(kgpu_set_uniform_grid(kg, lo, hi));
  CHECK(kgpu_set_minkowski_metric(kg));
  CHECK(kgpu_init_orszag_tang(kg));
  CHECK(kgpu_begin_run(kg));
  return kg;
}

static kgpu_ctx *make_torus(int nx, int ny, int nz, kgpu_config *cfg) {
  kgpu_torus_params tp;
  kgpu_ctx *kg;
  CHECK(kgpu_default_torus_params(&tp));
  CHECK(kgpu_default_config(cfg, nx, ny, nz));
  cfg->ng = 4;
  cfg->int_order = KGPU_MP5;
  cfg->fluxmethod = KGPU_HLL;
  cfg->axisym_metric = 1;
  cfg->bc[0] = KGPU_BC_OUTFLOW;
  cfg->bc[1] = KGPU_BC_REFLECT;
  cfg->bc[2] = KGPU_BC_PERIODIC_COPY;
  cfg->gamma = 13. / 9.;
  cfg->tsteplim = 0.5;
  cfg->uurhoratiomin = 1e-10;
  cfg->uurhoratiomax = 1e2;
  cfg->b2rhoratiomax = 100.;
  CHECK(kgpu_create(cfg, &kg));
  CHECK(kgpu_init_fm_torus(kg, &tp));
  return kg;
}

static size_t state_doubles(const kgpu_config *c) {
  const int sx = c->nx + 2 * c->ng, sy = c->ny > 1 ? c->ny + 2 * c->ng : 1, sz = c->nz > 1 ? c->nz + 2 * c->ng : 1;
  return (size_t)sx * sy * sz * c->nv;
}

/* the per-operator loop on a against kgpu_rk2_steps on b, same start */
static int compare(const char *name, kgpu_ctx *a, kgpu_ctx *b, const kgpu_config *cfg, int nsteps) {
  const size_t n = state_doubles(cfg);
  double *ua = malloc(n * 8), *pa = malloc(n * 8), *ub = malloc(n * 8), *pb = malloc(n * 8);
  double t = 0., ta, tb;
  int s, bad;
  if (!ua || !pa || !ub || !pb) return 1;
  CHECK(kgpu_download_state(a, ua, pa));
  CHECK(kgpu_upload_state(b, ua, pa));
  CHECK(kgpu_get_tstepdenmax(a, &ta));
  CHECK(kgpu_set_tstepdenmax(b, ta));
  for (s = 0; s < nsteps; s++) rk2_step(a, &t);
  CHECK(kgpu_rk2_steps(b, nsteps));
  /* The loop ends on addi_u, which (as in the reference) updates domain
   * cells only: the ghost cells of u keep the values of the last set_bc
   * until the next op_explicit applies the boundary conditions first.  The
   * fused step applies them right after its combination.  Compare after
   * the set_bc that the next operator would run. */
  CHECK(kgpu_set_bc(a, t, 0));
  CHECK(kgpu_set_bc(b, t, 0));
  CHECK(kgpu_download_state(a, ua, pa));
  CHECK(kgpu_download_state(b, ub, pb));
  CHECK(kgpu_get_tstepdenmax(a, &ta));
  CHECK(kgpu_get_tstepdenmax(b, &tb));
  bad = memcmp(ua, ub, n * 8) != 0 || memcmp(pa, pb, n * 8) != 0 || memcmp(&ta, &tb, 8) != 0;
  printf("%s: %d RK2 steps operator by operator %s kgpu_rk2_steps (t = %.17g, 1/dt = %.17g)\n", name, nsteps,
         bad ? "DIFFER from" : "are bit-identical to", t, ta);
  free(ua); free(pa); free(ub); free(pb);
  return bad;
}

int main(void) {
  int bad = 0;
  kgpu_config cot, ctor;
  kgpu_ctx *a = make_ot(64), *b = make_ot(64);
  CHECK(kgpu_default_config(&cot, 64, 64, 1));
  cot.ng = 3;
  bad |= compare("Orszag-Tang 64x64", a, b, &cot, 10);
  kgpu_destroy(a);
  kgpu_destroy(b);
  a = make_torus(32, 16, 8, &ctor);
  b = make_torus(32, 16, 8, &ctor);
  bad |= compare("Kerr torus 32x16x8", a, b, &ctor, 10);
  kgpu_destroy(a);
  kgpu_destroy(b);
  return bad;
}
