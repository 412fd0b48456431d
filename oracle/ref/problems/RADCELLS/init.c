/* Placeholder state (the harness overwrites every cell): gas at rest with
 * rho = 1, u = 0.1, a weak field and radiation in equipartition at rest. */
{
  ldouble rc_pp[NV], rc_uu[NV];
  struct geometry rc_geom;
  int rc_iv;
  fill_geometry(ix, iy, iz, &rc_geom);
  for (rc_iv = 0; rc_iv < NV; rc_iv++) rc_pp[rc_iv] = 0.;
  rc_pp[RHO] = 1.;
  rc_pp[UU] = 0.1;
  rc_pp[B1] = 1.e-3;
  rc_pp[EE0] = 0.1;
  rc_pp[ENTR] = calc_Sfromu(rc_pp[RHO], rc_pp[UU]);
  p2u(rc_pp, rc_uu, &rc_geom);
  for (rc_iv = 0; rc_iv < NV; rc_iv++) {
    set_u(u, rc_iv, ix, iy, iz, rc_uu[rc_iv]);
    set_u(p, rc_iv, ix, iy, iz, rc_pp[rc_iv]);
  }
}
