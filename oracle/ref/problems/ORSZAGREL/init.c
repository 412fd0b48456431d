/* Initial state of the relativistic Orszag-Tang vortex, executed by
 * set_initial_profile() (problem.c:55-69) for every domain cell (ix,iy,iz).
 * rho = 25/(36 pi), p = 5/(12 pi) (u = p/(Gamma-1)),
 * coordinate three-velocity v = 0.5 (-sin y, sin x, 0) converted to the
 * relative four-velocity primitive, B = (-sin y, sin 2x, 0)/sqrt(4 pi) set
 * directly at cell centres. */
{
  ldouble ot_pp[NV], ot_uu[NV], ot_v[4];
  struct geometry ot_geom;
  int ot_iv;
  fill_geometry(ix, iy, iz, &ot_geom);

  ot_v[0] = 0.;
  ot_v[1] = -0.5 * sin(ot_geom.yy);
  ot_v[2] = 0.5 * sin(ot_geom.xx);
  ot_v[3] = 0.;
  conv_vels(ot_v, ot_v, VEL3, VELR, ot_geom.gg, ot_geom.GG);

  ot_pp[RHO] = 25. / (36. * M_PI);
  ot_pp[UU] = (5. / (12. * M_PI)) / GAMMAM1;
  ot_pp[VX] = ot_v[1];
  ot_pp[VY] = ot_v[2];
  ot_pp[VZ] = ot_v[3];
  ot_pp[B1] = -sin(ot_geom.yy) / sqrt(4. * M_PI);
  ot_pp[B2] = sin(2. * ot_geom.xx) / sqrt(4. * M_PI);
  ot_pp[B3] = 0.;
  ot_pp[ENTR] = calc_Sfromu(ot_pp[RHO], ot_pp[UU]);

  p2u(ot_pp, ot_uu, &ot_geom);

  for (ot_iv = 0; ot_iv < NV; ot_iv++) {
    set_u(u, ot_iv, ix, iy, iz, ot_uu[ot_iv]);
    set_u(p, ot_iv, ix, iy, iz, ot_pp[ot_iv]);
  }
  for (ot_iv = 0; ot_iv < NFLAGS; ot_iv++)
    set_cflag(ot_iv, ix, iy, iz, 0);
}
