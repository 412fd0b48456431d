/* Rescales the magnetic field so that max(pmag/pgas) over the domain is
 * TORUS_MAXBETA (beta_min = 1/TORUS_MAXBETA); included in main() after
 * calc_BfromA (ko.c:189-191). */
{
  int pi_ix, pi_iy, pi_iz, pi_iv;
  ldouble pi_maxbeta = 0.;
  for (pi_iz = 0; pi_iz < NZ; pi_iz++)
    for (pi_iy = 0; pi_iy < NY; pi_iy++)
      for (pi_ix = 0; pi_ix < NX; pi_ix++) {
        ldouble pi_pp[NV], pi_bcon[4], pi_bcov[4];
        struct geometry pi_geom;
        fill_geometry(pi_ix, pi_iy, pi_iz, &pi_geom);
        for (pi_iv = 0; pi_iv < NV; pi_iv++) pi_pp[pi_iv] = get_u(p, pi_iv, pi_ix, pi_iy, pi_iz);
        calc_bcon_prim(pi_pp, pi_bcon, &pi_geom);
        indices_21(pi_bcon, pi_bcov, pi_geom.gg);
        ldouble pi_pmag = dot(pi_bcon, pi_bcov) / 2.;
        ldouble pi_pgas = GAMMAM1 * pi_pp[UU];
        if (pi_pmag / pi_pgas > pi_maxbeta) pi_maxbeta = pi_pmag / pi_pgas;
      }
  ldouble pi_fac = sqrt(TORUS_MAXBETA / pi_maxbeta);
  for (pi_iz = 0; pi_iz < NZ; pi_iz++)
    for (pi_iy = 0; pi_iy < NY; pi_iy++)
      for (pi_ix = 0; pi_ix < NX; pi_ix++) {
        ldouble pi_pp[NV], pi_uu[NV];
        struct geometry pi_geom;
        fill_geometry(pi_ix, pi_iy, pi_iz, &pi_geom);
        for (pi_iv = 0; pi_iv < NV; pi_iv++) pi_pp[pi_iv] = get_u(p, pi_iv, pi_ix, pi_iy, pi_iz);
        pi_pp[B1] *= pi_fac;
        pi_pp[B2] *= pi_fac;
        pi_pp[B3] *= pi_fac;
        p2u(pi_pp, pi_uu, &pi_geom);
        for (pi_iv = 0; pi_iv < NV; pi_iv++) {
          set_u(p, pi_iv, pi_ix, pi_iy, pi_iz, pi_pp[pi_iv]);
          set_u(u, pi_iv, pi_ix, pi_iy, pi_iz, pi_uu[pi_iv]);
        }
      }
  mpi_exchangedata();
  calc_avgs_throughout();
  set_bc(0., 1);
}
