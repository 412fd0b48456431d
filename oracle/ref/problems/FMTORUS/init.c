/* Initial state of the magnetised Fishbone-Moncrief torus, executed by
 * set_initial_profile() (problem.c:55-69) for every domain cell.  Primitives
 * are built in Boyer-Lindquist coordinates and transformed to MKS2 with the
 * reference's own trans_pall_coco(); the azimuthal vector potential is put
 * into the B3 slot for calc_BfromA() (VECPOTGIVEN, magn.c:380-470). */
{
  ldouble fm_pp[NV], fm_uu[NV], fm_xx[4], fm_xxBL[4];
  struct geometry fm_geom, fm_geomBL;
  int fm_iv;
  fill_geometry(ix, iy, iz, &fm_geom);
  fill_geometry_arb(ix, iy, iz, &fm_geomBL, KERRCOORDS);
  get_xx(ix, iy, iz, fm_xx);
  coco_N(fm_xx, fm_xxBL, MYCOORDS, BLCOORDS);
  ldouble fm_r = fm_xxBL[1], fm_th = fm_xxBL[2];
  ldouble fm_a = BHSPIN;
  ldouble fm_l = fmtorus_lfish(fm_a, TORUS_RMAX);
  ldouble fm_lnh = fmtorus_lnh_raw(fm_a, fm_l, fm_r, fm_th) - fmtorus_lnh_raw(fm_a, fm_l, TORUS_RIN, M_PI / 2.);
  /* normalisation of the density maximum: h at (r_max, pi/2) */
  ldouble fm_lnhmax = fmtorus_lnh_raw(fm_a, fm_l, TORUS_RMAX, M_PI / 2.) - fmtorus_lnh_raw(fm_a, fm_l, TORUS_RIN, M_PI / 2.);
  ldouble fm_rhomax = pow((exp(fm_lnhmax) - 1.) * (GAMMA - 1.) / (TORUS_KAPPA * GAMMA), 1. / (GAMMA - 1.));

  /* atmosphere: normal observer, rho = 1e-4 r^-1.5, u = 1e-6 r^-2.5 */
  ldouble fm_rhoatm = ATM_RHO0 * pow(fm_r, -1.5);
  ldouble fm_uuatm = ATM_UU0 * pow(fm_r, -2.5);
  fm_pp[RHO] = fm_rhoatm;
  fm_pp[UU] = fm_uuatm;
  fm_pp[VX] = fm_pp[VY] = fm_pp[VZ] = 0.;
  fm_pp[B1] = fm_pp[B2] = fm_pp[B3] = 0.;

  if (fm_lnh > 0. && fm_r >= TORUS_RIN) {
    ldouble fm_h = exp(fm_lnh);
    ldouble fm_rho = pow((fm_h - 1.) * (GAMMA - 1.) / (TORUS_KAPPA * GAMMA), 1. / (GAMMA - 1.)) / fm_rhomax;
    ldouble fm_u = TORUS_KAPPA * pow(fm_rho * fm_rhomax, GAMMA) / (GAMMA - 1.) / fm_rhomax;
    int fm_gix, fm_giy, fm_giz;
    mpi_local2globalidx(ix, iy, iz, &fm_gix, &fm_giy, &fm_giz);
    unsigned long long fm_idx = (unsigned long long)fm_gix + (unsigned long long)TNX * ((unsigned long long)fm_giy + (unsigned long long)TNY * (unsigned long long)fm_giz);
    fm_u *= 1. + TORUS_NOISE * (2. * fmtorus_noise(TORUS_SEED, fm_idx) - 1.);

    /* BL velocity of the torus fluid, then to MKS2 */
    ldouble fm_ucon[4] = {0., 0., 0., fmtorus_uphi(fm_a, fm_l, fm_r, fm_th)};
    conv_vels(fm_ucon, fm_ucon, VEL4, VELPRIM, fm_geomBL.gg, fm_geomBL.GG);
    ldouble fm_pbl[NV];
    for (fm_iv = 0; fm_iv < NV; fm_iv++) fm_pbl[fm_iv] = 0.;
    fm_pbl[RHO] = my_max(fm_rho, fm_rhoatm);
    fm_pbl[UU] = my_max(fm_u, fm_uuatm);
    fm_pbl[VX] = fm_ucon[1];
    fm_pbl[VY] = fm_ucon[2];
    fm_pbl[VZ] = fm_ucon[3];
    trans_pall_coco(fm_pbl, fm_pp, KERRCOORDS, MYCOORDS, fm_xxBL, &fm_geomBL, &fm_geom);
    fm_pp[B1] = 0.;
    fm_pp[B2] = 0.;
    fm_pp[B3] = my_max(fm_rho - 0.2, 0.);   /* A_phi in MKS2, rho_max = 1 */
  }
  fm_pp[ENTR] = calc_Sfromu(fm_pp[RHO], fm_pp[UU]);
  p2u(fm_pp, fm_uu, &fm_geom);
  for (fm_iv = 0; fm_iv < NV; fm_iv++) {
    set_u(u, fm_iv, ix, iy, iz, fm_uu[fm_iv]);
    set_u(p, fm_iv, ix, iy, iz, fm_pp[fm_iv]);
  }
  for (fm_iv = 0; fm_iv < NFLAGS; fm_iv++)
    set_cflag(fm_iv, ix, iy, iz, 0);
}
