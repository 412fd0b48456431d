/* Initial state of the magnetised Fishbone-Moncrief torus, executed by
 * set_initial_profile() (problem.c:55-69) for every domain cell.  Primitives
 * are built in Boyer-Lindquist coordinates and transformed to MKS2 with the
 * reference's own trans_pmhd_coco(); the azimuthal vector potential is put
 * into the B3 slot for calc_BfromA() (VECPOTGIVEN, magn.c:380-470).  With
 * radiation the pressure of the torus is shared with radiation in thermal
 * equilibrium; the atmosphere gets radiation of TORUS_ERADATM times its
 * gas energy. */
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
  int fm_intorus = fm_lnh > 0. && fm_r >= TORUS_RIN;

  if (fm_intorus) {
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
    /* the MHD primitives alone: in a RADIATION build trans_pall_coco's
     * radiation step starts by copying all NV input values to the output
     * (trans_prad_coco, frames.c), which would put the untransformed BL
     * velocities back; the radiation is set after the transformation */
    trans_pmhd_coco(fm_pbl, fm_pp, KERRCOORDS, MYCOORDS, fm_xxBL, &fm_geomBL, &fm_geom);
    fm_pp[B1] = 0.;
    fm_pp[B2] = 0.;
    fm_pp[B3] = my_max(fm_rho - 0.2, 0.);   /* A_phi in MKS2, rho_max = 1 */
  }
#ifdef RADIATION
  /* local thermal equilibrium: the temperature T at which gas and radiation
   * together carry the pressure p of the torus, b T + a T^4 = p, by Newton
   * steps from the smaller of the one-component solutions (the root lies
   * below both and the function is convex, so the steps fall monotonically);
   * the radiation frame moves with the gas */
  if (fm_intorus || TORUS_ERADATM < 0.) {
    ldouble fm_P = GAMMAM1 * fm_pp[UU];
    ldouble fm_aa = 4. * SIGMA_RAD / 3., fm_bb = K_BOLTZ * fm_pp[RHO] / MU_GAS / M_PROTON;
    ldouble fm_T = my_min(fm_P / fm_bb, sqrt(sqrt(fm_P / fm_aa)));
    int fm_it;
    for (fm_it = 0; fm_it < 100; fm_it++)
      fm_T -= (fm_bb * fm_T + fm_aa * fm_T * fm_T * fm_T * fm_T - fm_P) / (fm_bb + 4. * fm_aa * fm_T * fm_T * fm_T);
    fm_pp[UU] = calc_PEQ_ufromTrho(fm_T, fm_pp[RHO]);
    fm_pp[EE0] = calc_LTE_EfromT(fm_T);
    fm_pp[FX0] = fm_pp[VX];
    fm_pp[FY0] = fm_pp[VY];
    fm_pp[FZ0] = fm_pp[VZ];
  } else {
    /* the atmosphere keeps its gas energy and carries a faint radiation
     * field at rest with it */
    fm_pp[EE0] = TORUS_ERADATM * fm_pp[UU];
    fm_pp[FX0] = fm_pp[FY0] = fm_pp[FZ0] = 0.;
  }
#endif
  fm_pp[ENTR] = calc_Sfromu(fm_pp[RHO], fm_pp[UU]);
  p2u(fm_pp, fm_uu, &fm_geom);
  for (fm_iv = 0; fm_iv < NV; fm_iv++) {
    set_u(u, fm_iv, ix, iy, iz, fm_uu[fm_iv]);
    set_u(p, fm_iv, ix, iy, iz, fm_pp[fm_iv]);
  }
  for (fm_iv = 0; fm_iv < NFLAGS; fm_iv++)
    set_cflag(fm_iv, ix, iy, iz, 0);
}
