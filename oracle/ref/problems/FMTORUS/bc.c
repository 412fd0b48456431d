/* Boundary conditions of the torus (calc_bc, problem.c:41-48), called by
 * set_bc_core() for every ghost cell of the six faces:
 *  - radial, both ends: copy of the nearest domain cell (outflow);
 *  - theta, both ends: reflection across the boundary with u^theta and B^theta
 *    (and the radiation frame's u^theta) reversed;
 *  - phi: periodic, conserved and primitives copied. */
{
  int bc_iv, bc_ix = ix, bc_iy = iy, bc_iz = iz;
  struct geometry bc_geom;
  if (ix >= NX || ix < 0) {
    bc_ix = ix < 0 ? 0 : NX - 1;
    for (bc_iv = 0; bc_iv < NV; bc_iv++) pp[bc_iv] = get_u(p, bc_iv, bc_ix, bc_iy, bc_iz);
    fill_geometry(ix, iy, iz, &bc_geom);
    p2u(pp, uu, &bc_geom);
    return 0;
  }
  if (iy < 0 || iy >= NY) {
    bc_iy = iy < 0 ? -iy - 1 : 2 * NY - iy - 1;
    for (bc_iv = 0; bc_iv < NV; bc_iv++) {
#ifdef RADIATION
      if (bc_iv == VY || bc_iv == B2 || bc_iv == FY0)
#else
      if (bc_iv == VY || bc_iv == B2)
#endif
        pp[bc_iv] = -get_u(p, bc_iv, bc_ix, bc_iy, bc_iz);
      else
        pp[bc_iv] = get_u(p, bc_iv, bc_ix, bc_iy, bc_iz);
    }
    fill_geometry(ix, iy, iz, &bc_geom);
    p2u(pp, uu, &bc_geom);
    return 0;
  }
  if (iz < 0) bc_iz = iz + NZ;
  if (iz > NZ - 1) bc_iz = iz - NZ;
  for (bc_iv = 0; bc_iv < NV; bc_iv++) {
    uu[bc_iv] = get_u(u, bc_iv, bc_ix, bc_iy, bc_iz);
    pp[bc_iv] = get_u(p, bc_iv, bc_ix, bc_iy, bc_iz);
  }
  return 0;
}
