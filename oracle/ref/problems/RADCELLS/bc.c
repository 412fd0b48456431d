/* Ghost cells copy the nearest domain cell (only storage: no transport is
 * run in this problem). */
{
  int rc_iv, rc_ix = ix < 0 ? 0 : (ix >= NX ? NX - 1 : ix), rc_iy = iy < 0 ? 0 : (iy >= NY ? NY - 1 : iy);
  for (rc_iv = 0; rc_iv < NV; rc_iv++) {
    pp[rc_iv] = get_u(p, rc_iv, rc_ix, rc_iy, 0);
    uu[rc_iv] = get_u(u, rc_iv, rc_ix, rc_iy, 0);
  }
  return 0;
}
