/* Helper routines of the torus plug-in (included into problem.c). */

/* Fishbone & Moncrief (1976) constant specific angular momentum of the
 * torus whose pressure maximum sits at r (Boyer-Lindquist, M = 1), from the
 * Keplerian circular orbit at r in a Kerr spacetime of spin a. */
ldouble fmtorus_lfish(ldouble a, ldouble r)
{
  ldouble sr = sqrt(r);
  ldouble x = r * r - 2. * a * sr + a * a;
  ldouble num = x * ((-2. * a * r * x) / sqrt(2. * a * sr + (-3. + r) * r) +
                     ((a + (-2. + r) * sr) * (r * r * r + a * a * (2. + r))) / sqrt(1. + (2. * a) / (r * sr) - 3. / r));
  ldouble den = r * r * r * sqrt(2. * a * sr + (-3. + r) * r) * (a * a + (-2. + r) * r);
  return num / den;
}

/* ln h of the FM torus at (r, theta), up to the constant fixed at r_in. */
ldouble fmtorus_lnh_raw(ldouble a, ldouble l, ldouble r, ldouble th)
{
  ldouble sth = sin(th), cth = cos(th);
  ldouble Sigma = r * r + a * a * cth * cth;
  ldouble Delta = r * r - 2. * r + a * a;
  ldouble A = (r * r + a * a) * (r * r + a * a) - Delta * a * a * sth * sth;
  ldouble q = sqrt(1. + 4. * l * l * Sigma * Sigma * Delta / (A * A * sth * sth));
  return 0.5 * log((1. + q) / (Sigma * Delta / A)) - 0.5 * q - 2. * a * r * l / A;
}

/* BL four-velocity u^phi of the torus fluid at (r, theta). */
ldouble fmtorus_uphi(ldouble a, ldouble l, ldouble r, ldouble th)
{
  ldouble sth = sin(th), cth = cos(th);
  ldouble Sigma = r * r + a * a * cth * cth;
  ldouble Delta = r * r - 2. * r + a * a;
  ldouble A = (r * r + a * a) * (r * r + a * a) - Delta * a * a * sth * sth;
  ldouble e2 = Sigma * Sigma * Delta / (A * A * sth * sth);
  ldouble up1 = sqrt((-1. + sqrt(1. + 4. * l * l * e2)) / 2.);
  return 2. * a * r * sqrt(1. + up1 * up1) / sqrt(A * Sigma * Delta) + sqrt(Sigma / A) * up1 / sth;
}

/* uniform [0,1) deviate from a 64-bit mix of (seed, global cell index):
 * the same cell gets the same number on every machine */
ldouble fmtorus_noise(unsigned long long seed, unsigned long long idx)
{
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (idx + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (ldouble)(z >> 11) * (1.0 / 9007199254740992.0);
}
