// Radiation physics of the per-cell implicit gas-radiation source solve:
// M1 closure (radiation stress tensor, conserved <-> primitives), the
// radiative four-force with Kramers-type absorption and electron
// scattering, the lab/fluid-frame residuals and the 4D Newton solver on
// hydro or radiation primitives, and the cascade of attempts KORAL tries per
// cell.  Host and device callable; the arithmetic follows the reference
// operation by operation (see the citations) so that results agree with it
// to rounding.
//
// State layout: 13 doubles per cell, the nine MHD variables followed by the
// radiation energy density in the radiation rest frame and the relative
// four-velocity of that frame (primitives), or R^t_t, R^t_i (conserved).
#pragma once

#include "kgpu_physics.cuh"

// Large routines of the implicit solve that are called from several places
// of its evaluation: out of line with -DKGPU_RAD_NOINLINE (one copy of each
// in the instruction stream), inlined by default.
#ifdef KGPU_RAD_NOINLINE
#define KG_RAD_CALL __noinline__
#else
#define KG_RAD_CALL
#endif

namespace kgpu {

constexpr int NVR = 13;
constexpr int EE0 = 9, FX0 = 10, FY0 = 11, FZ0 = 12;
constexpr double RAD_PI = 3.141592654;   // the reference's Pi (ko.h:47)

// which primitives the Newton iteration works on, which energy equation,
// which frame it is written in (rad.c:110-351)
enum ImpPrim { IMP_RAD = 0, IMP_MHD = 1 };
enum ImpEq { IMP_ENERGY = 0, IMP_ENTROPY = 1 };
enum ImpFrame { IMP_LAB = 0, IMP_FF = 1 };

// Constants and solver controls, in code units (kgpu_rad_params in the
// public header gives the meaning of each field).
struct RadParams {
  double gamma;
  double kb, mp, sigma, mu;          // K_BOLTZ, M_PROTON, SIGMA_RAD, MU_GAS
  double ggg, ccc, masscm;           // unit conversion of the opacity law
  double kramers, kes;               // opacity coefficients (cgs)
  double kes_gu;                     // kes in code units, folded as the reference's compiler does
  double gammamaxrad, eradfloor, gammasmalllimit, numepsilon;
  double eps, conv, entrconv, maxiter;
  double dampfac, maxdown, maxup, maxdamping, threshold;
  double u2pconv;
  double eerhoratiomin, eerhoratiomax, eeuuratiomin, eeuuratiomax;
};

struct RadGeom {
  Geom g;
  double alpha;   // sqrt(-1/g^tt), as fill_geometry sets it (metric.c:1661)
};

KG_HD void rad_geom(const double *g20, const double *G20, RadGeom &r) {
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 5; b++) {
      r.g.gg[a][b] = g20[a * 5 + b];
      r.g.GG[a][b] = G20[a * 5 + b];
    }
  r.g.gdet = r.g.gg[3][4];
  r.g.gttpert = r.g.GG[3][4];
  r.alpha = sqrt(-1. / r.g.GG[0][0]);
}

// ---------------------------------------------------------------------------
// gas temperature and opacities (physics.c:984-989, rad.c:11-37 with the
// Kramers + electron-scattering law of the radiating-cells problem)
// ---------------------------------------------------------------------------
KG_HD double peq_T_from_urho(const RadParams &R, double u, double rho) {
  double p = u * (R.gamma - 1.);
  return p / (R.kb * rho / R.mu / R.mp);
}
KG_HD double rad_kappa_abs(const RadParams &R, const double *pp) {
  double rho = pp[RHO];
  double T = peq_T_from_urho(R, pp[UU], pp[RHO]);
  double rhocgs = rho / R.ggg * R.ccc * R.ccc / R.masscm / R.masscm;
  return R.kramers * rhocgs * pow(T, -3.5) / R.ggg * R.ccc * R.ccc / R.masscm * rho;
}
KG_HD double rad_kappa_es(const RadParams &R, const double *pp) { return R.kes_gu * pp[RHO]; }

// ---------------------------------------------------------------------------
// M1 stress tensor and radiation conserved variables (rad.c:1943-1975,
// p2u.c:253-298)
// ---------------------------------------------------------------------------
KG_HD void rad_urf4(const double *pp, const Geom &g, double urf[4]) {
  double u1[4] = {0., pp[FX0], pp[FY0], pp[FZ0]}, ucov[4];
  velr_to_vel4(u1, urf, ucov, g);
}
KG_HD void calc_Rij_M1(const double *pp, const Geom &g, double Rij[4][4]) {
  double Erf = pp[EE0];
  double urf[4];
  rad_urf4(pp, g, urf);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) Rij[i][j] = 4. / 3. * Erf * urf[i] * urf[j] + 1. / 3. * Erf * g.GG[i][j];
}
KG_HD void p2u_rad(const double *pp, double *uu, const Geom &g) {
  double Erf = pp[EE0];
  double urf[4];
  rad_urf4(pp, g, urf);
  double Rt[4];
  Rt[0] = 4. / 3. * Erf * urf[0] * urf[0] + 1. / 3. * Erf * g.GG[0][0];
  Rt[1] = 4. / 3. * Erf * urf[0] * urf[1] + 1. / 3. * Erf * g.GG[0][1];
  Rt[2] = 4. / 3. * Erf * urf[0] * urf[2] + 1. / 3. * Erf * g.GG[0][2];
  Rt[3] = 4. / 3. * Erf * urf[0] * urf[3] + 1. / 3. * Erf * g.GG[0][3];
  lower(Rt, Rt, g.gg);
  const double gdetu = g.gdet;
  uu[EE0] = gdetu * Rt[0];
  uu[FX0] = gdetu * Rt[1];
  uu[FY0] = gdetu * Rt[2];
  uu[FZ0] = gdetu * Rt[3];
}
// p2u for the full 13-variable state (p2u.c:40-48)
KG_RAD_CALL KG_HD void p2u_rad_full(const Grid &G, const double *pp, double *uu, const Geom &g) {
  p2u_full(G, pp, uu, g);
  p2u_rad(pp, uu, g);
}

// fluid-frame radiation energy density -R^t_t and the gas four-velocity
// (calc_ff_Rtt, rad.c:2833-2860)
KG_RAD_CALL KG_HD void calc_ff_Rtt(const double *pp, const Geom &g, double &Rtt, double ucon[4]) {
  double ut[4] = {0., pp[VX], pp[VY], pp[VZ]}, ucov[4];
  velr_to_vel4(ut, ucon, ucov, g);
  double Rij[4][4], Rl[4][4];
  calc_Rij_M1(pp, g, Rij);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.;
      for (int k = 0; k < 4; k++) s += Rij[i][k] * g.gg[k][j];
      Rl[i][j] = s;
    }
  double r = 0.;
  for (int i1 = 0; i1 < 4; i1++)
    for (int i2 = 0; i2 < 4; i2++) r += -Rl[i1][i2] * ucon[i2] * ucov[i1];
  Rtt = r;
}

// Lorentz boost lab -> fluid frame of a contravariant vector, made
// orthonormal by the lapse (calc_Lorentz_lab2ff frames.c:393-437,
// boost2_lab2ff 807-850)
KG_HD void boost2_lab2ff(double A[4], const double *pp, const Geom &g) {
  double ut[4] = {0., pp[2], pp[3], pp[4]}, ucon[4], ucov[4];
  velr_to_vel4(ut, ucon, ucov, g);
  double alpha = sqrt(-1. / g.GG[0][0]);
  double wcov[4] = {-alpha, 0., 0., 0.}, wcon[4];
  raise(wcov, wcon, g.GG);
  double Om[4][4];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) Om[i][j] = ucon[i] * wcov[j] - wcon[i] * ucov[j];
  double gam = -dot4(wcon, ucov);
  double L[4][4];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double Omsum = 0.;
      for (int k = 0; k < 4; k++) Omsum += Om[i][k] * Om[k][j];
      L[i][j] = (i == j ? 1. : 0.) + 1. / (1. + gam) * Omsum + Om[i][j];
    }
  double At[4] = {A[0], A[1], A[2], A[3]};
  for (int i = 0; i < 4; i++) {
    double s = 0.;
    for (int k = 0; k < 4; k++) s += L[i][k] * At[k];
    A[i] = s;
  }
  double alpha2 = sqrt(-1. / g.GG[0][0]);
  for (int i = 0; i < 4; i++) A[i] *= alpha2;
}

// radiative four-force G^mu, lab frame (labframe = 1) or fluid frame with
// the time component rewritten (calc_Gi, rad.c:1787-1888; no Comptonisation)
KG_RAD_CALL KG_HD void calc_Gi(const RadParams &R, const double *pp, const Geom &g, double Gi[4], int labframe) {
  double Rij[4][4];
  calc_Rij_M1(pp, g, Rij);
  double ut[4] = {0., pp[2], pp[3], pp[4]}, ucon[4], ucov[4];
  velr_to_vel4(ut, ucon, ucov, g);
  double rho = pp[RHO];
  double u = pp[1];
  double p = (R.gamma - 1.) * u;
  double Tgas = p * R.mu * R.mp / R.kb / rho;
  double B = R.sigma * pw4(Tgas) / RAD_PI;
  double kappa = rad_kappa_abs(R, pp);
  double kappaes = rad_kappa_es(R, pp);
  double Ruu = 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) Ruu += Rij[i][j] * ucov[i] * ucov[j];
  double Ehatrad = Ruu;
  for (int i = 0; i < 4; i++) {
    double Ru = 0.;
    for (int j = 0; j < 4; j++) Ru += Rij[i][j] * ucov[j];
    Gi[i] = -(kappa + kappaes) * Ru - (kappaes * Ruu + kappa * 4. * RAD_PI * B) * ucon[i];
  }
  if (labframe == 0) {
    boost2_lab2ff(Gi, pp, g);
    Gi[0] = -kappa * 4. * RAD_PI * B + kappa * Ehatrad;
  }
}

// ---------------------------------------------------------------------------
// M1 closure: radiation conserved -> primitives (u2prad.c:9-411, 485-520).
// The closed forms are the reference's (generated by computer algebra);
// they are kept term for term so that the rounding is the same.
// ---------------------------------------------------------------------------
// pow(x, 2.) of the closed forms: the product, which is the correctly
// rounded square (a general pow is not always; the host library's almost
// always is)
KG_HD double m1_pow2(double x) { return pw2(x); }

// lab-frame gamma^2 of the radiation frame from R_t_mu (u2prad.c:116-250)
KG_RAD_CALL KG_HD double m1_gammarel2(const RadParams &R, const RadGeom &rg, const double Avcov[4]) {
  const auto &GG = rg.g.GG;
  double gn11 = GG[0][0], gn12 = GG[0][1], gn13 = GG[0][2], gn14 = GG[0][3], gn22 = GG[1][1], gn23 = GG[1][2],
         gn24 = GG[1][3], gn33 = GG[2][2], gn34 = GG[2][3], gn44 = GG[3][3];
  double Rdtt = Avcov[0], Rdtx = Avcov[1], Rdty = Avcov[2], Rdtz = Avcov[3];
  // the discriminant and the denominator shared by both roots
  auto disc = [&]() {
    return sqrt(4. * m1_pow2(gn11) * m1_pow2(Rdtt) + m1_pow2(gn12 * Rdtx + gn13 * Rdty + gn14 * Rdtz) +
                gn11 * (8. * gn12 * Rdtt * Rdtx + 3. * gn22 * m1_pow2(Rdtx) + 8. * gn13 * Rdtt * Rdty +
                        6. * gn23 * Rdtx * Rdty + 3. * gn33 * m1_pow2(Rdty) + 8. * gn14 * Rdtt * Rdtz +
                        6. * gn24 * Rdtx * Rdtz + 6. * gn34 * Rdty * Rdtz + 3. * gn44 * m1_pow2(Rdtz)));
  };
  auto den = [&]() {
    return gn11 * m1_pow2(Rdtt) + 2. * gn12 * Rdtt * Rdtx + gn22 * m1_pow2(Rdtx) + 2. * gn13 * Rdtt * Rdty +
           2. * gn23 * Rdtx * Rdty + gn33 * m1_pow2(Rdty) + 2. * (gn14 * Rdtt + gn24 * Rdtx + gn34 * Rdty) * Rdtz +
           gn44 * m1_pow2(Rdtz);
  };
  double gamma2a =
      (-0.25 * (2. * m1_pow2(gn11) * m1_pow2(Rdtt) +
                (gn12 * Rdtx + gn13 * Rdty + gn14 * Rdtz) * (gn12 * Rdtx + gn13 * Rdty + gn14 * Rdtz + disc()) +
                gn11 * (4. * gn12 * Rdtt * Rdtx + gn22 * m1_pow2(Rdtx) + 2. * gn23 * Rdtx * Rdty +
                        gn33 * m1_pow2(Rdty) + 2. * gn24 * Rdtx * Rdtz + 2. * gn34 * Rdty * Rdtz +
                        gn44 * m1_pow2(Rdtz) + Rdtt * (4. * gn13 * Rdty + 4. * gn14 * Rdtz + disc())))) /
      den();
  double gamma2;
  if (gamma2a < R.gammasmalllimit || !isfinite(gamma2a)) {
    double gamma2b =
        (0.25 * (-2. * m1_pow2(gn11) * m1_pow2(Rdtt) -
                 1. * gn11 *
                     (4. * gn12 * Rdtt * Rdtx + gn22 * m1_pow2(Rdtx) +
                      Rdty * (4. * gn13 * Rdtt + 2. * gn23 * Rdtx + gn33 * Rdty) +
                      2. * (2. * gn14 * Rdtt + gn24 * Rdtx + gn34 * Rdty) * Rdtz + gn44 * m1_pow2(Rdtz)) +
                 gn11 * Rdtt * disc() +
                 (gn12 * Rdtx + gn13 * Rdty + gn14 * Rdtz) *
                     (-1. * gn12 * Rdtx - 1. * gn13 * Rdty - 1. * gn14 * Rdtz + disc()))) /
        den();
    gamma2 = gamma2b;
  } else {
    gamma2 = gamma2a;
  }
  double alpha = rg.alpha;
  double gammarel2 = gamma2 * alpha * alpha;
  if ((gammarel2 > R.gammasmalllimit && gammarel2 < 1.0)) gammarel2 = 1.0;
  return gammarel2;
}

// cold solution at a prescribed gamma^2 (u2prad.c:9-105): new R_t, R^t, Erf
// and the relative four-velocity
KG_RAD_CALL KG_HD void m1_cold(const RadGeom &rg, double Avcon[4], double Avcov[4], double gammarel2, double &Erf,
                   double urfconrel[4]) {
  const auto &GG = rg.g.GG;
  double alpha = rg.alpha;
  double gn11 = GG[0][0], gn12 = GG[0][1], gn13 = GG[0][2], gn14 = GG[0][3], gn22 = GG[1][1], gn23 = GG[1][2],
         gn24 = GG[1][3], gn33 = GG[2][2], gn34 = GG[2][3], gn44 = GG[3][3];
  double Rdtx = Avcov[1], Rdty = Avcov[2], Rdtz = Avcov[3];
  double utsq = gammarel2 / (alpha * alpha);
  double q = (m1_pow2(gn12) * m1_pow2(Rdtx) + 2. * gn12 * Rdtx * (gn13 * Rdty + gn14 * Rdtz) +
              m1_pow2(gn13 * Rdty + gn14 * Rdtz) -
              1. * gn11 *
                  (gn22 * m1_pow2(Rdtx) + 2. * gn23 * Rdtx * Rdty + gn33 * m1_pow2(Rdty) + 2. * gn24 * Rdtx * Rdtz +
                   2. * gn34 * Rdty * Rdtz + gn44 * m1_pow2(Rdtz))) *
             utsq * (gn11 + utsq) * m1_pow2(gn11 + 4. * utsq);
  Avcov[0] = (0.25 * (-4. * (gn12 * Rdtx + gn13 * Rdty + gn14 * Rdtz) * utsq * (gn11 + utsq) + sqrt(q))) /
             (gn11 * utsq * (gn11 + utsq));
  Erf = (0.75 * sqrt(q)) / (utsq * (gn11 + utsq) * (gn11 + 4. * utsq));
  raise(Avcov, Avcon, GG);
  double gammarel = sqrt(gammarel2);
  for (int jj = 1; jj < 4; jj++) {
    if (Erf > 0.0)
      urfconrel[jj] = alpha * (Avcon[jj] + 1. / 3. * Erf * GG[0][jj] * (4.0 * gammarel2 - 1.0)) /
                      (4. / 3. * Erf * gammarel);
    else
      urfconrel[jj] = 0.0;
  }
}

// u2p_rad (u2prad.c:485-520 with get_m1closure_* 116-411).  Returns 0 or -1;
// corrected = 1 when the closure fell back to a cold solution.
KG_RAD_CALL KG_HD int u2p_rad(const RadParams &R, const double *uu, double *pp, const RadGeom &rg, int &corrected) {
  corrected = 0;
  const auto &GG = rg.g.GG;
  const double gdetu = rg.g.gdet;
  double Avcov[4] = {uu[EE0] / gdetu, uu[FX0] / gdetu, uu[FY0] / gdetu, uu[FZ0] / gdetu};
  double Avcon[4];
  raise(Avcov, Avcon, GG);
  double gammarel2 = m1_gammarel2(R, rg, Avcov);
  double alpha = rg.alpha;
  double Erf = 3. * Avcon[0] * alpha * alpha / (4. * gammarel2 - 1.0);
  double urf[4] = {0., 0., 0., 0.};
  const double gammamax = R.gammamaxrad;
  bool nonfailure = gammarel2 >= 1.0 && Erf > R.eradfloor &&
                    gammarel2 <= gammamax * gammamax / R.gammasmalllimit / R.gammasmalllimit;
  if (nonfailure) {
    double gammarel = sqrt(gammarel2);
    for (int ii = 0; ii < 4; ii++)
      urf[ii] = alpha * (Avcon[ii] + 1. / 3. * Erf * GG[0][ii] * (4.0 * gammarel2 - 1.0)) / (4. / 3. * Erf * gammarel);
  } else {
    double gs2 = pow(1.0 + 10.0 * R.numepsilon, 2.0);
    double cs[4], ks[4], us[4] = {0., 0., 0., 0.}, Es;
    double cf[4], kf[4], uf[4] = {0., 0., 0., 0.}, Ef;
    for (int j = 0; j < 4; j++) {
      cs[j] = cf[j] = Avcon[j];
      ks[j] = kf[j] = Avcov[j];
    }
    m1_cold(rg, cs, ks, gs2, Es, us);
    double gf2 = gammamax * gammamax;
    m1_cold(rg, cf, kf, gf2, Ef, uf);
    if (fabs(ks[0] - Avcov[0]) > fabs(kf[0] - Avcov[0])) {
      for (int j = 0; j < 4; j++) urf[j] = uf[j];
      gammarel2 = gf2;
      Erf = Ef;
    } else {
      for (int j = 0; j < 4; j++) urf[j] = us[j];
      gammarel2 = gs2;
      Erf = Es;
    }
    corrected = 1;
  }
  if (!isfinite(Erf) || !isfinite(gammarel2) || !isfinite(urf[1]) || !isfinite(urf[2]) || !isfinite(urf[3]))
    return -1;
  pp[EE0] = Erf;
  pp[FX0] = urf[1];
  pp[FY0] = urf[2];
  pp[FZ0] = urf[3];
  return 0;
}

// 4x4 inverse by cofactors (misc.c:500-602), the same products and sums in
// the same order; returns -1 on a NaN determinant or entry.
KG_RAD_CALL KG_HD int inverse_44(const double a[4][4], double ia[4][4]) {
  double s[16], d[16], t[12];
  for (int i = 0; i < 4; i++) {
    s[i] = a[i][0];
    s[i + 4] = a[i][1];
    s[i + 8] = a[i][2];
    s[i + 12] = a[i][3];
  }
  t[0] = s[10] * s[15]; t[1] = s[11] * s[14]; t[2] = s[9] * s[15];  t[3] = s[11] * s[13];
  t[4] = s[9] * s[14];  t[5] = s[10] * s[13]; t[6] = s[8] * s[15];  t[7] = s[11] * s[12];
  t[8] = s[8] * s[14];  t[9] = s[10] * s[12]; t[10] = s[8] * s[13]; t[11] = s[9] * s[12];
  d[0] = t[0] * s[5] + t[3] * s[6] + t[4] * s[7];   d[0] -= t[1] * s[5] + t[2] * s[6] + t[5] * s[7];
  d[1] = t[1] * s[4] + t[6] * s[6] + t[9] * s[7];   d[1] -= t[0] * s[4] + t[7] * s[6] + t[8] * s[7];
  d[2] = t[2] * s[4] + t[7] * s[5] + t[10] * s[7];  d[2] -= t[3] * s[4] + t[6] * s[5] + t[11] * s[7];
  d[3] = t[5] * s[4] + t[8] * s[5] + t[11] * s[6];  d[3] -= t[4] * s[4] + t[9] * s[5] + t[10] * s[6];
  d[4] = t[1] * s[1] + t[2] * s[2] + t[5] * s[3];   d[4] -= t[0] * s[1] + t[3] * s[2] + t[4] * s[3];
  d[5] = t[0] * s[0] + t[7] * s[2] + t[8] * s[3];   d[5] -= t[1] * s[0] + t[6] * s[2] + t[9] * s[3];
  d[6] = t[3] * s[0] + t[6] * s[1] + t[11] * s[3];  d[6] -= t[2] * s[0] + t[7] * s[1] + t[10] * s[3];
  d[7] = t[4] * s[0] + t[9] * s[1] + t[10] * s[2];  d[7] -= t[5] * s[0] + t[8] * s[1] + t[11] * s[2];
  t[0] = s[2] * s[7]; t[1] = s[3] * s[6]; t[2] = s[1] * s[7];  t[3] = s[3] * s[5];
  t[4] = s[1] * s[6]; t[5] = s[2] * s[5]; t[6] = s[0] * s[7];  t[7] = s[3] * s[4];
  t[8] = s[0] * s[6]; t[9] = s[2] * s[4]; t[10] = s[0] * s[5]; t[11] = s[1] * s[4];
  d[8] = t[0] * s[13] + t[3] * s[14] + t[4] * s[15];    d[8] -= t[1] * s[13] + t[2] * s[14] + t[5] * s[15];
  d[9] = t[1] * s[12] + t[6] * s[14] + t[9] * s[15];    d[9] -= t[0] * s[12] + t[7] * s[14] + t[8] * s[15];
  d[10] = t[2] * s[12] + t[7] * s[13] + t[10] * s[15];  d[10] -= t[3] * s[12] + t[6] * s[13] + t[11] * s[15];
  d[11] = t[5] * s[12] + t[8] * s[13] + t[11] * s[14];  d[11] -= t[4] * s[12] + t[9] * s[13] + t[10] * s[14];
  d[12] = t[2] * s[10] + t[5] * s[11] + t[1] * s[9];    d[12] -= t[4] * s[11] + t[0] * s[9] + t[3] * s[10];
  d[13] = t[8] * s[11] + t[0] * s[8] + t[7] * s[10];    d[13] -= t[6] * s[10] + t[9] * s[11] + t[1] * s[8];
  d[14] = t[6] * s[9] + t[11] * s[11] + t[3] * s[8];    d[14] -= t[10] * s[11] + t[2] * s[8] + t[7] * s[9];
  d[15] = t[10] * s[10] + t[4] * s[8] + t[9] * s[9];    d[15] -= t[8] * s[9] + t[11] * s[10] + t[5] * s[8];
  double det = s[0] * d[0] + s[1] * d[1] + s[2] * d[2] + s[3] * d[3];
  det = 1 / det;
  if (isnan(det)) return -1;
  for (int j = 0; j < 16; j++) d[j] *= det;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      ia[i][j] = d[i * 4 + j];
      if (isnan(ia[i][j])) return -1;
    }
  return 0;
}

// ---------------------------------------------------------------------------
// implicit gas-radiation coupling (rad.c:110-351, 376-1218, 1225-1570)
// ---------------------------------------------------------------------------
struct ImpParams {
  int prim, eq, frame;
};

// MHD u2p inside the residual: energy equation only (u2p_solver, u2p.c:1219)
// How the nested MHD inversion of an evaluation runs: by one lane alone,
// optionally with a cap on its W-function evaluations (a capped inversion
// that runs out returns U2P_OVER_CAP and the evaluation is repeated in the
// cooperative form), or by all 32 lanes of a warp on the same cell.
struct ImpInner {
  unsigned *stats;   // [0] Newton steps, [1] W-function evaluations, or null
  unsigned cap;      // 0: no cap
  bool warp;
  int warm_attempts; // attempts of the cascade run from the predicted iterate (1..6)
};

// inner: where and how the nested inversion runs (see ImpInner)
KG_RAD_CALL KG_HD int imp_u2p_hot(const RadParams &R, const double *uu, double *pp, const Geom &g, const ImpInner *inner = nullptr) {
  Grid G;
  G.gamma = R.gamma;
  G.u2pconv = R.u2pconv;
  G.nv = NVMAX;
  unsigned *st = inner ? inner->stats : nullptr;
#ifdef __CUDA_ARCH__
  if (inner && inner->warp) return u2p_solver_W_warp(G, uu, pp, g, 0, st, st ? st + 1 : nullptr);
#endif
  unsigned used = 0;
  const int r = u2p_solver_W(G, uu, pp, g, 0, st, &used, inner ? inner->cap : 0u);
  if (st) st[1] += used;
  return r;
}

KG_HD double rad_Sfromu(const RadParams &R, double rho, double u) { return calc_Sfromu(R.gamma, rho, u); }

// Conserved state that goes with the primitives pp when the other
// component takes the opposite change of energy-momentum, and the inversion
// of that other component (rad.c:140-198 and 883-960).  Returns u2p's
// verdict as the residual sees it: 0 or -1 usable, -2 failed; corr set
// when the M1 closure was corrected.
KG_HD int imp_counterpart(const RadParams &R, int prim, const double *uu0, double *pp, double *uu, const RadGeom &rg,
                          int &corr, const ImpInner *inner = nullptr) {
  Grid G;
  G.gamma = R.gamma;
  G.nv = NVMAX;
  p2u_rad_full(G, pp, uu, rg.g);
  uu[ENTR] = uu0[ENTR] - (uu[EE0] - uu0[EE0]);
  corr = 0;
  if (prim == IMP_RAD) {
    uu[RHO] = uu0[RHO];
    uu[1] = uu0[1] - (uu[EE0] - uu0[EE0]);
    uu[2] = uu0[2] - (uu[FX0] - uu0[FX0]);
    uu[3] = uu0[3] - (uu[FY0] - uu0[FY0]);
    uu[4] = uu0[4] - (uu[FZ0] - uu0[FZ0]);
    const int r = imp_u2p_hot(R, uu, pp, rg.g, inner);
    if (r == U2P_OVER_CAP) return r;
    return r < 0 ? -2 : 0;
  }
  uu[EE0] = uu0[EE0] - (uu[1] - uu0[1]);
  uu[FX0] = uu0[FX0] - (uu[2] - uu0[2]);
  uu[FY0] = uu0[FY0] - (uu[3] - uu0[3]);
  uu[FZ0] = uu0[FZ0] - (uu[4] - uu0[4]);
  return u2p_rad(R, uu, pp, rg, corr);
}

// density that follows the gas velocity when iterating MHD primitives
KG_HD void imp_rho_from_velocity(const double *uu0, double *pp, const Geom &g) {
  double ut[4] = {0., pp[2], pp[3], pp[4]}, ucon[4], ucov[4];
  velr_to_vel4(ut, ucon, ucov, g);
  pp[RHO] = (uu0[RHO]) / g.gdet / ucon[0];
}

// The part of every evaluation that precedes the residual (rad.c:130-198,
// 880-960): the density that follows the gas velocity when iterating MHD
// primitives, the entropy, the conserved state that goes with pp, and the
// inversion of the other component (which updates pp in place).
KG_HD int imp_prepare(const RadParams &R, const ImpParams &P, const double *uu0, double *pp, double *uu,
                      const RadGeom &rg, int &corr, const ImpInner *inner = nullptr) {
  if (P.prim == IMP_MHD) imp_rho_from_velocity(uu0, pp, rg.g);
  pp[ENTR] = rad_Sfromu(R, pp[RHO], pp[UU]);
  return imp_counterpart(R, P.prim, uu0, pp, uu, rg, corr, inner);
}

// residual f[4] and its relative size from a prepared state (the rest of
// f_implicit_lab_4dprim, rad.c:199-351).  Returns -1 on failure, 1 when the
// closure was corrected, else 0.
KG_RAD_CALL KG_HD int imp_residual(const RadParams &R, const ImpParams &P, double *pp, const double *uu, const double *uu0,
                       const double *pp00, double dt, const RadGeom &rg, int u2pret, int corr, double f[4],
                       double &err0) {
  const Geom &g = rg.g;
  const double gdetu = g.gdet;
  int ret = corr != 0 ? 1 : 0;
  if (u2pret < -1) return -1;
  double err[4] = {0., 0., 0., 0.};
  double Gi[4];
  calc_Gi(R, pp, g, Gi, 1);
  lower(Gi, Gi, g.gg);
  if (P.prim == IMP_MHD) {
    for (int k = 1; k < 4; k++) {
      f[k] = uu[k + 1] - uu0[k + 1] - dt * gdetu * Gi[k];
      if (fabs(f[k]) > SMALL)
        err[k] = fabs(f[k]) / (fabs(uu[k + 1]) + fabs(uu0[k + 1]) + fabs(dt * gdetu * Gi[k]));
      else
        err[k] = 0.;
    }
  } else {
    for (int k = 1; k < 4; k++) {
      f[k] = uu[EE0 + k] - uu0[EE0 + k] + dt * gdetu * Gi[k];
      if (fabs(f[k]) > SMALL)
        err[k] = fabs(f[k]) / (fabs(uu[EE0 + k]) + fabs(uu0[EE0 + k]) + fabs(dt * gdetu * Gi[k]));
      else
        err[k] = 0.;
    }
  }
  if (P.frame == IMP_LAB) {
    int iv;
    bool plus;
    if (P.prim == IMP_RAD) {
      iv = P.eq == IMP_ENERGY ? EE0 : ENTR;
      plus = true;
    } else {
      iv = P.eq == IMP_ENERGY ? UU : ENTR;
      plus = false;
    }
    if (plus) f[0] = uu[iv] - uu0[iv] + dt * gdetu * Gi[0];
    else f[0] = uu[iv] - uu0[iv] - dt * gdetu * Gi[0];
    if (fabs(f[0]) > SMALL)
      err[0] = fabs(f[0]) / (fabs(uu[iv]) + fabs(uu0[iv]) + fabs(dt * gdetu * Gi[0]));
    else
      err[0] = 0.;
  } else {
    double pp0[NVR];
    for (int i = 0; i < NVR; i++) pp0[i] = pp00[i];
    calc_Gi(R, pp, g, Gi, 0);
    double uconf[4], Rtt0, Rtt;
    calc_ff_Rtt(pp0, g, Rtt0, uconf);
    calc_ff_Rtt(pp, g, Rtt, uconf);
    double Ehat = -Rtt;
    double Ehat0 = -Rtt0;
    double dtau = dt / uconf[0];
    if (P.prim == IMP_RAD) {
      if (P.eq == IMP_ENERGY) {
        f[0] = Ehat - Ehat0 + dtau * Gi[0];
        err[0] = fabs(f[0]) / (fabs(Ehat) + fabs(Ehat0) + fabs(dtau * Gi[0]));
      } else {
        pp[ENTR] = rad_Sfromu(R, pp[RHO], pp[UU]);
        f[0] = pp[ENTR] - pp0[ENTR] - dtau * Gi[0];
        err[0] = fabs(f[0]) / (fabs(pp[ENTR]) + fabs(pp0[ENTR]) + fabs(dtau * Gi[0]));
      }
    } else {
      if (P.eq == IMP_ENERGY) {
        f[0] = pp[UU] - pp0[UU] - dtau * Gi[0];
        err[0] = fabs(f[0]) / (fabs(pp[UU]) + fabs(pp0[UU]) + fabs(dtau * Gi[0]));
      } else {
        pp0[ENTR] = rad_Sfromu(R, pp0[RHO], pp0[UU]);
        pp[ENTR] = rad_Sfromu(R, pp[RHO], pp[UU]);
        f[0] = pp[ENTR] - pp0[ENTR] - dtau * Gi[0];
        err[0] = fabs(f[0]) / (fabs(pp[ENTR]) + fabs(pp0[ENTR]) + fabs(dtau * Gi[0]));
      }
    }
  }
  if (!isfinite(f[0]) || !isfinite(f[1]) || !isfinite(f[2]) || !isfinite(f[3])) return -1;
  double e01 = err[0] > err[1] ? err[0] : err[1];
  double e23 = err[2] > err[3] ? err[2] : err[3];
  err0 = e01 > e23 ? e01 : e23;
  return ret;
}

// The attempts solve_implicit_lab makes (rad.c:1404-1505), in order.  The
// primitive set of attempts 0, 1, 4 is `startwith`, of 2, 3, 5 the other.
constexpr int IMP_NATTEMPTS = 6;
KG_HD ImpParams imp_attempt(int a, int startwith) {
  int other = startwith == IMP_RAD ? IMP_MHD : IMP_RAD;
  switch (a) {
    case 0: return ImpParams{startwith, IMP_ENERGY, IMP_LAB};
    case 1: return ImpParams{startwith, IMP_ENERGY, IMP_FF};
    case 2: return ImpParams{other, IMP_ENERGY, IMP_LAB};
    case 3: return ImpParams{other, IMP_ENERGY, IMP_FF};
    case 4: return ImpParams{startwith, IMP_ENTROPY, IMP_LAB};
    default: return ImpParams{other, IMP_ENTROPY, IMP_LAB};
  }
}

// which primitive set the cascade starts with (rad.c:1395-1397)
KG_HD int imp_startwith(const RadParams &R, const double *pp0, const Geom &g) {
  double ugas0[4], Rtt0;
  calc_ff_Rtt(pp0, g, Rtt0, ugas0);
  double Ehat = -Rtt0;
  return Ehat < R.threshold * pp0[UU] ? IMP_RAD : IMP_MHD;
}

// ---------------------------------------------------------------------------
// The cascade as a state machine that advances one evaluation at a time.
//
// solve_implicit_lab_4dprim (rad.c:376-1218) evaluates, per Newton
// iteration, the residual at the iterate (base), at four perturbed iterates
// (Jacobian columns, a column tried with the other sign after a failure),
// and the inversion of the other component at damped trial points until
// one is accepted; after convergence the final state is inverted once more.
// Written as nested loops, the threads of a warp sit in different loops
// and take turns.  Here every call of imp_advance performs exactly one of
// those evaluations — the preparation and inversion of the other component
// are common to all of them, the residual is added for base and Jacobian
// evaluations — and then moves the cell's state to the next one, so all
// lanes of a warp run the expensive part together whatever phase their cell
// is in.  The sequence of operations per cell is the reference's.
// ---------------------------------------------------------------------------
enum ImpPhase { PH_BASE = 0, PH_JAC = 1, PH_DAMP = 2, PH_FINAL = 3 };
enum ImpAdvance { IMP_RUNNING = 0, IMP_DONE_OK = 1, IMP_DONE_FAIL = 2, IMP_PAUSE = 3, IMP_OVER_CAP = 4 };

struct ImpState {
  double pp[NVR];      // the iterate
  double ppp[NVR];     // the iterate at the start of the iteration
  double f1[4];        // residual at ppp
  double J[4][4];      // Jacobian; its inverse once complete
  double xiapp;        // damping factor of the update
  double sign;         // side of the finite difference of column j
  int iter;            // Newton iterations of the running attempt
  int att, sw;         // running attempt (0..5), primitives the cascade starts with
  int phase, j;
  int warm;            // the first attempt runs from a predicted iterate
  unsigned evals;      // evaluations performed (statistics)
  unsigned inner[2];   // nested MHD inversions: Newton steps, W-function evaluations (statistics)
};

KG_HD void imp_begin(const RadParams &R, const double *pp00, const Geom &g, ImpState &s) {
  for (int i = 0; i < NVR; i++) s.pp[i] = pp00[i];
  s.iter = 0;
  s.att = 0;
  s.sw = imp_startwith(R, pp00, g);
  s.phase = PH_BASE;
  s.j = 0;
  s.sign = -1.;
  s.xiapp = 1.;
  s.warm = 0;
  s.evals = 0;
  s.inner[0] = s.inner[1] = 0;
}

// The attempt failed: the next one starts afresh, from the cell's guess, or
// from the predicted iterate while the learned warm start is on.  When the
// warm cascade has failed in every attempt, the reference cascade runs
// from the guess (the fallback), so a cell fails only where the reference
// fails.
// With a warm start the first warm_attempts attempts run from the predicted
// iterate; then the reference cascade runs from the reference guess.
KG_HD int imp_next_attempt(const double *pp00, const double *warm_guess, ImpState &s,
                           int warm_attempts = IMP_NATTEMPTS) {
  s.att++;
  if (s.warm && s.att >= warm_attempts) {
    s.warm = 0;
    s.att = 0;
  } else if (s.att >= IMP_NATTEMPTS) {
    return IMP_DONE_FAIL;
  }
  const double *start = s.warm ? warm_guess : pp00;
  for (int i = 0; i < NVR; i++) s.pp[i] = start[i];
  s.iter = 0;
  s.phase = PH_BASE;
  return IMP_RUNNING;
}

// Evaluations done ahead of the state machine: the base evaluation of a
// Newton iteration and its four Jacobian columns on either side depend only
// on the iterate at the start of the iteration, so other lanes of a warp can
// compute them together from the same inputs (imp_input) with the same code
// (imp_eval_entry).  imp_advance then takes the entry for its phase, column
// and side instead of evaluating, and counts it as the evaluation it
// replaces; entries the sequence does not reach are dropped.
struct ImpEval {
  double pin[NVR];   // the input after the evaluation (the other component inverted into it)
  double f[4];
  double err;
  int u2pret, corr, fret;
  unsigned inner[2];
};
constexpr int IMP_NCACHE = 9;   // [0] base, [1+j] column j at sign -1, [5+j] column j at sign +1
struct ImpCache {
  const ImpEval *e;
  unsigned valid;   // bit i: entry i present
};

// The input of an evaluation in phase PH_BASE or PH_JAC (column s.j on side
// s.sign), as imp_advance forms it.
KG_HD void imp_input(const RadParams &R, int sh, const ImpState &s, const RadGeom &rg, double *pin) {
  if (s.phase == PH_BASE) {
    for (int i = 0; i < NVR; i++) pin[i] = s.pp[i];
    return;
  }
  for (int i = 0; i < NVR; i++) pin[i] = s.ppp[i];
  const int j = s.j;
  double del;
  if (j == 0) {
    del = s.sign * R.eps * s.ppp[sh];
  } else {
    double x = s.ppp[j + sh];
    double sg = x > 0. ? 1. : (x < 0. ? -1. : (x == 0. ? 1. : 0.));
    double lim = 1.e-6 / sqrt(rg.g.gg[j][j]);
    double ax = fabs(x);
    double veleps = R.eps * sg * (lim > ax ? lim : ax);
    del = x >= 0. ? s.sign * veleps : -s.sign * veleps;
  }
  pin[j + sh] = s.ppp[j + sh] + del;
}

// Entry `slot` of the iteration that cell state s (in phase PH_BASE) is
// about to start.  With cap > 0 a nested inversion that passes cap
// W-function evaluations is abandoned and false returned: the entry is not
// valid, and the state machine evaluates it itself.
KG_HD bool imp_eval_entry(const RadParams &R, const double *uu0, const double *pp00, double dt, const RadGeom &rg,
                          const ImpState &s, int slot, ImpEval &e, unsigned cap = 0u) {
  const ImpParams P = imp_attempt(s.att, s.sw);
  const int sh = P.prim == IMP_MHD ? UU : EE0;
  ImpState t = s;
  for (int i = 0; i < NVR; i++) t.ppp[i] = t.pp[i];
  if (slot == 0) {
    t.phase = PH_BASE;
  } else {
    t.phase = PH_JAC;
    t.j = (slot - 1) & 3;
    t.sign = slot < 5 ? -1. : 1.;
  }
  imp_input(R, sh, t, rg, e.pin);
  double uu[NVR];
  e.inner[0] = e.inner[1] = 0;
  ImpInner in{e.inner, cap, false, IMP_NATTEMPTS};
  e.corr = 0;
  e.u2pret = imp_prepare(R, P, uu0, e.pin, uu, rg, e.corr, &in);
  if (e.u2pret == U2P_OVER_CAP) return false;
  for (int i = 0; i < 4; i++) e.f[i] = 0.;
  e.err = 0.;
  e.fret = imp_residual(R, P, e.pin, uu, uu0, pp00, dt, rg, e.u2pret, e.corr, e.f, e.err);
  return true;
}

// One evaluation and the transition that follows it.  `budget` counts the
// Newton iterations the cell may still start in this call sequence; at the
// start of an iteration with no budget left the cell pauses (IMP_PAUSE)
// with its state intact.
// `how` sets how the nested MHD inversion runs (ImpInner); when a capped
// inversion runs out the evaluation is abandoned with the state as before
// the call (IMP_OVER_CAP), to be repeated in the cooperative form.
KG_HD int imp_advance(const RadParams &R, const double *uu0, const double *pp00, double dt, const RadGeom &rg,
                      ImpState &s, int &budget, const double *warm_guess = nullptr, const ImpInner *how = nullptr,
                      const ImpCache *cache = nullptr) {
  const ImpParams P = imp_attempt(s.att, s.sw);
  const int sh = P.prim == IMP_MHD ? UU : EE0;
  const double CONV = P.eq == IMP_ENTROPY ? R.entrconv : R.conv;
  double pin[NVR], uu[NVR], f[4] = {0., 0., 0., 0.}, err = 0., xxx0 = 0.;
  // input of this evaluation
  if (s.phase == PH_BASE) {
    if (budget <= 0) return IMP_PAUSE;
    budget--;
    s.iter++;
    for (int i = 0; i < NVR; i++) s.ppp[i] = s.pp[i];
    imp_input(R, sh, s, rg, pin);
  } else if (s.phase == PH_JAC) {
    imp_input(R, sh, s, rg, pin);
  } else if (s.phase == PH_DAMP) {
    double xxx[4];
    for (int i = 0; i < 4; i++) xxx[i] = s.ppp[i + sh];
    for (int i = 0; i < 4; i++)
      for (int k = 0; k < 4; k++) xxx[i] -= s.xiapp * s.J[i][k] * s.f1[k];
    for (int i = 0; i < NVR; i++) pin[i] = s.pp[i];
    for (int i = 0; i < 4; i++) pin[i + sh] = xxx[i];
    xxx0 = xxx[0];
  } else {
    for (int i = 0; i < NVR; i++) pin[i] = s.pp[i];
  }
  // the evaluation: other component's inversion, residual where needed
  const int wa = how ? how->warm_attempts : IMP_NATTEMPTS;
  int slot = -1;
  if (cache && s.phase == PH_BASE) slot = 0;
  else if (cache && s.phase == PH_JAC) slot = (s.sign < 0. ? 1 : 5) + s.j;
  if (slot >= 0 && !((cache->valid >> slot) & 1u)) slot = -1;
  int corr = 0, u2pret, fret = 0;
  if (slot >= 0) {   // evaluated ahead from the same input
    const ImpEval &e = cache->e[slot];
    for (int i = 0; i < NVR; i++) pin[i] = e.pin[i];
    for (int i = 0; i < 4; i++) f[i] = e.f[i];
    err = e.err;
    u2pret = e.u2pret;
    corr = e.corr;
    fret = e.fret;
    s.inner[0] += e.inner[0];
    s.inner[1] += e.inner[1];
    s.evals++;
  } else {
    ImpInner in{s.inner, how ? how->cap : 0u, how ? how->warp : false, IMP_NATTEMPTS};
    u2pret = imp_prepare(R, P, uu0, pin, uu, rg, corr, &in);
    if (u2pret == U2P_OVER_CAP) {
      if (s.phase == PH_BASE) {   // undo the start of the iteration
        budget++;
        s.iter--;
      }
      return IMP_OVER_CAP;
    }
    s.evals++;
    if (s.phase == PH_BASE || s.phase == PH_JAC)
      fret = imp_residual(R, P, pin, uu, uu0, pp00, dt, rg, u2pret, corr, f, err);
  }
  // transition
  if (s.phase == PH_BASE) {
    if (fret < 0) return imp_next_attempt(pp00, warm_guess, s, wa);
    if (err < CONV) {
      if (s.iter > R.maxiter) return imp_next_attempt(pp00, warm_guess, s, wa);   // converged past the limit (rad.c:1051)
      s.phase = PH_FINAL;
      return IMP_RUNNING;
    }
    for (int i = 0; i < 4; i++) s.f1[i] = f[i];
    s.j = 0;
    s.sign = -1.;
    s.phase = PH_JAC;
    return IMP_RUNNING;
  }
  if (s.phase == PH_JAC) {
    const int j = s.j;
    if (fret < 0) {
      if (s.sign > 0.) return imp_next_attempt(pp00, warm_guess, s, wa);
      s.sign = 1.;
      return IMP_RUNNING;
    }
    for (int i = 0; i < 4; i++) s.J[i][j] = (f[i] - s.f1[i]) / (pin[j + sh] - s.ppp[j + sh]);
    s.j = j + 1;
    s.sign = -1.;
    if (s.j == 4) {
      double iJ[4][4];
      if (inverse_44(s.J, iJ) < 0) return imp_next_attempt(pp00, warm_guess, s, wa);
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) s.J[a][b] = iJ[a][b];
      s.xiapp = 1.;
      s.phase = PH_DAMP;
    }
    return IMP_RUNNING;
  }
  if (s.phase == PH_DAMP) {
    for (int i = 0; i < NVR; i++) s.pp[i] = pin[i];   // the trial and its inversion stay in the iterate
    if (P.prim == IMP_MHD && corr > 0) u2pret = -1;
    const double edenmin = s.ppp[sh] / R.maxdown;
    const double edenmax = s.ppp[sh] * R.maxup;
    if (xxx0 > edenmin && xxx0 < edenmax && u2pret >= -1) {
      if (s.iter > R.maxiter) return imp_next_attempt(pp00, warm_guess, s, wa);
      s.phase = PH_BASE;
      return IMP_RUNNING;
    }
    if (xxx0 <= 0.) {
      s.xiapp *= s.ppp[sh] / (s.ppp[sh] + fabs(xxx0));
      s.xiapp *= 1.e-1;
    } else {
      s.xiapp /= R.dampfac;
    }
    if (s.xiapp < R.maxdamping) return imp_next_attempt(pp00, warm_guess, s, wa);
    return IMP_RUNNING;
  }
  // final inversion of the converged state (rad.c:1088-1150)
  for (int i = 0; i < NVR; i++) s.pp[i] = pin[i];
  if (P.prim == IMP_MHD && corr > 0) u2pret = -2;
  if (u2pret < -1) return imp_next_attempt(pp00, warm_guess, s, wa);
  return IMP_DONE_OK;
}

// ---------------------------------------------------------------------------
// M1 radiation inside the grid step: characteristic speeds, face fluxes,
// floors
// ---------------------------------------------------------------------------

// Lab-frame speeds of the radiative characteristics per direction
// (calc_rad_wavespeeds, rad.c:2451-2557, analytic branch): the rest-frame
// speed 1/sqrt(3), limited by the optical depth tautot of the cell when
// `limiter` is set, boosted with the HARM quadratic; co-going speeds zeroed
// as calc_wavespeeds_lr_pure does (physics.c:209-226).
KG_HD void rad_wavespeeds(const double *pp, const Geom &g, const double tautot[3], bool limiter, double al[3],
                          double ar[3]) {
  double urf[4];
  rad_urf4(pp, g, urf);
  const double rv2rad = 1. / 3.;
  for (int dim = 0; dim < 3; dim++) {
    double rv2 = rv2rad;
    if (limiter && tautot[dim] > 0.) {
      double rv2tau = 4. / 3. / tautot[dim] * 4. / 3. / tautot[dim];
      rv2 = dmin(rv2rad, rv2tau);
    }
    double Acov[4] = {0., 0., 0., 0.}, Acon[4], Bcov[4] = {1., 0., 0., 0.}, Bcon[4];
    Acov[dim + 1] = 1.;
    raise(Acov, Acon, g.GG);
    raise(Bcov, Bcon, g.GG);
    double Asq = dot4(Acon, Acov);
    double Bsq = dot4(Bcon, Bcov);
    double Au = dot4(Acov, urf);
    double Bu = dot4(Bcov, urf);
    double AB = dot4(Acon, Bcov);
    double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
    double wspeed2 = rv2;
    double B = 2. * (AuBu * (1.0 - wspeed2) - AB * wspeed2);
    double A = Bu2 * (1.0 - wspeed2) - Bsq * wspeed2;
    double discr = 4.0 * wspeed2 *
                   ((AB * AB - Asq * Bsq) * wspeed2 + (2.0 * AB * Au * Bu - Asq * Bu2 - Bsq * Au2) * (wspeed2 - 1.0));
    if (discr < 0.) discr = 0.;
    discr = sqrt(discr);
    double cst1 = -(-B + discr) / (2. * A);
    double cst2 = -(-B - discr) / (2. * A);
    double l = dmin(cst1, cst2), r = dmax(cst1, cst2);
    al[dim] = l > 0. ? 0. : l;
    ar[dim] = r < 0. ? 0. : r;
  }
}

// Total opacity times the cell's proper size per direction (calc_tautot,
// rad.c:55-65, with the sizes of calc_wavespeeds_lr_pure, physics.c:180-184:
// the larger of this cell's and the next cell's).
KG_HD void rad_tautot(const RadParams &R, const double *pp, const Geom &g, const double size_lo[3],
                      const double size_hi[3], double tautot[3]) {
  double chi = rad_kappa_abs(R, pp) + rad_kappa_es(R, pp);
  for (int d = 0; d < 3; d++) {
    double sq = sqrt(g.gg[d + 1][d + 1]);
    tautot[d] = chi * dmax(size_lo[d] * sq, size_hi[d] * sq);
  }
}

// gdet R^{idim+1}_j, j = 0..3: the radiative fluxes through a face
// (f_flux_prime_rad, rad.c:3280-3330, with f_flux_prime_rad_total
// 3125-3160 and indices_2221 frames.c:1966-1993 restricted to one row)
KG_HD void rad_flux(const double *pp, int idim, const Geom &g, double ff[4]) {
  double urf[4];
  rad_urf4(pp, g, urf);
  const double Erf = pp[EE0];
  const int i = idim + 1;
  double Ri[4];
  for (int k = 0; k < 4; k++) Ri[k] = 4. / 3. * Erf * urf[i] * urf[k] + 1. / 3. * Erf * g.GG[i][k];
  for (int j = 0; j < 4; j++) {
    double s = 0.;
    for (int k = 0; k < 4; k++) s += Ri[k] * g.gg[k][j];
    ff[j] = g.gdet * s;
  }
}

// R^k_l of the cell (calc_Rij then indices_2221), for the metric source
KG_HD void rad_Rmixed(const double *pp, const Geom &g, double Rl[4][4]) {
  double Rij[4][4];
  calc_Rij_M1(pp, g, Rij);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.;
      for (int k = 0; k < 4; k++) s += Rij[i][k] * g.gg[k][j];
      Rl[i][j] = s;
    }
}

// check_floors_rad (u2prad.c:687-790; the magnetic-pressure branch is not
// compiled in a build with the magnetic field evolved): the radiation
// energy floor, then the fluid-frame radiation energy against density and
// gas energy.  Returns -1 when a floor acted.
KG_HD int check_floors_rad(const RadParams &R, double *pp, const Geom &g) {
  int ret = 0;
  double Rtt, ugas[4];
  calc_ff_Rtt(pp, g, Rtt, ugas);
  const double Ehat = -Rtt;
  const double Eratio = pp[EE0] / Ehat;
  if (pp[EE0] < R.eradfloor) {
    pp[EE0] = R.eradfloor;
    ret = -1;
  }
  if (Ehat < R.eerhoratiomin * pp[0]) {
    pp[EE0] = Eratio * R.eerhoratiomin * pp[0];
    ret = -1;
  }
  if (Ehat > R.eerhoratiomax * pp[0]) {
    pp[0] = 1. / R.eerhoratiomax * Ehat;
    ret = -1;
  }
  if (Ehat < R.eeuuratiomin * pp[1]) {
    pp[EE0] = Eratio * R.eeuuratiomin * pp[1];
    ret = -1;
  }
  if (Ehat > R.eeuuratiomax * pp[1]) {
    pp[1] = 1. / R.eeuuratiomax * Ehat;
    ret = -1;
  }
  return ret;
}

}  // namespace kgpu
