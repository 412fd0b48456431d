// Learned warm start of the implicit radiation source solve: the network's
// inputs (16 features of a cell's state before the solve) and outputs (5
// numbers from which the initial iterate is built), host and device
// callable.
//
// Features (each brought to order one):
//   0  log10 rho / 4 + 1           1  log10(u_gas / rho) / 4
//   2  log10(E_rad / rho) / 6      3-5  gas relative 4-velocity x sqrt(g_ii), asinh
//   6-8  radiation-frame relative 4-velocity x sqrt(g_ii), asinh
//   9  log10(kappa_abs dt) / 5     10  log10(kappa_es dt) / 5
//   11 lapse                       12  g_tt + 1
//   13 log10 sqrt(g_33) / 2        14  1 when the cascade starts on gas primitives, else 0
//   15 log10(E_rad / u_gas) / 6
// Outputs 0-4, the change from the state before the solve to the converged
// one:
//   0  ln(u_gas' / u_gas)          1  ln(E_rad' / E_rad)
//   2-4  change of the velocity the first attempt iterates (the gas's when
//        it works on gas primitives, the radiation frame's otherwise),
//        x sqrt(g_ii)
// and two scores of how the cascade goes (trained on 0/1 targets):
//   5  the first attempt fails     6  the first two attempts fail
// Each output is standardised with a mean and a scale kept with the weights
// (the scores with mean 0 and scale 1).
#pragma once

#include "kgpu_rad.cuh"

namespace kgpu {

constexpr int MLP_IN = 16, MLP_H = 128, MLP_OUT = 7, MLP_OUTP = 8;
constexpr int MLP_NREG = 5;   // outputs that build the initial iterate

KG_HD double mlp_safe_log10(double x) { return log10(x > 1e-300 ? x : 1e-300); }

KG_HD void mlp_features(const RadParams &R, const double *pp, const RadGeom &rg, double dt, int startwith,
                        float x[MLP_IN]) {
  const auto &gg = rg.g.gg;
  const double rho = pp[RHO], ug = pp[UU], Er = pp[EE0];
  x[0] = (float)(mlp_safe_log10(rho) / 4. + 1.);
  x[1] = (float)(mlp_safe_log10(ug / rho) / 4.);
  x[2] = (float)(mlp_safe_log10(Er / rho) / 6.);
  for (int i = 0; i < 3; i++) {
    x[3 + i] = (float)asinh(pp[VX + i] * sqrt(gg[i + 1][i + 1]));
    x[6 + i] = (float)asinh(pp[FX0 + i] * sqrt(gg[i + 1][i + 1]));
  }
  x[9] = (float)(mlp_safe_log10(rad_kappa_abs(R, pp) * dt) / 5.);
  x[10] = (float)(mlp_safe_log10(rad_kappa_es(R, pp) * dt) / 5.);
  x[11] = (float)rg.alpha;
  x[12] = (float)rg.g.gttpert;
  x[13] = (float)(mlp_safe_log10(sqrt(gg[3][3])) / 2.);
  x[14] = startwith == IMP_MHD ? 1.f : 0.f;
  x[15] = (float)(mlp_safe_log10(Er / ug) / 6.);
}

// raw (unstandardised) targets from the state before and after the solve
// and the attempt that succeeded (-1: none)
KG_HD void mlp_targets(const double *pp0, const double *pp1, const RadGeom &rg, int startwith, int attempt,
                       double t[MLP_OUT]) {
  const auto &gg = rg.g.gg;
  t[0] = log(pp1[UU] / pp0[UU]);
  t[1] = log(pp1[EE0] / pp0[EE0]);
  const int v = startwith == IMP_MHD ? VX : FX0;
  for (int i = 0; i < 3; i++) t[2 + i] = (pp1[v + i] - pp0[v + i]) * sqrt(gg[i + 1][i + 1]);
  t[5] = attempt != 0 ? 1. : 0.;
  t[6] = (attempt < 0 || attempt >= 2) ? 1. : 0.;
}

// The attempt a warm-started cascade begins with: the energy-equation
// attempts the network expects to fail are skipped (all four solve the
// same equation to the same tolerance; the entropy attempts are never
// skipped to)
KG_HD int mlp_first_attempt(const double t[MLP_OUT]) {
  if (t[6] > 0.5) return 2;
  if (t[5] > 0.5) return 1;
  return 0;
}

// initial iterate from the (unstandardised) prediction
KG_HD void mlp_guess(const double *pp0, const RadGeom &rg, int startwith, const double t[MLP_NREG], double *guess) {
  const auto &gg = rg.g.gg;
  for (int i = 0; i < NVR; i++) guess[i] = pp0[i];
  guess[UU] = pp0[UU] * exp(t[0]);
  guess[EE0] = pp0[EE0] * exp(t[1]);
  // the predicted velocity is used for the radiation frame only: a gas
  // velocity guess moved by the prediction slows the gas-primitive Newton
  // iteration down (measured), the radiation one speeds it up
  if (startwith == IMP_RAD)
    for (int i = 0; i < 3; i++) guess[FX0 + i] = pp0[FX0 + i] + t[2 + i] / sqrt(gg[i + 1][i + 1]);
}

// ---------------------------------------------------------------------------
// The same network as the warm start of the MHD inversion (u2p).  Inputs:
// the invariants of the conserved state that u2p_setup forms (D, the
// normal-frame energy E = -Q.n, |Q_perp|^2, B^2, (Q.B)^2, the entropy
// density), the reference's starting W (u2p.c:2093-2112) with the energy
// residual and Newton step there, and the metric at the cell:
//   0  log10 D / 4 + 1              1  log10(E / D - 1) / 4
//   2  |Q_perp| / E                 3  log10(1 - Q_perp^2 / E^2) / 4
//   4  log10(B^2 / D) / 4           5  (Q.B)^2 / (B^2 Q_perp^2)
//   6  log10(W_guess / D) / 4       7  asinh(f(W_guess) / E)
//   8  asinh(-f / (f' W_guess))     9  log10(u / rho) / 4 of the guess
//   10 log10(gamma^2) / 2 of the guess   11 lapse
//   12 g_tt + 1                     13 log10 sqrt(g_33) / 2
//   14 asinh(S_c / D) / 4           15 log10(E / W_guess)
// Outputs: 0  ln(W / W_guess), W the root the plain inversion reached;
//          1  1 when the plain inversion needed the entropy equation.
// ---------------------------------------------------------------------------
KG_HD double mlp_clip_log10(double x, double lo) { return log10(x > lo ? x : lo); }

KG_HD void u2p_features(double GAMMA, const double *uu, const double *pp0, const Geom &g, float x[MLP_IN]) {
  U2PState s;
  u2p_setup(uu, g, s);
  const double D = s.c.D > 1e-300 ? s.c.D : 1e-300;
  const double E = -s.c.Qn;
  const double Ep = fabs(E) > 1e-300 ? fabs(E) : 1e-300;
  const double W0 = u2p_initial_w(GAMMA, pp0, g);
  double f0 = 0., df0 = 0., err0 = 0.;
  f_u2p(GAMMA, 0, W0 - s.c.D, s.c, f0, df0, err0);
  const double q2 = s.c.Qt2 / (Ep * Ep);
  x[0] = (float)(mlp_clip_log10(D, 1e-300) / 4. + 1.);
  x[1] = (float)(mlp_clip_log10(E / D - 1., 1e-30) / 4.);
  x[2] = (float)sqrt(q2 < 1. ? q2 : 1.);
  x[3] = (float)(mlp_clip_log10(1. - q2, 1e-12) / 4.);
  x[4] = (float)(mlp_clip_log10(s.c.Bsq / D, 1e-12) / 4.);
  x[5] = (float)(s.c.Bsq * s.c.Qt2 > 0. ? s.c.QdotBsq / (s.c.Bsq * s.c.Qt2) : 0.);
  x[6] = (float)(mlp_clip_log10(W0 / D, 1e-30) / 4.);
  x[7] = (float)asinh(f0 / Ep);
  x[8] = (float)(df0 != 0. && isfinite(f0 / df0) ? asinh(-f0 / (df0 * W0)) : 0.);
  x[9] = (float)(mlp_clip_log10(pp0[UU] / pp0[RHO], 1e-30) / 4.);
  x[10] = (float)(mlp_clip_log10(W0 / (pp0[RHO] + GAMMA * pp0[UU]), 1.) / 2.);
  x[11] = (float)sqrt(-1. / g.GG[0][0]);
  x[12] = (float)g.gttpert;
  x[13] = (float)(mlp_clip_log10(sqrt(g.gg[3][3]), 1e-300) / 2.);
  x[14] = (float)(asinh(s.c.Sc / D) / 4.);
  x[15] = (float)mlp_clip_log10(Ep / W0, 1e-30);
  for (int f = 0; f < MLP_IN; f++)
    if (!isfinite(x[f])) x[f] = 0.f;
}

KG_HD void u2p_targets(double GAMMA, const double *pp0, const double *pp1, const Geom &g, int status,
                       double t[MLP_OUT]) {
  for (int o = 0; o < MLP_OUT; o++) t[o] = 0.;
  t[0] = log(u2p_initial_w(GAMMA, pp1, g) / u2p_initial_w(GAMMA, pp0, g));
  t[1] = status != 0 ? 1. : 0.;
}

// the starting W of a warm-started inversion (0 when the prediction gives
// no usable value)
KG_HD double u2p_warm_w(double GAMMA, const double *pp0, const Geom &g, float y0) {
  const double W = u2p_initial_w(GAMMA, pp0, g) * exp((double)y0);
  return (isfinite(W) && W > 0.) ? W : 0.;
}

}  // namespace kgpu
