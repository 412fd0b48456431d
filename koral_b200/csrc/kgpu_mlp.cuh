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

}  // namespace kgpu
