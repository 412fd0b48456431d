// Set-up of the Kerr torus problem: metric tables in modified Kerr-Schild
// coordinates (MKS2) and Fishbone-Moncrief initial data, on the host (KORAL
// layout, for comparison with the reference and for upload) and on the
// device (straight into the device layout, no host work or upload).
//
// KORAL evaluates its MKS2 metric and connection from machine-generated
// closed forms (metric.c:259-1640).  This file derives them independently:
// the Kerr-Schild metric g_KS(r, theta) and its first derivatives are
// written out analytically, the MKS2 metric follows from the diagonal
// coordinate map r = exp(x1) + R0, theta = pi/2 (1 + cot(pi H0/2)
// tan(pi H0 (x2 - 1/2))) by the chain rule, and the Christoffel symbols come
// from the metric derivatives, Gamma^m_{nl} = g^{ms}(d_n g_{sl} + d_l g_{sn}
// - d_s g_{nl})/2.  Afterwards the traces Gamma^m_{km} are corrected so that
// they equal the finite-difference derivative of ln(sqrt(-g)) across the
// cell, as calc_Krzysie_at_center does (metric.c:828-905), which keeps the
// discrete update of a static metric exactly balanced.
//
// The tables use KORAL's layout (20 doubles of g_{mu nu}/d ln gdet/gdet per
// point, 20 of g^{mu nu}/g_tt perturbation, 64 Christoffels) so they can be
// compared with the reference's and uploaded through kgpu_upload_metric.
//
// Every per-point and per-cell formula below is one __host__ __device__
// function that the host loops and the device kernels both call; the two
// paths differ only in the math library behind sin, cos, tan, exp, log and
// pow (glibc on the host, CUDA on the device).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/koral_b200.h"
#include "kgpu_rad.cuh"
#include "kgpu_setup.cuh"

namespace {

struct MKS2 {
  double a, R0, H0;
  // coordinate map and its first two derivatives
  KG_HD double r(double x1) const { return exp(x1) + R0; }
  KG_HD double drdx1(double x1) const { return exp(x1); }
  KG_HD double d2rdx1(double x1) const { return exp(x1); }
  KG_HD double th(double x2) const { return 0.5 * M_PI * (1. + tan(H0 * M_PI * (x2 - 0.5)) / tan(0.5 * M_PI * H0)); }
  KG_HD double dthdx2(double x2) const {
    double c = cos(H0 * M_PI * (x2 - 0.5));
    return 0.5 * M_PI * H0 * M_PI / (tan(0.5 * M_PI * H0) * c * c);
  }
  KG_HD double d2thdx2(double x2) const {
    double arg = H0 * M_PI * (x2 - 0.5);
    double c = cos(arg);
    return 0.5 * M_PI * (H0 * M_PI) * (H0 * M_PI) * 2. * tan(arg) / (tan(0.5 * M_PI * H0) * c * c);
  }
};

// Kerr-Schild g_{mu nu}(r, theta) with its r- and theta-derivatives
struct KSPoint {
  double g[4][4], dgr[4][4], dgth[4][4], G[4][4];
  double gdet;
};

KG_HD void ks_point(double a, double r, double th, KSPoint &k) {
  double s = sin(th), c = cos(th), s2 = s * s, a2 = a * a;
  double Sig = r * r + a2 * c * c;
  double dSr = 2. * r, dSth = -2. * a2 * c * s;
  double q = 2. * r / Sig;
  double dqr = 2. * (Sig - 2. * r * r) / (Sig * Sig);
  double dqth = -2. * r * dSth / (Sig * Sig);
  double ds2 = 2. * s * c;   // d(sin^2)/dtheta
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) k.g[i][j] = k.dgr[i][j] = k.dgth[i][j] = k.G[i][j] = 0.;
  k.g[0][0] = -(1. - q);
  k.g[0][1] = k.g[1][0] = q;
  k.g[0][3] = k.g[3][0] = -a * s2 * q;
  k.g[1][1] = 1. + q;
  k.g[1][3] = k.g[3][1] = -a * s2 * (1. + q);
  k.g[2][2] = Sig;
  k.g[3][3] = s2 * (Sig + a2 * s2 * (1. + q));
  k.dgr[0][0] = dqr;
  k.dgr[0][1] = k.dgr[1][0] = dqr;
  k.dgr[0][3] = k.dgr[3][0] = -a * s2 * dqr;
  k.dgr[1][1] = dqr;
  k.dgr[1][3] = k.dgr[3][1] = -a * s2 * dqr;
  k.dgr[2][2] = dSr;
  k.dgr[3][3] = s2 * (dSr + a2 * s2 * dqr);
  k.dgth[0][0] = dqth;
  k.dgth[0][1] = k.dgth[1][0] = dqth;
  k.dgth[0][3] = k.dgth[3][0] = -a * (ds2 * q + s2 * dqth);
  k.dgth[1][1] = dqth;
  k.dgth[1][3] = k.dgth[3][1] = -a * (ds2 * (1. + q) + s2 * dqth);
  k.dgth[2][2] = dSth;
  k.dgth[3][3] = ds2 * (Sig + a2 * s2 * (1. + q)) + s2 * (dSth + a2 * (ds2 * (1. + q) + s2 * dqth));
  double Del = r * r - 2. * r + a2;
  k.G[0][0] = -(1. + q);
  k.G[0][1] = k.G[1][0] = q;
  k.G[1][1] = Del / Sig;
  k.G[1][3] = k.G[3][1] = a / Sig;
  k.G[2][2] = 1. / Sig;
  k.G[3][3] = 1. / (Sig * s2);
  k.gdet = Sig * fabs(s);   // sqrt(-g) > 0 also beyond the pole (theta < 0 or > pi)
}

// metric of one MKS2 point: the 20-double g and G entries of KORAL's table
// and the (uncorrected) Christoffels
KG_HD void mks2_point(const MKS2 &m, double x1, double x2, double *g20, double *G20, double Kr[4][4][4],
                      double &gdet) {
  double r = m.r(x1), th = m.th(x2);
  KSPoint k;
  ks_point(m.a, r, th, k);
  double J[4] = {1., m.drdx1(x1), m.dthdx2(x2), 1.};
  double dJ1 = m.d2rdx1(x1), dJ2 = m.d2thdx2(x2);
  double g[4][4], Gi[4][4], dg[4][4][4];   // dg[l][i][j] = d_l g_ij (MKS2)
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      g[i][j] = k.g[i][j] * J[i] * J[j];
      Gi[i][j] = k.G[i][j] / (J[i] * J[j]);
      dg[0][i][j] = dg[3][i][j] = 0.;
      double dJJ1 = (i == 1 ? dJ1 * J[j] : 0.) + (j == 1 ? J[i] * dJ1 : 0.);
      double dJJ2 = (i == 2 ? dJ2 * J[j] : 0.) + (j == 2 ? J[i] * dJ2 : 0.);
      dg[1][i][j] = k.dgr[i][j] * J[1] * J[i] * J[j] + k.g[i][j] * dJJ1;
      dg[2][i][j] = k.dgth[i][j] * J[2] * J[i] * J[j] + k.g[i][j] * dJJ2;
    }
  gdet = k.gdet * J[1] * J[2];
  for (int mu = 0; mu < 4; mu++)
    for (int n = 0; n < 4; n++)
      for (int l = 0; l < 4; l++) {
        double sum = 0.;
        for (int s = 0; s < 4; s++) sum += Gi[mu][s] * (dg[n][s][l] + dg[l][s][n] - dg[s][n][l]);
        Kr[mu][n][l] = 0.5 * sum;
      }
  // d ln gdet / dx^i (KORAL stores these in g[i][4], i < 3)
  double s = sin(th), c = cos(th), Sig = r * r + m.a * m.a * c * c;
  double dl1 = (2. * r / Sig) * J[1] + dJ1 / J[1];
  double dl2 = (-2. * m.a * m.a * c * s / Sig + c / s) * J[2] + dJ2 / J[2];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 5; j++) {
      g20[i * 5 + j] = j < 4 ? g[i][j] : 0.;
      G20[i * 5 + j] = j < 4 ? Gi[i][j] : 0.;
    }
  g20[0 * 5 + 4] = dl1;
  g20[1 * 5 + 4] = dl2;
  g20[2 * 5 + 4] = 0.;
  g20[3 * 5 + 4] = gdet;
  G20[3 * 5 + 4] = 2. * r / Sig;   // g_tt + 1 in Kerr-Schild time
}

KG_HD double gdet_at(const MKS2 &m, double x1, double x2) {
  double r = m.r(x1), th = m.th(x2), c = cos(th);
  return (r * r + m.a * m.a * c * c) * fabs(sin(th)) * m.drdx1(x1) * m.dthdx2(x2);
}

KG_HD double x_centre(const double *xb, int ng, int i) { return .5 * (xb[i + 1 + ng] + xb[i + ng]); }
KG_HD double x_face(const double *xb, int ng, int i) { return xb[i + ng]; }

// Centre point (ix, iy, izm) of the metric tables (izm counts the metric's
// own phi planes): g, G and the Christoffels kr64[i*16 + j*4 + k] with the
// flux-consistent traces (calc_Krzysie_at_center, metric.c:828-905).
KG_HD void mks2_centre(const MKS2 &m, const double *xbx, const double *xby, const double *xbz, int ng, int ix, int iy,
                       int izm, double *g20, double *G20, double *kr64) {
  double Kr[4][4][4], gd;
  double x1 = x_centre(xbx, ng, ix), x2 = x_centre(xby, ng, iy);
  mks2_point(m, x1, x2, g20, G20, Kr, gd);
  const double *xbs[3] = {xbx, xby, xbz};
  int ic[3] = {ix, iy, izm};
  for (int kap = 1; kap <= 3; kap++) {
    double Ck = Kr[0][kap][0] + Kr[1][kap][1] + Kr[2][kap][2] + Kr[3][kap][3];
    double Sk = 1.e-300 + fabs(Kr[0][kap][0]) + fabs(Kr[1][kap][1]) + fabs(Kr[2][kap][2]) + fabs(Kr[3][kap][3]);
    double W[4];
    for (int mu = 0; mu < 4; mu++) W[mu] = fabs(Kr[mu][kap][mu]) / Sk;
    double g0 = gdet_at(m, x1, x2), gu, gl, dxk;
    const double *xbk = xbs[kap - 1];
    int i = ic[kap - 1];
    if (kap == 1) { gu = gdet_at(m, x_face(xbx, ng, ix + 1), x2); gl = gdet_at(m, x_face(xbx, ng, ix), x2); }
    else if (kap == 2) { gu = gdet_at(m, x1, x_face(xby, ng, iy + 1)); gl = gdet_at(m, x1, x_face(xby, ng, iy)); }
    else { gu = g0; gl = g0; }
    dxk = xbk[i + 1 + ng] - xbk[i + ng];
    double D = (gu - gl) / (dxk * g0);
    for (int mu = 0; mu < 4; mu++) {
      Kr[mu][kap][mu] += (D - Ck) * W[mu];
      Kr[mu][mu][kap] = Kr[mu][kap][mu];
    }
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) kr64[i * 16 + j * 4 + k] = Kr[i][j][k];
}

// Face point of direction d at (ix, iy): the face's own coordinate along d,
// centre coordinates across (the metric does not depend on phi).
KG_HD void mks2_face(const MKS2 &m, const double *xbx, const double *xby, int ng, int d, int ix, int iy, double *g20,
                     double *G20) {
  double Kr[4][4][4], gd;
  double x1 = d == 0 ? x_face(xbx, ng, ix) : x_centre(xbx, ng, ix);
  double x2 = d == 1 ? x_face(xby, ng, iy) : x_centre(xby, ng, iy);
  mks2_point(m, x1, x2, g20, G20, Kr, gd);
}

}  // namespace

extern "C" int kgpu_mks2_metric_tables(double a, double R0, double H0, int nx, int ny, int nz, int ng, int axisym,
                                       const double *xbx, const double *xby, const double *xbz, double *g,
                                       double *G, double *gKr, double *gbx, double *gby, double *gbz, double *Gbx,
                                       double *Gby, double *Gbz) {
  if (!xbx || !xby || !xbz || !g || !G || !gKr || !gbx || !gby || !gbz || !Gbx || !Gby || !Gbz) return KGPU_EINVAL;
  if (nx < 1 || ny < 1 || nz < 1 || ng < 1) return KGPU_EINVAL;
  MKS2 m{a, R0, H0};
  const int sx = nx + 2 * ng, sy = ny > 1 ? ny + 2 * ng : 1, sz = nz > 1 ? nz + 2 * ng : 1;
  const int ngy = ny > 1 ? ng : 0, ngz = nz > 1 ? ng : 0;
  const int szm = axisym ? 1 : sz, ngzm = axisym ? 0 : ngz;
  for (int kz = 0; kz < szm; kz++)
    for (int ky = 0; ky < sy; ky++)
      for (int kx = 0; kx < sx; kx++) {
        long pt = kx + (long)ky * sx + (long)kz * sx * sy;
        mks2_centre(m, xbx, xby, xbz, ng, kx - ng, ky - ngy, kz - ngzm, g + pt * 20, G + pt * 20, gKr + pt * 64);
      }
  // faces: (sx+1) x sy x szm along x, sx x (sy+1) x szm along y,
  // sx x sy x (szm+1) along z
  double *gb[3] = {gbx, gby, gbz}, *Gb[3] = {Gbx, Gby, Gbz};
  for (int d = 0; d < 3; d++) {
    const int ex = sx + (d == 0), ey = sy + (d == 1), ez = szm + (d == 2);
    for (int kz = 0; kz < ez; kz++)
      for (int ky = 0; ky < ey; ky++)
        for (int kx = 0; kx < ex; kx++) {
          long f = kx + (long)ky * ex + (long)kz * ex * ey;
          mks2_face(m, xbx, xby, ng, d, kx - ng, ky - ngy, gb[d] + f * 20, Gb[d] + f * 20);
        }
  }
  return 0;
}

// Device form of kgpu_mks2_metric_tables, written in the device layout
// ([component][point]; g in 0..19, G in 20..39 of the 40 per point).
namespace {

__global__ void k_setup_metric_centre(kgpu::Grid G, MKS2 m, int ngy, int ngzm) {
  const long pt = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (pt >= G.nmet) return;
  const int kx = (int)(pt % G.sx), ky = (int)((pt / G.sx) % G.sy), kz = (int)(pt / ((long)G.sx * G.sy));
  double g20[20], G20[20], kr[64];
  mks2_centre(m, G.xb[0], G.xb[1], G.xb[2], G.ng, kx - G.ng, ky - ngy, kz - ngzm, g20, G20, kr);
  double *mc = (double *)G.met_c, *gk = (double *)G.gkr;
  for (int k = 0; k < 20; k++) {
    mc[k * G.nmet + pt] = g20[k];
    mc[(20 + k) * G.nmet + pt] = G20[k];
  }
  for (int k = 0; k < 64; k++) gk[k * G.nmet + pt] = kr[k];
}

__global__ void k_setup_metric_face(kgpu::Grid G, MKS2 m, int d, int ngy) {
  const long n = G.nfmet[d];
  const long f = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (f >= n) return;
  const int ex = G.sx + (d == 0), ey = G.sy + (d == 1);
  const int kx = (int)(f % ex), ky = (int)((f / ex) % ey);
  double g20[20], G20[20];
  mks2_face(m, G.xb[0], G.xb[1], G.ng, d, kx - G.ng, ky - ngy, g20, G20);
  double *mf = (double *)G.met_f[d];
  for (int k = 0; k < 20; k++) {
    mf[k * n + f] = g20[k];
    mf[(20 + k) * n + f] = G20[k];
  }
}

unsigned setup_blocks(long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

int kgpu::setup_mks2_metric_device(const Grid &G, double a, double r0, double h0, cudaStream_t st) {
  if (G.nx < 1 || G.ny < 1 || G.nz < 1 || G.ng < 1) return KGPU_EINVAL;
  MKS2 m{a, r0, h0};
  const int ngy = G.ny > 1 ? G.ng : 0, ngz = G.nz > 1 ? G.ng : 0, ngzm = G.axisym ? 0 : ngz;
  k_setup_metric_centre<<<setup_blocks(G.nmet, 128), 128, 0, st>>>(G, m, ngy, ngzm);
  for (int d = 0; d < 3; d++) k_setup_metric_face<<<setup_blocks(G.nfmet[d], 128), 128, 0, st>>>(G, m, d, ngy);
  return cudaGetLastError() == cudaSuccess ? 4 : KGPU_ECUDA;
}

// ---------------------------------------------------------------------------
// Fishbone & Moncrief (1976) torus: constant specific angular momentum l,
// enthalpy from the first integral of hydrostatic equilibrium in Kerr
// (Boyer-Lindquist, M = 1).  Same construction as the KORAL plug-in used by
// the oracle (oracle/ref/problems/FMTORUS).
// ---------------------------------------------------------------------------
namespace {

using kgpu::Geom;
using kgpu::Grid;

KG_HD double fm_lfish(double a, double r) {
  double sr = sqrt(r);
  double x = r * r - 2. * a * sr + a * a;
  double num = x * ((-2. * a * r * x) / sqrt(2. * a * sr + (-3. + r) * r) +
                    ((a + (-2. + r) * sr) * (r * r * r + a * a * (2. + r))) / sqrt(1. + (2. * a) / (r * sr) - 3. / r));
  double den = r * r * r * sqrt(2. * a * sr + (-3. + r) * r) * (a * a + (-2. + r) * r);
  return num / den;
}
KG_HD double fm_lnh_raw(double a, double l, double r, double th) {
  double sth = sin(th), cth = cos(th);
  double Sigma = r * r + a * a * cth * cth;
  double Delta = r * r - 2. * r + a * a;
  double A = (r * r + a * a) * (r * r + a * a) - Delta * a * a * sth * sth;
  double q = sqrt(1. + 4. * l * l * Sigma * Sigma * Delta / (A * A * sth * sth));
  return 0.5 * log((1. + q) / (Sigma * Delta / A)) - 0.5 * q - 2. * a * r * l / A;
}
KG_HD double fm_uphi(double a, double l, double r, double th) {
  double sth = sin(th), cth = cos(th);
  double Sigma = r * r + a * a * cth * cth;
  double Delta = r * r - 2. * r + a * a;
  double A = (r * r + a * a) * (r * r + a * a) - Delta * a * a * sth * sth;
  double e2 = Sigma * Sigma * Delta / (A * A * sth * sth);
  double up1 = sqrt((-1. + sqrt(1. + 4. * l * l * e2)) / 2.);
  return 2. * a * r * sqrt(1. + up1 * up1) / sqrt(A * Sigma * Delta) + sqrt(Sigma / A) * up1 / sth;
}
KG_HD double fm_noise(unsigned long long seed, unsigned long long idx) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (idx + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Constants of one torus: specific angular momentum, ln h at the inner
// edge, the density maximum the code density is normalised by.
struct TorusK {
  double l, lnh0, rhomax;
};
TorusK torus_consts(const kgpu_torus_params &tp, double GAM) {
  TorusK K;
  K.l = fm_lfish(tp.spin, tp.rmax);
  K.lnh0 = fm_lnh_raw(tp.spin, K.l, tp.rin, M_PI / 2.);
  const double lnhmax = fm_lnh_raw(tp.spin, K.l, tp.rmax, M_PI / 2.) - K.lnh0;
  K.rhomax = pow((exp(lnhmax) - 1.) * (GAM - 1.) / (tp.kappa * GAM), 1. / (GAM - 1.));
  return K;
}

// Primitives of domain cell (ix, iy, iz) without the field, and the vector
// potential A_phi there.  With rad.on (13 variables) the torus pressure is
// shared by gas and radiation in thermal equilibrium and the atmosphere gets
// radiation of rad.eradatm times its gas energy, at rest with it (as the
// radiative build of the torus plug-in sets it up).
KG_HD double torus_cell_prims(const kgpu_torus_params &tp, const MKS2 &m, double GAM, const TorusK &K,
                              const kgpu::TorusRadConsts &rad, int nx, int ny, int ix, int iy, int iz, double x1,
                              double x2, const Geom &gm, double *pp) {
  using namespace kgpu;
  const double a = tp.spin;
  double r = m.r(x1), th = m.th(x2);
  double aphi = 0.;
  double rhoatm = tp.atm_rho0 * pow(r, -1.5), uuatm = tp.atm_uu0 * pow(r, -2.5);
  pp[RHO] = rhoatm;
  pp[UU] = uuatm;
  pp[VX] = pp[VY] = pp[VZ] = 0.;
  pp[B1] = pp[B2] = pp[B3] = 0.;
  double lnh = fm_lnh_raw(a, K.l, r, th) - K.lnh0;
  const bool intorus = lnh > 0. && r >= tp.rin;
  if (intorus) {
    double h = exp(lnh);
    double rho = pow((h - 1.) * (GAM - 1.) / (tp.kappa * GAM), 1. / (GAM - 1.)) / K.rhomax;
    double ui = tp.kappa * pow(rho * K.rhomax, GAM) / (GAM - 1.) / K.rhomax;
    unsigned long long idx = (unsigned long long)ix + (unsigned long long)nx * ((unsigned long long)iy + (unsigned long long)ny * (unsigned long long)iz);
    ui *= 1. + tp.noise * (2. * fm_noise(tp.seed, idx) - 1.);
    // Boyer-Lindquist u^phi with u^r = u^theta = 0: the Kerr-Schild and
    // MKS2 components equal the BL ones, u^t from the normalisation in
    // the MKS2 metric; then the relative four-velocity
    double uph = fm_uphi(a, K.l, r, th);
    double A2 = gm.gg[0][0], B2 = 2. * gm.gg[0][3] * uph, C2 = gm.gg[3][3] * uph * uph + 1.;
    double ut = (-B2 - sqrt(B2 * B2 - 4. * A2 * C2)) / (2. * A2);
    if (ut < 0.) ut = (-B2 + sqrt(B2 * B2 - 4. * A2 * C2)) / (2. * A2);
    double ucon[4] = {ut, 0., 0., uph};
    double v[4];
    for (int i = 1; i < 4; i++) v[i] = ucon[i] - ucon[0] * gm.GG[0][i] / gm.GG[0][0];
    pp[RHO] = rho > rhoatm ? rho : rhoatm;
    pp[UU] = ui > uuatm ? ui : uuatm;
    pp[VX] = v[1]; pp[VY] = v[2]; pp[VZ] = v[3];
    aphi = rho - 0.2 > 0. ? rho - 0.2 : 0.;
  }
  if (rad.on) {
    if (intorus || rad.eradatm < 0.) {
      // the temperature at which gas and radiation carry the torus
      // pressure together, b T + a T^4 = p: Newton steps from the
      // smaller one-component solution fall monotonically onto it
      const double P = (GAM - 1.) * pp[UU];
      const double aa = 4. * rad.sigma / 3., bb = rad.kb * pp[RHO] / rad.mu / rad.mp;
      double T = P / bb, T4 = sqrt(sqrt(P / aa));
      if (T4 < T) T = T4;
      for (int it = 0; it < 100; it++) T -= (bb * T + aa * T * T * T * T - P) / (bb + 4. * aa * T * T * T);
      pp[UU] = rad.kb * pp[RHO] * T / rad.mu / rad.mp / (GAM - 1.);
      pp[EE0] = 4. * rad.sigma * T * T * T * T;
      pp[FX0] = pp[VX];
      pp[FY0] = pp[VY];
      pp[FZ0] = pp[VZ];
    } else {
      pp[EE0] = rad.eradatm * pp[UU];
      pp[FX0] = pp[FY0] = pp[FZ0] = 0.;
    }
  }
  pp[ENTR] = calc_Sfromu(GAM, pp[RHO], pp[UU]);
  return aphi;
}

// A_phi with the ghost layers the torus boundaries give it (radial copy,
// theta mirror, periodic phi); only domain values are ever stored.
KG_HD double torus_aphi(const Grid &Gr, const double *Aphi, int ix, int iy, int iz) {
  const int nx = Gr.nx, ny = Gr.ny, nz = Gr.nz;
  if (ix < 0) ix = 0;
  if (ix > nx - 1) ix = nx - 1;
  if (iy < 0) iy = -iy - 1;
  if (iy > ny - 1) iy = 2 * ny - iy - 1;
  if (iz < 0) iz += nz;
  if (iz > nz - 1) iz -= nz;
  return Aphi[kgpu::cell_index(Gr, ix, iy, iz)];
}
// corner value: mean of the eight cells around the corner
KG_HD double torus_aphi_corner(const Grid &Gr, const double *Ap, int ix, int iy, int iz) {
  return 1. / 8. * (torus_aphi(Gr, Ap, ix, iy, iz) + torus_aphi(Gr, Ap, ix, iy - 1, iz) +
                    torus_aphi(Gr, Ap, ix - 1, iy, iz) + torus_aphi(Gr, Ap, ix - 1, iy - 1, iz) +
                    torus_aphi(Gr, Ap, ix, iy, iz - 1) + torus_aphi(Gr, Ap, ix, iy - 1, iz - 1) +
                    torus_aphi(Gr, Ap, ix - 1, iy, iz - 1) + torus_aphi(Gr, Ap, ix - 1, iy - 1, iz - 1));
}

// The field of cell (ix, iy, iz) from the curl of A_phi with one-sided
// corner differences (calc_BfromA, magn.c:380-586), before normalisation;
// returns the cell's p_mag / p_gas.
KG_HD double torus_cell_field(const Grid &Gr, const double *Ap, const double *xbx, const double *xby, int ix, int iy,
                              int iz, const Geom &gm, double *pp) {
  using namespace kgpu;
  const int ng = Gr.ng;
  double dx = xbx[ix + 1 + ng] - xbx[ix + ng], dy = xby[iy + 1 + ng] - xby[iy + ng];
  auto Ac = [&](int jx, int jy, int jz) { return torus_aphi_corner(Gr, Ap, jx, jy, jz); };
  double dA32 = (Ac(ix, iy + 1, iz) - Ac(ix, iy, iz) + Ac(ix + 1, iy + 1, iz) - Ac(ix + 1, iy, iz) +
                 Ac(ix, iy + 1, iz + 1) - Ac(ix, iy, iz + 1) + Ac(ix + 1, iy + 1, iz + 1) - Ac(ix + 1, iy, iz + 1)) /
                (4. * dy);
  double dA31 = (Ac(ix + 1, iy, iz) - Ac(ix, iy, iz) + Ac(ix + 1, iy + 1, iz) - Ac(ix, iy + 1, iz) +
                 Ac(ix + 1, iy, iz + 1) - Ac(ix, iy, iz + 1) + Ac(ix + 1, iy + 1, iz + 1) - Ac(ix, iy + 1, iz + 1)) /
                (4. * dx);
  pp[B1] = (0. - dA32) / gm.gdet;
  pp[B2] = (dA31 - 0.) / gm.gdet;
  pp[B3] = 0.;
  Kin k;
  kinematics(pp, gm, true, k);
  double pmag = k.bsq / 2., pgas = (Gr.gamma - 1.) * pp[UU];
  return pmag / pgas;
}

// Normalised field and the conserved variables of the cell.
KG_HD void torus_cell_finish(const Grid &Gr, double fac, bool rad, double *pp, double *uu, const Geom &gm) {
  pp[kgpu::B1] *= fac;
  pp[kgpu::B2] *= fac;
  pp[kgpu::B3] *= fac;
  kgpu::p2u_full(Gr, pp, uu, gm);
  if (rad) kgpu::p2u_rad(pp, uu, gm);
}

double torus_field_factor(const kgpu_torus_params &tp, double maxbeta) {
  return maxbeta > 0. ? sqrt(tp.maxbeta / maxbeta) : 0.;
}

}  // namespace

// Primitive and conserved arrays (KORAL layout, whole padded grid) of the
// magnetised torus.  g and G are the centre tables of kgpu_mks2_metric_tables
// for the same grid.  Ghost cells are left zero: the caller applies the
// boundary conditions (kgpu_set_bc) after uploading.  With rp (nv = 13) the
// radiative torus of torus_cell_prims.
static int fm_torus_state(const kgpu_torus_params *tp, const kgpu_config *cfg, const kgpu_rad_params *rp,
                          double eradatm, const double *xbx, const double *xby, const double *xbz, const double *g,
                          const double *G, double *u, double *p) {
  using namespace kgpu;
  if (!tp || !cfg || !xbx || !xby || !xbz || !g || !G || !u || !p) return KGPU_EINVAL;
  const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, ng = cfg->ng, nv = cfg->nv;
  if (nv != (rp ? 13 : 9) || ny < 2 || nz < 2) return KGPU_EINVAL;
  Grid Gr;
  memset(&Gr, 0, sizeof(Gr));
  Gr.nx = nx; Gr.ny = ny; Gr.nz = nz; Gr.ng = ng; Gr.nv = nv;
  Gr.sx = nx + 2 * ng; Gr.sy = ny + 2 * ng; Gr.sz = nz + 2 * ng;
  Gr.ngcx = Gr.ngcy = Gr.ngcz = ng;
  Gr.axisym = cfg->axisym_metric; Gr.ngczmet = Gr.axisym ? 0 : ng;
  Gr.gamma = cfg->gamma;
  const double GAM = cfg->gamma;
  MKS2 m{tp->spin, tp->r0, tp->h0};
  TorusRadConsts rad{0, 0., 0., 0., 0., 0.};
  if (rp) rad = TorusRadConsts{1, rp->sigma, rp->kb, rp->mu, rp->mp, eradatm};
  const TorusK K = torus_consts(*tp, GAM);
  const long ncell = (long)Gr.sx * Gr.sy * Gr.sz;
  for (long i = 0; i < ncell * nv; i++) u[i] = p[i] = 0.;
  auto geom_at = [&](int ix, int iy, int iz, Geom &gm) {
    long pt = met_index(Gr, ix, iy, iz);
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 5; j++) {
        gm.gg[i][j] = g[pt * 20 + i * 5 + j];
        gm.GG[i][j] = G[pt * 20 + i * 5 + j];
      }
    gm.gdet = gm.gg[3][4];
    gm.gttpert = gm.GG[3][4];
  };
  std::vector<double> Aphi(ncell, 0.);
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++) {
        Geom gm;
        geom_at(ix, iy, iz, gm);
        long c = cell_index(Gr, ix, iy, iz);
        Aphi[c] = torus_cell_prims(*tp, m, GAM, K, rad, nx, ny, ix, iy, iz, x_centre(xbx, ng, ix),
                                   x_centre(xby, ng, iy), gm, p + c * nv);
      }
  double maxbeta = 0.;
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++) {
        Geom gm;
        geom_at(ix, iy, iz, gm);
        long c = cell_index(Gr, ix, iy, iz);
        double beta = torus_cell_field(Gr, Aphi.data(), xbx, xby, ix, iy, iz, gm, p + c * nv);
        if (beta > maxbeta) maxbeta = beta;
      }
  const double fac = torus_field_factor(*tp, maxbeta);
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++) {
        long c = cell_index(Gr, ix, iy, iz);
        Geom gm;
        geom_at(ix, iy, iz, gm);
        torus_cell_finish(Gr, fac, rad.on, p + c * nv, u + c * nv, gm);
      }
  return 0;
}

// Device form: the same three sweeps as kernels over the domain cells, on
// the context's own grid, metric (already on the device) and state arrays
// ([variable][cell]).  A_phi goes to scratch[0..ncell), the largest
// p_mag/p_gas to the bits of scratch[ncell] (a maximum of non-negative
// doubles is a maximum of their bit patterns, so the atomic reduction is
// exact and independent of order).
namespace {

__device__ inline void setup_cell_of(const Grid &G, long i, int &ix, int &iy, int &iz) {
  ix = (int)(i % G.nx);
  iy = (int)((i / G.nx) % G.ny);
  iz = (int)(i / ((long)G.nx * G.ny));
}

__global__ void k_setup_torus_prims(Grid G, kgpu_torus_params tp, MKS2 m, TorusK K, kgpu::TorusRadConsts rad,
                                    double *Aphi) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)G.nx * G.ny * G.nz) return;
  int ix, iy, iz;
  setup_cell_of(G, i, ix, iy, iz);
  Geom gm;
  kgpu::geom_centre(G, ix, iy, iz, gm);
  double pp[kgpu::NVR];
  const long c = kgpu::cell_index(G, ix, iy, iz);
  Aphi[c] = torus_cell_prims(tp, m, G.gamma, K, rad, G.nx, G.ny, ix, iy, iz, x_centre(G.xb[0], G.ng, ix),
                             x_centre(G.xb[1], G.ng, iy), gm, pp);
  for (int v = 0; v < G.nv; v++) G.p[v * G.ncell + c] = pp[v];
}

__global__ void k_setup_torus_field(Grid G, const double *Aphi, unsigned long long *maxbeta_bits) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)G.nx * G.ny * G.nz) return;
  int ix, iy, iz;
  setup_cell_of(G, i, ix, iy, iz);
  Geom gm;
  kgpu::geom_centre(G, ix, iy, iz, gm);
  const long c = kgpu::cell_index(G, ix, iy, iz);
  double pp[kgpu::NVR];
  for (int v = 0; v < G.nv; v++) pp[v] = G.p[v * G.ncell + c];
  double beta = torus_cell_field(G, Aphi, G.xb[0], G.xb[1], ix, iy, iz, gm, pp);
  G.p[kgpu::B1 * G.ncell + c] = pp[kgpu::B1];
  G.p[kgpu::B2 * G.ncell + c] = pp[kgpu::B2];
  G.p[kgpu::B3 * G.ncell + c] = pp[kgpu::B3];
  if (beta > 0.) atomicMax(maxbeta_bits, (unsigned long long)__double_as_longlong(beta));
}

__global__ void k_setup_torus_finish(Grid G, kgpu_torus_params tp, const unsigned long long *maxbeta_bits) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)G.nx * G.ny * G.nz) return;
  int ix, iy, iz;
  setup_cell_of(G, i, ix, iy, iz);
  const double maxbeta = __longlong_as_double((long long)*maxbeta_bits);
  const double fac = maxbeta > 0. ? sqrt(tp.maxbeta / maxbeta) : 0.;
  Geom gm;
  kgpu::geom_centre(G, ix, iy, iz, gm);
  const long c = kgpu::cell_index(G, ix, iy, iz);
  double pp[kgpu::NVR], uu[kgpu::NVR];
  for (int v = 0; v < G.nv; v++) pp[v] = G.p[v * G.ncell + c];
  torus_cell_finish(G, fac, G.nv == kgpu::NVR, pp, uu, gm);
  for (int v = 0; v < G.nv; v++) {
    G.p[v * G.ncell + c] = pp[v];
    G.u[v * G.ncell + c] = uu[v];
  }
}

}  // namespace

int kgpu::setup_fm_torus_device(const Grid &G, const kgpu_torus_params &tp, const TorusRadConsts &rad, double *scratch,
                                cudaStream_t st) {
  if (G.ny < 2 || G.nz < 2 || G.nv != (rad.on ? NVR : 9) || !scratch) return KGPU_EINVAL;
  const long n = (long)G.nx * G.ny * G.nz;
  MKS2 m{tp.spin, tp.r0, tp.h0};
  const TorusK K = torus_consts(tp, G.gamma);
  unsigned long long *bits = (unsigned long long *)(scratch + G.ncell);
  if (cudaMemsetAsync(G.u, 0, G.nv * G.ncell * sizeof(double), st) != cudaSuccess ||
      cudaMemsetAsync(G.p, 0, G.nv * G.ncell * sizeof(double), st) != cudaSuccess ||
      cudaMemsetAsync(scratch, 0, (G.ncell + 1) * sizeof(double), st) != cudaSuccess)
    return KGPU_ECUDA;
  k_setup_torus_prims<<<setup_blocks(n, 128), 128, 0, st>>>(G, tp, m, K, rad, scratch);
  k_setup_torus_field<<<setup_blocks(n, 128), 128, 0, st>>>(G, scratch, bits);
  k_setup_torus_finish<<<setup_blocks(n, 128), 128, 0, st>>>(G, tp, bits);
  return cudaGetLastError() == cudaSuccess ? 3 : KGPU_ECUDA;
}

extern "C" int kgpu_fm_torus_state(const kgpu_torus_params *tp, const kgpu_config *cfg, const double *xbx,
                                   const double *xby, const double *xbz, const double *g, const double *G, double *u,
                                   double *p) {
  return fm_torus_state(tp, cfg, nullptr, 0., xbx, xby, xbz, g, G, u, p);
}

extern "C" int kgpu_fm_radtorus_state(const kgpu_torus_params *tp, const kgpu_rad_params *rp, double eradatm,
                                      const kgpu_config *cfg, const double *xbx, const double *xby, const double *xbz,
                                      const double *g, const double *G, double *u, double *p) {
  if (!rp) return KGPU_EINVAL;
  return fm_torus_state(tp, cfg, rp, eradatm, xbx, xby, xbz, g, G, u, p);
}

// Density floor rho >= atm_rho0 * r^-1.5 tabulated per x-index at cell
// centres and x-faces (the form of RHOFLOOR_BH, u2p.c:546-557).
extern "C" int kgpu_fm_torus_floor(const kgpu_torus_params *tp, int nx, int ng, const double *xbx, double *centres,
                                   double *xfaces) {
  if (!tp || !xbx || !centres || !xfaces) return KGPU_EINVAL;
  MKS2 m{tp->spin, tp->r0, tp->h0};
  double rh = 1. + sqrt(1 - tp->spin * tp->spin);
  double norm = tp->atm_rho0 / pow(rh, 1.5);
  for (int ix = -ng; ix < nx + ng; ix++) {
    double rr = m.r(.5 * (xbx[ix + 1 + ng] + xbx[ix + ng])) / rh;
    centres[ix + ng] = norm / sqrt(rr * rr * rr);
  }
  for (int ix = -ng; ix <= nx + ng; ix++) {
    double rr = m.r(xbx[ix + ng]) / rh;
    xfaces[ix + ng] = norm / sqrt(rr * rr * rr);
  }
  return 0;
}

extern "C" int kgpu_default_torus_params(kgpu_torus_params *tp) {
  if (!tp) return KGPU_EINVAL;
  tp->spin = 0.9;
  tp->r0 = 0.;
  tp->h0 = 0.6;
  tp->r_lo = 1.8;
  tp->r_hi = 1000.;
  tp->x2_lo = 0.005;
  tp->x2_hi = 0.995;
  tp->rin = 6.;
  tp->rmax = 12.;
  tp->kappa = 1.e-3;
  tp->noise = 0.02;
  tp->seed = 12345ULL;
  tp->atm_rho0 = 1.e-4;
  tp->atm_uu0 = 1.e-6;
  tp->maxbeta = 0.01;
  return 0;
}

extern "C" int kgpu_ks_metric(double a, double r, double th, double *g20, double *G20) {
  if (!g20 || !G20 || !(r > 0.)) return KGPU_EINVAL;
  KSPoint k;
  ks_point(a, r, th, k);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      g20[i * 5 + j] = k.g[i][j];
      G20[i * 5 + j] = k.G[i][j];
    }
  double s = sin(th), c = cos(th), Sig = r * r + a * a * c * c;
  g20[0 * 5 + 4] = 2. * r / Sig;                          // d ln(Sigma sin) / dr
  g20[1 * 5 + 4] = -2. * a * a * c * s / Sig + c / s;     // d ln(Sigma sin) / dtheta
  g20[2 * 5 + 4] = 0.;
  g20[3 * 5 + 4] = k.gdet;
  G20[0 * 5 + 4] = G20[1 * 5 + 4] = G20[2 * 5 + 4] = 0.;
  G20[3 * 5 + 4] = 2. * r / Sig;                          // g_tt + 1
  return 0;
}

extern "C" int kgpu_ks_metric_batch(double a, int n, const double *r, const double *th, double *g20, double *G20) {
  if (n < 0 || (n > 0 && (!r || !th || !g20 || !G20))) return KGPU_EINVAL;
  for (int k = 0; k < n; k++) {
    int e = kgpu_ks_metric(a, r[k], th[k], g20 + 20L * k, G20 + 20L * k);
    if (e) return e;
  }
  return 0;
}

