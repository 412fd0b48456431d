// Device-side per-cell physics of KORAL's MHD hot path for sm_100a.
//
// Every routine restates a reference routine (file:line given beside it) in
// the reference's floating-point evaluation order.  The translation units
// that include this header are compiled with --fmad=false, so each
// +,-,*,/ and sqrt rounds exactly as the reference's x86-64 build does and
// the results agree bit for bit; only the transcendental calls (log, pow in
// the entropy) may differ in the last place from the host C library.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "kgpu_math.cuh"

namespace kgpu {

#define KG_HD __host__ __device__ inline

constexpr int NVMAX = 9;           // MHD variables (no radiation on this path)
constexpr bool kMagn = NVMAX > 8;  // the magnetic field is always carried
constexpr int RHO = 0, UU = 1, VX = 2, VY = 3, VZ = 4, ENTR = 5, B1 = 6, B2 = 7, B3 = 8;
constexpr double SMALL = 1.e-50, BIG = 1. / SMALL;

struct RadParams;   // radiation constants (kgpu_rad.cuh)

// Run-time description of one grid, passed by value to every kernel.
struct Grid {
  int nx, ny, nz, ng, nv;
  int sx, sy, sz;            // padded extents (sy = 1 when ny == 1, ...)
  int ngcx, ngcy, ngcz;
  int axisym, szmet, ngczmet;
  long ncell;                // sx*sy*sz
  long nmet;                 // sx*sy*szmet
  long nfmet[3];             // metric points per face set
  double gamma, tsteplim;
  int int_order, fluxmethod;
  double rhofloor, uurhoratiomin, uurhoratiomax, b2rhoratiomax, gammamaxhd, u2pconv;
  // device arrays
  double *u, *p, *ut0, *ut1;         // [nv][ncell]
  double *pfix, *ufix;               // fixup staging [nv][ncell]
  const double *xb[3];               // cell faces, index ic+ng
  const double *met_c;               // centre metric, [40][nmet]: g 0..19, G 20..39
  const double *met_f[3];            // face metric, [40][nfmet[d]]
  const double *gkr;                 // Christoffels, [64][nmet]
  double *flb[3];                    // face fluxes [nv][nface[d]]
  long nface[3];
  double *emf;                       // [3][(nx+1)(ny+1)(nz+1)]
  double *al[3], *ar[3];             // wavespeeds per cell and direction
  int *flag;                         // HD fixup request per cell
  int *fq[3];                        // faces whose magnetic floor the face flux left to k_flux_fix
  int *fqn;                          // their number per direction
  const double *rhofl_c, *rhofl_f;   // density floor per x-index (centres, x-faces), or null
  int bc[3];                         // boundary kind per axis (KGPU_BC_*)
  double *scal;                      // device scalars (see ScalarSlot)
  unsigned long long *cnt;           // device counters
  // radiation (nv == 13): variables EE0..FZ0 follow the nine MHD ones
  int rad;                           // radiation carried
  int rad_limiter;                   // optical-depth limiter of the radiative wave speeds
  const RadParams *radp;             // device copy of the radiation constants
  double *arl[3], *arr[3];           // radiative wave speeds per cell and direction
  // polar-axis correction (CORRECT_POLARAXIS / _3D): the cells within
  // polar_nc rows of either theta boundary are corrected, not evolved
  // (0: none); polar_emf: flux-CT's EMFs zeroed on the polar edges
  int polar_nc, polar_emf;
};

// is_cell_corrected_polaraxis (finite.c:5604-5625)
KG_HD bool polar_cell(const Grid &G, int iy) {
  return G.polar_nc > 0 && (iy < G.polar_nc || iy > G.ny - G.polar_nc - 1);
}

enum ScalarSlot { S_TSTEPDENMAX = 0, S_TSTEPDENMIN = 1, S_DT = 2, S_T = 3, S_NSCAL = 8 };
enum CounterSlot {
  C_FIXUP = 0, C_ENTROPY = 1, C_FAIL = 2, C_NEGRHO = 3,
  C_ITERS_HOT = 4,   // Newton steps of energy-equation solves
  C_ITERS_ENT = 5,   // Newton steps of entropy-equation solves
  C_SLOW = 6,        // energy solves paused after the first pass and resumed
  C_ENTQ = 7,        // cells handed to the entropy equation
  C_RADCOR = 8,      // M1 inversions that needed a correction (U2PRAD fixup requests)
  C_RADIMP_FAIL = 9, // implicit source solves where every attempt failed
  C_IMP_ITERS = 10,  // Newton iterations of the implicit solves, all attempts
  C_IMP_PASSES = 11, // passes of the batched solver that had work
  C_IMP_FALLBACK = 12,  // warm-started solves that fell back to the reference cascade
  C_IMP_EVALS = 13,  // residual evaluations of the implicit solves
  C_IMP_INNER = 14,  // Newton steps of the MHD inversions nested in those evaluations
  C_IMP_INNER_F = 15,   // their W-function evaluations (bracketing, steps, damped trials)
  C_IMP_COOP = 16,   // evaluations handed to a whole warp (nested inversion over its cap)
                     // (10..16 are the solver's own statistics, in its order)
  C_IMP_SOLVES = 17, // implicit source solves
  C_RADFLOOR = 18,   // cells whose radiation floors acted
  C_FACE_FLOOR = 19, // faces whose state needed the magnetic floor (computed by k_flux_fix)
  C_NCNT = 20
};

// ---------------------------------------------------------------------------
// index helpers (ko.h:190-230 and 505-560, with the same collapse of unused
// dimensions: an index along a dimension of size one always maps to 0)
// ---------------------------------------------------------------------------
KG_HD long cell_index(const Grid &G, int ix, int iy, int iz) {
  int ky = (G.ny > 1 ? iy : 0) + G.ngcy, kz = (G.nz > 1 ? iz : 0) + G.ngcz;
  return (long)(ix + G.ngcx) + (long)ky * G.sx + (long)kz * G.sx * G.sy;
}
KG_HD long met_index(const Grid &G, int ix, int iy, int iz) {
  int ky = (G.ny > 1 ? iy : 0) + G.ngcy;
  int kz = G.axisym ? 0 : (G.nz > 1 ? iz : 0) + G.ngcz;
  return (long)(ix + G.ngcx) + (long)ky * G.sx + (long)kz * G.sx * G.sy;
}
KG_HD long face_index(const Grid &G, int ix, int iy, int iz, int d) {
  long kx = ix + G.ngcx, ky = (G.ny > 1 ? iy : 0) + G.ngcy, kz = (G.nz > 1 ? iz : 0) + G.ngcz;
  if (d == 0) return kx + ky * (G.sx + 1) + kz * (long)G.sy * (G.sx + 1);
  if (d == 1) return kx + ky * G.sx + kz * (long)(G.sy + 1) * G.sx;
  return kx + ky * G.sx + kz * (long)G.sy * G.sx;
}
KG_HD long facemet_index(const Grid &G, int ix, int iy, int iz, int d) {
  long kx = ix + G.ngcx, ky = (G.ny > 1 ? iy : 0) + G.ngcy;
  // an axisymmetric metric keeps one phi plane for every face set
  // (iZMET(iz) = 0 in get_gb, ko.h:125)
  long kz = G.axisym ? 0 : (long)((G.nz > 1 ? iz : 0) + G.ngcz);
  if (d == 0) return kx + ky * (G.sx + 1) + kz * (long)G.sy * (G.sx + 1);
  if (d == 1) return kx + ky * G.sx + kz * (long)(G.sy + 1) * G.sx;
  return kx + ky * G.sx + kz * (long)G.sy * G.sx;
}
KG_HD long emf_index(const Grid &G, int ix, int iy, int iz) {
  return (long)ix + (long)iy * (G.nx + 1) + (long)iz * (G.ny + 1) * (G.nx + 1);
}
__device__ inline double size_x(const Grid &G, int ic, int d) {   // finite.c:2248
  return G.xb[d][ic + 1 + G.ng] - G.xb[d][ic + G.ng];
}

// ---------------------------------------------------------------------------
// geometry (struct geometry, ko.h:336-353; fill_geometry metric.c:1643-1748)
// ---------------------------------------------------------------------------
struct Geom {
  double gg[4][5];
  double GG[4][5];
  double gdet, gttpert;
};

__device__ inline void load_geom(const double *met, long npts, long i, Geom &g) {
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 5; b++) {
      g.gg[a][b] = __ldg(met + (long)(a * 5 + b) * npts + i);
      g.GG[a][b] = __ldg(met + (long)(20 + a * 5 + b) * npts + i);
    }
  g.gdet = g.gg[3][4];
  g.gttpert = g.GG[3][4];
}
__device__ inline void geom_centre(const Grid &G, int ix, int iy, int iz, Geom &g) {
  load_geom(G.met_c, G.nmet, met_index(G, ix, iy, iz), g);
}
__device__ inline void geom_face(const Grid &G, int ix, int iy, int iz, int d, Geom &g) {
  load_geom(G.met_f[d], G.nfmet[d], facemet_index(G, ix, iy, iz, d), g);
}

// ---------------------------------------------------------------------------
// small helpers (misc.c:56-92, ko.h:332)
// ---------------------------------------------------------------------------
KG_HD double dmin(double a, double b) { return a < b ? a : b; }
KG_HD double dmax(double x, double y) { return x > y ? x : y; }
KG_HD double dsign(double x) {
  if (x > 0.) return 1.;
  if (x < 0.) return -1.;
  if (x == 0.) return 1.;
  return 0.;
}
KG_HD double dot4(const double *A, const double *B) {
  return A[0] * B[0] + A[1] * B[1] + A[2] * B[2] + A[3] * B[3];
}

// frames.c:2086-2106 (A^i -> A_i)
KG_HD void lower(const double A1[4], double A2[4], const double gg[4][5]) {
  double At[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    At[i] = 0.;
#pragma unroll
    for (int k = 0; k < 4; k++) At[i] += A1[k] * gg[i][k];
  }
#pragma unroll
  for (int i = 0; i < 4; i++) A2[i] = At[i];
}
// frames.c:2057-2085 (A_i -> A^i)
KG_HD void raise(const double A1[4], double A2[4], const double GG[4][5]) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 4; k++) s += A1[k] * GG[i][k];
    A2[i] = s;
  }
}

// relative four-velocity -> four-velocity and its covariant form
// (conv_vels_both VELR->VEL4, relele.c:64-91 and 309-327)
KG_HD void velr_to_vel4(const double u1[4], double ucon[4], double ucov[4], const Geom &g) {
  double qsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++)
#pragma unroll
    for (int j = 1; j < 4; j++) qsq += u1[i] * u1[j] * g.gg[i][j];
  double gamma2 = (1. + qsq);
  double alpha2 = (-1. / g.GG[0][0]);
  double alpgam = sqrt(alpha2 * gamma2);
  double uc[4];
  uc[0] = sqrt(gamma2 / alpha2);
  uc[1] = u1[1] - alpgam * g.GG[0][1];
  uc[2] = u1[2] - alpgam * g.GG[0][2];
  uc[3] = u1[3] - alpgam * g.GG[0][3];
  double uo[4];
  lower(uc, uo, g.gg);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    ucon[i] = uc[i];
    ucov[i] = uo[i];
  }
}

// magn.c:7-23
KG_HD void bcon_4vel(const double *pr, const double ucon[4], const double ucov[4], double bcon[4]) {
  bcon[0] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
#pragma unroll
  for (int j = 1; j < 4; j++) bcon[j] = (pr[B1 - 1 + j] + bcon[0] * ucon[j]) / ucon[0];
}

// 1 + u_t from the relative velocity (p2u.c:548-580)
KG_HD double calc_utp1(const double vcon[4], const Geom &g) {
  double qsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++)
#pragma unroll
    for (int j = 1; j < 4; j++) qsq += vcon[i] * vcon[j] * g.gg[i][j];
  double gamma2 = (1. + qsq);
  double alphasq = (-1. / g.GG[0][0]);
  double alpgam = sqrt(alphasq * gamma2);
  double betasqoalphasq = g.gg[0][1] * g.GG[0][1] + g.gg[0][2] * g.GG[0][2] + g.gg[0][3] * g.GG[0][3];
  double ud0tilde = 0.0;
#pragma unroll
  for (int j = 1; j < 4; j++) ud0tilde += vcon[j] * g.gg[0][j];
  return ud0tilde + (g.gttpert - alphasq * (betasqoalphasq + qsq)) / (1.0 + alpgam);
}

// Per-state kinematics shared by the flux, p2u and wavespeed formulas.
struct Kin {
  double ucon[4], ucov[4], bcon[4], bcov[4], bsq;
};
KG_HD void kinematics(const double *pp, const Geom &g, bool magn, Kin &k) {
  double v[4] = {0., pp[VX], pp[VY], pp[VZ]};
  velr_to_vel4(v, k.ucon, k.ucov, g);
  if (magn) {
    bcon_4vel(pp, k.ucon, k.ucov, k.bcon);
    lower(k.bcon, k.bcov, g.gg);
    k.bsq = dot4(k.bcon, k.bcov);
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++) k.bcon[i] = k.bcov[i] = 0.;
    k.bsq = 0.;
  }
}

// primitives -> conserved (p2u_mhd, p2u.c:56-156)
KG_HD void p2u_mhd(const Grid &G, const double *p, double *u, const Geom &g, const Kin &k) {
  double gdetu = g.gdet;
  double rho = p[0], uu = p[1], S = p[5];
  double vcon[4] = {0., p[2], p[3], p[4]};
  double ut = k.ucon[0];
  double rhout = rho * ut;
  double Sut = S * ut;
  double pre = (G.gamma - 1.) * uu;
  double w = rho + uu + pre;
  double eta = w + k.bsq;
  double etap = uu + pre + k.bsq;
  double ptot = pre + 0.5 * k.bsq;
  double utp1 = calc_utp1(vcon, g);
  double Tttt = etap * k.ucon[0] * k.ucov[0] + rho * k.ucon[0] * utp1 + ptot - k.bcon[0] * k.bcov[0];
  double Ttr = eta * k.ucon[0] * k.ucov[1] - k.bcon[0] * k.bcov[1];
  double Ttth = eta * k.ucon[0] * k.ucov[2] - k.bcon[0] * k.bcov[2];
  double Ttph = eta * k.ucon[0] * k.ucov[3] - k.bcon[0] * k.bcov[3];
  double pb1 = p[B1], pb2 = p[B2], pb3 = p[B3];   // read before u[] is written (u may alias p)
  u[0] = gdetu * rhout;
  u[1] = gdetu * Tttt;
  u[2] = gdetu * Ttr;
  u[3] = gdetu * Ttth;
  u[4] = gdetu * Ttph;
  u[5] = gdetu * Sut;
  if (kMagn) {
    u[B1] = gdetu * pb1;
    u[B2] = gdetu * pb2;
    u[B3] = gdetu * pb3;
  }
}
KG_HD void p2u_full(const Grid &G, const double *p, double *u, const Geom &g) {
  Kin k;
  kinematics(p, g, kMagn, k);
  p2u_mhd(G, p, u, g, k);
}

// physics.c:913-917
KG_HD double calc_Sfromu(double gamma, double rho, double u) {
  double gammam1 = gamma - 1.;
  double indexn = 1.0 / gammam1;
  return rho * log(pow(gammam1 * u, indexn) / pow(rho, indexn + 1.0));
}

// T^{mu}_{nu} row (idim+1) and the face flux (f_flux_prime, physics.c:687-820,
// calc_Tij 827-892, indices_2221 frames.c:1966-1999)
KG_HD void flux_prime(const Grid &G, const double *pp, int idim, const Geom &g, const Kin &k, double *ff) {
  double rho = pp[0], u = pp[1], S = pp[5];
  double pre = (G.gamma - 1.) * u;
  double w = rho + u + pre;
  double eta = w + k.bsq;
  double ptot = pre + 0.5 * k.bsq;
  // T^{a b} for a = idim+1 only, then lower the second index
  const int a = idim + 1;
  double Tup[4];
#pragma unroll
  for (int j = 0; j < 4; j++) Tup[j] = eta * k.ucon[a] * k.ucon[j] + ptot * g.GG[a][j] - k.bcon[a] * k.bcon[j];
  double Tmix[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    double s = 0.;
#pragma unroll
    for (int kk = 0; kk < 4; kk++) s += Tup[kk] * g.gg[kk][j];
    Tmix[j] = s;
  }
  double gdetu = g.gdet;
  double etap = u + pre + k.bsq;
  double vcon[4] = {0., pp[2], pp[3], pp[4]};
  double utp1 = calc_utp1(vcon, g);
  ff[0] = gdetu * rho * k.ucon[a];
  ff[1] = gdetu * (etap * k.ucon[a] * k.ucov[0] + rho * k.ucon[a] * utp1);
  if (kMagn) ff[1] += -gdetu * k.bcon[a] * k.bcov[0];
  ff[2] = gdetu * (Tmix[1]);
  ff[3] = gdetu * (Tmix[2]);
  ff[4] = gdetu * (Tmix[3]);
  ff[5] = gdetu * S * k.ucon[a];
  if (kMagn) {
    ff[B1] = gdetu * (k.bcon[1] * k.ucon[a] - k.bcon[a] * k.ucon[1]);
    ff[B2] = gdetu * (k.bcon[2] * k.ucon[a] - k.bcon[a] * k.ucon[2]);
    ff[B3] = gdetu * (k.bcon[3] * k.ucon[a] - k.bcon[a] * k.ucon[3]);
  }
}

// HARM-style fast magnetosonic speeds (calc_wavespeeds_lr_core, physics.c:9-56)
KG_HD void wavespeed_core(const double ucon[4], const Geom &g, double wspeed2, int idim, double &al,
                                      double &ar) {
  double Acov[4] = {0., 0., 0., 0.}, Acon[4], Bcov[4] = {1., 0., 0., 0.}, Bcon[4];
  Acov[idim + 1] = 1.;
  raise(Acov, Acon, g.GG);
  raise(Bcov, Bcon, g.GG);
  double Asq = dot4(Acon, Acov);
  double Bsq = dot4(Bcon, Bcov);
  double Au = dot4(Acov, ucon);
  double Bu = dot4(Bcov, ucon);
  double AB = dot4(Acon, Bcov);
  double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  double B = 2. * (AuBu * (1.0 - wspeed2) - AB * wspeed2);
  double A = Bu2 * (1.0 - wspeed2) - Bsq * wspeed2;
  double discr = 4.0 * wspeed2 * ((AB * AB - Asq * Bsq) * wspeed2 + (2.0 * AB * Au * Bu - Asq * Bu2 - Bsq * Au2) * (wspeed2 - 1.0));
  if (discr < 0.) return;   // previous values kept, as the reference does
  discr = sqrt(discr);
  al = -(-B + discr) / (2. * A);
  ar = -(-B - discr) / (2. * A);
}

// left/right speeds per direction, co-going speeds zeroed
// (calc_wavespeeds_lr_pure, physics.c:61-241, MHD part)
KG_HD void wavespeeds(const Grid &G, const double *pp, const Geom &g, double al[3], double ar[3]) {
  Kin k;
  kinematics(pp, g, kMagn, k);
  double rho = pp[RHO], uu = pp[UU];
  double pre = (G.gamma - 1.) * uu;
  double cs2 = G.gamma * pre / (rho + uu + pre);
  if (cs2 < 0.) cs2 = 0.;
  double va2 = 0.;
  if (kMagn) {
    double EF = rho + G.gamma * uu;
    double EEloc = k.bsq + EF;
    va2 = k.bsq / EEloc;
    if (va2 < 0.) va2 = 0.;
  }
  double vtot2 = cs2 + va2 - cs2 * va2;
  double l = 0., r = 0.;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    wavespeed_core(k.ucon, g, vtot2, d, l, r);
    al[d] = l > 0. ? 0. : l;
    ar[d] = r < 0. ? 0. : r;
  }
}

// ---------------------------------------------------------------------------
// conserved -> primitives: the W Newton solver with the Noble energy
// equation and the entropy equation (u2p_solver_W u2p.c:1965-2352,
// f_u2p_hot 733-814, f_u2p_entropy 914-974)
// ---------------------------------------------------------------------------
struct U2PCons {
  double Qn, Qt2, D, QdotBsq, Bsq, Sc;
};

KG_HD void f_u2p(double GAMMA, int Etype, double Wp, const U2PCons &c, double &f, double &df, double &err) {
  double GAMMAM1 = GAMMA - 1.;
  double Qn = c.Qn, Qtsq = c.Qt2, D = c.D, QdotBsq = c.QdotBsq, Bsq = c.Bsq, Sc = c.Sc;
  double W = Wp + D;
  double X = Bsq + W;
  double Wsq = W * W;
  double W3 = Wsq * W;
  double X2 = X * X;
  double Xsq = X2;
  double X3 = X2 * X;
  double v2 = (Wsq * Qtsq + QdotBsq * (Bsq + 2. * W)) / (Wsq * Xsq);
  double gamma2 = 1. / (1. - v2);
  double gamma = sqrt(gamma2);
  double rho0 = D / gamma;
  double wmrho0 = Wp / gamma2 - D * v2 / (1. + gamma);
  double dvsq = (-2.0 / X3 * (Qtsq + QdotBsq * (3.0 * W * X + Bsq * Bsq) / W3));
  double dwmrho0dvsq = (D * (gamma * 0.5 - 1.0) - Wp);
  double drho0dvsq = -D * gamma * 0.5;
  if (Etype == 0) {
    double u = wmrho0 / GAMMA;
    double p = (GAMMA - 1) * u;
    f = Qn + W - p + 0.5 * Bsq * (1. + v2) - QdotBsq / 2. / Wsq;
    err = fabs(f) / (fabs(Qn) + fabs(W) + fabs(p) + fabs(0.5 * Bsq * (1. + v2)) + fabs(QdotBsq / 2. / Wsq));
    double dp1 = ((GAMMA - 1.) * (1. - v2) / GAMMA);
    double idwmrho0dp = GAMMAM1 / GAMMA;
    double idrho0dp = 0.0;
    double dp2 = drho0dvsq * idrho0dp + dwmrho0dvsq * idwmrho0dp;
    double dpdW = dp1 + dp2 * dvsq;
    df = 1. - dpdW + QdotBsq / (Wsq * W) + 0.5 * Bsq * dvsq;
  } else {
    double pressure = (GAMMAM1 / GAMMA) * wmrho0;
    double indexn = 1.0 / GAMMAM1;
    double insideentropy = pow(pressure, indexn) / pow(rho0, indexn + 1.0);
    double Ssofchi = log(insideentropy);
    f = -Sc + D * Ssofchi;
    err = fabs(f) / (fabs(Sc) + fabs(D * Ssofchi));
    double dSsdrho = GAMMA / ((1.0 - GAMMA) * rho0);
    double dSsdchi = 1.0 / (GAMMAM1 * wmrho0);
    double dwmrho0dW = 1.0 / gamma;
    double drho0dW = 0.0;
    double dSsdW = drho0dW * dSsdrho + dwmrho0dW * dSsdchi;
    double dSsdvsq = drho0dvsq * dSsdrho + dwmrho0dvsq * dSsdchi;
    double dSsdWp = dSsdW + dSsdvsq * dvsq;
    df = D * dSsdWp;
  }
}

KG_HD bool u2p_bad_w(double W, double Bsq, double QdotBsq, double Qtsq, double f, double df) {
  return ((W * W * W * (W + 2. * Bsq) - QdotBsq * (2. * W + Bsq)) <= W * W * (Qtsq - Bsq * Bsq)) || !isfinite(f) ||
         !isfinite(df);
}

// The W solver in resumable pieces.  U2PState holds everything the solver
// derives from the conserved variables and the metric; the Newton loop's
// only carried state is (W, iter), so a solve stopped after some iterations
// and resumed later takes exactly the same steps as an uninterrupted one.
struct U2PState {
  U2PCons c;
  double Qtcon[4], Bcon[4], QdotB;
};

KG_HD void u2p_setup(const double *uu, const Geom &g, U2PState &s) {
  const double gdetu = g.gdet;
  double alpha = sqrt(-1. / g.GG[0][0]);
  double D = uu[0] / gdetu * alpha;
  double Sc = uu[5] / gdetu * alpha;
  double Qcov[4], Qcon[4];
  Qcov[0] = (uu[1] / gdetu - uu[0] / gdetu) * alpha;
  Qcov[1] = uu[2] / gdetu * alpha;
  Qcov[2] = uu[3] / gdetu * alpha;
  Qcov[3] = uu[4] / gdetu * alpha;
  raise(Qcov, Qcon, g.GG);
  double Bcov[4], Bsq = 0., QdotB = 0., QdotBsq = 0.;
  s.Bcon[0] = s.Bcon[1] = s.Bcon[2] = s.Bcon[3] = 0.;
  if (kMagn) {
    s.Bcon[1] = uu[B1] / gdetu * alpha;
    s.Bcon[2] = uu[B2] / gdetu * alpha;
    s.Bcon[3] = uu[B3] / gdetu * alpha;
    lower(s.Bcon, Bcov, g.gg);
    Bsq = dot4(s.Bcon, Bcov);
    QdotB = dot4(Qcov, s.Bcon);
    QdotBsq = QdotB * QdotB;
  }
  double ncov[4] = {-alpha, 0., 0., 0.}, ncon[4];
  raise(ncov, ncon, g.GG);
  double Qn = Qcon[0] * ncov[0];
  double Qtcov[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double sum = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) sum += ((i == j ? 1 : 0) + ncon[i] * ncov[j]) * Qcon[j];
    s.Qtcon[i] = sum;
  }
  lower(s.Qtcon, Qtcov, g.gg);
  double Qt2 = dot4(s.Qtcon, Qtcov);
  s.QdotB = QdotB;
  s.c = U2PCons{Qn, Qt2, D, QdotBsq, Bsq, Sc};
}

// initial W from the primitive guess (u2p.c:2100-2110)
KG_HD double u2p_initial_w(double GAMMA, const double *pp, const Geom &g) {
  double qsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++)
#pragma unroll
    for (int j = 1; j < 4; j++) qsq += pp[1 + i] * pp[1 + j] * g.gg[i][j];
  double gamma2 = 1. + qsq;
  return (pp[0] + GAMMA * pp[1]) * gamma2;
}

// W x 10 until the state is physical (u2p.c:2117-2135); 0 or -150
KG_HD int u2p_bracket(double GAMMA, int Etype, const U2PCons &c, double &W, unsigned *fevals = nullptr) {
  double f0, dfdW, err;
  int i_increase = 0;
  while (true) {
    f0 = dfdW = 0.;
    if (fevals) (*fevals)++;
    f_u2p(GAMMA, Etype, W - c.D, c, f0, dfdW, err);
    if (u2p_bad_w(W, c.Bsq, c.QdotBsq, c.Qt2, f0, dfdW) && (i_increase < 50)) {
      W *= 10.;
      i_increase++;
      continue;
    }
    break;
  }
  return i_increase >= 50 ? -150 : 0;
}

constexpr int U2P_PAUSED = 1;
// returned by a capped W solve that used up its function evaluations (the
// caller repeats the whole inversion another way; nothing is kept)
constexpr int U2P_OVER_CAP = 7;

// Newton iterations (u2p.c:2140-2200) until convergence, failure, or a
// pause: at the top of an iteration once iter reaches `stop`, or before an
// iteration whose damped step would need `damp_budget` or more halvings
// (the iteration is then undone, (W, iter) as before it).  A paused solve
// resumed with larger limits takes exactly the steps an uninterrupted one
// takes.  Returns 0 when the loop has ended (the caller finishes with
// u2p_final), U2P_PAUSED, or a negative reference status on failure.
KG_HD int u2p_newton(double GAMMA, double CONV, int Etype, const U2PCons &c, double &W, int &iter, int stop,
                     int damp_budget = 1 << 30, unsigned *fevals = nullptr, unsigned fcap = 0) {
  const double D = c.D;
  double f0, dfdW, err;
  while (true) {
    if (iter >= stop && iter < 50) return U2P_PAUSED;
    if (fcap && *fevals >= fcap) return U2P_OVER_CAP;
    double Wprev = W;
    iter++;
    if (fevals) (*fevals)++;
    f_u2p(GAMMA, Etype, W - D, c, f0, dfdW, err);
    if (err < CONV) break;
    if (dfdW == 0.) {
      W *= 1.1;
      if (iter < 50) continue;
      break;
    }
    double Wnew = W - f0 / dfdW;
    int idump = 0;
    double dumpfac = 1.;
    while (true) {
      double f0t = 0., dft = 0., errt;
      if (fevals) (*fevals)++;
      f_u2p(GAMMA, Etype, Wnew - D, c, f0t, dft, errt);
      if (u2p_bad_w(Wnew, c.Bsq, c.QdotBsq, c.Qt2, f0t, dft) && (idump < 100)) {
        if (fcap && *fevals >= fcap) return U2P_OVER_CAP;
        idump++;
        if (idump >= damp_budget) {
          W = Wprev;
          iter--;
          return U2P_PAUSED;
        }
        dumpfac /= 2.;
        Wnew = W - dumpfac * f0 / dfdW;
        continue;
      }
      break;
    }
    if (idump >= 100) return -101;
    W = Wnew;
    if (fabs(W) > BIG) return -103;
    if (fabs((W - Wprev) / Wprev) < CONV && err < 1.e-1) break;
    if (!(iter < 50)) break;
  }
  return 0;
}

#ifdef __CUDACC__
// The same iterations carried out by a whole warp on one cell (all lanes
// hold the same state): the damped step's trial points, which the scalar
// loop tries one after another, are tried 32 at a time and the first
// acceptable one is taken.  Trial k is W - 2^-k f/f' as in the scalar loop
// (2^-k is the exact result of its repeated halving), so the result is the
// same bit for bit.  Every lane returns the same values.
__device__ inline int u2p_newton_warp(double GAMMA, double CONV, int Etype, const U2PCons &c, double &W, int &iter) {
  const int lane = threadIdx.x & 31;
  const double D = c.D;
  double f0, dfdW, err;
  while (true) {
    double Wprev = W;
    iter++;
    f_u2p(GAMMA, Etype, W - D, c, f0, dfdW, err);
    if (err < CONV) break;
    if (dfdW == 0.) {
      W *= 1.1;
      if (iter < 50) continue;
      break;
    }
    double Wnew = 0.;
    int found = -1;
    for (int base = 0; base <= 100 && found < 0; base += 32) {
      const int k = base + lane;
      double Wk = 0.;
      bool accept = false;
      if (k == 0) {
        Wk = W - f0 / dfdW;
      } else if (k <= 100) {
        const double dumpfac = ldexp(1.0, -k);
        Wk = W - dumpfac * f0 / dfdW;
      }
      if (k == 100) {
        accept = true;   // the scalar loop stops here whatever the state
      } else if (k < 100) {
        double f0t = 0., dft = 0., errt;
        f_u2p(GAMMA, Etype, Wk - D, c, f0t, dft, errt);
        accept = !u2p_bad_w(Wk, c.Bsq, c.QdotBsq, c.Qt2, f0t, dft);
      }
      const unsigned m = __ballot_sync(0xffffffffu, accept);
      if (m) {
        const int L = __ffs(m) - 1;
        found = base + L;
        Wnew = __shfl_sync(0xffffffffu, Wk, L);
      }
    }
    if (found >= 100) return -101;
    W = Wnew;
    if (fabs(W) > BIG) return -103;
    if (fabs((W - Wprev) / Wprev) < CONV && err < 1.e-1) break;
    if (!(iter < 50)) break;
  }
  return 0;
}
#endif

#ifdef __CUDACC__
KG_HD int u2p_final(double GAMMA, const struct U2PState &s, double W, int iter, const double *uu, double *pp,
                    const Geom &g);
// u2p_solver_W with all 32 lanes of a warp on the same cell: the damped
// trials of a Newton step are tried 32 at a time; same result.
__device__ inline int u2p_solver_W_warp(const Grid &G, const double *uu, double *pp, const Geom &g, int Etype,
                                        unsigned *iters = nullptr, unsigned *fevals = nullptr) {
  U2PState s;
  u2p_setup(uu, g, s);
  double W = u2p_initial_w(G.gamma, pp, g);
  if (u2p_bracket(G.gamma, Etype, s.c, W, fevals)) return -150;
  int iter = 0;
  int r = u2p_newton_warp(G.gamma, G.u2pconv, Etype, s.c, W, iter);
  if (iters) *iters += (unsigned)iter;
  if (r < 0) return r;
  return u2p_final(G.gamma, s, W, iter, uu, pp, g);
}
#endif

// checks and primitives from the converged W (u2p.c:2205-2292)
KG_HD int u2p_final(double GAMMA, const U2PState &s, double W, int iter, const double *uu, double *pp, const Geom &g) {
  if (iter >= 50) return -102;
  if (!isfinite(W)) return -103;
  const double gdetu = g.gdet;
  const double Bsq = s.c.Bsq, QdotBsq = s.c.QdotBsq, Qtsq = s.c.Qt2, D = s.c.D, QdotB = s.QdotB;
  double Wsq = W * W;
  double Xsq = (Bsq + W) * (Bsq + W);
  double v2 = (Wsq * Qtsq + QdotBsq * (Bsq + 2. * W)) / (Wsq * Xsq);
  double gamma2 = 1. / (1. - v2);
  double gamma = sqrt(gamma2);
  double rho = D / gamma;
  double uint = 1. / GAMMA * (W / gamma2 - rho);
  double ut1 = gamma / (W + Bsq) * (s.Qtcon[1] + QdotB * s.Bcon[1] / W);
  double ut2 = gamma / (W + Bsq) * (s.Qtcon[2] + QdotB * s.Bcon[2] / W);
  double ut3 = gamma / (W + Bsq) * (s.Qtcon[3] + QdotB * s.Bcon[3] / W);
  if (!isfinite(ut1)) return -120;
  if (uint < 0. || gamma2 < 0. || isnan(W) || !isfinite(W)) return -104;
  pp[0] = rho;
  pp[1] = uint;
  pp[2] = ut1;
  pp[3] = ut2;
  pp[4] = ut3;
  if (rho < 0.) return -105;
  pp[5] = calc_Sfromu(GAMMA, rho, uint);
  if (kMagn) {
    pp[B1] = uu[B1] / gdetu;
    pp[B2] = uu[B2] / gdetu;
    pp[B3] = uu[B3] / gdetu;
  }
  return 0;
}

// Returns 0 on success or the reference's negative status codes.
// Iteration counts are bounded exactly as in the reference (50 bracket
// expansions, 50 Newton steps, 100 halvings), so every call terminates.
// iters, when given, accumulates the Newton steps taken, fevals the
// evaluations of the W function (bracketing, steps, damped trials); with
// fcap the solve gives up (U2P_OVER_CAP, pp untouched) once *fevals reaches
// fcap during the Newton steps
KG_HD int u2p_solver_W(const Grid &G, const double *uu, double *pp, const Geom &g, int Etype,
                       unsigned *iters = nullptr, unsigned *fevals = nullptr, unsigned fcap = 0) {
  U2PState s;
  u2p_setup(uu, g, s);
  double W = u2p_initial_w(G.gamma, pp, g);
  if (u2p_bracket(G.gamma, Etype, s.c, W, fevals)) return -150;
  int iter = 0;
  int r = u2p_newton(G.gamma, G.u2pconv, Etype, s.c, W, iter, 1 << 30, 1 << 30, fevals, fcap);
  if (r == U2P_OVER_CAP) return r;
  if (iters) *iters += (unsigned)iter;
  if (r < 0) return r;
  return u2p_final(G.gamma, s, W, iter, uu, pp, g);
}

// high-level inversion with entropy fallback and "keep old" last resort
// (u2p, u2p.c:176-485).  Returns the reference's status: 0 hot, -1 entropy,
// -2 entropy after negative density, -3 failure (old primitives kept).
KG_HD int u2p(const Grid &G, const double *uu0, double *pp, const Geom &g, int &fixup) {
  double uu[NVMAX], ppbak[NVMAX];
  constexpr int nv = NVMAX;
#pragma unroll
  for (int iv = 0; iv < nv; iv++) {
    uu[iv] = uu0[iv];
    ppbak[iv] = pp[iv];
  }
  int ret = 0, u2pret = -1;
  if (uu[0] / g.gdet < 0.) {
    pp[0] = G.rhofloor;
    uu[0] = G.rhofloor * g.gdet;
    ret = -2;
  }
  u2pret = u2p_solver_W(G, uu, pp, g, 0);
  if (u2pret < 0) {
    ret = -1;
    u2pret = u2p_solver_W(G, uu, pp, g, 1);
    if (u2pret < 0) ret = -2;
  }
  if (u2pret < 0) {
    ret = -3;
#pragma unroll
    for (int iv = 0; iv < nv; iv++) pp[iv] = ppbak[iv];
  }
  fixup = (ret < -1) ? 1 : 0;
  return ret;
}

// density, internal-energy, magnetisation and Lorentz-factor floors
// (check_floors_mhd, u2p.c:492-695, B2RHOFLOORFRAME = ZAMO)
// kout (optional): the four-velocity and magnetic four-vector the floor
// computes for the magnetic test; *kvalid tells whether they still hold for
// the returned primitives (neither the magnetic floor nor the Lorentz-factor
// ceiling changed velocities or field; the density and energy floors do
// not enter them), so a caller can skip computing them again.
// defer (optional): where the magnetic floor applies, set *defer and return
// at once, leaving pp part-floored; the caller then discards pp and runs
// the whole floor again without defer (the face flux hands such faces to a
// second kernel so that the floor's nested inversion stays out of its
// register budget).
KG_HD int check_floors_mhd(const Grid &G, double *pp, const Geom &g, double rhofloor_bh = -1., Kin *kout = nullptr,
                           bool *kvalid = nullptr, bool *defer = nullptr) {
  int ret = 0;
  if (kvalid) *kvalid = false;
  const bool magn = kMagn;
  // the reference converts the incoming primitives first (u2p.c:505); the
  // conserved state is only read by the magnetic floor, so it is computed
  // there, from a copy of the incoming primitives
  double pin[NVMAX];
#pragma unroll
  for (int iv = 0; iv < NVMAX; iv++) pin[iv] = pp[iv];
  if (pp[0] < G.rhofloor) {
    pp[0] = G.rhofloor;
    ret = -1;
  }
  // radius-dependent floor (RHOFLOOR_BH, u2p.c:546-557), tabulated per x-index
  if (rhofloor_bh > 0. && pp[0] < rhofloor_bh) {
    pp[0] = rhofloor_bh;
    ret = -1;
  }
  if (pp[1] < G.uurhoratiomin * pp[0]) {
    pp[1] = G.uurhoratiomin * pp[0];
    ret = -1;
  }
  if (pp[1] > G.uurhoratiomax * pp[0]) {
    pp[1] = G.uurhoratiomax * pp[0];
    ret = -1;
  }
  if (magn) {
    double v[4] = {0., pp[2], pp[3], pp[4]}, ucond[4], ucovd[4], bcond[4], bcovd[4];
    velr_to_vel4(v, ucond, ucovd, g);
    lower(ucond, ucovd, g.gg);
    bcon_4vel(pp, ucond, ucovd, bcond);
    lower(bcond, bcovd, g.gg);
    const double bsq = dot4(bcond, bcovd);
    double magpre = bsq / 2.;
    if (kout) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        kout->ucon[i] = ucond[i];
        kout->ucov[i] = ucovd[i];
        kout->bcon[i] = bcond[i];
        kout->bcov[i] = bcovd[i];
      }
      kout->bsq = bsq;
      if (kvalid) *kvalid = true;
    }
    if (magpre > G.b2rhoratiomax * pp[RHO]) {
      if (kvalid) *kvalid = false;
      if (defer) {
        *defer = true;
        return -1;
      }
      // normal observer as a relative velocity (relele.c:569-575, 282-307)
      double alp = 1. / sqrt(-g.GG[0][0]);
      double ncov[4] = {-alp, 0., 0., 0.}, etacon[4];
      raise(ncov, etacon, g.GG);
      double f = magpre / (G.b2rhoratiomax * pp[RHO]);
      double dpp[NVMAX], duu[NVMAX];
      double drho = pp[RHO] * (f - 1.);
      for (int iv = 0; iv < NVMAX; iv++) dpp[iv] = 0.0;
      dpp[RHO] = drho;
      dpp[UU] = pp[UU] * drho / pp[RHO];
      dpp[VX] = etacon[1] - etacon[0] * g.GG[0][1] / g.GG[0][0];
      dpp[VY] = etacon[2] - etacon[0] * g.GG[0][2] / g.GG[0][0];
      dpp[VZ] = etacon[3] - etacon[0] * g.GG[0][3] / g.GG[0][0];
      p2u_full(G, dpp, duu, g);
      double uu[NVMAX];
      p2u_full(G, pin, uu, g);
      for (int iv = 0; iv < NVMAX; iv++) uu[iv] += duu[iv];
      int rt = u2p_solver_W(G, uu, pp, g, 0);
      if (rt < 0) u2p_solver_W(G, uu, pp, g, 1);
      ret = -1;
    }
  }
  {
    double qsq = 0.;
#pragma unroll
    for (int i = 1; i < 4; i++)
#pragma unroll
      for (int j = 1; j < 4; j++) qsq += pp[1 + i] * pp[1 + j] * g.gg[i][j];
    double gamma2 = 1. + qsq;
    if (gamma2 > G.gammamaxhd * G.gammamaxhd) {
      double qsqmax = G.gammamaxhd * G.gammamaxhd - 1.;
      double A = sqrt(qsqmax / qsq);
      for (int j = 1; j < 4; j++) pp[1 + j] *= A;
      ret = -1;
      if (kvalid) *kvalid = false;
    }
  }
  if (ret < 0) pp[5] = calc_Sfromu(G.gamma, pp[0], pp[1]);
  return ret;
}

// ---------------------------------------------------------------------------
// reconstruction (avg2point, finite.c:89-289): one variable at a time
// ---------------------------------------------------------------------------
KG_HD double DMM(double X, double Y) { return .5 * (dsign(X) + dsign(Y)) * dmin(fabs(X), fabs(Y)); }
KG_HD double DM4(double W, double X, double Y, double Z) {
  return 0.125 * (dsign(W) + dsign(X)) * fabs((dsign(W) + dsign(Y)) * (dsign(W) + dsign(Z))) *
         dmin(dmin(fabs(W), fabs(X)), dmin(fabs(Y), fabs(Z)));
}

// PPM on a non-uniform grid (finite.c:142-225); returns the left (ul) and
// right (ur) face values of the centre cell.
KG_HD void ppm(double um2, double um1, double u0, double up1, double up2, double dxm2, double dxm1,
                           double dx0, double dxp1, double dxp2, double &ul, double &ur) {
  double Z1 = (dxm1 + dx0) / (2. * dx0 + dxp1);
  double Z2 = (dxp2 + dxp1) / (2. * dxp1 + dx0);
  double DX = dxm1 + dx0 + dxp1 + dxp2;
  double dri = dx0 / (dxm1 + dx0 + dxp1) *
               ((2. * dxm1 + dx0) / (dxp1 + dx0) * (up1 - u0) + (dx0 + 2. * dxp1) / (dxm1 + dx0) * (u0 - um1));
  double drip1 = dxp1 / (dx0 + dxp1 + dxp2) *
                 ((2. * dx0 + dxp1) / (dxp2 + dxp1) * (up2 - up1) + (dxp1 + 2. * dxp2) / (dx0 + dxp1) * (up1 - u0));
  double drim1 = dxm1 / (dxm2 + dxm1 + dx0) *
                 ((2. * dxm2 + dxm1) / (dx0 + dxm1) * (u0 - um1) + (dxm1 + 2. * dx0) / (dxm2 + dxm1) * (um1 - um2));
  if ((up1 - u0) * (u0 - um1) > 0.) dri = dmin(fabs(dri), dmin(2. * fabs(u0 - um1), 2. * fabs(u0 - up1))) * dsign(dri);
  else dri = 0.;
  if ((up2 - up1) * (up1 - u0) > 0.) drip1 = dmin(fabs(drip1), dmin(2. * fabs(up1 - u0), 2. * fabs(up1 - up2))) * dsign(drip1);
  else drip1 = 0.;
  if ((u0 - um1) * (um1 - um2) > 0.) drim1 = dmin(fabs(drim1), dmin(2. * fabs(um1 - um2), 2. * fabs(um1 - u0))) * dsign(drim1);
  else drim1 = 0.;
  ur = u0 + dx0 / (dx0 + dxp1) * (up1 - u0) +
       1. / DX * ((2. * dxp1 * dx0) / (dxp1 + dx0) * (Z1 - Z2) * (up1 - u0) - dx0 * Z1 * drip1 + dxp1 * Z2 * dri);
  Z1 = (dxm2 + dxm1) / (2. * dxm1 + dx0);
  Z2 = (dxp1 + dx0) / (2. * dx0 + dxm1);
  DX = dxm2 + dxm1 + dx0 + dxp1;
  ul = um1 + dxm1 / (dxm1 + dx0) * (u0 - um1) +
       1. / DX * ((2. * dx0 * dxm1) / (dx0 + dxm1) * (Z1 - Z2) * (u0 - um1) - dxm1 * Z1 * dri + dx0 * Z2 * drim1);
  if ((ur - u0) * (u0 - ul) <= 0.) {
    ul = u0;
    ur = u0;
  }
  if ((ur - ul) * (ul - (3. * u0 - 2. * ur)) < 0.) ul = 3. * u0 - 2. * ur;
  if ((ur - ul) * ((3. * u0 - 2. * ul) - ur) < 0.) ur = 3. * u0 - 2. * ul;
}

// MP5 (finite.c:226-286), uniform spacing.  One face value: pass the
// stencil in the direction of the face (a = far side, e = near side).
KG_HD double mp5_face(double um2, double um1, double u0, double up1, double up2) {
  const double alpha = 4., epsm = 1.e-10, BB2 = 1.3333333;
  double VOR = (3. * um2 - 20. * um1 + 90. * u0 + 60. * up1 - 5. * up2) / 128.;
  double VMP = u0 + DMM(up1 - u0, alpha * (u0 - um1));
  if ((VOR - u0) * (VOR - VMP) < epsm) return VOR;
  double DJM1 = um2 - 2. * um1 + u0;
  double DJ = um1 - 2. * u0 + up1;
  double DJP1 = u0 - 2. * up1 + up2;
  double DM4JPH = DM4(4. * DJ - DJP1, 4. * DJP1 - DJ, DJ, DJP1);
  double DM4JMH = DM4(4. * DJ - DJM1, 4. * DJM1 - DJ, DJ, DJM1);
  double VUL = u0 + alpha * (u0 - um1);
  double VAV = 0.5 * (u0 + up1);
  double VMD = VAV - 0.5 * DM4JPH;
  double VLC = u0 + 0.5 * (u0 - um1) + BB2 * DM4JMH;
  double VMIN = dmax(dmin(u0, dmin(up1, VMD)), dmin(u0, dmin(VUL, VLC)));
  double VMAX = dmin(dmax(u0, dmax(up1, VMD)), dmax(u0, dmax(VUL, VLC)));
  return VOR + DMM(VMIN - VOR, VMAX - VOR);
}

}  // namespace kgpu
