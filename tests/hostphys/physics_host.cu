// The library's per-cell physics (koral_b200/csrc/kgpu_physics.cuh and
// kgpu_rad.cuh, the same source the kernels are built from) compiled for
// the host, behind C entry points for tests/test_host_physics.py, which
// compares them on the CPU with the oracle and the reference build.  Cells
// are independent: [n][9] or [n][13] states, [n][20] + [n][20] metric
// points in KORAL's layout.  Test infrastructure only.
#include "../../koral_b200/csrc/kgpu_physics.cuh"
#include "../../koral_b200/csrc/kgpu_rad.cuh"
#include "../../include/koral_b200.h"

using namespace kgpu;

// the library's conversion of the public radiation constants
kgpu::RadParams kgpu_rad_device_params(const kgpu_rad_params &p);

namespace {

Grid mhd_grid(double gamma, double b2rho) {
  Grid G{};
  G.nv = NVMAX;
  G.gamma = gamma;
  G.rhofloor = 1e-50;
  G.uurhoratiomin = 1e-50;
  G.uurhoratiomax = 100.;
  G.b2rhoratiomax = b2rho;
  G.gammamaxhd = 100.;
  G.u2pconv = 1e-10;
  return G;
}

Geom geom_of(const double *g, const double *Gm, long i) {
  Geom o;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 5; b++) {
      o.gg[a][b] = g[i * 20 + a * 5 + b];
      o.GG[a][b] = Gm[i * 20 + a * 5 + b];
    }
  o.gdet = o.gg[3][4];
  o.gttpert = o.GG[3][4];
  return o;
}

}  // namespace

extern "C" {

// what: 0 p2u; 1..3 the flux row of direction what-1; 4 wavespeeds
// (out[n][6]: al_x, ar_x, al_y, ar_y, al_z, ar_z)
void hp_mhd_point(long n, int what, double gamma, const double *pp, const double *g, const double *Gm, double *out) {
  const Grid G = mhd_grid(gamma, 100.);
  for (long i = 0; i < n; i++) {
    const Geom geo = geom_of(g, Gm, i);
    const double *p = pp + i * NVMAX;
    if (what == 4) {
      double al[3], ar[3];
      wavespeeds(G, p, geo, al, ar);
      for (int d = 0; d < 3; d++) {
        out[i * 6 + 2 * d] = al[d];
        out[i * 6 + 2 * d + 1] = ar[d];
      }
      continue;
    }
    Kin k;
    kinematics(p, geo, kMagn, k);
    if (what == 0) p2u_mhd(G, p, out + i * NVMAX, geo, k);
    else flux_prime(G, p, what - 1, geo, k, out + i * NVMAX);
  }
}

// u2p (u2p.c:176, the MHD part) or, with floors = 1, check_floors_mhd
void hp_u2p(long n, int floors, double gamma, double b2rho, const double *uu, double *pp, const double *g,
            const double *Gm, int *ret, int *fixup) {
  const Grid G = mhd_grid(gamma, b2rho);
  for (long i = 0; i < n; i++) {
    const Geom geo = geom_of(g, Gm, i);
    if (floors) {
      ret[i] = check_floors_mhd(G, pp + i * NVMAX, geo);
      fixup[i] = 0;
    } else {
      ret[i] = u2p(G, uu + i * NVMAX, pp + i * NVMAX, geo, fixup[i]);
    }
  }
}

// one face value of each cell's stencil u[n][5] (cells i-2..i+2): PPM
// (order 2, widths dx[n][5]) gives both faces of cell i, MP5 (order 4) the
// right face of cell i
void hp_recon(long n, int order, const double *u, const double *dx, double *left, double *right) {
  for (long i = 0; i < n; i++) {
    const double *v = u + i * 5, *d = dx + i * 5;
    if (order == 2) {
      ppm(v[0], v[1], v[2], v[3], v[4], d[0], d[1], d[2], d[3], d[4], left[i], right[i]);
    } else {
      right[i] = mp5_face(v[0], v[1], v[2], v[3], v[4]);
      left[i] = mp5_face(v[4], v[3], v[2], v[1], v[0]);
    }
  }
}

// radiation: 0 p2u of the 13 variables (out uu[n][13]); 1 u2p_rad
// (pp in/out, status, corrected)
void hp_rad_cells(long n, int what, const kgpu_rad_params *rp, const double *uu, double *pp, const double *g,
                  const double *Gm, double *out, int *status, int *corrected) {
  const RadParams R = kgpu_rad_device_params(*rp);
  Grid G{};
  G.gamma = R.gamma;
  G.nv = NVMAX;
  for (long i = 0; i < n; i++) {
    RadGeom rg;
    rad_geom(g + i * 20, Gm + i * 20, rg);
    if (what == 0) {
      p2u_rad_full(G, pp + i * NVR, out + i * NVR, rg.g);
    } else {
      int c = 0;
      status[i] = u2p_rad(R, uu + i * NVR, pp + i * NVR, rg, c);
      corrected[i] = c;
    }
  }
}

// the implicit source solve of each cell, one cell after another as the
// one-thread-per-cell kernel runs it (kgpu_rad.cu k_rad_plain)
void hp_rad_implicit(long n, const kgpu_rad_params *rp, const double *uu, const double *pp, const double *g,
                     const double *Gm, const double *dt, double *pp_out, double *uu_out, int *status, int *attempt,
                     int *iters) {
  const RadParams R = kgpu_rad_device_params(*rp);
  Grid G{};
  G.gamma = R.gamma;
  G.nv = NVMAX;
  for (long k = 0; k < n; k++) {
    RadGeom rg;
    rad_geom(g + 20 * k, Gm + 20 * k, rg);
    const double *u0 = uu + k * NVR, *p0 = pp + k * NVR;
    ImpState s;
    imp_begin(R, p0, rg.g, s);
    int budget = 1 << 30;
    int r;
    while ((r = imp_advance(R, u0, p0, dt[k], rg, s, budget)) == IMP_RUNNING) {
    }
    if (r == IMP_DONE_OK) {
      p2u_rad_full(G, s.pp, uu_out + k * NVR, rg.g);
      for (int i = 0; i < NVR; i++) pp_out[k * NVR + i] = s.pp[i];
      status[k] = 0;
      attempt[k] = s.att;
      iters[k] = s.iter;
    } else {
      for (int i = 0; i < NVR; i++) {
        pp_out[k * NVR + i] = p0[i];
        uu_out[k * NVR + i] = u0[i];
      }
      status[k] = -1;
      attempt[k] = -1;
      iters[k] = 0;
    }
  }
}

}  // extern "C"
