// Learned warm start of the MHD inversion (u2p) on independent cells.
//
// KORAL's u2p (u2p.c:176-485) starts its Newton iteration on
// W = w gamma^2 from the primitives it is handed (u2p.c:2093-2112), and
// tries the energy equation first and the entropy equation when that
// fails.  Here the same network as the implicit solve's warm start
// (16 -> 128 -> 128 -> 8, BF16 tensor-core kernels in kgpu_mlp.cu) predicts
// from the conserved state, the guess and the metric (u2p_features in
// kgpu_mlp.cuh):
//   output 0  ln(W / W_guess), W the root the plain inversion converges to
//   output 1  a score (trained on 0/1) that the energy equation fails
// and the inversion starts from W_guess exp(output 0): with the energy
// equation unless the score says it fails, then the entropy equation; if
// neither converges from the prediction, the reference's inversion runs
// from the reference's guess (the fallback), so the set of cells that
// invert is never smaller than the reference's.  Every Newton step is the
// unchanged FP64 one and ends on the same residual test (U2PCONV).
//
// Without a prediction the kernel is the reference's u2p itself (the same
// function as kgpu_u2p_cells, same bits), with its Newton iterations
// counted.
#include <cuda_runtime.h>
#include <string.h>

#include "../../include/koral_b200.h"
#include "kgpu_mlp.cuh"

using namespace kgpu;

int kgpu_report_cuda(const char *what, cudaError_t e);

namespace {

#define WCK(call)                                              \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return kgpu_report_cuda(#call, e_); \
  } while (0)

struct U2PParams {
  double gamma, u2pconv, rhofloor;
};

__device__ inline void cell_geom(const double *g20, const double *G20, long i, Geom &g) {
  RadGeom rg;
  rad_geom(g20 + 20 * i, G20 + 20 * i, rg);
  g = rg.g;
}

__device__ inline Grid u2p_grid(const U2PParams &P) {
  Grid G;
  memset(&G, 0, sizeof(G));
  G.gamma = P.gamma;
  G.u2pconv = P.u2pconv;
  G.rhofloor = P.rhofloor;
  G.nv = NVMAX;
  return G;
}

// u2p_solver_W from a given initial W (the bracketing, Newton steps and
// final checks of u2p.c:2117-2292); counts Newton steps and W evaluations
__device__ int solve_from(const Grid &G, const double *uu, double *pp, const Geom &g, int Etype, double W,
                          unsigned &iters, unsigned &fevals) {
  U2PState s;
  u2p_setup(uu, g, s);
  if (u2p_bracket(G.gamma, Etype, s.c, W, &fevals)) return -150;
  int iter = 0;
  const int r = u2p_newton(G.gamma, G.u2pconv, Etype, s.c, W, iter, 1 << 30, 1 << 30, &fevals, 0u);
  iters += (unsigned)iter;
  if (r < 0) return r;
  return u2p_final(G.gamma, s, W, iter, uu, pp, g);
}

// u2p (u2p.c:176-485) with both solves started from W0 when W0 > 0, from
// the reference's guess (the primitives pp) otherwise; the same sequence
// of operations as kgpu::u2p when W0 <= 0
__device__ int u2p_counted(const Grid &G, const double *uu0, double *pp, const Geom &g, int &fixup, double W0,
                           bool skip_energy, unsigned &iters, unsigned &fevals) {
  double uu[NVMAX], ppbak[NVMAX];
  for (int iv = 0; iv < NVMAX; iv++) {
    uu[iv] = uu0[iv];
    ppbak[iv] = pp[iv];
  }
  int ret = 0, u2pret = -1;
  if (uu[0] / g.gdet < 0.) {
    pp[0] = G.rhofloor;
    uu[0] = G.rhofloor * g.gdet;
    ret = -2;
  }
  if (!skip_energy) u2pret = solve_from(G, uu, pp, g, 0, W0 > 0. ? W0 : u2p_initial_w(G.gamma, pp, g), iters, fevals);
  if (u2pret < 0) {
    ret = -1;
    // the reference's entropy solve reads its guess from pp again (which a
    // failed energy solve may have changed: u2p.c:2281-2293 writes the
    // primitives before the negative-density check)
    u2pret = solve_from(G, uu, pp, g, 1, W0 > 0. ? W0 : u2p_initial_w(G.gamma, pp, g), iters, fevals);
    if (u2pret < 0) ret = -2;
  }
  if (u2pret < 0) {
    ret = -3;
    for (int iv = 0; iv < NVMAX; iv++) pp[iv] = ppbak[iv];
  }
  fixup = (ret < -1) ? 1 : 0;
  return ret;
}

__global__ void k_u2p_warm_cells(U2PParams P, int n, int nv, const double *uu, double *pp, const double *g20,
                                 const double *G20, const float *ypred, float wgate, float sgate, int *status,
                                 int *fixup, int *iters, unsigned long long *stats) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned it = 0, fe = 0, fell = 0;
  if (i < n) {
    const Grid G = u2p_grid(P);
    Geom g;
    cell_geom(g20, G20, i, g);
    double u[NVMAX], p[NVMAX], p0[NVMAX];
    for (int iv = 0; iv < NVMAX; iv++) {
      u[iv] = uu[(long)i * nv + iv];
      p[iv] = p0[iv] = pp[(long)i * nv + iv];
    }
    int fix = 0, ret;
    if (!ypred) {
      ret = u2p_counted(G, u, p, g, fix, -1., false, it, fe);
    } else {
      const float *y = ypred + (long)i * MLP_OUTP;
      // a predicted change of W smaller than wgate is within the network's
      // own error: the guess's W is kept; the energy equation is skipped
      // where the score passes sgate
      const double W0 = fabsf(y[0]) >= wgate ? u2p_warm_w(G.gamma, p0, g, y[0]) : u2p_initial_w(G.gamma, p0, g);
      ret = W0 > 0. ? u2p_counted(G, u, p, g, fix, W0, y[1] > sgate, it, fe) : -3;
      if (ret < -1) {
        // fallback: the reference's inversion from the reference's guess
        fell = 1;
        for (int iv = 0; iv < NVMAX; iv++) p[iv] = p0[iv];
        ret = u2p_counted(G, u, p, g, fix, -1., false, it, fe);
      }
    }
    for (int iv = 0; iv < NVMAX; iv++) pp[(long)i * nv + iv] = p[iv];
    status[i] = ret;
    fixup[i] = fix;
    if (iters) iters[i] = (int)it;
  }
  if (stats) {
    // per-warp sums, one atomic per warp and counter
    unsigned long long a = it, b = fell, c = fe;
    for (int o = 16; o; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
      if (a) atomicAdd(&stats[0], a);
      if (b) atomicAdd(&stats[1], b);
      if (c) atomicAdd(&stats[2], c);
    }
  }
}

__global__ void k_u2p_features(U2PParams P, int n, int nv, const double *uu, const double *pp, const double *g20,
                               const double *G20, float *X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Geom g;
  cell_geom(g20, G20, i, g);
  float x[MLP_IN];
  u2p_features(P.gamma, uu + (long)i * nv, pp + (long)i * nv, g, x);
  for (int f = 0; f < MLP_IN; f++) X[(long)i * MLP_IN + f] = x[f];
}

__global__ void k_u2p_targets(U2PParams P, int n, int nv, const double *pp0, const double *pp1, const double *g20,
                              const double *G20, const int *status, float *T) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Geom g;
  cell_geom(g20, G20, i, g);
  double t[MLP_OUT];
  const bool ok = status[i] == 0 || status[i] == -1;
  u2p_targets(P.gamma, pp0 + (long)i * nv, pp1 + (long)i * nv, g, status[i], t);
  for (int o = 0; o < MLP_OUT; o++) T[(long)i * MLP_OUT + o] = ok ? (float)t[o] : __int_as_float(0x7fc00000);
}

bool params_of(const kgpu_config *cfg, int nv, U2PParams &P) {
  if (!cfg || nv < NVMAX) return false;
  if (!(cfg->gamma > 1.) || !(cfg->u2pconv > 0.)) return false;
  P.gamma = cfg->gamma;
  P.u2pconv = cfg->u2pconv;
  P.rhofloor = cfg->rhofloor;
  return true;
}

}  // namespace

extern "C" int kgpu_u2p_features_device(int n, const kgpu_config *cfg, int nv, const double *uu, const double *pp,
                                        const double *g, const double *G, float *X, void *stream) {
  U2PParams P;
  if (n < 0 || !params_of(cfg, nv, P) || (n > 0 && (!uu || !pp || !g || !G || !X))) return KGPU_EINVAL;
  if (n == 0) return 0;
  k_u2p_features<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(P, n, nv, uu, pp, g, G, X);
  WCK(cudaGetLastError());
  return 0;
}

extern "C" int kgpu_u2p_targets_device(int n, const kgpu_config *cfg, int nv, const double *pp, const double *pp1,
                                       const double *g, const double *G, const int *status, float *T,
                                       void *stream) {
  U2PParams P;
  if (n < 0 || !params_of(cfg, nv, P) || (n > 0 && (!pp || !pp1 || !g || !G || !status || !T))) return KGPU_EINVAL;
  if (n == 0) return 0;
  k_u2p_targets<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(P, n, nv, pp, pp1, g, G, status, T);
  WCK(cudaGetLastError());
  return 0;
}

extern "C" int kgpu_u2p_cells_device(int n, const kgpu_config *cfg, int nv, const double *uu, double *pp,
                                     const double *g, const double *G, const float *ypred, float wgate, float sgate,
                                     int *status, int *fixup, int *iters, void *stream, unsigned long long *stats,
                                     int nstats) {
  U2PParams P;
  if (n < 0 || !params_of(cfg, nv, P) || nstats < 0 || nstats > 3 || (nstats > 0 && !stats)) return KGPU_EINVAL;
  if (!(wgate >= 0.f) || !(sgate >= 0.f)) return KGPU_EINVAL;
  if (n > 0 && (!uu || !pp || !g || !G || !status || !fixup)) return KGPU_EINVAL;
  for (int k = 0; k < nstats; k++) stats[k] = 0;
  if (n == 0) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned long long *dstats = nullptr;
  if (nstats > 0) {
    WCK(cudaMallocAsync(&dstats, 3 * sizeof(unsigned long long), s));
    WCK(cudaMemsetAsync(dstats, 0, 3 * sizeof(unsigned long long), s));
  }
  k_u2p_warm_cells<<<(n + 127) / 128, 128, 0, s>>>(P, n, nv, uu, pp, g, G, ypred, wgate, sgate, status, fixup, iters,
                                                    dstats);
  cudaError_t e = cudaGetLastError();
  if (dstats) {
    unsigned long long h[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, dstats, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(dstats, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (int k = 0; k < nstats; k++) stats[k] = h[k];
  }
  WCK(e);
  return 0;
}
