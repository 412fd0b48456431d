// Kernels and C-ABI of the B200 implementation of KORAL's MHD hot path.
//
// Data layout in HBM: every cell array is structure-of-arrays,
// [variable][z][y][x] with KORAL's ghost padding, so that a warp reads 32
// consecutive x-cells of one variable in one coalesced transaction.  The
// metric tables are [component][point]; with an axisymmetric metric only one
// phi slice is stored, which keeps them L2-resident.
//
// One explicit operator (op_explicit, finite.c:646-1234) is four launches:
//   k_wavespeeds  cell speeds of loop_1 + the CFL maximum (atomic on bits)
//   k_flux<d>     per face: reconstruction of both sides, floors, fluxes,
//                 p2u of both states and the LLF/HLL combination, fused; the
//                 reference's face-state and one-sided-flux arrays never
//                 reach HBM
//   k_emf         corner EMFs of flux-CT (magn.c:199-297)
//   k_update      metric source terms and the unsplit update; the
//                 magnetic-field fluxes that flux_ct() rewrites are formed
//                 here directly from the EMFs (magn.c:300-337)
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/koral_b200.h"
#include "kgpu_rad.cuh"
#include "kgpu_setup.cuh"
#include "kgpu_diag.cuh"
#include "kgpu_avg.cuh"

using namespace kgpu;

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------
static thread_local char g_lasterr[256] = "";
static int set_err(const char *what, cudaError_t e) {
  snprintf(g_lasterr, sizeof(g_lasterr), "%s: %s", what, cudaGetErrorString(e));
  return KGPU_ECUDA;
}
#define CK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return set_err(#call, e_); \
  } while (0)
#define CKL(what)                                 \
  do {                                            \
    cudaError_t e_ = cudaGetLastError();          \
    if (e_ != cudaSuccess) return set_err(what, e_); \
  } while (0)

extern "C" const char *kgpu_last_error(void) { return g_lasterr; }
// for the other translation units of the library
int kgpu_report_cuda(const char *what, cudaError_t e) { return set_err(what, e); }
extern "C" int kgpu_abi_version(void) { return KGPU_ABI_VERSION; }

// ---------------------------------------------------------------------------
// launch geometry: a 3D index box flattened with x fastest
// ---------------------------------------------------------------------------
struct Box {
  int x0, y0, z0, nx, ny, nz;
  __host__ __device__ long n() const { return (long)nx * ny * nz; }
};
__device__ inline bool box_coord(const Box &b, long t, int &ix, int &iy, int &iz) {
  if (t >= (long)b.nx * b.ny * b.nz) return false;
  ix = b.x0 + (int)(t % b.nx);
  long r = t / b.nx;
  iy = b.y0 + (int)(r % b.ny);
  iz = b.z0 + (int)(r / b.ny);
  return true;
}
static inline unsigned nblocks(long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ inline bool in_domain(const Grid &G, int ix, int iy, int iz) {
  return ix >= 0 && ix < G.nx && iy >= 0 && iy < G.ny && iz >= 0 && iz < G.nz;
}
// finite.c:2641-2666: ghost cells that touch the domain through a face only
__device__ inline bool outside_gc(const Grid &G, int ix, int iy, int iz) {
  bool inx = ix >= 0 && ix < G.nx, iny = iy >= 0 && iy < G.ny, inz = iz >= 0 && iz < G.nz;
  return !((!inx && iny && inz) || (inx && !iny && inz) || (inx && iny && !inz) || (inx && iny && inz));
}

// every kernel carries the NVMAX MHD variables (kgpu_create rejects others)
__device__ inline void load_cell(const double *arr, long ncell, long c, double *v) {
#pragma unroll
  for (int iv = 0; iv < NVMAX; iv++) v[iv] = arr[iv * ncell + c];
}
__device__ inline void store_cell(double *arr, long ncell, long c, const double *v) {
#pragma unroll
  for (int iv = 0; iv < NVMAX; iv++) arr[iv * ncell + c] = v[iv];
}
// the four radiation variables (EE0..FZ0) of a 13-variable grid
__device__ inline void load_rad(const double *arr, long ncell, long c, double *v) {
#pragma unroll
  for (int iv = EE0; iv <= FZ0; iv++) v[iv] = arr[iv * ncell + c];
}
__device__ inline void store_rad(double *arr, long ncell, long c, const double *v) {
#pragma unroll
  for (int iv = EE0; iv <= FZ0; iv++) arr[iv * ncell + c] = v[iv];
}

// ---------------------------------------------------------------------------
// boundary conditions (set_bc, finite.c:2752-2803; set_bc_core 2673-2748)
// ---------------------------------------------------------------------------
__global__ void k_bc_faces(Grid G, Box b) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  if (in_domain(G, ix, iy, iz) || outside_gc(G, ix, iy, iz)) return;
  int d = (ix < 0 || ix >= G.nx) ? 0 : ((iy < 0 || iy >= G.ny) ? 1 : 2);
  int c3[3] = {ix, iy, iz}, n3[3] = {G.nx, G.ny, G.nz};
  int s3[3] = {ix, iy, iz};
  const int kind = G.bc[d];
  const int i = c3[d], n = n3[d];
  bool flip = false;
  if (kind == KGPU_BC_OUTFLOW) {
    s3[d] = i < 0 ? 0 : n - 1;
  } else if (kind == KGPU_BC_REFLECT) {
    s3[d] = i < 0 ? -i - 1 : 2 * n - i - 1;
    flip = true;
  } else {
    if (i < 0) s3[d] = i + n;
    if (i > n - 1) s3[d] = i - n;
    if (d > 0 && n < G.ng) s3[d] = 0;   // finite.c:2705, 2720
  }
  long c = cell_index(G, ix, iy, iz), s = cell_index(G, s3[0], s3[1], s3[2]);
  double pp[NVR], uu[NVR];
  load_cell(G.p, G.ncell, s, pp);
  if (G.rad) load_rad(G.p, G.ncell, s, pp);
  if (flip) {
    // the component normal to the boundary: VX/B1 for x, VY/B2 for y, VZ/B3
    // for z, and the radiation frame's FX0/FY0/FZ0
    pp[VX + d] = -pp[VX + d];
    pp[B1 + d] = -pp[B1 + d];
    if (G.rad) pp[FX0 + d] = -pp[FX0 + d];
  }
  if (kind == KGPU_BC_PERIODIC_COPY) {
    load_cell(G.u, G.ncell, s, uu);
    if (G.rad) load_rad(G.u, G.ncell, s, uu);
  } else {
    Geom g;
    geom_centre(G, ix, iy, iz, g);
    p2u_full(G, pp, uu, g);
    if (G.rad) p2u_rad(pp, uu, g);
  }
  store_cell(G.p, G.ncell, c, pp);
  store_cell(G.u, G.ncell, c, uu);
  if (G.rad) {
    store_rad(G.p, G.ncell, c, pp);
    store_rad(G.u, G.ncell, c, uu);
  }
}

// Corners of a 2D periodic domain, filled as the reference does
// (finite.c:3075-3328): the first NG-1 cells of the two edges next to each
// corner copy the adjacent edge ghost row/column, the diagonal cells take
// the periodic image (written there as the mean of two equal cells).
__device__ inline void corner2d_op(const Grid &G, int op, int &tx, int &ty, int &ax, int &ay, int &bx, int &by) {
  const int NX = G.nx, NY = G.ny, NG = G.ng;
  int per = 2 * NG;             // ops per corner
  int corner = op / per, k = op % per;
  // within a corner: k < 2(NG-1): copies (two per i); then the two diagonal cells
  if (k < 2 * (NG - 1)) {
    int i = k / 2, second = k % 2;
    switch (corner) {
      case 0:  // bottom-left
        if (!second) { tx = -NG + i; ty = -1; ax = bx = -NG + i; ay = by = 0; }
        else { tx = -1; ty = -NG + i; ax = bx = 0; ay = by = -NG + i; }
        break;
      case 1:  // top-left
        if (!second) { tx = -NG + i; ty = NY; ax = bx = -NG + i; ay = by = NY - 1; }
        else { tx = -1; ty = NY + i + 1; ax = bx = 0; ay = by = NY + i + 1; }
        break;
      case 2:  // bottom-right
        if (!second) { tx = NX + i + 1; ty = -1; ax = bx = NX + i + 1; ay = by = 0; }
        else { tx = NX; ty = -NG + i; ax = bx = NX - 1; ay = by = -NG + i; }
        break;
      default:  // top-right
        if (!second) { tx = NX + i + 1; ty = NY; ax = bx = NX + i + 1; ay = by = NY - 1; }
        else { tx = NX; ty = NY + i + 1; ax = bx = NX - 1; ay = by = NY + i + 1; }
        break;
    }
    return;
  }
  int j = k - 2 * (NG - 1);    // 0: first diagonal cell, 1: second
  switch (corner) {
    case 0: tx = -1 - j; ty = -1 - j; ax = bx = NX - 1 - j; ay = by = -1 - j; break;
    case 1: tx = -1 - j; ty = NY + j; ax = bx = NX - 1 - j; ay = by = NY + j; break;
    case 2: tx = NX + j; ty = -1 - j; ax = bx = 0 + j; ay = by = -1 - j; break;
    default: tx = NX + j; ty = NY + j; ax = bx = 0 + j; ay = by = NY + j; break;
  }
}
__global__ void k_bc_corners2d(Grid G) {
  int op = blockIdx.x * blockDim.x + threadIdx.x;
  if (op >= 8 * G.ng) return;
  int tx, ty, ax, ay, bx, by;
  corner2d_op(G, op, tx, ty, ax, ay, bx, by);
  int k = op % (2 * G.ng);
  bool avg = k >= 2 * (G.ng - 1);
  long ca = cell_index(G, ax, ay, 0), cb = cell_index(G, bx, by, 0), c = cell_index(G, tx, ty, 0);
  double pp[NVR], uu[NVR];
  const int nv = G.rad ? NVR : NVMAX;
  for (int iv = 0; iv < nv; iv++) {
    double a = G.p[iv * G.ncell + ca];
    pp[iv] = avg ? .5 * (a + G.p[iv * G.ncell + cb]) : a;
  }
  Geom g;
  geom_centre(G, tx, ty, 0, g);
  p2u_full(G, pp, uu, g);
  store_cell(G.p, G.ncell, c, pp);
  store_cell(G.u, G.ncell, c, uu);
  if (G.rad) {
    p2u_rad(pp, uu, g);
    store_rad(G.p, G.ncell, c, pp);
    store_rad(G.u, G.ncell, c, uu);
  }
}

// Edges and corners of a 3D domain with physical boundaries, in the
// reference's order (finite.c:3330-3705): edges elongated along z, then
// along y, then along x, each filling the first NG-1 cells of the two faces
// next to the edge from the adjacent ghost row and two diagonal cells as
// means of their neighbours; then the eight NG^3 corner blocks copy the
// nearest domain corner cell.  A pass reads only cells that earlier passes
// (or the face fill) wrote, so the lines of one pass run in parallel.
__device__ inline void set_from(const Grid &G, int tx, int ty, int tz, int s1x, int s1y, int s1z, int s2x, int s2y,
                                int s2z, bool avg) {
  long c = cell_index(G, tx, ty, tz), a = cell_index(G, s1x, s1y, s1z), b = cell_index(G, s2x, s2y, s2z);
  double pp[NVR], uu[NVR];
  const int nv = G.rad ? NVR : NVMAX;
  for (int iv = 0; iv < nv; iv++) {
    double va = G.p[iv * G.ncell + a];
    pp[iv] = avg ? .5 * (va + G.p[iv * G.ncell + b]) : va;
  }
  Geom g;
  geom_centre(G, tx, ty, tz, g);
  p2u_full(G, pp, uu, g);
  store_cell(G.p, G.ncell, c, pp);
  store_cell(G.u, G.ncell, c, uu);
  if (G.rad) {
    p2u_rad(pp, uu, g);
    store_rad(G.p, G.ncell, c, pp);
    store_rad(G.u, G.ncell, c, uu);
  }
}
// one line of one elongated-edge pass.  Edge axis c, the two other axes
// (a, b); corner k: bit 1 = high end of a, bit 0 = high end of b; position t
// along c in [-NG, N_c+NG).  In (a, b) coordinates, with the ghost layers
// counted outwards, the reference writes for i = 0..NG-2
//   lo,lo: (-NG+i,-1)<-(-NG+i,0)      (-1,-NG+i)<-(0,-NG+i)
//   lo,hi: (-NG+i,NB)<-(-NG+i,NB-1)   (-1,NB+i+1)<-(0,NB+i+1)
//   hi,lo: (NA,-NG+i)<-(NA-1,-NG+i)   (NA+i+1,-1)<-(NA+i+1,0)
//   hi,hi: (NA+i+1,NB)<-(NA+i+1,NB-1) (NA,NB+i+1)<-(NA-1,NB+i+1)
// and then the two diagonal cells as means of their inner neighbours.
// (x, y, z) of the cell at (va, vb) in the (a, b) plane and t along c;
// plain selects, no indexed local array
__device__ inline void at3(int c, int a, int b, int t, int va, int vb, int &x, int &y, int &z) {
  x = a == 0 ? va : (b == 0 ? vb : t);
  y = a == 1 ? va : (b == 1 ? vb : t);
  z = a == 2 ? va : (b == 2 ? vb : t);
  (void)c;
}
// target (ta, tb) and source (sa, sb) of copy j of ghost layer i
__device__ inline void edge_copy(bool hiA, bool hiB, int NG, int NA, int NB, int i, int j, int &ta, int &tb, int &sa,
                                 int &sb) {
  if (!hiA && !hiB) {
    if (j == 0) { ta = -NG + i; tb = -1; sa = -NG + i; sb = 0; }
    else { ta = -1; tb = -NG + i; sa = 0; sb = -NG + i; }
  } else if (!hiA && hiB) {
    if (j == 0) { ta = -NG + i; tb = NB; sa = -NG + i; sb = NB - 1; }
    else { ta = -1; tb = NB + i + 1; sa = 0; sb = NB + i + 1; }
  } else if (hiA && !hiB) {
    if (j == 0) { ta = NA; tb = -NG + i; sa = NA - 1; sb = -NG + i; }
    else { ta = NA + i + 1; tb = -1; sa = NA + i + 1; sb = 0; }
  } else {
    if (j == 0) { ta = NA + i + 1; tb = NB; sa = NA + i + 1; sb = NB - 1; }
    else { ta = NA; tb = NB + i + 1; sa = NA - 1; sb = NB + i + 1; }
  }
}
__global__ void k_bc_edges3d(Grid G, int c, int a, int b) {
  const int NG = G.ng;
  const int NA = a == 0 ? G.nx : (a == 1 ? G.ny : G.nz);
  const int NB = b == 0 ? G.nx : (b == 1 ? G.ny : G.nz);
  const int NC = c == 0 ? G.nx : (c == 1 ? G.ny : G.nz);
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  int len = NC + 2 * NG;
  if (tid >= 4 * len) return;
  const int k = tid / len, t = tid % len - NG;
  const bool hiA = (k >> 1) & 1, hiB = k & 1;
  int x, y, z, x1, y1, z1, x2, y2, z2;
  for (int i = 0; i < NG - 1; i++)
    for (int j = 0; j < 2; j++) {
      int ta, tb, sa, sb;
      edge_copy(hiA, hiB, NG, NA, NB, i, j, ta, tb, sa, sb);
      at3(c, a, b, t, ta, tb, x, y, z);
      at3(c, a, b, t, sa, sb, x1, y1, z1);
      set_from(G, x, y, z, x1, y1, z1, x1, y1, z1, false);
    }
  // diagonal cells: g1 = first ghost layer in both a and b, g2 = second;
  // mean of (g.a, g.b - sB) and (g.a - sA, g.b), s pointing out of the domain
  const int sA = hiA ? 1 : -1, sB = hiB ? 1 : -1;
  const int g1a = hiA ? NA : -1, g1b = hiB ? NB : -1;
  at3(c, a, b, t, g1a, g1b, x, y, z);
  at3(c, a, b, t, g1a, g1b - sB, x1, y1, z1);
  at3(c, a, b, t, g1a - sA, g1b, x2, y2, z2);
  set_from(G, x, y, z, x1, y1, z1, x2, y2, z2, true);
  const int g2a = g1a + sA, g2b = g1b + sB;
  at3(c, a, b, t, g2a, g2b, x, y, z);
  at3(c, a, b, t, g2a, g2b - sB, x1, y1, z1);
  at3(c, a, b, t, g2a - sA, g2b, x2, y2, z2);
  set_from(G, x, y, z, x1, y1, z1, x2, y2, z2, true);
}
__global__ void k_bc_corners3d(Grid G) {
  const int NG = G.ng;
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  int per = NG * NG * NG;
  if (tid >= 8 * per) return;
  int k = tid / per, r = tid % per;
  bool hx = k & 1, hy = (k >> 1) & 1, hz = (k >> 2) & 1;
  int ox = r % NG, oy = (r / NG) % NG, oz = r / (NG * NG);
  int tx = hx ? G.nx + ox : -NG + ox, ty = hy ? G.ny + oy : -NG + oy, tz = hz ? G.nz + oz : -NG + oz;
  int sx = hx ? G.nx - 1 : 0, sy = hy ? G.ny - 1 : 0, sz = hz ? G.nz - 1 : 0;
  set_from(G, tx, ty, tz, sx, sy, sz, sx, sy, sz, false);
}

// ---------------------------------------------------------------------------
// wavespeeds and the CFL reduction (calc_wavespeeds finite.c:567-599,
// save_wavespeeds 295-398)
// ---------------------------------------------------------------------------
__device__ inline void atomic_max_pos(double *addr, double v) {
  if (!(v == v)) return;   // NaN never wins, as with the reference's '>' test
  atomicMax((long long *)addr, __double_as_longlong(v));
}

__global__ void k_wavespeeds(Grid G, Box b) {
  int ix, iy, iz;
  double tsd = -1.;
  if (box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) {
    long c = cell_index(G, ix, iy, iz);
    double pp[NVR];
    load_cell(G.p, G.ncell, c, pp);
    Geom g;
    geom_centre(G, ix, iy, iz, g);
    double al[3], ar[3];
    wavespeeds(G, pp, g, al, ar);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      G.al[d][c] = al[d];
      G.ar[d][c] = ar[d];
    }
    double wsx = dmax(fabs(al[0]), fabs(ar[0]));
    double wsy = dmax(fabs(al[1]), fabs(ar[1]));
    double wsz = dmax(fabs(al[2]), fabs(ar[2]));
    if (G.rad) {
      // radiative characteristics (physics.c:170-197), stored apart for
      // the radiation fluxes; the time step takes the faster of the two
      load_rad(G.p, G.ncell, c, pp);
      double tau[3] = {0., 0., 0.};
      if (G.rad_limiter) {
        const int ic[3] = {ix, iy, iz};
        double lo[3], hi[3];
        for (int d = 0; d < 3; d++) {
          lo[d] = size_x(G, ic[d], d);
          hi[d] = size_x(G, ic[d] + 1, d);
        }
        rad_tautot(*G.radp, pp, g, lo, hi, tau);
      }
      double rl[3], rr[3];
      rad_wavespeeds(pp, g, tau, G.rad_limiter != 0, rl, rr);
      for (int d = 0; d < 3; d++) {
        G.arl[d][c] = rl[d];
        G.arr[d][c] = rr[d];
      }
      wsx = dmax(wsx, dmax(fabs(rl[0]), fabs(rr[0])));
      wsy = dmax(wsy, dmax(fabs(rl[1]), fabs(rr[1])));
      wsz = dmax(wsz, dmax(fabs(rl[2]), fabs(rr[2])));
    }
    if (in_domain(G, ix, iy, iz)) {
      double dx = size_x(G, ix, 0), dy = size_x(G, iy, 1), dz = size_x(G, iz, 2);
      double tstepden;
      if (G.nz > 1 && G.ny > 1) tstepden = wsx / dx + wsy / dy + wsz / dz;
      else if (G.nz == 1 && G.ny > 1) tstepden = wsx / dx + wsy / dy;
      else if (G.ny == 1 && G.nz > 1) tstepden = wsx / dx + wsz / dz;
      else tstepden = wsx / dx;
      tsd = tstepden / G.tsteplim;
    }
  }
  // warp-level maximum, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) {
    double other = __shfl_xor_sync(0xffffffffu, tsd, o);
    tsd = other > tsd ? other : tsd;
  }
  if ((threadIdx.x & 31) == 0 && tsd > 0.) atomic_max_pos(&G.scal[S_TSTEPDENMAX], tsd);
}

// ---------------------------------------------------------------------------
// fused face flux (finite.c:694-1014 and 1297-1624)
// ---------------------------------------------------------------------------
// Two threads per face, one per side: lane pair (2k, 2k+1) handles face k,
// the even lane the left state (right-face value of cell i-1), the odd lane
// the right state (left-face value of cell i).  Each lane reconstructs,
// floors and evaluates its own state; the pair then swaps fluxes and
// conserved values with shuffles and each lane stores every other variable.
// Per face the arithmetic is exactly that of the one-thread form.
// blocks per SM the face-flux, update and first inversion kernels are
// compiled for (registers per thread = 65536 / (128 x this)); they are
// FP64-latency bound, so occupancy is traded against spills (measured on the
// 192x96x64 torus, x faces: 0.66 ms at 4 blocks, 128 registers without DRAM
// spill traffic; 0.558 ms at 5 blocks, 96 registers; 0.538 ms at 6, 80
// registers; 0.525 ms at 7, 72 registers; 0.56 ms at 8 blocks, 64
// registers, whose spills then reach DRAM: 1.2 GB written per launch)
#ifndef KGPU_FLUX_MIN_BLOCKS
#define KGPU_FLUX_MIN_BLOCKS 7
#endif
#ifndef KGPU_UPDATE_MIN_BLOCKS
#define KGPU_UPDATE_MIN_BLOCKS 4
#endif
#ifndef KGPU_U2P_MIN_BLOCKS
#define KGPU_U2P_MIN_BLOCKS 5
#endif
// The face states of direction D (avg2point, finite.c:89-289) on their
// own: one thread per face of box b and variable, both sides (the left
// state is the right value of cell i-1, the right state the left value of
// cell i), stored [variable][face of the box] for k_flux<.., true>.  The
// same functions and operations as the reconstruction inside k_flux.
template <int D>
__global__ void __launch_bounds__(256) k_recon(Grid G, Box b, double *sl, double *sr) {
  const long nb = b.n();
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= nb * NVMAX) return;
  const int iv = (int)(t / nb);
  const long fi = t - (long)iv * nb;
  int ix, iy, iz;
  box_coord(b, fi, ix, iy, iz);
  const int i = D == 0 ? ix : (D == 1 ? iy : iz);
  const long stride = D == 0 ? 1 : (D == 1 ? (long)G.sx : (long)G.sx * G.sy);
  const long cR = cell_index(G, ix, iy, iz);
  const double *pv = G.p + iv * G.ncell + cR;
  double left, right;
  if (G.int_order == 4) {
    left = mp5_face(pv[-3 * stride], pv[-2 * stride], pv[-stride], pv[0], pv[stride]);
    right = mp5_face(pv[2 * stride], pv[stride], pv[0], pv[-stride], pv[-2 * stride]);
  } else {
    double dx[6];
#pragma unroll
    for (int k = 0; k < 6; k++) dx[k] = size_x(G, i - 3 + k, D);
    double ul, ur;
    ppm(pv[-3 * stride], pv[-2 * stride], pv[-stride], pv[0], pv[stride], dx[0], dx[1], dx[2], dx[3], dx[4], ul, ur);
    left = ur;
    ppm(pv[-2 * stride], pv[-stride], pv[0], pv[stride], pv[2 * stride], dx[1], dx[2], dx[3], dx[4], dx[5], ul, ur);
    right = ul;
  }
  sl[(long)iv * nb + fi] = left;
  sr[(long)iv * nb + fi] = right;
}

// The flux of face fi of box b, computed by the lane pair (side 0, side 1)
// of pairmask.  SPLIT: the face states come from k_recon (sl, sr) instead
// of being reconstructed here; the rest is the same.  DEFER: a face where
// either side's state needs the magnetic floor (magnetic pressure above
// B2RHORATIOMAX rho, u2p.c:617-671: a nested W inversion, rare and only in
// the magnetised funnel) is appended to G.fq[D] and left; k_flux_fix
// computes it, whole and with the same arithmetic, without DEFER.  The
// floor's inversion then no longer sets the register budget of the common
// path.
template <int D, bool SPLIT, bool DEFER>
__device__ __forceinline__ void face_flux(const Grid &G, const Box &b, const double *sl, const double *sr, long fi,
                                          int side, unsigned pairmask) {
  int ix, iy, iz;
  box_coord(b, fi, ix, iy, iz);
  constexpr int nv = NVMAX;
  const int i = D == 0 ? ix : (D == 1 ? iy : iz);
  const long stride = D == 0 ? 1 : (D == 1 ? (long)G.sx : (long)G.sx * G.sy);
  const long cR = cell_index(G, ix, iy, iz);     // cell i (right of the face)
  const long cL = cR - stride;                   // cell i-1

  // reconstruction (avg2point, finite.c:89-289) of this lane's side
  double ps[NVMAX];
  if (SPLIT) {
    const long nb = b.n();
    const double *src = side ? sr : sl;
#pragma unroll
    for (int iv = 0; iv < nv; iv++) ps[iv] = src[(long)iv * nb + fi];
  } else if (G.int_order == 4) {
    // left: MP5 centred on i-1 over cells i-3..i+1; right: centred on i,
    // stencil mirrored, cells i+2..i-2
    const long c0 = side ? cR + 2 * stride : cR - 3 * stride;
    const long st = side ? -stride : stride;
#pragma unroll
    for (int iv = 0; iv < nv; iv++) {
      const double *pv = G.p + iv * G.ncell + c0;
      ps[iv] = mp5_face(pv[0], pv[st], pv[2 * st], pv[3 * st], pv[4 * st]);
    }
  } else {
    // PPM of cell i-1 (its right value) or of cell i (its left value)
    const int i0 = i - 3 + side;
    double dx[5];
#pragma unroll
    for (int k = 0; k < 5; k++) dx[k] = size_x(G, i0 + k, D);
    const long c0 = cR + (side - 3) * stride;
#pragma unroll
    for (int iv = 0; iv < nv; iv++) {
      const double *pv = G.p + iv * G.ncell + c0;
      double ul, ur;
      ppm(pv[0], pv[stride], pv[2 * stride], pv[3 * stride], pv[4 * stride], dx[0], dx[1], dx[2], dx[3], dx[4], ul,
          ur);
      ps[iv] = side ? ul : ur;
    }
  }

  Geom g;
  geom_face(G, ix, iy, iz, D, g);
  // density floor of this face: x-faces sit at xb[ix], the others at x[ix]
  const double rfl = G.rhofl_c ? (D == 0 ? G.rhofl_f[ix + G.ng] : G.rhofl_c[ix + G.ng]) : -1.;
  double fs[NVMAX], us[NVMAX];
  {
    Kin k;
    bool kv;
    if (DEFER) {
      bool need = false;
      check_floors_mhd(G, ps, g, rfl, &k, &kv, &need);
      const bool pairneed = (__shfl_xor_sync(pairmask, (int)need, 1) | (int)need) != 0;
      const unsigned defer = __ballot_sync(pairmask, pairneed);
      if (pairneed) {
        // one queue slot per deferred face, taken by its side-0 lane; one
        // atomic per warp
        const unsigned app = defer & 0x55555555u;
        const int lane = (int)(threadIdx.x & 31), leader = __ffs(app) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(G.fqn + D, __popc(app));
        base = __shfl_sync(defer, base, leader);
        if (side == 0) G.fq[D][base + __popc(app & ((1u << lane) - 1u))] = (int)fi;
        return;
      }
      pairmask &= ~defer;
    } else {
      check_floors_mhd(G, ps, g, rfl, &k, &kv);
    }
    if (!kv) kinematics(ps, g, kMagn, k);
    flux_prime(G, ps, D, g, k, fs);
    p2u_mhd(G, ps, us, g, k);
  }
  double ap1l = G.al[D][cR], ap1r = G.ar[D][cR], am1l = G.al[D][cL], am1r = G.ar[D][cL];
  double ap1 = dmax(fabs(ap1l), fabs(ap1r)), am1 = dmax(fabs(am1l), fabs(am1r));
  double ag = dmax(ap1, am1);
  double al = dmin(ap1l, am1l);
  double ar = dmax(ap1r, am1r);
  const long f = face_index(G, ix, iy, iz, D);
  double *out = G.flb[D] + f;
  const long nf = G.nface[D];
#pragma unroll
  for (int iv = 0; iv < nv; iv++) {
    const double fo = __shfl_xor_sync(pairmask, fs[iv], 1);
    const double uo = __shfl_xor_sync(pairmask, us[iv], 1);
    const double fL = side ? fo : fs[iv], fR = side ? fs[iv] : fo;
    const double uL = side ? uo : us[iv], uR = side ? us[iv] : uo;
    if ((iv & 1) != side) continue;
    double fl;
    if (G.fluxmethod == 0) {
      fl = .5 * (fR + fL - ag * (uR - uL));
    } else {
      if (al > 0.) fl = fL;
      else if (ar < 0.) fl = fL;   // the reference takes the left flux here too (finite.c:1410)
      else fl = (-al * fR + ar * fL + al * ar * (uR - uL)) / (ar - al);
    }
    out[iv * nf] = fl;
  }
}

template <int D, int MB = KGPU_FLUX_MIN_BLOCKS, bool SPLIT = false>
__global__ void __launch_bounds__(128, MB) k_flux(Grid G, Box b, const double *sl, const double *sr) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const bool valid = t < 2 * b.n();
  const unsigned pairmask = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  face_flux<D, SPLIT, true>(G, b, sl, sr, t >> 1, (int)(t & 1), pairmask);
}

// The faces k_flux left to the magnetic floor: a lane pair per face, all
// registers the floor's inversion wants.  The loop runs warp-uniformly.
template <int D, bool SPLIT>
__global__ void __launch_bounds__(128) k_flux_fix(Grid G, Box b, const double *sl, const double *sr) {
  const int n = *(volatile int *)(G.fqn + D);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(G.cnt + C_FACE_FLOOR, (unsigned long long)n);
  const long warp = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  const int lane = (int)(threadIdx.x & 31);
  for (long base = warp * 16; base < n; base += nwarps * 16) {
    const long q = base + (lane >> 1);
    const unsigned pairmask = __ballot_sync(0xffffffffu, q < n);
    if (q < n) face_flux<D, SPLIT, false>(G, b, sl, sr, G.fq[D][q], lane & 1, pairmask);
  }
}

// Radiative face fluxes (the EE0..FZ0 part of the same face loop): the
// reference reconstructs all thirteen variables together, but nothing of
// the radiation flux depends on the gas state of the face (the face floors
// touch gas variables only, f_flux_prime_rad and the conserved variables
// of the Riemann solver read the radiation primitives and the metric), so
// the radiation runs as its own kernel with the same two-lane layout and
// its own characteristic speeds (f_calc_fluxes_at_faces, finite.c:1379-1395).
template <int D>
__global__ void __launch_bounds__(128) k_flux_rad(Grid G, Box b) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int side = (int)(t & 1);
  int ix, iy, iz;
  const bool valid = box_coord(b, t >> 1, ix, iy, iz);
  const unsigned pairmask = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  const int i = D == 0 ? ix : (D == 1 ? iy : iz);
  const long stride = D == 0 ? 1 : (D == 1 ? (long)G.sx : (long)G.sx * G.sy);
  const long cR = cell_index(G, ix, iy, iz);
  const long cL = cR - stride;
  double ps[NVR];
  if (G.int_order == 4) {
    const long c0 = side ? cR + 2 * stride : cR - 3 * stride;
    const long st = side ? -stride : stride;
#pragma unroll
    for (int iv = EE0; iv <= FZ0; iv++) {
      const double *pv = G.p + iv * G.ncell + c0;
      ps[iv] = mp5_face(pv[0], pv[st], pv[2 * st], pv[3 * st], pv[4 * st]);
    }
  } else {
    const int i0 = i - 3 + side;
    double dx[5];
#pragma unroll
    for (int k = 0; k < 5; k++) dx[k] = size_x(G, i0 + k, D);
    const long c0 = cR + (side - 3) * stride;
#pragma unroll
    for (int iv = EE0; iv <= FZ0; iv++) {
      const double *pv = G.p + iv * G.ncell + c0;
      double ul, ur;
      ppm(pv[0], pv[stride], pv[2 * stride], pv[3 * stride], pv[4 * stride], dx[0], dx[1], dx[2], dx[3], dx[4], ul,
          ur);
      ps[iv] = side ? ul : ur;
    }
  }
  Geom g;
  geom_face(G, ix, iy, iz, D, g);
  double fs[4], us[NVR];
  rad_flux(ps, D, g, fs);
  p2u_rad(ps, us, g);
  double ap1l = G.arl[D][cR], ap1r = G.arr[D][cR], am1l = G.arl[D][cL], am1r = G.arr[D][cL];
  double ap1 = dmax(fabs(ap1l), fabs(ap1r)), am1 = dmax(fabs(am1l), fabs(am1r));
  double ag = dmax(ap1, am1);
  double al = dmin(ap1l, am1l);
  double ar = dmax(ap1r, am1r);
  const long f = face_index(G, ix, iy, iz, D);
  double *out = G.flb[D] + f;
  const long nf = G.nface[D];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const double fo = __shfl_xor_sync(pairmask, fs[j], 1);
    const double uo = __shfl_xor_sync(pairmask, us[EE0 + j], 1);
    const double fL = side ? fo : fs[j], fR = side ? fs[j] : fo;
    const double uL = side ? uo : us[EE0 + j], uR = side ? us[EE0 + j] : uo;
    if ((j & 1) != side) continue;
    double fl;
    if (G.fluxmethod == 0) {
      fl = .5 * (fR + fL - ag * (uR - uL));
    } else {
      if (al > 0.) fl = fL;
      else if (ar < 0.) fl = fL;
      else fl = (-al * fR + ar * fL + al * ar * (uR - uL)) / (ar - al);
    }
    out[(EE0 + j) * nf] = fl;
  }
}

// zero fluxes outside the Riemann range (finite.c:1520, 1620): only needed
// for directions of size one, whose face fluxes the update reads
__global__ void k_zero_flux(Grid G, int d) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  long n = G.nface[d] * G.nv;
  if (t < n) G.flb[d][t] = 0.;
}

// ---------------------------------------------------------------------------
// flux-CT corner EMFs (magn.c:199-297)
// ---------------------------------------------------------------------------
struct Acc {
  double s;
  bool first;
  __device__ Acc() : s(0.), first(true) {}
  __device__ void add(double v, bool neg) {
    if (first) { s = neg ? -v : v; first = false; }
    else s = neg ? s - v : s + v;
  }
};

__global__ void k_emf(Grid G, Box b) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const int NX = G.nx, NY = G.ny, NZ = G.nz;
  const double *fx = G.flb[0], *fy = G.flb[1], *fz = G.flb[2];
  const long nfx = G.nface[0], nfy = G.nface[1], nfz = G.nface[2];
#define FXV(iv, a, b2, c) fx[(iv)*nfx + face_index(G, a, b2, c, 0)]
#define FYV(iv, a, b2, c) fy[(iv)*nfy + face_index(G, a, b2, c, 1)]
#define FZV(iv, a, b2, c) fz[(iv)*nfz + face_index(G, a, b2, c, 2)]
  const long ne = (long)(NX + 1) * (NY + 1) * (NZ + 1);
  const long e = emf_index(G, ix, iy, iz);
  double c1 = ((NY > 1) && (NZ > 1)) ? 0.25 : 0.5;
  double c2 = ((NX > 1) && (NZ > 1)) ? 0.25 : 0.5;
  double c3 = ((NX > 1) && (NY > 1)) ? 0.25 : 0.5;
  if ((NY > 1) || (NZ > 1)) {
    Acc a;
    if (NY > 1) { a.add(FYV(B3, ix, iy, iz), false); a.add(FYV(B3, ix, iy, iz - 1), false); }
    if (NZ > 1) { a.add(FZV(B2, ix, iy, iz), true); a.add(FZV(B2, ix, iy - 1, iz), true); }
    G.emf[0 * ne + e] = c1 * (a.s);
  } else G.emf[0 * ne + e] = 0.;
  if ((NX > 1) || (NZ > 1)) {
    Acc a;
    if (NZ > 1) { a.add(FZV(B1, ix, iy, iz), false); a.add(FZV(B1, ix - 1, iy, iz), false); }
    if (NX > 1) { a.add(FXV(B3, ix, iy, iz), true); a.add(FXV(B3, ix, iy, iz - 1), true); }
    G.emf[1 * ne + e] = c2 * (a.s);
  } else G.emf[1 * ne + e] = 0.;
  if ((NX > 1) || (NY > 1)) {
    Acc a;
    if (NX > 1) { a.add(FXV(B2, ix, iy, iz), false); a.add(FXV(B2, ix, iy - 1, iz), false); }
    if (NY > 1) { a.add(FYV(B1, ix, iy, iz), true); a.add(FYV(B1, ix - 1, iy, iz), true); }
    G.emf[2 * ne + e] = c3 * (a.s);
  } else G.emf[2 * ne + e] = 0.;
#undef FXV
#undef FYV
#undef FZV
}

// ---------------------------------------------------------------------------
// unsplit update with metric source terms (finite.c:1062-1160,
// f_metric_source_term_arb physics.c:324-465)
// ---------------------------------------------------------------------------
template <int MB = KGPU_UPDATE_MIN_BLOCKS>
__global__ void __launch_bounds__(128, MB) k_update(Grid G, Box b, const double *dtp, double fac,
                                                                        double *save) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  constexpr int nv = NVMAX;
  const long c = cell_index(G, ix, iy, iz);
  const double dt = fac * dtp[0];
  double pp[NVMAX];
  load_cell(G.p, G.ncell, c, pp);
  Geom g;
  geom_centre(G, ix, iy, iz, g);
  Kin k;
  kinematics(pp, g, nv > B3, k);
  // T^{mu nu} (calc_Tij) then T^mu_nu (indices_2221)
  double T[4][4];
  {
    double rho = pp[0], uu = pp[1];
    double pr = (G.gamma - 1.) * uu;
    double w = rho + uu + pr;
    double eta = w + k.bsq;
    double ptot = pr + 0.5 * k.bsq;
    double Tu[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int bb = 0; bb < 4; bb++) Tu[a][bb] = eta * k.ucon[a] * k.ucon[bb] + ptot * g.GG[a][bb] - k.bcon[a] * k.bcon[bb];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int bb = 0; bb < 4; bb++) {
        double s = 0.;
#pragma unroll
        for (int kk = 0; kk < 4; kk++) s += Tu[a][kk] * g.gg[kk][bb];
        T[a][bb] = s;
      }
  }
  double ms[NVMAX];
  for (int iv = 0; iv < nv; iv++) ms[iv] = 0.;
  {
    const long mi = met_index(G, ix, iy, iz);
    const double gdetu = g.gdet;
    double s1 = 0., s2 = 0., s3 = 0., s4 = 0.;
    for (int kk = 0; kk < 4; kk++)
      for (int l = 0; l < 4; l++) {
        double gt = gdetu * T[kk][l];
        const double *K = G.gkr + (long)(l * 16 + kk) * G.nmet + mi;
        s1 += gt * __ldg(K + 0 * 4 * G.nmet);
        s2 += gt * __ldg(K + 1 * 4 * G.nmet);
        s3 += gt * __ldg(K + 2 * 4 * G.nmet);
        s4 += gt * __ldg(K + 3 * 4 * G.nmet);
      }
    ms[1] = s1; ms[2] = s2; ms[3] = s3; ms[4] = s4;
  }
  const double dx = size_x(G, ix, 0), dy = size_x(G, iy, 1), dz = size_x(G, iz, 2);
  const long fxl = face_index(G, ix, iy, iz, 0), fxr = face_index(G, ix + 1, iy, iz, 0);
  const long fyl = face_index(G, ix, iy, iz, 1), fyr = face_index(G, ix, iy + 1, iz, 1);
  const long fzl = face_index(G, ix, iy, iz, 2), fzr = face_index(G, ix, iy, iz + 1, 2);
  const long ne = (long)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
#define EMFV(comp, a, b2, c2) G.emf[((comp)-1) * ne + emf_index(G, a, b2, c2)]
#pragma unroll
  for (int iv = 0; iv < nv; iv++) {
    double flxl = G.flb[0][iv * G.nface[0] + fxl], flxr = G.flb[0][iv * G.nface[0] + fxr];
    double flyl = G.flb[1][iv * G.nface[1] + fyl], flyr = G.flb[1][iv * G.nface[1] + fyr];
    double flzl = G.flb[2][iv * G.nface[2] + fzl], flzr = G.flb[2][iv * G.nface[2] + fzr];
    if (nv > B3 && iv >= B1) {
      // fluxes rewritten by flux_ct (magn.c:300-337)
      if (G.nx > 1) {
        if (iv == B1) { flxl = 0.; flxr = 0.; }
        if (iv == B2) {
          flxl = 0.5 * (EMFV(3, ix, iy, iz) + EMFV(3, ix, iy + 1, iz));
          flxr = 0.5 * (EMFV(3, ix + 1, iy, iz) + EMFV(3, ix + 1, iy + 1, iz));
        }
        if (iv == B3) {
          flxl = -0.5 * (EMFV(2, ix, iy, iz) + EMFV(2, ix, iy, iz + 1));
          flxr = -0.5 * (EMFV(2, ix + 1, iy, iz) + EMFV(2, ix + 1, iy, iz + 1));
        }
      }
      if (G.ny > 1) {
        if (iv == B1) {
          flyl = -0.5 * (EMFV(3, ix, iy, iz) + EMFV(3, ix + 1, iy, iz));
          flyr = -0.5 * (EMFV(3, ix, iy + 1, iz) + EMFV(3, ix + 1, iy + 1, iz));
        }
        if (iv == B2) { flyl = 0.; flyr = 0.; }
        if (iv == B3) {
          flyl = 0.5 * (EMFV(1, ix, iy, iz) + EMFV(1, ix, iy, iz + 1));
          flyr = 0.5 * (EMFV(1, ix, iy + 1, iz) + EMFV(1, ix, iy + 1, iz + 1));
        }
      }
      if (G.nz > 1) {
        if (iv == B1) {
          flzl = 0.5 * (EMFV(2, ix, iy, iz) + EMFV(2, ix + 1, iy, iz));
          flzr = 0.5 * (EMFV(2, ix, iy, iz + 1) + EMFV(2, ix + 1, iy, iz + 1));
        }
        if (iv == B2) {
          flzl = -0.5 * (EMFV(1, ix, iy, iz) + EMFV(1, ix, iy + 1, iz));
          flzr = -0.5 * (EMFV(1, ix, iy, iz + 1) + EMFV(1, ix, iy + 1, iz + 1));
        }
        if (iv == B3) { flzl = 0.; flzr = 0.; }
      }
    }
    double du = -(flxr - flxl) * dt / dx - (flyr - flyl) * dt / dy - (flzr - flzl) * dt / dz;
    double uold = G.u[iv * G.ncell + c];
    double val = uold + du + ms[iv] * dt;
    if (save) save[iv * G.ncell + c] = uold;
    G.u[iv * G.ncell + c] = val;
  }
#undef EMFV
}

// The radiation variables of the update (the same loop of finite.c:1062-1160
// over EE0..FZ0): flux divergence plus the radiative metric source
// gdet R^k_l Gamma^l_{jk} (f_metric_source_term_arb, physics.c:383-405).
__global__ void __launch_bounds__(128) k_update_rad(Grid G, Box b, const double *dtp, double fac) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  const double dt = fac * dtp[0];
  double pp[NVR];
  load_rad(G.p, G.ncell, c, pp);
  Geom g;
  geom_centre(G, ix, iy, iz, g);
  double Rl[4][4];
  rad_Rmixed(pp, g, Rl);
  double ms[4];
  {
    const long mi = met_index(G, ix, iy, iz);
    const double gdetu = g.gdet;
    double s0 = 0., s1 = 0., s2 = 0., s3 = 0.;
    for (int kk = 0; kk < 4; kk++)
      for (int l = 0; l < 4; l++) {
        double gt = gdetu * Rl[kk][l];
        const double *K = G.gkr + (long)(l * 16 + kk) * G.nmet + mi;
        s0 += gt * __ldg(K + 0 * 4 * G.nmet);
        s1 += gt * __ldg(K + 1 * 4 * G.nmet);
        s2 += gt * __ldg(K + 2 * 4 * G.nmet);
        s3 += gt * __ldg(K + 3 * 4 * G.nmet);
      }
    ms[0] = s0; ms[1] = s1; ms[2] = s2; ms[3] = s3;
  }
  const double dx = size_x(G, ix, 0), dy = size_x(G, iy, 1), dz = size_x(G, iz, 2);
  const long fxl = face_index(G, ix, iy, iz, 0), fxr = face_index(G, ix + 1, iy, iz, 0);
  const long fyl = face_index(G, ix, iy, iz, 1), fyr = face_index(G, ix, iy + 1, iz, 1);
  const long fzl = face_index(G, ix, iy, iz, 2), fzr = face_index(G, ix, iy, iz + 1, 2);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int iv = EE0 + j;
    double flxl = G.flb[0][iv * G.nface[0] + fxl], flxr = G.flb[0][iv * G.nface[0] + fxr];
    double flyl = G.flb[1][iv * G.nface[1] + fyl], flyr = G.flb[1][iv * G.nface[1] + fyr];
    double flzl = G.flb[2][iv * G.nface[2] + fzl], flzr = G.flb[2][iv * G.nface[2] + fzr];
    double du = -(flxr - flxl) * dt / dx - (flyr - flyl) * dt / dy - (flzr - flzl) * dt / dz;
    double uold = G.u[iv * G.ncell + c];
    G.u[iv * G.ncell + c] = uold + du + ms[j] * dt;
  }
}

// ---------------------------------------------------------------------------
// conserved -> primitives over the domain (calc_u2p finite.c:501-561,
// calc_primitives u2p.c:13-133) and neighbour-average fixups
// (cell_fixup finite.c:4467-4631)
// ---------------------------------------------------------------------------
// Warp-aggregated counter increment: one atomic per converged group of lanes.
__device__ inline void count_lanes(unsigned long long *ctr, bool pred) {
  const unsigned m = __activemask();
  const unsigned bits = __ballot_sync(m, pred);
  if (bits && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(ctr, (unsigned long long)__popc(bits));
}

// Floors, conserved from primitives and the stores that end a cell's
// inversion (calc_primitives u2p.c:82-127).
__device__ inline void u2p_finish(const Grid &G, long c, int ix, double *pp, double *uu, const Geom &g, int fix) {
  Kin k;
  bool kv;
  check_floors_mhd(G, pp, g, G.rhofl_c ? G.rhofl_c[ix + G.ng] : -1., &k, &kv);
  if (!kv) kinematics(pp, g, kMagn, k);
  p2u_mhd(G, pp, uu, g, k);
  store_cell(G.p, G.ncell, c, pp);
  store_cell(G.u, G.ncell, c, uu);
  G.flag[c] = fix;
}

// Warp-aggregated append to a work queue of box indices.
__device__ inline void queue_push(int *queue, int *qcount, bool pred, int item) {
  const unsigned m = __activemask();
  const unsigned bits = __ballot_sync(m, pred);
  if (!bits) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(qcount, __popc(bits));
  base = __shfl_sync(m, base, leader);
  if (pred) queue[base + __popc(bits & ((1u << lane) - 1u))] = item;
}

__device__ inline void count_sum(unsigned long long *ctr, unsigned v) {
  const unsigned m = __activemask();
  const unsigned sum = __reduce_add_sync(m, v);
  if (sum && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(ctr, (unsigned long long)sum);
}

// Queues of one inversion stage, reset by k_commit at the end of the stage.
struct U2PQueues {
  int *slow, *ent, *slow_ent;      // box indices
  int *n;                          // counts: [0] slow, [1] ent, [2] slow_ent
  double *w;                       // saved W of a paused solve, per cell
  int *it;                         // saved iteration count, per cell
};

// Cell state at the start of u2p (u2p.c:187-215): the conserved variables
// (with the negative-density fix applied by the caller), the primitive
// guess, the metric.
struct U2PCell {
  long c;
  int ix, iy, iz;
  bool negrho;
  double uc[NVMAX], pp[NVMAX];
  Geom g;
};

__device__ inline void u2p_load(const Grid &G, int ix, int iy, int iz, const double *guess, U2PCell &x) {
  x.ix = ix; x.iy = iy; x.iz = iz;
  x.c = cell_index(G, ix, iy, iz);
  load_cell(G.u, G.ncell, x.c, x.uc);
  load_cell(guess, G.ncell, x.c, x.pp);
  geom_centre(G, ix, iy, iz, x.g);
  x.negrho = x.uc[0] / x.g.gdet < 0.;
}

// u2p (u2p.c:176-485) as a sequence of passes over work queues, so that the
// few cells that need many Newton steps, heavy damping or the entropy
// fallback do not hold back whole warps:
//   k_u2p          energy equation, at most a few Newton steps and damping
//                  halvings per cell;
//   k_u2p_resume   continues the paused energy solves, one warp per cell;
//   k_u2p_entropy  entropy equation for the cells whose energy solve failed,
//                  with the same limits;
//   k_u2p_resume   continues the paused entropy solves.
// A paused solve keeps (W, iter) and resumes with exactly the steps it would
// have taken, so per cell the arithmetic is that of u2p.  A cell whose
// energy solve fails leaves its guess, as the solver left it, in pfix
// (free until the fixup pass).
__device__ inline void u2p_energy_done(const Grid &G, U2PQueues Q, int item, U2PCell &x, int r, int iter) {
  count_sum(&G.cnt[C_ITERS_HOT], (unsigned)iter);
  const bool failed = r < 0;
  queue_push(Q.ent, Q.n + 1, failed, item);
  count_lanes(&G.cnt[C_ENTQ], failed);
  if (failed) {
    store_cell(G.pfix, G.ncell, x.c, x.pp);
    return;
  }
  const int fix = x.negrho ? 1 : 0;   // u2p's status stays -2 after a negative density
  count_lanes(&G.cnt[C_FIXUP], fix != 0);
  double uo[NVMAX];
  u2p_finish(G, x.c, x.ix, x.pp, uo, x.g, fix);
}

__device__ inline void u2p_entropy_done(const Grid &G, U2PCell &x, int r, int iter) {
  count_sum(&G.cnt[C_ITERS_ENT], (unsigned)iter);
  int ret = -1;
  if (r < 0) {
    ret = -3;   // -2 from the entropy failure, then -3: old primitives kept
    load_cell(G.p, G.ncell, x.c, x.pp);
  }
  count_lanes(&G.cnt[C_ENTROPY], ret == -1);
  count_lanes(&G.cnt[C_FAIL], ret == -3);
  const int fix = ret < -1 ? 1 : 0;
  count_lanes(&G.cnt[C_FIXUP], fix != 0);
  double uo[NVMAX];
  u2p_finish(G, x.c, x.ix, x.pp, uo, x.g, fix);
}

// Damped-step halvings a first-pass solve may need before it is paused and
// left to the warp-cooperative resumption pass.
constexpr int U2P_DAMP_BUDGET = 4;

// One solve of the given equation from its start (paused after `stop`
// Newton steps or at the damping budget).  Returns U2P_PAUSED, 0
// (primitives in x.pp) or a negative status.
__device__ inline int u2p_run(const Grid &G, int Etype, U2PCell &x, int stop, double &W, int &iter) {
  U2PState st;
  u2p_setup(x.uc, x.g, st);
  W = u2p_initial_w(G.gamma, x.pp, x.g);
  iter = 0;
  if (u2p_bracket(G.gamma, Etype, st.c, W)) return -150;
  int r = u2p_newton(G.gamma, G.u2pconv, Etype, st.c, W, iter, stop, U2P_DAMP_BUDGET);
  if (r) return r;
  return u2p_final(G.gamma, st, W, iter, x.uc, x.pp, x.g);
}

template <int MB = KGPU_U2P_MIN_BLOCKS>
__global__ void __launch_bounds__(128, MB) k_u2p(Grid G, Box b, U2PQueues Q, int stop) {
  int ix, iy, iz;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (!box_coord(b, t, ix, iy, iz)) return;
  if (polar_cell(G, iy)) {
    // a corrected polar cell: only its field is inverted (u2p_solver_Bonly,
    // u2p.c:2356-2377), no floors, no fixup, conserved state as it is
    // (calc_primitives, u2p.c:49-101)
    const long c = cell_index(G, ix, iy, iz);
    const double gdet = G.met_c[(long)(3 * 5 + 4) * G.nmet + met_index(G, ix, iy, iz)];
    for (int iv = B1; iv <= B3; iv++) G.p[iv * G.ncell + c] = G.u[iv * G.ncell + c] / gdet;
    G.flag[c] = 0;
    return;
  }
  U2PCell x;
  u2p_load(G, ix, iy, iz, G.p, x);
  if (x.negrho) {
    x.pp[0] = G.rhofloor;
    x.uc[0] = G.rhofloor * x.g.gdet;
  }
  count_lanes(&G.cnt[C_NEGRHO], x.negrho);
  double W;
  int iter;
  const int r = u2p_run(G, 0, x, stop, W, iter);
  const bool paused = r == U2P_PAUSED;
  queue_push(Q.slow, Q.n + 0, paused, (int)t);
  count_lanes(&G.cnt[C_SLOW], paused);
  if (paused) {
    Q.w[x.c] = W;
    Q.it[x.c] = iter;
    return;
  }
  u2p_energy_done(G, Q, (int)t, x, r, iter);
}

// Paused solves, one warp per cell (Etype 0: energy, 1: entropy).  All
// lanes carry the cell; lane 0 writes the outcome.
__global__ void __launch_bounds__(128) k_u2p_resume(Grid G, Box b, U2PQueues Q, int Etype) {
  const int n = Q.n[Etype == 0 ? 0 : 2];
  const int *queue = Etype == 0 ? Q.slow : Q.slow_ent;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < n; q += nwarps) {
    int ix, iy, iz;
    const int item = queue[q];
    box_coord(b, item, ix, iy, iz);
    U2PCell x;
    u2p_load(G, ix, iy, iz, Etype == 0 ? G.p : G.pfix, x);
    if (x.negrho) {
      if (Etype == 0) x.pp[0] = G.rhofloor;
      x.uc[0] = G.rhofloor * x.g.gdet;
    }
    U2PState st;
    u2p_setup(x.uc, x.g, st);
    double W = Q.w[x.c];
    int iter = Q.it[x.c];
    int r = u2p_newton_warp(G.gamma, G.u2pconv, Etype, st.c, W, iter);
    if (r == 0) r = u2p_final(G.gamma, st, W, iter, x.uc, x.pp, x.g);
    if (lane == 0) {
      if (Etype == 0) u2p_energy_done(G, Q, item, x, r, iter);
      else u2p_entropy_done(G, x, r, iter);
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(128) k_u2p_entropy(Grid G, Box b, U2PQueues Q, int stop) {
  const int n = Q.n[1];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    const int item = Q.ent[q];
    box_coord(b, item, ix, iy, iz);
    U2PCell x;
    u2p_load(G, ix, iy, iz, G.pfix, x);
    if (x.negrho) x.uc[0] = G.rhofloor * x.g.gdet;
    double W;
    int iter;
    const int r = u2p_run(G, 1, x, stop, W, iter);
    const bool paused = r == U2P_PAUSED;
    queue_push(Q.slow_ent, Q.n + 2, paused, item);
    if (paused) {
      Q.w[x.c] = W;
      Q.it[x.c] = iter;
      continue;
    }
    u2p_entropy_done(G, x, r, iter);
  }
}

// The radiation part of calc_primitives (u2p.c:13-133, with u2p_rad called
// from u2p, u2p.c:432): after the MHD inversion and its floors, the M1
// inversion of the radiation conserved variables, the radiation floors
// (which may raise the density or the gas energy) and the conserved
// variables of the final primitives.  Runs after the MHD passes and before
// the neighbour fixup, whose averages read these primitives.  The U2PRAD
// fixup the reference then requests changes no data (cell_fixup,
// finite.c:4599-4604, stores only the first NVMHD variables, and those
// were not averaged for this kind), so a correction is only counted.
__global__ void __launch_bounds__(128) k_u2p_rad(Grid G, Box b) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  if (polar_cell(G, iy)) return;   // corrected polar cells: field only (u2p.c:49-101)
  const long c = cell_index(G, ix, iy, iz);
  double uu[NVR], pp[NVR];
  load_rad(G.u, G.ncell, c, uu);
  load_cell(G.p, G.ncell, c, pp);
  load_rad(G.p, G.ncell, c, pp);
  RadGeom rg;
  geom_centre(G, ix, iy, iz, rg.g);
  rg.alpha = sqrt(-1. / rg.g.GG[0][0]);
  const RadParams &R = *G.radp;
  int corr = 0;
  u2p_rad(R, uu, pp, rg, corr);
  count_lanes(&G.cnt[C_RADCOR], corr != 0);
  const double rho0 = pp[RHO], u0 = pp[UU];
  const int fl = check_floors_rad(R, pp, rg.g);
  count_lanes(&G.cnt[C_RADFLOOR], fl < 0);
  if (pp[RHO] != rho0 || pp[UU] != u0) {
    double um[NVMAX];
    p2u_full(G, pp, um, rg.g);
    store_cell(G.p, G.ncell, c, pp);
    store_cell(G.u, G.ncell, c, um);
  }
  p2u_rad(pp, uu, rg.g);
  store_rad(G.p, G.ncell, c, pp);
  store_rad(G.u, G.ncell, c, uu);
}

// ---------------------------------------------------------------------------
// implicit radiation source step over the domain (op_implicit,
// finite.c:1242-1292): the domain cells are gathered into the batched
// solver's cell-major arrays, solved, and scattered back; cells where every
// attempt failed keep their state and get the RADIMP neighbour fixup.
// ---------------------------------------------------------------------------
// metric of each domain cell, 20 + 20 doubles (done once per metric)
__global__ void k_imp_pack_metric(Grid G, Box b, double *g20, double *G20) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  int ix, iy, iz;
  if (!box_coord(b, k, ix, iy, iz)) return;
  const long mi = met_index(G, ix, iy, iz);
  for (int a = 0; a < 20; a++) {
    g20[k * 20 + a] = G.met_c[(long)a * G.nmet + mi];
    G20[k * 20 + a] = G.met_c[(long)(20 + a) * G.nmet + mi];
  }
}
// conserved state after the explicit part, primitive guess and time step
// (solve_implicit_lab, rad.c:1230-1260; implicit_lab_rad_source_term is
// called with dt times the unit multi-step multiplier)
__global__ void k_imp_gather(Grid G, Box b, const double *dtp, double fac, double *uu, double *pp, double *dt) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  int ix, iy, iz;
  if (!box_coord(b, k, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
#pragma unroll
  for (int iv = 0; iv < NVR; iv++) {
    uu[k * NVR + iv] = G.u[iv * G.ncell + c];
    pp[k * NVR + iv] = G.p[iv * G.ncell + c];
  }
  dt[k] = (dtp[0] * fac) * 1.;
}
__global__ void k_imp_scatter(Grid G, Box b, const double *pp, const double *uu, const int *status) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  int ix, iy, iz;
  if (!box_coord(b, k, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  if (polar_cell(G, iy)) {   // op_implicit skips corrected polar cells (finite.c:1270-1272)
    G.flag[c] = 0;
    return;
  }
  const bool ok = status[k] == 0;
  count_lanes(&G.cnt[C_RADIMP_FAIL], !ok);
  count_lanes(&G.cnt[C_IMP_SOLVES], true);
  G.flag[c] = ok ? 0 : 1;
  if (!ok) return;
#pragma unroll
  for (int iv = 0; iv < NVR; iv++) {
    G.p[iv * G.ncell + c] = pp[k * NVR + iv];
    G.u[iv * G.ncell + c] = uu[k * NVR + iv];
  }
}

// ---------------------------------------------------------------------------
// RK2IMEX combinations over the domain, all thirteen variables, each in the
// reference's operation order (ko.c:444-570)
// ---------------------------------------------------------------------------
// d = (1/(dt f)) u + (-1/(dt f)) base; optionally copy = u
__global__ void k_imex_rate(Grid G, Box b, const double *dtp, double f, const double *base, double *d, double *copy) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  const double dtcell = dtp[0];
  const double a = 1. / (dtcell * f), m = -1. / (dtcell * f);
  for (int iv = 0; iv < NVR; iv++) {
    const long i = iv * G.ncell + c;
    const double u = G.u[i];
    d[i] = a * u + m * base[i];
    if (copy) copy[i] = 1. * u;
  }
}
// dut1 = (1/dt) u + (-1/dt) ut1, then u = ut0 + dt dut1 + dt (1 - 2 gamma) drt1,
// and the copy of the new u that the second implicit stage starts from
__global__ void k_imex_stage1(Grid G, Box b, const double *dtp, double gam, const double *ut0, const double *ut1,
                              double *dut1, const double *drt1, double *copy) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  const double dtcell = dtp[0];
  for (int iv = 0; iv < NVR; iv++) {
    const long i = iv * G.ncell + c;
    const double d = (1. / (dtcell)) * G.u[i] + (-1. / (dtcell)) * ut1[i];
    dut1[i] = d;
    const double un = ut0[i] + (dtcell) * d + (dtcell * (1. - 2. * gam)) * drt1[i];
    G.u[i] = un;
    copy[i] = 1. * un;
  }
}
// dut2 = (1/dt) u + (-1/dt) ut2; u = ut0 + dt/2 dut1 + dt/2 dut2, then
// u += dt/2 drt1 + dt/2 drt2
__global__ void k_imex_final(Grid G, Box b, const double *dtp, const double *ut0, const double *ut2,
                             const double *dut1, const double *drt1, const double *drt2) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  const double dtcell = dtp[0];
  for (int iv = 0; iv < NVR; iv++) {
    const long i = iv * G.ncell + c;
    const double dut2 = (1. / (dtcell)) * G.u[i] + (-1. / (dtcell)) * ut2[i];
    const double ue = ut0[i] + (dtcell / 2.) * dut1[i] + (dtcell / 2.) * dut2;
    G.u[i] = ue + (dtcell / 2.) * drt1[i] + (dtcell / 2.) * drt2[i];
  }
}

// The reference visits cells in loop_0 order (x outer, z inner) and clears
// each flag as it goes, so a neighbour that precedes the cell in that order
// always counts as good, one that follows counts when its own inversion
// succeeded.  Neighbour values are the post-inversion primitives.
__global__ void k_fixup(Grid G, Box b, int *fixmark) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  if (G.flag[c] == 0) return;
  const int NX = G.nx, NY = G.ny, NZ = G.nz;
  constexpr int nv = NVMAX;
  int nb[6][3] = {{ix - 1, iy, iz}, {ix + 1, iy, iz}, {ix, iy - 1, iz}, {ix, iy + 1, iz}, {ix, iy, iz - 1}, {ix, iy, iz + 1}};
  bool inr[6] = {ix - 1 >= 0, ix + 1 < NX, iy - 1 >= 0, iy + 1 < NY, iz - 1 >= 0, iz + 1 < NZ};
  bool before[6] = {true, false, true, false, true, false};
  int in = 0;
  long nbc[6];
  for (int k = 0; k < 6; k++) {
    if (!inr[k]) continue;
    long n = cell_index(G, nb[k][0], nb[k][1], nb[k][2]);
    if (before[k] || G.flag[n] == 0) nbc[in++] = n;
  }
  fixmark[c] = 0;
  if (!((NZ == 1 && NY == 1 && in >= 1) || (NZ == 1 && in >= 2) || (NY == 1 && in >= 2) || in >= 3)) return;
  double pp[NVMAX], uu[NVMAX];
  for (int iv = 0; iv < nv; iv++) {
    if (iv != RHO && iv < B1) {
      double s = 0.;
      for (int k = 0; k < in; k++) s += G.p[iv * G.ncell + nbc[k]];
      pp[iv] = s / (double)in;
    } else
      pp[iv] = G.p[iv * G.ncell + c];
  }
  Geom g;
  geom_centre(G, ix, iy, iz, g);
  p2u_full(G, pp, uu, g);
  store_cell(G.pfix, G.ncell, c, pp);
  store_cell(G.ufix, G.ncell, c, uu);
  fixmark[c] = 1;
}

// apply fixups; optionally finish an RK2 step: u = ut0 + (u - ut1)
// (addi_u pair of ko.c:614-615)
__global__ void k_commit(Grid G, Box b, const int *fixmark, int combine, int *qcount) {
  if (blockIdx.x == 0 && threadIdx.x < 3) qcount[threadIdx.x] = 0;   // the inversion queues of this stage are spent
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  constexpr int nv = NVMAX;
  if (G.flag[c] != 0) {
    if (fixmark[c]) {
      for (int iv = 0; iv < nv; iv++) {
        G.p[iv * G.ncell + c] = G.pfix[iv * G.ncell + c];
        G.u[iv * G.ncell + c] = G.ufix[iv * G.ncell + c];
      }
    }
    G.flag[c] = 0;
  }
  if (combine) {
    for (int iv = 0; iv < nv; iv++) {
      long i = iv * G.ncell + c;
      double ut2 = 1. * G.u[i] + (-1.) * G.ut1[i];
      G.u[i] = 1. * G.ut0[i] + 1. * ut2;
    }
  }
}

__global__ void k_begin_step(Grid G) {
  G.scal[S_DT] = 1. / G.scal[S_TSTEPDENMAX];
  G.scal[S_TSTEPDENMAX] = -1.;
}

// copyi_u, addi_u, addi_u_3 (finite.c:2492-2620): domain cells, all NV
// variables, the reference's products and sums in its order
__global__ void k_copy_domain(Grid G, Box b, double f, const double *src, double *dst) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  long c = cell_index(G, ix, iy, iz);
  for (int iv = 0; iv < G.nv; iv++) dst[iv * G.ncell + c] = f * src[iv * G.ncell + c];
}
__global__ void k_add_domain(Grid G, Box b, double f1, const double *a, double f2, const double *bb, double *c3) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  long c = cell_index(G, ix, iy, iz);
  for (int iv = 0; iv < G.nv; iv++) c3[iv * G.ncell + c] = f1 * a[iv * G.ncell + c] + f2 * bb[iv * G.ncell + c];
}
__global__ void k_add3_domain(Grid G, Box b, double f1, const double *a, double f2, const double *bb, double f3,
                              const double *cc, double *d4) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  long c = cell_index(G, ix, iy, iz);
  for (int iv = 0; iv < G.nv; iv++) {
    const long i = iv * G.ncell + c;
    d4[i] = f1 * a[i] + f2 * bb[i] + f3 * cc[i];
  }
}

// The second half of flux_ct (magn.c:297-337): the magnetic components of
// the face fluxes rewritten from the corner EMFs, over the corner box
// (loop_4: 0..NX x 0..NY x 0..NZ).  op_explicit applies the same values
// inside k_update without storing them; this kernel stores them in the
// face-flux arrays, as the reference leaves its flbx/flby/flbz.
__global__ void k_flux_ct_rewrite(Grid G, Box b) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const int NX = G.nx, NY = G.ny, NZ = G.nz;
  const long ne = (long)(NX + 1) * (NY + 1) * (NZ + 1);
#define EMFV(comp, a, b2, c2) G.emf[((comp)-1) * ne + emf_index(G, a, b2, c2)]
  if (NX > 1 && iy < NY && iz < NZ) {
    double *f = G.flb[0];
    const long n = G.nface[0], i = face_index(G, ix, iy, iz, 0);
    f[B1 * n + i] = 0.;
    f[B2 * n + i] = 0.5 * (EMFV(3, ix, iy, iz) + EMFV(3, ix, iy + 1, iz));
    f[B3 * n + i] = -0.5 * (EMFV(2, ix, iy, iz) + EMFV(2, ix, iy, iz + 1));
  }
  if (NY > 1 && ix < NX && iz < NZ) {
    double *f = G.flb[1];
    const long n = G.nface[1], i = face_index(G, ix, iy, iz, 1);
    f[B1 * n + i] = -0.5 * (EMFV(3, ix, iy, iz) + EMFV(3, ix + 1, iy, iz));
    f[B2 * n + i] = 0.;
    f[B3 * n + i] = 0.5 * (EMFV(1, ix, iy, iz) + EMFV(1, ix, iy, iz + 1));
  }
  if (NZ > 1 && ix < NX && iy < NY) {
    double *f = G.flb[2];
    const long n = G.nface[2], i = face_index(G, ix, iy, iz, 2);
    f[B1 * n + i] = 0.5 * (EMFV(2, ix, iy, iz) + EMFV(2, ix + 1, iy, iz));
    f[B2 * n + i] = -0.5 * (EMFV(1, ix, iy, iz) + EMFV(1, ix, iy + 1, iz));
    f[B3 * n + i] = 0.;
  }
#undef EMFV
}

// ---------------------------------------------------------------------------
// polar-axis corrections (do_correct, finite.c:605-640)
// ---------------------------------------------------------------------------
// cell-centre code coordinate along d (set_x of set_grid, finite.c:1646-1664)
__device__ inline double centre_x(const Grid &G, int ic, int d) {
  return .5 * (G.xb[d][ic + 1 + G.ng] + G.xb[d][ic + G.ng]);
}
// writes pp and its conserved state into cell c except the magnetic field
__device__ inline void polar_store(const Grid &G, long c, const double *pp, const Geom &g) {
  double uu[NVR];
  if (G.rad) p2u_rad_full(G, pp, uu, g);
  else p2u_full(G, pp, uu, g);
  for (int iv = 0; iv < G.nv; iv++) {
    if (iv >= B1 && iv <= B3) continue;   // the field is not overwritten
    G.p[iv * G.ncell + c] = pp[iv];
    G.u[iv * G.ncell + c] = uu[iv];
  }
}
// correct_polaraxis (finite.c:4923-5166, spherical-like coordinates;
// mode 1) and correct_polaraxis_3d without POLARAXISAVGIN3D
// (finite.c:5170-5474; mode 2): each of the nc most polar cells of a
// column takes its state from the cell nc rows from the axis; mode 1 scales
// the theta velocities by the distance from the axis.  One thread per
// (ix, iz, ic, side); the source cells are not written.
__global__ void k_correct_polar(Grid G, int nc, int mode) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long n = (long)G.nx * G.nz * nc * 2;
  if (t >= n) return;
  const int ix = (int)(t % G.nx);
  long r = t / G.nx;
  const int iz = (int)(r % G.nz);
  r /= G.nz;
  const int ic = (int)(r % nc);
  const int lower = (int)(r / nc);
  const int iy = lower ? G.ny - 1 - ic : ic;
  const int iysrc = lower ? G.ny - 1 - nc : nc;
  const long c = cell_index(G, ix, iy, iz), cs = cell_index(G, ix, iysrc, iz);
  Geom g;
  geom_centre(G, ix, iy, iz, g);
  double pp[NVR];
  if (mode == 2) {
    for (int iv = 0; iv < G.nv; iv++) pp[iv] = G.p[iv * G.ncell + cs];
  } else {
    const double thaxis = G.xb[1][(lower ? G.ny : 0) + G.ng];
    const double th = centre_x(G, iy, 1), thsrc = centre_x(G, iysrc, 1);
    for (int iv = 0; iv < G.nv; iv++) pp[iv] = G.p[iv * G.ncell + c];
    const double f = fabs((th - thaxis) / (thsrc - thaxis));
    pp[RHO] = G.p[RHO * G.ncell + cs];
    pp[UU] = G.p[UU * G.ncell + cs];
    pp[ENTR] = G.p[ENTR * G.ncell + cs];
    pp[VX] = G.p[VX * G.ncell + cs];
    pp[VZ] = G.p[VZ * G.ncell + cs];
    pp[VY] = f * G.p[VY * G.ncell + cs];
    if (G.rad) {
      pp[EE0] = G.p[EE0 * G.ncell + cs];
      pp[FX0] = G.p[FX0 * G.ncell + cs];
      pp[FZ0] = G.p[FZ0 * G.ncell + cs];
      pp[FY0] = f * G.p[FY0 * G.ncell + cs];
    }
  }
  polar_store(G, c, pp, g);
}
// smooth_polaraxis (finite.c:4832-4921): each of the nc most polar rows
// takes, in every cell, the phi average of the row (summed in phi order),
// with the cell's own magnetic field.  One thread per (ix, ic, side), so
// the row is read in full before it is written.
__global__ void k_smooth_polar(Grid G, int nc) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)G.nx * nc * 2) return;
  const int ix = (int)(t % G.nx);
  const int ic = (int)((t / G.nx) % nc);
  const int lower = (int)(t / ((long)G.nx * nc));
  const int iy = lower ? G.ny - 1 - ic : ic;
  double pp[NVR];
  for (int iv = 0; iv < G.nv; iv++) pp[iv] = 0.;
  for (int iz = 0; iz < G.nz; iz++) {
    const long c = cell_index(G, ix, iy, iz);
    for (int iv = 0; iv < G.nv; iv++) pp[iv] += G.p[iv * G.ncell + c];
  }
  for (int iv = 0; iv < G.nv; iv++) pp[iv] /= G.nz;
  for (int iz = 0; iz < G.nz; iz++) {
    const long c = cell_index(G, ix, iy, iz);
    Geom g;
    geom_centre(G, ix, iy, iz, g);
    pp[B1] = G.p[B1 * G.ncell + c];
    pp[B2] = G.p[B2 * G.ncell + c];
    pp[B3] = G.p[B3 * G.ncell + c];
    polar_store(G, c, pp, g);
  }
}
// adjust_fluxcttoth_emfs (magn.c:343-376, CORRECT_POLARAXIS): EMF
// components 1 and 3 vanish on the corners of both polar edges
__global__ void k_emf_polar(Grid G) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long ne = (long)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
  if (t >= (long)(G.nx + 1) * (G.nz + 1) * 2) return;
  const int ix = (int)(t % (G.nx + 1));
  const int iz = (int)((t / (G.nx + 1)) % (G.nz + 1));
  const int iy = t / ((long)(G.nx + 1) * (G.nz + 1)) ? G.ny : 0;
  const long e = emf_index(G, ix, iy, iz);
  G.emf[0 * ne + e] = 0.;
  G.emf[2 * ne + e] = 0.;
}

// KORAL layout [cell][var] <-> device [var][cell]
__global__ void k_aos_to_soa(const double *aos, double *soa, long n, int nv) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n * nv) return;
  long c = t / nv;
  int iv = (int)(t % nv);
  soa[iv * n + c] = aos[t];
}
__global__ void k_soa_to_aos(const double *soa, double *aos, long n, int nv) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n * nv) return;
  long c = t / nv;
  int iv = (int)(t % nv);
  aos[t] = soa[iv * n + c];
}
__global__ void k_minkowski(double *met, long npts) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= npts) return;
  for (int k = 0; k < 40; k++) met[k * npts + t] = 0.;
  met[0 * npts + t] = -1.;
  met[6 * npts + t] = 1.;
  met[12 * npts + t] = 1.;
  met[18 * npts + t] = 1.;
  met[19 * npts + t] = 1.;         // gdet
  met[20 * npts + t] = -1.;
  met[26 * npts + t] = 1.;
  met[32 * npts + t] = 1.;
  met[38 * npts + t] = 1.;
}
// cells c0 .. c0+m-1 of a [nv][n] array into [m][nv]
__global__ void k_soa_slab_to_aos(const double *soa, long n, long c0, long m, int nv, double *aos) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= m * nv) return;
  const long cc = t / nv;
  const int v = (int)(t - cc * nv);
  aos[t] = soa[(long)v * n + c0 + cc];
}
__global__ void k_fill(double *a, long n, double v) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < n) a[t] = v;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
enum KernelId { K_BC = 0, K_WAVESPEEDS, K_FLUX0, K_FLUX1, K_FLUX2, K_EMF, K_UPDATE, K_U2P, K_U2P_RESUME,
                K_U2P_ENT, K_U2P_RESUME_ENT, K_FIXUP, K_COMMIT, K_BEGIN, K_FLUXRAD0, K_FLUXRAD1, K_FLUXRAD2,
                K_UPDATE_RAD, K_U2P_RAD, K_IMP_GATHER, K_IMP_WARM, K_IMP_SOLVE, K_IMP_SCATTER, K_IMEX, K_RECON0,
                K_RECON1, K_RECON2, K_AVG, K_NKERNELS };
static const char *kKernelNames[K_NKERNELS] = {"k_bc", "k_wavespeeds", "k_flux_x", "k_flux_y", "k_flux_z", "k_emf",
                                               "k_update", "k_u2p", "k_u2p_resume", "k_u2p_entropy",
                                               "k_u2p_resume_entropy", "k_fixup", "k_commit", "k_begin_step",
                                               "k_flux_rad_x", "k_flux_rad_y", "k_flux_rad_z", "k_update_rad",
                                               "k_u2p_rad", "k_imp_gather", "k_imp_warm_start", "k_imp_solve",
                                               "k_imp_scatter", "k_imex", "k_recon_x", "k_recon_y", "k_recon_z",
                                               "k_save_avg"};

int kgpu_rad_solve_enqueue(int n, const kgpu_rad_params *rp, const double *uu, const double *pp, const double *g,
                           const double *G, const double *dt, const float *ypred, double *pp_out, double *uu_out,
                           int *status, int *attempt, int *iters, int mode, void *work, void *stream,
                           unsigned long long *acc, long long *launches, int gate,
                           const kgpu_rad_solver_opts *opts);
kgpu::RadParams kgpu_rad_device_params(const kgpu_rad_params &p);
bool kgpu_rad_opts_valid(const kgpu_rad_solver_opts &o);

// Variants of the face-flux, update and first inversion kernels compiled
// for different numbers of resident blocks per SM (registers traded
// against occupancy); the context picks one of each (kgpu_set_tuning,
// kgpu_autotune).  Every variant performs the same arithmetic.
template <int D>
static void launch_flux(int mb, unsigned nb, cudaStream_t st, const Grid &G, Box b) {
  switch (mb) {
    case 5: k_flux<D, 5><<<nb, 128, 0, st>>>(G, b, nullptr, nullptr); break;
    case 6: k_flux<D, 6><<<nb, 128, 0, st>>>(G, b, nullptr, nullptr); break;
    case 8: k_flux<D, 8><<<nb, 128, 0, st>>>(G, b, nullptr, nullptr); break;
    default: k_flux<D, 7><<<nb, 128, 0, st>>>(G, b, nullptr, nullptr); break;
  }
}
template <int D>
static void launch_flux_split(int mb, unsigned nb, cudaStream_t st, const Grid &G, Box b, const double *sl,
                              const double *sr) {
  switch (mb) {
    case 5: k_flux<D, 5, true><<<nb, 128, 0, st>>>(G, b, sl, sr); break;
    case 6: k_flux<D, 6, true><<<nb, 128, 0, st>>>(G, b, sl, sr); break;
    case 8: k_flux<D, 8, true><<<nb, 128, 0, st>>>(G, b, sl, sr); break;
    default: k_flux<D, 7, true><<<nb, 128, 0, st>>>(G, b, sl, sr); break;
  }
}
// the faces of direction D that k_flux left to the magnetic floor: two
// blocks per SM loop over the queue (empty on most steps)
template <int D>
static void launch_flux_fix(bool split, int sms, cudaStream_t st, const Grid &G, Box b, const double *sl,
                            const double *sr) {
  if (split) k_flux_fix<D, true><<<2 * sms, 128, 0, st>>>(G, b, sl, sr);
  else k_flux_fix<D, false><<<2 * sms, 128, 0, st>>>(G, b, sl, sr);
}
static void launch_update(int mb, unsigned nb, cudaStream_t st, const Grid &G, Box b, const double *dtp, double fac,
                          double *save) {
  switch (mb) {
    case 3: k_update<3><<<nb, 128, 0, st>>>(G, b, dtp, fac, save); break;
    case 5: k_update<5><<<nb, 128, 0, st>>>(G, b, dtp, fac, save); break;
    default: k_update<4><<<nb, 128, 0, st>>>(G, b, dtp, fac, save); break;
  }
}
static void launch_u2p_first(int mb, unsigned nb, cudaStream_t st, const Grid &G, Box b, U2PQueues Q, int stop) {
  switch (mb) {
    case 4: k_u2p<4><<<nb, 128, 0, st>>>(G, b, Q, stop); break;
    case 6: k_u2p<6><<<nb, 128, 0, st>>>(G, b, Q, stop); break;
    default: k_u2p<5><<<nb, 128, 0, st>>>(G, b, Q, stop); break;
  }
}
static bool tuning_valid(const kgpu_tuning &t) {
  return t.flux_blocks >= 5 && t.flux_blocks <= 8 && (t.flux_split == 0 || t.flux_split == 1) && t.update_blocks >= 3 && t.update_blocks <= 5 &&
         t.u2p_blocks >= 4 && t.u2p_blocks <= 6 && t.u2p_pass_iters >= 1 &&
         (t.implicit_mode == KGPU_RAD_PLAIN || t.implicit_mode == KGPU_RAD_BATCHED ||
          t.implicit_mode == KGPU_RAD_PERSISTENT) &&
         kgpu_rad_opts_valid(t.implicit);
}

struct ProfRec {
  int id;
  cudaEvent_t a, b;
};

struct kgpu_ctx {
  kgpu_config cfg;
  bool profiling = false;
  std::vector<ProfRec> prof;        // events of the launches since the last read
  std::vector<cudaEvent_t> evpool;  // recycled events
  double prof_ms[K_NKERNELS] = {0};
  long long prof_n[K_NKERNELS] = {0};
  long long launches = 0;           // kernels launched by this context
  long long graph_launches = 0;     // kernels in one captured RK2 step
  Grid G;
  cudaStream_t stream;
  std::vector<void *> allocs;
  double *stage;        // AoS staging for uploads / downloads
  double *ut2 = nullptr; // RK2's k2 array of the per-operator loop (KGPU_ARR_UT2)
  bool flux_ct_done = false;  // the face fluxes already hold flux_ct's rewrite
  int *fixmark;
  U2PQueues u2pq;                // work queues of the inversion passes
  int u2p_pass_iters = 8;        // Newton steps before a solve is queued for resumption
  int flux_blocks = KGPU_FLUX_MIN_BLOCKS, update_blocks = KGPU_UPDATE_MIN_BLOCKS, u2p_blocks = KGPU_U2P_MIN_BLOCKS;
  int flux_split = 0;            // face states by k_recon, then the flux kernel reads them
  double *fsl = nullptr, *fsr = nullptr;   // face states of one direction [NVMAX][faces of its box]
  int sm_count;
  double *rhofl_c = nullptr, *rhofl_f = nullptr;
  double min_dx, min_dy, min_dz;
  bool have_grid, have_metric;
  std::vector<double> hxb[3];
  cudaGraph_t graph;
  cudaGraphExec_t graph_exec;
  bool graph_ready;
  int graph_kind = 0;            // 0: RK2 step, 1: RK2IMEX step
  // radiation (nv == 13)
  kgpu_rad_params rp;
  double *drt1 = nullptr, *dut1 = nullptr, *drt2 = nullptr, *dut2 = nullptr;   // RK2IMEX rates
  long nimp = 0;                 // domain cells of the implicit solve
  double *imp_uu = nullptr, *imp_pp = nullptr, *imp_g = nullptr, *imp_G = nullptr, *imp_dt = nullptr;
  double *imp_ppo = nullptr, *imp_uuo = nullptr;
  int *imp_status = nullptr, *imp_att = nullptr, *imp_it = nullptr;
  void *imp_work = nullptr;
  float *imp_X = nullptr, *imp_Y = nullptr;
  int imp_mode = KGPU_RAD_BATCHED;
  kgpu_rad_solver_opts imp_opts;  // this context's solver tuning
  kgpu_mlp *warm = nullptr;      // warm-start network, or none
  int warm_gate = -1;            // warm-start only cells whose previous solve took more than this (-1: all)
  long long metric_gen = 0, packed_gen = -1;
  double *diag_work = nullptr, *diag_out = nullptr;   // calc_scalars on the device
  // time averages (save_avg): running sums [NV + NAVGVARS][ncell], the
  // summed time, the unit constants of the averaged temperatures, and
  // whether the fused steps add to them once per step
  double *pavg = nullptr, *avgtime = nullptr;
  RadParams avg_units;
  bool avg_on = false, avg_ready = false;
  // polar-axis corrections of do_correct: KGPU_POLAR_* bits and the rows
  int polar_flags = 0, polar_nc = 2;
};

static cudaEvent_t pool_event(kgpu_ctx *c) {
  if (!c->evpool.empty()) {
    cudaEvent_t e = c->evpool.back();
    c->evpool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
// brackets one launch with events when profiling; counts every launch
struct LaunchScope {
  kgpu_ctx *c;
  ProfRec r;
  LaunchScope(kgpu_ctx *ctx, int id) : c(ctx) {
    c->launches++;
    if (c->profiling) {
      r.id = id;
      r.a = pool_event(c);
      r.b = pool_event(c);
      cudaEventRecord(r.a, c->stream);
    }
  }
  ~LaunchScope() {
    if (c->profiling) {
      cudaEventRecord(r.b, c->stream);
      c->prof.push_back(r);
    }
  }
};

static int dalloc(kgpu_ctx *c, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 8);
  if (e != cudaSuccess) {
    set_err("cudaMalloc", e);
    return KGPU_ENOMEM;
  }
  c->allocs.push_back(*p);
  return 0;
}

extern "C" int kgpu_default_config(kgpu_config *cfg, int nx, int ny, int nz) {
  if (!cfg || nx < 1 || ny < 1 || nz < 1) return KGPU_EINVAL;
  memset(cfg, 0, sizeof(*cfg));
  cfg->nx = nx; cfg->ny = ny; cfg->nz = nz;
  cfg->ng = 3; cfg->nv = 9;
  cfg->int_order = KGPU_PPM;
  cfg->fluxmethod = KGPU_LAXF;
  cfg->axisym_metric = 0;
  cfg->bc[0] = cfg->bc[1] = cfg->bc[2] = KGPU_BC_PERIODIC;
  cfg->gamma = 5. / 3.;
  cfg->tsteplim = 0.5;
  cfg->rhofloor = 1.e-50;          // choices.h:319-329
  cfg->uurhoratiomin = 1.e-50;     // choices.h:55-58
  cfg->uurhoratiomax = 1.e2;       // choices.h:65-68
  cfg->b2rhoratiomax = 100.;       // choices.h:110-113
  cfg->gammamaxhd = 100.;          // choices.h:331-333
  cfg->u2pconv = 1.e-10;           // choices.h:457-459
  return 0;
}

static void fill_grid_params(Grid &G, const kgpu_config &c) {
  memset(&G, 0, sizeof(G));
  G.nx = c.nx; G.ny = c.ny; G.nz = c.nz; G.ng = c.ng; G.nv = c.nv;
  G.sx = c.nx + 2 * c.ng; G.ngcx = c.ng;
  G.sy = c.ny > 1 ? c.ny + 2 * c.ng : 1; G.ngcy = c.ny > 1 ? c.ng : 0;
  G.sz = c.nz > 1 ? c.nz + 2 * c.ng : 1; G.ngcz = c.nz > 1 ? c.ng : 0;
  G.axisym = c.axisym_metric;
  G.szmet = G.axisym ? 1 : G.sz;
  G.ngczmet = G.axisym ? 0 : G.ngcz;
  G.ncell = (long)G.sx * G.sy * G.sz;
  G.nmet = (long)G.sx * G.sy * G.szmet;
  G.nfmet[0] = (long)(G.sx + 1) * G.sy * G.szmet;
  G.nfmet[1] = (long)G.sx * (G.sy + 1) * G.szmet;
  G.nfmet[2] = (long)G.sx * G.sy * (G.szmet + 1);
  G.nface[0] = (long)(G.sx + 1) * G.sy * G.sz;
  G.nface[1] = (long)G.sx * (G.sy + 1) * G.sz;
  G.nface[2] = (long)G.sx * G.sy * (G.sz + 1);
  G.gamma = c.gamma; G.tsteplim = c.tsteplim;
  G.int_order = c.int_order; G.fluxmethod = c.fluxmethod;
  G.rhofloor = c.rhofloor; G.uurhoratiomin = c.uurhoratiomin; G.uurhoratiomax = c.uurhoratiomax;
  G.b2rhoratiomax = c.b2rhoratiomax; G.gammamaxhd = c.gammamaxhd; G.u2pconv = c.u2pconv;
  for (int d = 0; d < 3; d++) G.bc[d] = c.bc[d];
  G.rhofl_c = G.rhofl_f = nullptr;
}

static int check_config(const kgpu_config *c) {
  if (!c || c->nx < 1 || c->ny < 1 || c->nz < 1) return KGPU_EINVAL;
  if (c->nv != 9 && c->nv != 13) return KGPU_EINVAL;   // MHD with magnetic field, optionally M1 radiation
  if (c->int_order != KGPU_PPM && c->int_order != KGPU_MP5) return KGPU_EINVAL;
  if (c->int_order == KGPU_PPM && c->ng < 3) return KGPU_EINVAL;
  if (c->int_order == KGPU_MP5 && c->ng < 4) return KGPU_EINVAL;
  if (c->fluxmethod != KGPU_LAXF && c->fluxmethod != KGPU_HLL) return KGPU_EINVAL;
  if (c->nx < c->ng) return KGPU_EINVAL;
  if (!(c->gamma > 1.) || !(c->tsteplim > 0.)) return KGPU_EINVAL;
  return 0;
}

extern "C" int kgpu_create(const kgpu_config *cfg, kgpu_ctx **out) {
  if (!out) return KGPU_EINVAL;
  *out = nullptr;
  int r = check_config(cfg);
  if (r) return r;
  for (int d = 0; d < 3; d++)
    if (cfg->bc[d] < KGPU_BC_PERIODIC || cfg->bc[d] > KGPU_BC_PERIODIC_COPY) return KGPU_EINVAL;
  // the 2D corner fill follows the reference's periodic treatment only
  if (cfg->nz == 1 && cfg->ny > 1 && (cfg->bc[0] != KGPU_BC_PERIODIC || cfg->bc[1] != KGPU_BC_PERIODIC))
    return KGPU_EINVAL;
  kgpu_ctx *c = new kgpu_ctx();
  c->cfg = *cfg;
  kgpu_rad_default_solver_opts(&c->imp_opts);
  fill_grid_params(c->G, *cfg);
  Grid &G = c->G;
  c->have_grid = c->have_metric = false;
  c->graph_ready = false;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return set_err("cudaStreamCreate", e);
  }
  {
    int dev = 0;
    c->sm_count = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, dev);
  }
  const size_t d8 = sizeof(double);
  const long ncv = G.ncell * G.nv;
  void *p;
#define AL(ptr, bytes)                           \
  do {                                           \
    if ((r = dalloc(c, &p, (bytes))) != 0) {     \
      kgpu_destroy(c);                           \
      return r;                                  \
    }                                            \
    ptr = (decltype(ptr))p;                      \
  } while (0)
  AL(G.u, ncv * d8); AL(G.p, ncv * d8); AL(G.ut0, ncv * d8); AL(G.ut1, ncv * d8); AL(c->ut2, ncv * d8);
  AL(G.pfix, ncv * d8); AL(G.ufix, ncv * d8); AL(c->stage, ncv * d8);
  int n[3] = {G.nx, G.ny, G.nz};
  {
    long fmax = G.nface[0] > G.nface[1] ? G.nface[0] : G.nface[1];
    if (G.nface[2] > fmax) fmax = G.nface[2];
    AL(c->fsl, fmax * NVMAX * d8);
    AL(c->fsr, fmax * NVMAX * d8);
  }
  for (int d = 0; d < 3; d++) {
    double *xb;
    AL(xb, (n[d] + 1 + 2 * G.ng) * d8);
    G.xb[d] = xb;
    AL(G.flb[d], G.nface[d] * G.nv * d8);
    AL(G.al[d], G.ncell * d8);
    AL(G.ar[d], G.ncell * d8);
    double *mf;
    AL(mf, G.nfmet[d] * 40 * d8);
    G.met_f[d] = mf;
  }
  double *mc, *kr;
  AL(mc, G.nmet * 40 * d8); G.met_c = mc;
  AL(kr, G.nmet * 64 * d8); G.gkr = kr;
  AL(G.emf, 3L * (G.nx + 1) * (G.ny + 1) * (G.nz + 1) * d8);
  AL(G.flag, G.ncell * sizeof(int));
  for (int d = 0; d < 3; d++) AL(G.fq[d], G.nface[d] * sizeof(int));
  AL(G.fqn, 3 * sizeof(int));
  AL(c->fixmark, G.ncell * sizeof(int));
  AL(c->u2pq.slow, G.ncell * sizeof(int));
  AL(c->u2pq.ent, G.ncell * sizeof(int));
  AL(c->u2pq.slow_ent, G.ncell * sizeof(int));
  AL(c->u2pq.n, 4 * sizeof(int));
  AL(c->u2pq.w, G.ncell * d8);
  AL(c->u2pq.it, G.ncell * sizeof(int));
  AL(G.scal, S_NSCAL * d8);
  AL(G.cnt, C_NCNT * sizeof(unsigned long long));
  if (G.nv == NVR) {
    for (int d = 0; d < 3; d++) {
      AL(G.arl[d], G.ncell * d8);
      AL(G.arr[d], G.ncell * d8);
    }
    AL(c->drt1, ncv * d8); AL(c->dut1, ncv * d8); AL(c->drt2, ncv * d8); AL(c->dut2, ncv * d8);
  }
#undef AL
  CK(cudaMemsetAsync(G.u, 0, ncv * d8, c->stream));
  CK(cudaMemsetAsync(G.p, 0, ncv * d8, c->stream));
  CK(cudaMemsetAsync(G.ut0, 0, ncv * d8, c->stream));
  CK(cudaMemsetAsync(G.ut1, 0, ncv * d8, c->stream));
  for (int d = 0; d < 3; d++) {
    CK(cudaMemsetAsync(G.flb[d], 0, G.nface[d] * G.nv * d8, c->stream));
    CK(cudaMemsetAsync(G.al[d], 0, G.ncell * d8, c->stream));
    CK(cudaMemsetAsync(G.ar[d], 0, G.ncell * d8, c->stream));
  }
  CK(cudaMemsetAsync(G.emf, 0, 3L * (G.nx + 1) * (G.ny + 1) * (G.nz + 1) * d8, c->stream));
  CK(cudaMemsetAsync(G.flag, 0, G.ncell * sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->fixmark, 0, G.ncell * sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->u2pq.n, 0, 4 * sizeof(int), c->stream));
  CK(cudaMemsetAsync(G.scal, 0, S_NSCAL * d8, c->stream));
  CK(cudaMemsetAsync(G.cnt, 0, C_NCNT * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync((void *)G.gkr, 0, G.nmet * 64 * d8, c->stream));
  if (G.nv == NVR)
    for (int d = 0; d < 3; d++) {
      CK(cudaMemsetAsync(G.arl[d], 0, G.ncell * d8, c->stream));
      CK(cudaMemsetAsync(G.arr[d], 0, G.ncell * d8, c->stream));
    }
  CK(cudaStreamSynchronize(c->stream));
  *out = c;
  return 0;
}

// The captured step holds kernel arguments by value: drop it when they change.
static void drop_graph(kgpu_ctx *c) {
  if (c->graph_ready) {
    cudaGraphExecDestroy(c->graph_exec);
    cudaGraphDestroy(c->graph);
    c->graph_ready = false;
  }
}

extern "C" int kgpu_destroy(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  if (c->graph_ready) {
    cudaGraphExecDestroy(c->graph_exec);
    cudaGraphDestroy(c->graph);
  }
  cudaStreamSynchronize(c->stream);
  for (auto &r : c->prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : c->evpool) cudaEventDestroy(e);
  for (void *p : c->allocs) cudaFree(p);
  cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

// minimal cell sizes as set_grid computes them, including its comparison of
// dy and dz against the running minimum in x (finite.c:1672-1686)
static void min_sizes(kgpu_ctx *c) {
  const kgpu_config &k = c->cfg;
  double mdx = -1, mdy = -1, mdz = -1;
  auto sz = [&](int ic, int d) { return c->hxb[d][ic + 1 + k.ng] - c->hxb[d][ic + k.ng]; };
  for (int ix = 0; ix < k.nx; ix++)
    for (int iy = 0; iy < k.ny; iy++)
      for (int iz = 0; iz < k.nz; iz++) {
        double dx = sz(ix, 0), dy = sz(iy, 1), dz = sz(iz, 2);
        if ((dx < mdx || mdx < 0.)) mdx = dx;
        if ((dy < mdx || mdy < 0.)) mdy = dy;
        if ((dz < mdx || mdz < 0.)) mdz = dz;
      }
  c->min_dx = mdx; c->min_dy = mdy; c->min_dz = mdz;
}

extern "C" int kgpu_upload_grid(kgpu_ctx *c, const double *xbx, const double *xby, const double *xbz) {
  if (!c || !xbx || !xby || !xbz) return KGPU_EINVAL;
  const double *src[3] = {xbx, xby, xbz};
  int n[3] = {c->cfg.nx, c->cfg.ny, c->cfg.nz};
  for (int d = 0; d < 3; d++) {
    c->hxb[d].assign(src[d], src[d] + n[d] + 1 + 2 * c->cfg.ng);
    CK(cudaMemcpyAsync((void *)c->G.xb[d], src[d], (n[d] + 1 + 2 * c->cfg.ng) * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  min_sizes(c);
  c->have_grid = true;
  return 0;
}

extern "C" int kgpu_set_uniform_grid(kgpu_ctx *c, const double lo[3], const double hi[3]) {
  if (!c || !lo || !hi) return KGPU_EINVAL;
  int n[3] = {c->cfg.nx, c->cfg.ny, c->cfg.nz}, ng = c->cfg.ng;
  std::vector<double> xb[3];
  for (int d = 0; d < 3; d++) {
    double c0 = lo[d], c1 = hi[d], dc = (c1 - c0) / (double)n[d];   // problem.c:9-36
    xb[d].resize(n[d] + 1 + 2 * ng);
    for (int i = -ng; i <= n[d] + ng; i++) xb[d][i + ng] = c0 + (double)(i)*dc;
  }
  return kgpu_upload_grid(c, xb[0].data(), xb[1].data(), xb[2].data());
}

// KORAL metric tables ([point][20]) -> [component][point]
static int upload_met(kgpu_ctx *c, const double *g, const double *Gi, double *dst, long npts) {
  std::vector<double> h(npts * 40);
  for (long i = 0; i < npts; i++)
    for (int k = 0; k < 20; k++) {
      h[k * npts + i] = g[i * 20 + k];
      h[(20 + k) * npts + i] = Gi[i * 20 + k];
    }
  CK(cudaMemcpyAsync(dst, h.data(), npts * 40 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_upload_metric(kgpu_ctx *c, const double *g, const double *Gi, const double *gKr, const double *gbx,
                                  const double *gby, const double *gbz, const double *Gbx, const double *Gby,
                                  const double *Gbz) {
  if (!c || !g || !Gi || !gKr || !gbx || !gby || !gbz || !Gbx || !Gby || !Gbz) return KGPU_EINVAL;
  Grid &G = c->G;
  int r;
  if ((r = upload_met(c, g, Gi, (double *)G.met_c, G.nmet))) return r;
  const double *gb[3] = {gbx, gby, gbz}, *Gb[3] = {Gbx, Gby, Gbz};
  for (int d = 0; d < 3; d++)
    if ((r = upload_met(c, gb[d], Gb[d], (double *)G.met_f[d], G.nfmet[d]))) return r;
  std::vector<double> h(G.nmet * 64);
  for (long i = 0; i < G.nmet; i++)
    for (int k = 0; k < 64; k++) h[k * G.nmet + i] = gKr[i * 64 + k];
  CK(cudaMemcpyAsync((void *)G.gkr, h.data(), G.nmet * 64 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->have_metric = true;
  c->metric_gen++;
  return 0;
}

extern "C" int kgpu_set_density_floor(kgpu_ctx *c, const double *centres, const double *xfaces) {
  if (!c) return KGPU_EINVAL;
  Grid &G = c->G;
  if (!centres || !xfaces) {
    G.rhofl_c = G.rhofl_f = nullptr;
    return 0;
  }
  if (!c->rhofl_c) {
    void *p;
    int r;
    if ((r = dalloc(c, &p, G.sx * sizeof(double)))) return r;
    c->rhofl_c = (double *)p;
    if ((r = dalloc(c, &p, (G.sx + 1) * sizeof(double)))) return r;
    c->rhofl_f = (double *)p;
  }
  CK(cudaMemcpyAsync(c->rhofl_c, centres, G.sx * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->rhofl_f, xfaces, (G.sx + 1) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  G.rhofl_c = c->rhofl_c;
  G.rhofl_f = c->rhofl_f;
  drop_graph(c);   // kernels take the Grid by value: re-capture
  return 0;
}

extern "C" int kgpu_set_minkowski_metric(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  Grid &G = c->G;
  k_minkowski<<<nblocks(G.nmet, 256), 256, 0, c->stream>>>((double *)G.met_c, G.nmet);
  for (int d = 0; d < 3; d++)
    k_minkowski<<<nblocks(G.nfmet[d], 256), 256, 0, c->stream>>>((double *)G.met_f[d], G.nfmet[d]);
  k_fill<<<nblocks(G.nmet * 64, 256), 256, 0, c->stream>>>((double *)G.gkr, G.nmet * 64, 0.);
  CKL("k_minkowski");
  CK(cudaStreamSynchronize(c->stream));
  c->have_metric = true;
  c->metric_gen++;
  return 0;
}

extern "C" int kgpu_upload_state(kgpu_ctx *c, const double *u, const double *p) {
  if (!c || !u || !p) return KGPU_EINVAL;
  Grid &G = c->G;
  const long n = G.ncell;
  const double *src[2] = {u, p};
  double *dst[2] = {G.u, G.p};
  for (int k = 0; k < 2; k++) {
    CK(cudaMemcpyAsync(c->stage, src[k], n * G.nv * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_aos_to_soa<<<nblocks(n * G.nv, 256), 256, 0, c->stream>>>(c->stage, dst[k], n, G.nv);
    CKL("k_aos_to_soa");
  }
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

static double *arr_ptr(kgpu_ctx *c, int which) {
  switch (which) {
    case KGPU_ARR_U: return c->G.u;
    case KGPU_ARR_P: return c->G.p;
    case KGPU_ARR_UT0: return c->G.ut0;
    case KGPU_ARR_UT1: return c->G.ut1;
    case KGPU_ARR_UT2: return c->ut2;
    default: return nullptr;
  }
}

extern "C" int kgpu_download_array(kgpu_ctx *c, int which, double *out) {
  if (!c || !out) return KGPU_EINVAL;
  double *src = arr_ptr(c, which);
  if (!src) return KGPU_EINVAL;
  Grid &G = c->G;
  const long n = G.ncell;
  k_soa_to_aos<<<nblocks(n * G.nv, 256), 256, 0, c->stream>>>(src, c->stage, n, G.nv);
  CKL("k_soa_to_aos");
  CK(cudaMemcpyAsync(out, c->stage, n * G.nv * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_download_state(kgpu_ctx *c, double *u, double *p) {
  int r = kgpu_download_array(c, KGPU_ARR_U, u);
  if (r) return r;
  return kgpu_download_array(c, KGPU_ARR_P, p);
}

// ---------------------------------------------------------------------------
// operator launchers (all asynchronous on the context stream)
// ---------------------------------------------------------------------------
static Box domain_box(const Grid &G) { return Box{0, 0, 0, G.nx, G.ny, G.nz}; }

// ---------------------------------------------------------------------------
// restart files in the reference's serial binary format (fileop.c:910-1111)
// ---------------------------------------------------------------------------
// conserved variables of the domain cells from their primitives (the p2u
// of fread_restartfile_bin, fileop.c:1078-1092)
__global__ void k_p2u_domain(Grid G, Box b) {
  int ix, iy, iz;
  if (!box_coord(b, blockIdx.x * (long)blockDim.x + threadIdx.x, ix, iy, iz)) return;
  const long c = cell_index(G, ix, iy, iz);
  double pp[NVR], uu[NVR];
  load_cell(G.p, G.ncell, c, pp);
  Geom g;
  geom_centre(G, ix, iy, iz, g);
  p2u_full(G, pp, uu, g);
  store_cell(G.u, G.ncell, c, uu);
  if (G.rad) {
    load_rad(G.p, G.ncell, c, pp);
    p2u_rad(pp, uu, g);
    store_rad(G.u, G.ncell, c, uu);
  }
}

// KORAL's cell-major index of a domain cell in the padded arrays
static long aos_index(const Grid &G, int ix, int iy, int iz) {
  long ky = (G.ny > 1 ? iy : 0) + G.ngcy, kz = (G.nz > 1 ? iz : 0) + G.ngcz;
  return ((long)kz * G.sy + ky) * G.sx + ix + G.ngcx;
}

extern "C" int kgpu_write_restart(kgpu_ctx *c, const char *folder, int nout1, int nout2, double t, int problem) {
  if (!c || !folder || nout1 < 0) return KGPU_EINVAL;
  Grid &G = c->G;
  std::vector<double> p(G.ncell * G.nv);
  int r = kgpu_download_array(c, KGPU_ARR_P, p.data());
  if (r) return r;
  char name[4096];
  snprintf(name, sizeof(name), "%s/res%04d.head", folder, nout1);
  FILE *f = fopen(name, "w");
  if (!f) return KGPU_EIO;
  fprintf(f, "## %5d %5d %10.6e %5d %5d %5d %5d\n", nout1, nout2, t, problem, G.nx, G.ny, G.nz);
  if (fclose(f)) return KGPU_EIO;
  snprintf(name, sizeof(name), "%s/res%04d.dat", folder, nout1);
  f = fopen(name, "wb");
  if (!f) return KGPU_EIO;
  bool ok = true;
  // global indices first, x outer and z inner; then the primitives in the
  // same order
  for (int ix = 0; ix < G.nx && ok; ix++)
    for (int iy = 0; iy < G.ny && ok; iy++)
      for (int iz = 0; iz < G.nz && ok; iz++) {
        int gi[3] = {ix, iy, iz};
        ok = fwrite(gi, sizeof(int), 3, f) == 3;
      }
  for (int ix = 0; ix < G.nx && ok; ix++)
    for (int iy = 0; iy < G.ny && ok; iy++)
      for (int iz = 0; iz < G.nz && ok; iz++)
        ok = fwrite(p.data() + aos_index(G, ix, iy, iz) * G.nv, sizeof(double), G.nv, f) == (size_t)G.nv;
  if (fclose(f) || !ok) return KGPU_EIO;
  // reslast.* point at the newest files, as the reference's links do
  const char *ext[2] = {"dat", "head"};
  for (int k = 0; k < 2; k++) {
    char link[4096], target[64];
    snprintf(link, sizeof(link), "%s/reslast.%s", folder, ext[k]);
    snprintf(target, sizeof(target), "res%04d.%s", nout1, ext[k]);
    unlink(link);
    if (symlink(target, link)) return KGPU_EIO;
  }
  return 0;
}

extern "C" int kgpu_read_restart(kgpu_ctx *c, const char *folder, int nout1, double *t, int *nout1_next,
                                 int *nout2) {
  if (!c || !folder) return KGPU_EINVAL;
  if (!c->have_grid || !c->have_metric) return KGPU_ESTATE;
  int r;
  Grid &G = c->G;
  char name[4096], head[4096];
  if (nout1 >= 0) {
    snprintf(name, sizeof(name), "%s/res%04d.dat", folder, nout1);
    snprintf(head, sizeof(head), "%s/res%04d.head", folder, nout1);
  } else {
    snprintf(name, sizeof(name), "%s/reslast.dat", folder);
    snprintf(head, sizeof(head), "%s/reslast.head", folder);
  }
  FILE *f = fopen(head, "r");
  if (!f) return KGPU_EIO;
  int ip[6];
  double tt = 0.;
  int nr = fscanf(f, "## %d %d %lf %d %d %d %d\n", &ip[0], &ip[1], &tt, &ip[2], &ip[3], &ip[4], &ip[5]);
  fclose(f);
  if (nr != 7) return KGPU_EIO;
  if (ip[3] != G.nx || ip[4] != G.ny || ip[5] != G.nz) return KGPU_EINVAL;
  std::vector<double> u(G.ncell * G.nv), p(G.ncell * G.nv);
  if ((r = kgpu_download_state(c, u.data(), p.data()))) return r;
  f = fopen(name, "rb");
  if (!f) return KGPU_EIO;
  const long n = (long)G.nx * G.ny * G.nz;
  std::vector<int> idx(3 * n);
  bool ok = fread(idx.data(), sizeof(int), 3 * n, f) == (size_t)(3 * n);
  for (long k = 0; k < n && ok; k++) {
    const int gx = idx[3 * k], gy = idx[3 * k + 1], gz = idx[3 * k + 2];
    if (gx < 0 || gx >= G.nx || gy < 0 || gy >= G.ny || gz < 0 || gz >= G.nz) {
      ok = false;
      break;
    }
    ok = fread(p.data() + aos_index(G, gx, gy, gz) * G.nv, sizeof(double), G.nv, f) == (size_t)G.nv;
  }
  fclose(f);
  if (!ok) return KGPU_EIO;
  if ((r = kgpu_upload_state(c, u.data(), p.data()))) return r;
  Box db = domain_box(G);
  k_p2u_domain<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(G, db);
  CKL("k_p2u_domain");
  CK(cudaStreamSynchronize(c->stream));
  if (t) *t = tt;
  if (nout1_next) *nout1_next = ip[0] + 1;
  if (nout2) *nout2 = ip[1];
  return 0;
}

static int launch_bc(kgpu_ctx *c) {
  Grid &G = c->G;
  Box b{-G.ngcx, -G.ngcy, -G.ngcz, G.sx, G.sy, G.sz};
  { LaunchScope ls(c, K_BC); k_bc_faces<<<nblocks(b.n(), 128), 128, 0, c->stream>>>(G, b); }
  CKL("k_bc_faces");
  if (G.nz == 1 && G.ny > 1) {
    LaunchScope ls(c, K_BC);
    k_bc_corners2d<<<1, 8 * G.ng > 32 ? 64 : 32, 0, c->stream>>>(G);
    CKL("k_bc_corners2d");
  }
  if (G.nz > 1 && G.ny > 1) {
    // edges along z (a=x, b=y), along y (a=x, b=z), along x (a=y, b=z)
    const int axes[3][3] = {{2, 0, 1}, {1, 0, 2}, {0, 1, 2}};
    int n3[3] = {G.nx, G.ny, G.nz};
    for (int k = 0; k < 3; k++) {
      int cax = axes[k][0];
      int nthreads = 4 * (n3[cax] + 2 * G.ng);
      LaunchScope ls(c, K_BC);
      k_bc_edges3d<<<nblocks(nthreads, 128), 128, 0, c->stream>>>(G, cax, axes[k][1], axes[k][2]);
      CKL("k_bc_edges3d");
    }
    LaunchScope ls(c, K_BC);
    k_bc_corners3d<<<nblocks(8 * G.ng * G.ng * G.ng, 128), 128, 0, c->stream>>>(G);
    CKL("k_bc_corners3d");
  }
  return 0;
}

static int launch_explicit(kgpu_ctx *c, const double *dtp, double fac, double *save) {
  Grid &G = c->G;
  c->flux_ct_done = false;
  const int lim = G.int_order == 4 ? 2 : 1;
  int lx = G.nx > 1 ? lim : 0, ly = G.ny > 1 ? lim : 0, lz = G.nz > 1 ? lim : 0;
  Box wb{-lx, -ly, -lz, G.nx + 2 * lx, G.ny + 2 * ly, G.nz + 2 * lz};
  { LaunchScope ls(c, K_WAVESPEEDS); k_wavespeeds<<<nblocks(wb.n(), 128), 128, 0, c->stream>>>(G, wb); }
  CKL("k_wavespeeds");
  int ey0 = G.ny > 1 ? -1 : 0, eny = G.ny > 1 ? G.ny + 2 : 1;
  int ez0 = G.nz > 1 ? -1 : 0, enz = G.nz > 1 ? G.nz + 2 : 1;
  int ex0 = -1, enx = G.nx + 2;
  if (G.nx > 1) {
    Box b{0, ey0, ez0, G.nx + 1, eny, enz};
    CK(cudaMemsetAsync(G.fqn + 0, 0, sizeof(int), c->stream));
    if (c->flux_split) {
      { LaunchScope ls(c, K_RECON0);
        k_recon<0><<<nblocks(b.n() * NVMAX, 256), 256, 0, c->stream>>>(G, b, c->fsl, c->fsr); }
      CKL("k_recon<0>");
    }
    {
      // the face flux and its magnetic-floor pass, timed as one
      LaunchScope ls(c, K_FLUX0);
      if (c->flux_split) launch_flux_split<0>(c->flux_blocks, nblocks(2 * b.n(), 128), c->stream, G, b, c->fsl, c->fsr);
      else launch_flux<0>(c->flux_blocks, nblocks(2 * b.n(), 128), c->stream, G, b);
      CKL("k_flux<0>");
      c->launches++;
      launch_flux_fix<0>(c->flux_split != 0, c->sm_count, c->stream, G, b, c->fsl, c->fsr);
      CKL("k_flux_fix<0>");
    }
    if (G.rad) {
      LaunchScope ls(c, K_FLUXRAD0);
      k_flux_rad<0><<<nblocks(2 * b.n(), 128), 128, 0, c->stream>>>(G, b);
      CKL("k_flux_rad<0>");
    }
  }
  if (G.ny > 1) {
    Box b{ex0, 0, ez0, enx, G.ny + 1, enz};
    CK(cudaMemsetAsync(G.fqn + 1, 0, sizeof(int), c->stream));
    if (c->flux_split) {
      { LaunchScope ls(c, K_RECON1);
        k_recon<1><<<nblocks(b.n() * NVMAX, 256), 256, 0, c->stream>>>(G, b, c->fsl, c->fsr); }
      CKL("k_recon<1>");
    }
    {
      // the face flux and its magnetic-floor pass, timed as one
      LaunchScope ls(c, K_FLUX1);
      if (c->flux_split) launch_flux_split<1>(c->flux_blocks, nblocks(2 * b.n(), 128), c->stream, G, b, c->fsl, c->fsr);
      else launch_flux<1>(c->flux_blocks, nblocks(2 * b.n(), 128), c->stream, G, b);
      CKL("k_flux<1>");
      c->launches++;
      launch_flux_fix<1>(c->flux_split != 0, c->sm_count, c->stream, G, b, c->fsl, c->fsr);
      CKL("k_flux_fix<1>");
    }
    if (G.rad) {
      LaunchScope ls(c, K_FLUXRAD1);
      k_flux_rad<1><<<nblocks(2 * b.n(), 128), 128, 0, c->stream>>>(G, b);
      CKL("k_flux_rad<1>");
    }
  }
  if (G.nz > 1) {
    Box b{ex0, ey0, 0, enx, eny, G.nz + 1};
    CK(cudaMemsetAsync(G.fqn + 2, 0, sizeof(int), c->stream));
    if (c->flux_split) {
      { LaunchScope ls(c, K_RECON2);
        k_recon<2><<<nblocks(b.n() * NVMAX, 256), 256, 0, c->stream>>>(G, b, c->fsl, c->fsr); }
      CKL("k_recon<2>");
    }
    {
      // the face flux and its magnetic-floor pass, timed as one
      LaunchScope ls(c, K_FLUX2);
      if (c->flux_split) launch_flux_split<2>(c->flux_blocks, nblocks(2 * b.n(), 128), c->stream, G, b, c->fsl, c->fsr);
      else launch_flux<2>(c->flux_blocks, nblocks(2 * b.n(), 128), c->stream, G, b);
      CKL("k_flux<2>");
      c->launches++;
      launch_flux_fix<2>(c->flux_split != 0, c->sm_count, c->stream, G, b, c->fsl, c->fsr);
      CKL("k_flux_fix<2>");
    }
    if (G.rad) {
      LaunchScope ls(c, K_FLUXRAD2);
      k_flux_rad<2><<<nblocks(2 * b.n(), 128), 128, 0, c->stream>>>(G, b);
      CKL("k_flux_rad<2>");
    }
  }
  Box eb{0, 0, 0, G.nx + 1, G.ny + 1, G.nz + 1};
  { LaunchScope ls(c, K_EMF); k_emf<<<nblocks(eb.n(), 128), 128, 0, c->stream>>>(G, eb); }
  CKL("k_emf");
  if (G.polar_emf) {
    { LaunchScope ls(c, K_EMF); k_emf_polar<<<nblocks(2L * (G.nx + 1) * (G.nz + 1), 128), 128, 0, c->stream>>>(G); }
    CKL("k_emf_polar");
  }
  Box db = domain_box(G);
  { LaunchScope ls(c, K_UPDATE); launch_update(c->update_blocks, nblocks(db.n(), 128), c->stream, G, db, dtp, fac, save); }
  CKL("k_update");
  if (G.rad) {
    { LaunchScope ls(c, K_UPDATE_RAD); k_update_rad<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(G, db, dtp, fac); }
    CKL("k_update_rad");
  }
  return 0;
}

static int launch_u2p(kgpu_ctx *c, int combine) {
  Grid &G = c->G;
  Box db = domain_box(G);
  const int sweep = c->sm_count * 4;   // grid of the queue passes (grid-stride loops)
  { LaunchScope ls(c, K_U2P); launch_u2p_first(c->u2p_blocks, nblocks(db.n(), 128), c->stream, G, db, c->u2pq, c->u2p_pass_iters); }
  CKL("k_u2p");
  { LaunchScope ls(c, K_U2P_RESUME); k_u2p_resume<<<sweep, 128, 0, c->stream>>>(G, db, c->u2pq, 0); }
  CKL("k_u2p_resume");
  { LaunchScope ls(c, K_U2P_ENT); k_u2p_entropy<<<sweep, 128, 0, c->stream>>>(G, db, c->u2pq, c->u2p_pass_iters); }
  CKL("k_u2p_entropy");
  { LaunchScope ls(c, K_U2P_RESUME_ENT); k_u2p_resume<<<sweep, 128, 0, c->stream>>>(G, db, c->u2pq, 1); }
  CKL("k_u2p_resume_entropy");
  if (G.rad) {
    { LaunchScope ls(c, K_U2P_RAD); k_u2p_rad<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(G, db); }
    CKL("k_u2p_rad");
  }
  { LaunchScope ls(c, K_FIXUP); k_fixup<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(G, db, c->fixmark); }
  CKL("k_fixup");
  { LaunchScope ls(c, K_COMMIT); k_commit<<<nblocks(db.n(), 256), 256, 0, c->stream>>>(G, db, c->fixmark, combine, c->u2pq.n); }
  CKL("k_commit");
  return launch_bc(c);
}

static int ready(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  if (!c->have_grid || !c->have_metric) return KGPU_ESTATE;
  return 0;
}

extern "C" int kgpu_set_bc(kgpu_ctx *c, double t, int ifinit) {
  (void)t; (void)ifinit;
  int r = ready(c);
  if (r) return r;
  return launch_bc(c);
}

extern "C" int kgpu_op_explicit(kgpu_ctx *c, double t, double dt) {
  (void)t;
  int r = ready(c);
  if (r) return r;
  CK(cudaMemcpyAsync(c->G.scal + S_T, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if ((r = launch_bc(c))) return r;
  if ((r = launch_explicit(c, c->G.scal + S_T, 1., nullptr))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int kgpu_op_implicit_impl(kgpu_ctx *c, double dt);
extern "C" int kgpu_op_implicit(kgpu_ctx *c, double t, double dt) {
  (void)t;
  if (!c) return KGPU_EINVAL;
  if (!c->G.rad) return 0;   // no radiation: nothing to do, as in the reference
  return kgpu_op_implicit_impl(c, dt);
}

extern "C" int kgpu_calc_u2p(kgpu_ctx *c) {
  int r = ready(c);
  if (r) return r;
  if ((r = launch_u2p(c, 0))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_save_timesteps(kgpu_ctx *c) { return c ? 0 : KGPU_EINVAL; }

extern "C" int kgpu_copyi_u(kgpu_ctx *c, double factor, int src, int dst) {
  if (!c) return KGPU_EINVAL;
  double *a = arr_ptr(c, src), *b = arr_ptr(c, dst);
  if (!a || !b) return KGPU_EINVAL;
  Box db = domain_box(c->G);
  k_copy_domain<<<nblocks(db.n(), 256), 256, 0, c->stream>>>(c->G, db, factor, a, b);
  CKL("k_copy_domain");
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_addi_u(kgpu_ctx *c, double f1, int a, double f2, int b, int cc) {
  if (!c) return KGPU_EINVAL;
  double *pa = arr_ptr(c, a), *pb = arr_ptr(c, b), *pc = arr_ptr(c, cc);
  if (!pa || !pb || !pc) return KGPU_EINVAL;
  Box db = domain_box(c->G);
  k_add_domain<<<nblocks(db.n(), 256), 256, 0, c->stream>>>(c->G, db, f1, pa, f2, pb, pc);
  CKL("k_add_domain");
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_addi_u_3(kgpu_ctx *c, double f1, int a, double f2, int b, double f3, int cc, int d) {
  if (!c) return KGPU_EINVAL;
  double *pa = arr_ptr(c, a), *pb = arr_ptr(c, b), *pc = arr_ptr(c, cc), *pd = arr_ptr(c, d);
  if (!pa || !pb || !pc || !pd) return KGPU_EINVAL;
  Box db = domain_box(c->G);
  k_add3_domain<<<nblocks(db.n(), 256), 256, 0, c->stream>>>(c->G, db, f1, pa, f2, pb, f3, pc, pd);
  CKL("k_add3_domain");
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// do_correct (finite.c:605-640): the polar-axis corrections it runs exist
// only with CORRECT_POLARAXIS / CORRECT_POLARAXIS_3D / SMOOTH_POLARAXIS,
// which the configurations this library runs do not define; the problem's
// my_finger hook is host code and stays on the host.
static int launch_correct(kgpu_ctx *c);

extern "C" int kgpu_do_correct(kgpu_ctx *c) {
  int r = ready(c);
  if (r) return r;
  if (!c->polar_flags) return 0;
  if ((r = launch_correct(c))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_set_polar_correction(kgpu_ctx *c, int flags, int nc) {
  if (!c) return KGPU_EINVAL;
  if (flags & ~(KGPU_POLAR_CORRECT | KGPU_POLAR_CORRECT_3D | KGPU_POLAR_SMOOTH)) return KGPU_EINVAL;
  if (flags && (nc < 1 || c->G.ny < 2 * nc + 2)) return KGPU_EINVAL;
  c->polar_flags = flags;
  c->polar_nc = flags ? nc : 2;
  c->G.polar_nc = (flags & (KGPU_POLAR_CORRECT | KGPU_POLAR_CORRECT_3D)) ? nc : 0;
  c->G.polar_emf = (flags & KGPU_POLAR_CORRECT) ? 1 : 0;
  drop_graph(c);
  return 0;
}

extern "C" int kgpu_flux_ct(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  if (c->flux_ct_done) return KGPU_ESTATE;   // the EMFs come from the fluxes before the rewrite
  Grid &G = c->G;
  Box eb{0, 0, 0, G.nx + 1, G.ny + 1, G.nz + 1};
  k_emf<<<nblocks(eb.n(), 128), 128, 0, c->stream>>>(G, eb);
  CKL("k_emf");
  if (G.polar_emf) {
    k_emf_polar<<<nblocks(2L * (G.nx + 1) * (G.nz + 1), 128), 128, 0, c->stream>>>(G);
    CKL("k_emf_polar");
  }
  k_flux_ct_rewrite<<<nblocks(eb.n(), 128), 128, 0, c->stream>>>(G, eb);
  CKL("k_flux_ct_rewrite");
  c->flux_ct_done = true;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_begin_run(kgpu_ctx *c) {
  int r = ready(c);
  if (r) return r;
  double mws = 10000., tsd;
  const kgpu_config &k = c->cfg;
  if (k.nz > 1) tsd = mws / c->min_dx + mws / c->min_dy + mws / c->min_dz;
  else if (k.ny > 1) tsd = mws / c->min_dx + mws / c->min_dy;
  else tsd = mws / c->min_dx;
  tsd /= k.tsteplim;
  return kgpu_set_tstepdenmax(c, tsd);
}

extern "C" int kgpu_set_tstepdenmax(kgpu_ctx *c, double v) {
  if (!c) return KGPU_EINVAL;
  CK(cudaMemcpyAsync(c->G.scal + S_TSTEPDENMAX, &v, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_get_tstepdenmax(kgpu_ctx *c, double *out) {
  if (!c || !out) return KGPU_EINVAL;
  CK(cudaMemcpyAsync(out, c->G.scal + S_TSTEPDENMAX, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_begin_step(kgpu_ctx *c, double *dt_out) {
  if (!c) return KGPU_EINVAL;
  k_begin_step<<<1, 1, 0, c->stream>>>(c->G);
  CKL("k_begin_step");
  if (dt_out) CK(cudaMemcpyAsync(dt_out, c->G.scal + S_DT, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// one RK2 step (ko.c:571-626) with dt in device memory
// do_correct (finite.c:605-640) on the stream: the polar-axis corrections
// the context has switched on, in the reference's order
static int launch_correct(kgpu_ctx *c) {
  Grid &G = c->G;
  const int nc = c->polar_nc;
  if (c->polar_flags & KGPU_POLAR_CORRECT) {
    k_correct_polar<<<nblocks(2L * G.nx * G.nz * nc, 128), 128, 0, c->stream>>>(G, nc, 1);
    CKL("k_correct_polar");
  }
  if (c->polar_flags & KGPU_POLAR_CORRECT_3D) {
    k_correct_polar<<<nblocks(2L * G.nx * G.nz * nc, 128), 128, 0, c->stream>>>(G, nc, 2);
    CKL("k_correct_polar");
  }
  if (c->polar_flags & KGPU_POLAR_SMOOTH) {
    k_smooth_polar<<<nblocks(2L * G.nx * nc, 128), 128, 0, c->stream>>>(G, nc);
    CKL("k_smooth_polar");
  }
  return 0;
}

// save_avg (fileop.c:10-70) on the stream: the face fluxes get flux_ct's
// rewrite from the corner EMFs of the last op_explicit (the reference's
// flbx/flby/flbz hold it when its loop calls save_avg), then every domain
// cell adds its p2avg quantities times dt (device memory) to the sums.
static int enqueue_avg(kgpu_ctx *c, const double *dtp) {
  Grid &G = c->G;
  if (!c->flux_ct_done) {
    Box eb{0, 0, 0, G.nx + 1, G.ny + 1, G.nz + 1};
    { LaunchScope ls(c, K_AVG); k_flux_ct_rewrite<<<nblocks(eb.n(), 128), 128, 0, c->stream>>>(G, eb); }
    CKL("k_flux_ct_rewrite");
    c->flux_ct_done = true;
  }
  int r;
  { LaunchScope ls(c, K_AVG); r = avg_enqueue(G, c->avg_units, dtp, c->pavg, c->avgtime, c->stream); }
  if (r < 0) return set_err("k_save_avg", cudaGetLastError());
  return 0;
}

static int enqueue_rk2(kgpu_ctx *c) {
  Grid &G = c->G;
  int r;
  { LaunchScope ls(c, K_BEGIN); k_begin_step<<<1, 1, 0, c->stream>>>(G); }
  CKL("k_begin_step");
  if (c->polar_flags) {
    // copyi_u(1.,u,ut0) before do_correct (ko.c:577-579): ut0 keeps the
    // uncorrected state
    CK(cudaMemcpyAsync(G.ut0, G.u, G.ncell * G.nv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if ((r = launch_correct(c))) return r;
    // op_explicit begins with set_bc (finite.c:672), here after the
    // corrected cells changed the ghosts' sources
    if ((r = launch_bc(c))) return r;
    if ((r = launch_explicit(c, G.scal + S_DT, 0.5, nullptr))) return r;
  } else if ((r = launch_explicit(c, G.scal + S_DT, 0.5, G.ut0))) {   // ut0 = U^n
    return r;
  }
  if ((r = launch_u2p(c, 0))) return r;
  if ((r = launch_explicit(c, G.scal + S_DT, 1.0, G.ut1))) return r;   // ut1 = U^{n+1/2}
  if ((r = launch_u2p(c, 1))) return r;                                // u = ut0 + (u - ut1)
  // save_avg(dt) after the second stage's inversion (ko.c:606-610); the
  // combination above changed u only, and p2avg reads p
  if (c->avg_on && (r = enqueue_avg(c, G.scal + S_DT))) return r;
  return 0;
}

extern "C" int kgpu_rk2_steps(kgpu_ctx *c, int nsteps) {
  int r = ready(c);
  if (r) return r;
  if (nsteps < 1) return KGPU_EINVAL;
  for (int s = 0; s < nsteps; s++)
    if ((r = enqueue_rk2(c))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// Captures one step of the given kind into a CUDA graph (kept until the
// kernel arguments change) and replays it nsteps times.
static int run_graph(kgpu_ctx *c, int nsteps, int kind, int (*enqueue)(kgpu_ctx *)) {
  if (c->graph_ready && c->graph_kind != kind) drop_graph(c);
  if (!c->graph_ready) {
    bool prof = c->profiling;
    c->profiling = false;
    long long before = c->launches;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int r = enqueue(c);
    c->graph_launches = c->launches - before;
    c->launches = before;
    c->profiling = prof;
    cudaGraph_t gph;
    cudaError_t e = cudaStreamEndCapture(c->stream, &gph);
    if (r) return r;
    if (e != cudaSuccess) return set_err("cudaStreamEndCapture", e);
    CK(cudaGraphInstantiate(&c->graph_exec, gph, 0));
    c->graph = gph;
    c->graph_ready = true;
    c->graph_kind = kind;
  }
  for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(c->graph_exec, c->stream));
  c->launches += c->graph_launches * nsteps;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_rk2_steps_graph(kgpu_ctx *c, int nsteps) {
  int r = ready(c);
  if (r) return r;
  if (nsteps < 1) return KGPU_EINVAL;
  return run_graph(c, nsteps, 0, enqueue_rk2);
}

// ---------------------------------------------------------------------------
// radiation: the implicit source operator and the RK2IMEX step
// ---------------------------------------------------------------------------
extern "C" int kgpu_set_radiation(kgpu_ctx *c, const kgpu_rad_params *rp, int wavespeed_limiter) {
  if (!c || !rp) return KGPU_EINVAL;
  Grid &G = c->G;
  if (G.nv != NVR) return KGPU_EINVAL;
  if (!(rp->gamma == G.gamma)) return KGPU_EINVAL;   // one adiabatic index for the grid and the solver
  int r;
  void *p;
  if (!G.radp) {
    if ((r = dalloc(c, &p, sizeof(RadParams)))) return r;
    G.radp = (const RadParams *)p;
  }
  c->rp = *rp;
  RadParams R = kgpu_rad_device_params(*rp);
  CK(cudaMemcpyAsync((void *)G.radp, &R, sizeof(R), cudaMemcpyHostToDevice, c->stream));
  if (!c->imp_uu) {
    const long n = (long)G.nx * G.ny * G.nz;
    if (n > 0x7fffffffL) return KGPU_EINVAL;
    c->nimp = n;
    const size_t d8 = sizeof(double);
#define AL(ptr, bytes)                                  \
  do {                                                  \
    if ((r = dalloc(c, &p, (bytes))) != 0) return r;    \
    ptr = (decltype(ptr))p;                             \
  } while (0)
    AL(c->imp_uu, n * NVR * d8); AL(c->imp_pp, n * NVR * d8);
    AL(c->imp_ppo, n * NVR * d8); AL(c->imp_uuo, n * NVR * d8);
    AL(c->imp_g, n * 20 * d8); AL(c->imp_G, n * 20 * d8); AL(c->imp_dt, n * d8);
    AL(c->imp_status, n * sizeof(int)); AL(c->imp_att, n * sizeof(int)); AL(c->imp_it, n * sizeof(int));
    CK(cudaMemsetAsync(c->imp_att, 0, n * sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->imp_it, 0, n * sizeof(int), c->stream));
    AL(c->imp_work, kgpu_rad_work_bytes((int)n));
#undef AL
  }
  CK(cudaStreamSynchronize(c->stream));
  G.rad = 1;
  G.rad_limiter = wavespeed_limiter ? 1 : 0;
  c->packed_gen = -1;
  drop_graph(c);
  return 0;
}

extern "C" int kgpu_set_implicit_options(kgpu_ctx *c, const kgpu_rad_solver_opts *o) {
  if (!c || !o) return KGPU_EINVAL;
  if (!kgpu_rad_opts_valid(*o)) return KGPU_EINVAL;
  c->imp_opts = *o;
  drop_graph(c);
  return 0;
}

extern "C" int kgpu_get_implicit_options(kgpu_ctx *c, kgpu_rad_solver_opts *o) {
  if (!c || !o) return KGPU_EINVAL;
  *o = c->imp_opts;
  return 0;
}

extern "C" int kgpu_set_implicit_solver(kgpu_ctx *c, int mode, kgpu_mlp *warm) {
  if (!c || (mode != KGPU_RAD_PLAIN && mode != KGPU_RAD_BATCHED && mode != KGPU_RAD_PERSISTENT)) return KGPU_EINVAL;
  if (warm && mode == KGPU_RAD_PLAIN) return KGPU_EINVAL;   // the warm start runs in the queued solvers
  if (!c->G.rad) return KGPU_ESTATE;
  if (warm && !c->imp_X) {
    void *p;
    int r;
    if ((r = dalloc(c, &p, c->nimp * 16 * sizeof(float)))) return r;
    c->imp_X = (float *)p;
    if ((r = dalloc(c, &p, c->nimp * 8 * sizeof(float)))) return r;
    c->imp_Y = (float *)p;
  }
  c->imp_mode = mode;
  c->warm = warm;
  drop_graph(c);
  return 0;
}

extern "C" int kgpu_set_warm_gate(kgpu_ctx *c, int iters) {
  if (!c || iters < -1) return KGPU_EINVAL;
  c->warm_gate = iters;
  drop_graph(c);
  return 0;
}

// the per-cell metric of the domain for the solver, once per metric
static int ensure_packed(kgpu_ctx *c) {
  if (c->packed_gen == c->metric_gen) return 0;
  Box db = domain_box(c->G);
  k_imp_pack_metric<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(c->G, db, c->imp_g, c->imp_G);
  CKL("k_imp_pack_metric");
  CK(cudaStreamSynchronize(c->stream));
  c->packed_gen = c->metric_gen;
  return 0;
}

// op_implicit with time step fac * dtp[0]: solve, scatter, RADIMP fixup
static int enqueue_implicit(kgpu_ctx *c, const double *dtp, double fac) {
  Grid &G = c->G;
  Box db = domain_box(G);
  const int n = (int)c->nimp;
  { LaunchScope ls(c, K_IMP_GATHER);
    k_imp_gather<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(G, db, dtp, fac, c->imp_uu, c->imp_pp, c->imp_dt); }
  CKL("k_imp_gather");
  const float *ypred = nullptr;
  if (c->warm) {
    LaunchScope ls(c, K_IMP_WARM);
    int r = kgpu_rad_features_device(n, &c->rp, c->imp_pp, c->imp_g, c->imp_G, c->imp_dt, c->imp_X, c->stream);
    if (!r) r = kgpu_mlp_forward(c->warm, c->imp_X, n, c->imp_Y, c->stream);
    if (r) return r;
    c->launches += 1;   // two kernels under one scope
    ypred = c->imp_Y;
  }
  {
    LaunchScope ls(c, K_IMP_SOLVE);
    long long nl = 0;
    int r = kgpu_rad_solve_enqueue(n, &c->rp, c->imp_uu, c->imp_pp, c->imp_g, c->imp_G, c->imp_dt, ypred, c->imp_ppo,
                                   c->imp_uuo, c->imp_status, c->imp_att, c->imp_it, c->imp_mode, c->imp_work,
                                   c->stream, G.cnt + C_IMP_ITERS, &nl, c->warm_gate, &c->imp_opts);
    if (r) return r;
    c->launches += nl - 1;
  }
  { LaunchScope ls(c, K_IMP_SCATTER);
    k_imp_scatter<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(G, db, c->imp_ppo, c->imp_uuo, c->imp_status); }
  CKL("k_imp_scatter");
  { LaunchScope ls(c, K_FIXUP); k_fixup<<<nblocks(db.n(), 128), 128, 0, c->stream>>>(G, db, c->fixmark); }
  CKL("k_fixup");
  { LaunchScope ls(c, K_COMMIT); k_commit<<<nblocks(db.n(), 256), 256, 0, c->stream>>>(G, db, c->fixmark, 0, c->u2pq.n); }
  CKL("k_commit");
  return 0;
}

// one RK2IMEX step (ko.c:444-570) with dt in device memory
static int enqueue_rk2imex(kgpu_ctx *c) {
  Grid &G = c->G;
  const double gam = 1. - 1. / sqrt(2.);
  const double *dtp = G.scal + S_DT;
  Box db = domain_box(G);
  const unsigned nb = nblocks(db.n(), 128);
  int r;
  { LaunchScope ls(c, K_BEGIN); k_begin_step<<<1, 1, 0, c->stream>>>(G); }
  CKL("k_begin_step");
  CK(cudaMemcpyAsync(G.ut0, G.u, G.ncell * G.nv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if ((r = enqueue_implicit(c, dtp, gam))) return r;                       // U(1) = implicit from U(n)
  { LaunchScope ls(c, K_IMEX); k_imex_rate<<<nb, 128, 0, c->stream>>>(G, db, dtp, gam, G.ut0, c->drt1, G.ut1); }
  CKL("k_imex_rate");                                                       // R(U(1)); ut1 = U(1)
  if ((r = launch_u2p(c, 0))) return r;
  if (c->polar_flags && ((r = launch_correct(c)) || (r = launch_bc(c)))) return r;
  if ((r = launch_explicit(c, dtp, 1.0, nullptr))) return r;
  { LaunchScope ls(c, K_IMEX);
    k_imex_stage1<<<nb, 128, 0, c->stream>>>(G, db, dtp, gam, G.ut0, G.ut1, c->dut1, c->drt1, G.ut1); }
  CKL("k_imex_stage1");                                                     // F(U(1)); u; uforget = u
  if ((r = launch_u2p(c, 0))) return r;
  if (c->polar_flags && (r = launch_correct(c))) return r;
  if ((r = enqueue_implicit(c, dtp, gam))) return r;                       // U(2)
  if (c->avg_on && (r = enqueue_avg(c, dtp))) return r;                    // save_avg(dt), ko.c:504-507
  { LaunchScope ls(c, K_IMEX); k_imex_rate<<<nb, 128, 0, c->stream>>>(G, db, dtp, gam, G.ut1, c->drt2, G.ut1); }
  CKL("k_imex_rate");                                                       // R(U(2)); ut2 = U(2)
  if ((r = launch_u2p(c, 0))) return r;
  if (c->polar_flags && ((r = launch_correct(c)) || (r = launch_bc(c)))) return r;
  if ((r = launch_explicit(c, dtp, 1.0, nullptr))) return r;
  { LaunchScope ls(c, K_IMEX);
    k_imex_final<<<nb, 128, 0, c->stream>>>(G, db, dtp, G.ut0, G.ut1, c->dut1, c->drt1, c->drt2); }
  CKL("k_imex_final");
  if ((r = launch_u2p(c, 0))) return r;
  if (c->polar_flags && (r = launch_correct(c))) return r;
  return 0;
}

static int ready_rad(kgpu_ctx *c) {
  int r = ready(c);
  if (r) return r;
  if (!c->G.rad) return KGPU_ESTATE;
  return ensure_packed(c);
}

extern "C" int kgpu_get_implicit_buffers(kgpu_ctx *c, int *n, const double **pp_in, const double **uu_in,
                                         const double **pp_out, const double **g20, const double **G20,
                                         const double **dt, const int **status, const int **attempt,
                                         const int **iters) {
  if (!c || !n) return KGPU_EINVAL;
  if (!c->G.rad) return KGPU_ESTATE;
  *n = (int)c->nimp;
  if (pp_in) *pp_in = c->imp_pp;
  if (uu_in) *uu_in = c->imp_uu;
  if (pp_out) *pp_out = c->imp_ppo;
  if (g20) *g20 = c->imp_g;
  if (G20) *G20 = c->imp_G;
  if (dt) *dt = c->imp_dt;
  if (status) *status = c->imp_status;
  if (attempt) *attempt = c->imp_att;
  if (iters) *iters = c->imp_it;
  return 0;
}

extern "C" int kgpu_rk2imex_steps(kgpu_ctx *c, int nsteps) {
  int r = ready_rad(c);
  if (r) return r;
  if (nsteps < 1) return KGPU_EINVAL;
  for (int s = 0; s < nsteps; s++)
    if ((r = enqueue_rk2imex(c))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int kgpu_op_implicit_impl(kgpu_ctx *c, double dt) {
  int r = ready_rad(c);
  if (r) return r;
  CK(cudaMemcpyAsync(c->G.scal + S_T, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if ((r = enqueue_implicit(c, c->G.scal + S_T, 1.0))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_rk2imex_steps_graph(kgpu_ctx *c, int nsteps) {
  int r = ready_rad(c);
  if (r) return r;
  if (nsteps < 1) return KGPU_EINVAL;
  return run_graph(c, nsteps, 1, enqueue_rk2imex);
}

// ---------------------------------------------------------------------------
// tuning and the autotuner
// ---------------------------------------------------------------------------
extern "C" int kgpu_get_tuning(kgpu_ctx *c, kgpu_tuning *t) {
  if (!c || !t) return KGPU_EINVAL;
  t->flux_blocks = c->flux_blocks;
  t->flux_split = c->flux_split;
  t->update_blocks = c->update_blocks;
  t->u2p_blocks = c->u2p_blocks;
  t->u2p_pass_iters = c->u2p_pass_iters;
  t->implicit_mode = c->imp_mode;
  t->implicit = c->imp_opts;
  return 0;
}

extern "C" int kgpu_set_tuning(kgpu_ctx *c, const kgpu_tuning *t) {
  if (!c || !t || !tuning_valid(*t)) return KGPU_EINVAL;
  if (c->warm && t->implicit_mode == KGPU_RAD_PLAIN) return KGPU_EINVAL;
  c->flux_blocks = t->flux_blocks;
  c->flux_split = t->flux_split;
  c->update_blocks = t->update_blocks;
  c->u2p_blocks = t->u2p_blocks;
  c->u2p_pass_iters = t->u2p_pass_iters;
  c->imp_mode = t->implicit_mode;
  c->imp_opts = t->implicit;
  drop_graph(c);
  return 0;
}

extern "C" int kgpu_tune_select(int n, const double *ms, int incumbent, double min_gain) {
  if (n < 1 || !ms || incumbent < 0 || incumbent >= n || !(min_gain >= 0.)) return KGPU_EINVAL;
  int best = -1;
  for (int i = 0; i < n; i++)
    if (std::isfinite(ms[i]) && ms[i] >= 0. && (best < 0 || ms[i] < ms[best])) best = i;
  if (best < 0 || best == incumbent) return incumbent;
  const double inc = ms[incumbent];
  if (!(std::isfinite(inc) && inc >= 0.)) return best;   // the incumbent's trial failed
  return ms[best] < inc * (1. - min_gain) ? best : incumbent;
}

namespace {
struct DevMemRaii {
  void *p = nullptr;
  ~DevMemRaii() {
    if (p) cudaFree(p);
  }
};
struct TuneKey {
  int dev, nx, ny, nz, nv, int_order, fluxmethod, rad;
  bool operator<(const TuneKey &o) const {
    return std::tie(dev, nx, ny, nz, nv, int_order, fluxmethod, rad) <
           std::tie(o.dev, o.nx, o.ny, o.nz, o.nv, o.int_order, o.fluxmethod, o.rad);
  }
};
std::map<TuneKey, kgpu_tuning> g_tuned;   // choices of this process
std::mutex g_tuned_mutex;

// One knob of kgpu_tuning: candidate values and access to the field.
struct Knob {
  int *(*field)(kgpu_tuning &);
  std::vector<int> values;
};
}  // namespace

// time per step (ms) of `steps` steps from the saved state under tuning t;
// a negative value when a step fails
static double tune_trial(kgpu_ctx *c, const kgpu_tuning &t, int steps, const double *u0, const double *p0,
                         double tsd, cudaEvent_t ea, cudaEvent_t eb) {
  if (kgpu_set_tuning(c, &t)) return -1.;
  Grid &G = c->G;
  const size_t bytes = (size_t)G.ncell * G.nv * sizeof(double);
  if (cudaMemcpyAsync(G.u, u0, bytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) return -1.;
  if (cudaMemcpyAsync(G.p, p0, bytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) return -1.;
  if (cudaMemcpyAsync(G.scal + S_TSTEPDENMAX, &tsd, sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    return -1.;
  if (cudaEventRecord(ea, c->stream) != cudaSuccess) return -1.;
  for (int i = 0; i < steps; i++)
    if ((G.rad ? enqueue_rk2imex(c) : enqueue_rk2(c)) != 0) return -1.;
  if (cudaEventRecord(eb, c->stream) != cudaSuccess) return -1.;
  if (cudaEventSynchronize(eb) != cudaSuccess) return -1.;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ea, eb) != cudaSuccess) return -1.;
  return (double)ms / steps;
}

extern "C" int kgpu_autotune(kgpu_ctx *c, int steps, double min_gain, int reuse, kgpu_tuning *chosen, double *ms_out) {
  if (!c || steps < 1 || !(min_gain >= 0.)) return KGPU_EINVAL;
  int r = c->G.rad ? ready_rad(c) : ready(c);
  if (r) return r;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  const kgpu_config &k = c->cfg;
  const TuneKey key{dev, k.nx, k.ny, k.nz, k.nv, k.int_order, k.fluxmethod, c->G.rad};
  kgpu_tuning cur;
  kgpu_get_tuning(c, &cur);
  if (reuse) {
    std::lock_guard<std::mutex> lock(g_tuned_mutex);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      kgpu_tuning t = it->second;
      t.implicit.warm_attempts = cur.implicit.warm_attempts;   // a choice of the caller, not of the tuner
      if (c->warm && t.implicit_mode == KGPU_RAD_PLAIN) t.implicit_mode = cur.implicit_mode;
      if ((r = kgpu_set_tuning(c, &t))) return r;
      if (chosen) *chosen = t;
      if (ms_out) ms_out[0] = ms_out[1] = -1.;
      return 0;
    }
  }
  // the state the trials start from, and what the trials change besides it
  Grid &G = c->G;
  const size_t bytes = (size_t)G.ncell * G.nv * sizeof(double);
  DevMemRaii save_u, save_p;
  CK(cudaMalloc(&save_u.p, bytes));
  CK(cudaMalloc(&save_p.p, bytes));
  CK(cudaMemcpyAsync(save_u.p, G.u, bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(save_p.p, G.p, bytes, cudaMemcpyDeviceToDevice, c->stream));
  double tsd = 0.;
  unsigned long long cnt[C_NCNT];
  CK(cudaMemcpyAsync(&tsd, G.scal + S_TSTEPDENMAX, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(cnt, G.cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const bool prof = c->profiling;
  c->profiling = false;
  const long long launches = c->launches;
  cudaEvent_t ea, eb;
  CK(cudaEventCreate(&ea));
  CK(cudaEventCreate(&eb));
  std::vector<Knob> knobs = {
      {[](kgpu_tuning &t) { return &t.flux_split; }, {0, 1}},
      {[](kgpu_tuning &t) { return &t.flux_blocks; }, {5, 6, 7, 8}},
      {[](kgpu_tuning &t) { return &t.update_blocks; }, {3, 4, 5}},
      {[](kgpu_tuning &t) { return &t.u2p_blocks; }, {4, 5, 6}},
      {[](kgpu_tuning &t) { return &t.u2p_pass_iters; }, {4, 8, 16}},
  };
  if (G.rad) {
    knobs.push_back({[](kgpu_tuning &t) { return &t.implicit_mode; }, {KGPU_RAD_BATCHED, KGPU_RAD_PERSISTENT}});
    knobs.push_back({[](kgpu_tuning &t) { return &t.implicit.inner_cap; }, {32, 64, 128}});
  }
  kgpu_tuning best = cur;
  if (best.implicit_mode == KGPU_RAD_PLAIN && G.rad && !c->warm) best.implicit_mode = KGPU_RAD_BATCHED;
  const double ms_start = tune_trial(c, cur, steps, (const double *)save_u.p, (const double *)save_p.p, tsd, ea, eb);
  double ms_best = ms_start;
  int status = 0;
  for (size_t ki = 0; ki < knobs.size() && !status; ki++) {
    std::vector<Knob> round = {knobs[ki]};
    // the settings that belong to the solver form just chosen
    if (G.rad && knobs[ki].field(best) == &best.implicit.inner_cap) {
      if (best.implicit_mode == KGPU_RAD_BATCHED) {
        round.push_back({[](kgpu_tuning &t) { return &t.implicit.pass_iters; }, {4, 8, 16}});
        round.push_back({[](kgpu_tuning &t) { return &t.implicit.tail; }, {0, 4, 8, 16}});
        round.push_back({[](kgpu_tuning &t) { return &t.implicit.hard; }, {-1, 8, 16, 32}});
      } else {
        round.push_back({[](kgpu_tuning &t) { return &t.implicit.thin; }, {4, 8, 16}});
      }
    }
    for (const Knob &kn : round) {
      std::vector<double> ms;
      int inc = -1;
      for (size_t i = 0; i < kn.values.size(); i++) {
        kgpu_tuning t = best;
        *kn.field(t) = kn.values[i];
        if (*kn.field(t) == *kn.field(best)) inc = (int)i;
        ms.push_back(tune_trial(c, t, steps, (const double *)save_u.p, (const double *)save_p.p, tsd, ea, eb));
      }
      if (inc < 0) {   // the incumbent value is not a candidate: time it as one more
        ms.push_back(tune_trial(c, best, steps, (const double *)save_u.p, (const double *)save_p.p, tsd, ea, eb));
        inc = (int)ms.size() - 1;
      }
      const int pick = kgpu_tune_select((int)ms.size(), ms.data(), inc, min_gain);
      if (pick < 0) { status = KGPU_EINVAL; break; }
      if (pick != inc) {
        *kn.field(best) = kn.values[pick];
        ms_best = ms[pick];
      } else {
        ms_best = ms[inc];
      }
    }
  }
  cudaEventDestroy(ea);
  cudaEventDestroy(eb);
  // back to the saved state with the choice applied
  int r2 = kgpu_set_tuning(c, &best);
  CK(cudaMemcpyAsync(G.u, save_u.p, bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(G.p, save_p.p, bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(G.scal + S_TSTEPDENMAX, &tsd, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(G.cnt, cnt, sizeof(cnt), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->profiling = prof;
  c->launches = launches;
  if (status) return status;
  if (r2) return r2;
  if (ms_start < 0. || ms_best < 0.) return set_err("kgpu_autotune: a trial step failed", cudaErrorUnknown);
  {
    std::lock_guard<std::mutex> lock(g_tuned_mutex);
    g_tuned[key] = best;
  }
  if (chosen) *chosen = best;
  if (ms_out) {
    ms_out[0] = ms_start;
    ms_out[1] = ms_best;
  }
  return 0;
}

extern "C" int kgpu_get_counters(kgpu_ctx *c, unsigned long long out[4]) {
  if (!c || !out) return KGPU_EINVAL;
  unsigned long long h[C_NCNT];
  CK(cudaMemcpyAsync(h, c->G.cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < 4; i++) out[i] = h[i];
  return 0;
}

extern "C" int kgpu_get_counters_ex(kgpu_ctx *c, unsigned long long *out, int n) {
  if (!c || !out || n < 0) return KGPU_EINVAL;
  unsigned long long h[C_NCNT];
  CK(cudaMemcpyAsync(h, c->G.cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n && i < C_NCNT; i++) out[i] = h[i];
  return n < C_NCNT ? n : C_NCNT;
}

extern "C" int kgpu_set_u2p_pass_iters(kgpu_ctx *c, int n) {
  if (!c || n < 1) return KGPU_EINVAL;
  c->u2p_pass_iters = n;
  drop_graph(c);
  return 0;
}

extern "C" int kgpu_reset_counters(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  CK(cudaMemsetAsync(c->G.cnt, 0, C_NCNT * sizeof(unsigned long long), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// ---------------------------------------------------------------------------
// problem set-up on the host (same arithmetic as the reference plug-in, run
// with the host C library) then uploaded
// ---------------------------------------------------------------------------
extern "C" int kgpu_init_orszag_tang(kgpu_ctx *c) {
  int r = ready(c);
  if (r) return r;
  const kgpu_config &k = c->cfg;
  Grid &G = c->G;
  const long n = G.ncell;
  std::vector<double> u(n * G.nv, 0.), p(n * G.nv, 0.);
  Geom g;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 5; b++) g.gg[a][b] = g.GG[a][b] = 0.;
  g.gg[0][0] = -1.; g.gg[1][1] = g.gg[2][2] = g.gg[3][3] = 1.; g.gg[3][4] = 1.;
  g.GG[0][0] = -1.; g.GG[1][1] = g.GG[2][2] = g.GG[3][3] = 1.; g.GG[3][4] = 0.;
  g.gdet = 1.; g.gttpert = 0.;
  for (int ix = 0; ix < k.nx; ix++)
    for (int iy = 0; iy < k.ny; iy++)
      for (int iz = 0; iz < k.nz; iz++) {
        // cell centres, finite.c:1647: x = (xb[i+1] + xb[i]) / 2
        double xx = .5 * (c->hxb[0][ix + 1 + k.ng] + c->hxb[0][ix + k.ng]);
        double yy = .5 * (c->hxb[1][iy + 1 + k.ng] + c->hxb[1][iy + k.ng]);
        // VEL3 -> VELR (relele.c:208-232) for the coordinate three-velocity
        double v3[4] = {0., -0.5 * sin(yy), 0.5 * sin(xx), 0.};
        double a = 0., b = 0., uc[4];
        for (int i = 1; i < 4; i++) {
          a += 2. * v3[i] * g.gg[0][i];
          for (int j = 1; j < 4; j++) b += v3[i] * v3[j] * g.gg[i][j];
        }
        uc[0] = sqrt(-1. / (g.gg[0][0] + a + b));
        for (int i = 1; i < 4; i++) uc[i] = v3[i] * uc[0];
        for (int i = 1; i < 4; i++) uc[i] = uc[i] - uc[0] * g.GG[0][i] / g.GG[0][0];
        double pp[NVMAX], uu[NVMAX];
        pp[RHO] = 25. / (36. * M_PI);
        pp[UU] = (5. / (12. * M_PI)) / (k.gamma - 1.);
        pp[VX] = uc[1]; pp[VY] = uc[2]; pp[VZ] = uc[3];
        pp[B1] = -sin(yy) / sqrt(4. * M_PI);
        pp[B2] = sin(2. * xx) / sqrt(4. * M_PI);
        pp[B3] = 0.;
        pp[ENTR] = calc_Sfromu(k.gamma, pp[RHO], pp[UU]);
        p2u_full(G, pp, uu, g);
        long cidx = cell_index(G, ix, iy, iz);
        for (int iv = 0; iv < G.nv; iv++) {
          u[cidx * G.nv + iv] = uu[iv];
          p[cidx * G.nv + iv] = pp[iv];
        }
      }
  if ((r = kgpu_upload_state(c, u.data(), p.data()))) return r;
  if ((r = launch_bc(c))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// ---------------------------------------------------------------------------
// batched per-cell solvers
// ---------------------------------------------------------------------------
__global__ void k_u2p_cells(Grid G, int n, const double *uu, double *pp, const double *met, int *status, int *fixup) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Geom g;
  load_geom(met, n, i, g);
  double u[NVMAX], p[NVMAX];
  for (int iv = 0; iv < NVMAX; iv++) {
    u[iv] = uu[(long)iv * n + i];
    p[iv] = pp[(long)iv * n + i];
  }
  int fix = 0;
  int ret = u2p(G, u, p, g, fix);
  for (int iv = 0; iv < NVMAX; iv++) pp[(long)iv * n + i] = p[iv];
  status[i] = ret;
  fixup[i] = fix;
}
__global__ void k_p2u_cells(Grid G, int n, const double *pp, double *uu, const double *met) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Geom g;
  load_geom(met, n, i, g);
  double u[NVMAX], p[NVMAX];
  for (int iv = 0; iv < NVMAX; iv++) p[iv] = pp[(long)iv * n + i];
  p2u_full(G, p, u, g);
  for (int iv = 0; iv < NVMAX; iv++) uu[(long)iv * n + i] = u[iv];
}

static void to_soa(const double *aos, std::vector<double> &soa, int n, int m) {
  soa.resize((size_t)n * m);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < m; k++) soa[(size_t)k * n + i] = aos[(size_t)i * m + k];
}

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

extern "C" int kgpu_u2p_cells(int n, const kgpu_config *cfg, const double *uu, double *pp, const double *g,
                              const double *Gi, int *status, int *fixup) {
  if (n < 0 || !cfg || (n > 0 && (!uu || !pp || !g || !Gi || !status || !fixup))) return KGPU_EINVAL;
  if (cfg->nv != 9) return KGPU_EINVAL;
  if (n == 0) return 0;
  Grid G;
  fill_grid_params(G, *cfg);
  std::vector<double> su, sp, sm((size_t)n * 40), tmp;
  to_soa(uu, su, n, G.nv);
  to_soa(pp, sp, n, G.nv);
  to_soa(g, tmp, n, 20);
  memcpy(sm.data(), tmp.data(), (size_t)n * 20 * sizeof(double));
  to_soa(Gi, tmp, n, 20);
  memcpy(sm.data() + (size_t)n * 20, tmp.data(), (size_t)n * 20 * sizeof(double));
  DevBuf du, dp, dm, ds, df;
  CK(cudaMalloc(&du.p, su.size() * 8)); CK(cudaMalloc(&dp.p, sp.size() * 8));
  CK(cudaMalloc(&dm.p, sm.size() * 8)); CK(cudaMalloc(&ds.p, n * 4)); CK(cudaMalloc(&df.p, n * 4));
  CK(cudaMemcpy(du.p, su.data(), su.size() * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dp.p, sp.data(), sp.size() * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dm.p, sm.data(), sm.size() * 8, cudaMemcpyHostToDevice));
  k_u2p_cells<<<nblocks(n, 128), 128>>>(G, n, (double *)du.p, (double *)dp.p, (double *)dm.p, (int *)ds.p, (int *)df.p);
  CKL("k_u2p_cells");
  CK(cudaMemcpy(sp.data(), dp.p, sp.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(status, ds.p, n * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(fixup, df.p, n * 4, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; i++)
    for (int k = 0; k < G.nv; k++) pp[(size_t)i * G.nv + k] = sp[(size_t)k * n + i];
  return 0;
}

// u2p (u2p.c:176-485) with all its outputs on cells in KORAL's cell-major
// layout: the MHD inversion, then (with radiation) u2p_rad, and the
// corrected/fixups flags as the reference sets them
__global__ void k_u2p_cells_full(Grid G, RadParams R, int hasrad, int n, const double *uu, double *pp,
                                 const double *g20, const double *G20, int *status, int *corrected, int *fixups) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  RadGeom rg;
  rad_geom(g20 + 20L * i, G20 + 20L * i, rg);
  const int nv = G.nv;
  double u[NVR], p[NVR];
  for (int iv = 0; iv < nv; iv++) {
    u[iv] = uu[(long)i * nv + iv];
    p[iv] = pp[(long)i * nv + iv];
  }
  int fix = 0;
  const int ret = u2p(G, u, p, rg.g, fix);
  int radcor = 0;
  if (hasrad) u2p_rad(R, u, p, rg, radcor);
  for (int iv = 0; iv < nv; iv++) pp[(long)i * nv + iv] = p[iv];
  status[i] = ret;
  corrected[3L * i + 0] = ret < 0 ? 1 : 0;
  corrected[3L * i + 1] = radcor > 0 ? 1 : 0;
  corrected[3L * i + 2] = 0;
  fixups[2L * i + 0] = fix;
  fixups[2L * i + 1] = radcor > 0 ? 1 : 0;
}

extern "C" int kgpu_u2p_cells_full(int n, const kgpu_config *cfg, const kgpu_rad_params *rp, const double *uu,
                                   double *pp, const double *g, const double *Gi, int *status, int *corrected,
                                   int *fixups) {
  if (n < 0 || !cfg || (n > 0 && (!uu || !pp || !g || !Gi || !status || !corrected || !fixups))) return KGPU_EINVAL;
  if (!((cfg->nv == 9 && !rp) || (cfg->nv == NVR && rp))) return KGPU_EINVAL;
  if (rp && !(rp->gamma == cfg->gamma)) return KGPU_EINVAL;
  if (n == 0) return 0;
  Grid G;
  fill_grid_params(G, *cfg);
  RadParams R;
  memset(&R, 0, sizeof(R));
  if (rp) R = kgpu_rad_device_params(*rp);
  const size_t bs = (size_t)n * cfg->nv * 8, bm = (size_t)n * 20 * 8;
  DevBuf du, dp, dg, dG, ds, dc, df;
  CK(cudaMalloc(&du.p, bs)); CK(cudaMalloc(&dp.p, bs)); CK(cudaMalloc(&dg.p, bm)); CK(cudaMalloc(&dG.p, bm));
  CK(cudaMalloc(&ds.p, (size_t)n * 4)); CK(cudaMalloc(&dc.p, (size_t)n * 12)); CK(cudaMalloc(&df.p, (size_t)n * 8));
  CK(cudaMemcpy(du.p, uu, bs, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dp.p, pp, bs, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dg.p, g, bm, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dG.p, Gi, bm, cudaMemcpyHostToDevice));
  k_u2p_cells_full<<<nblocks(n, 128), 128>>>(G, R, rp ? 1 : 0, n, (const double *)du.p, (double *)dp.p,
                                             (const double *)dg.p, (const double *)dG.p, (int *)ds.p, (int *)dc.p,
                                             (int *)df.p);
  CKL("k_u2p_cells_full");
  CK(cudaMemcpy(pp, dp.p, bs, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(status, ds.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(corrected, dc.p, (size_t)n * 12, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(fixups, df.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int kgpu_p2u_cells(int n, const kgpu_config *cfg, const double *pp, double *uu, const double *g,
                              const double *Gi) {
  if (n < 0 || !cfg || (n > 0 && (!uu || !pp || !g || !Gi))) return KGPU_EINVAL;
  if (cfg->nv != 9) return KGPU_EINVAL;
  if (n == 0) return 0;
  Grid G;
  fill_grid_params(G, *cfg);
  std::vector<double> sp, sm((size_t)n * 40), tmp, su((size_t)n * G.nv);
  to_soa(pp, sp, n, G.nv);
  to_soa(g, tmp, n, 20);
  memcpy(sm.data(), tmp.data(), (size_t)n * 20 * sizeof(double));
  to_soa(Gi, tmp, n, 20);
  memcpy(sm.data() + (size_t)n * 20, tmp.data(), (size_t)n * 20 * sizeof(double));
  DevBuf du, dp, dm;
  CK(cudaMalloc(&du.p, su.size() * 8)); CK(cudaMalloc(&dp.p, sp.size() * 8)); CK(cudaMalloc(&dm.p, sm.size() * 8));
  CK(cudaMemcpy(dp.p, sp.data(), sp.size() * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dm.p, sm.data(), sm.size() * 8, cudaMemcpyHostToDevice));
  k_p2u_cells<<<nblocks(n, 128), 128>>>(G, n, (double *)dp.p, (double *)du.p, (double *)dm.p);
  CKL("k_p2u_cells");
  CK(cudaMemcpy(su.data(), du.p, su.size() * 8, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; i++)
    for (int k = 0; k < G.nv; k++) uu[(size_t)i * G.nv + k] = su[(size_t)k * n + i];
  return 0;
}

// ---------------------------------------------------------------------------
// instrumentation
// ---------------------------------------------------------------------------
extern "C" int kgpu_get_stream(kgpu_ctx *c, void **stream) {
  if (!c || !stream) return KGPU_EINVAL;
  *stream = (void *)c->stream;
  return 0;
}

extern "C" int kgpu_profile_enable(kgpu_ctx *c, int on) {
  if (!c) return KGPU_EINVAL;
  c->profiling = on != 0;
  return 0;
}

static int drain_profile(kgpu_ctx *c) {
  CK(cudaStreamSynchronize(c->stream));
  for (auto &r : c->prof) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, r.a, r.b));
    c->prof_ms[r.id] += ms;
    c->prof_n[r.id] += 1;
    c->evpool.push_back(r.a);
    c->evpool.push_back(r.b);
  }
  c->prof.clear();
  return 0;
}

extern "C" int kgpu_profile_read(kgpu_ctx *c, int kernel, double *total_ms, long long *count, const char **name) {
  if (!c || kernel < 0 || kernel >= K_NKERNELS) return KGPU_EINVAL;
  int r = drain_profile(c);
  if (r) return r;
  if (total_ms) *total_ms = c->prof_ms[kernel];
  if (count) *count = c->prof_n[kernel];
  if (name) *name = kKernelNames[kernel];
  return 0;
}

extern "C" int kgpu_profile_reset(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  int r = drain_profile(c);
  if (r) return r;
  for (int k = 0; k < K_NKERNELS; k++) {
    c->prof_ms[k] = 0.;
    c->prof_n[k] = 0;
  }
  return 0;
}

extern "C" int kgpu_launch_count(kgpu_ctx *c, long long *out) {
  if (!c || !out) return KGPU_EINVAL;
  *out = c->launches;
  return 0;
}

extern "C" int kgpu_num_kernels(void) { return K_NKERNELS; }

// ---------------------------------------------------------------------------
// torus set-up on a context
// ---------------------------------------------------------------------------
// grid of the torus: uniform in x1 = ln(r - r0), x2 in [x2_lo, x2_hi], phi
static int torus_grid(kgpu_ctx *c, const kgpu_torus_params *tp) {
  double lo[3] = {log(tp->r_lo - tp->r0), tp->x2_lo, 0.}, hi[3] = {log(tp->r_hi - tp->r0), tp->x2_hi, 2. * M_PI};
  return kgpu_set_uniform_grid(c, lo, hi);
}

static int torus_floor(kgpu_ctx *c, const kgpu_torus_params *tp) {
  const Grid &G = c->G;
  std::vector<double> fc(G.sx), ff(G.sx + 1);
  int r;
  if ((r = kgpu_fm_torus_floor(tp, c->cfg.nx, c->cfg.ng, c->hxb[0].data(), fc.data(), ff.data()))) return r;
  return kgpu_set_density_floor(c, fc.data(), ff.data());
}

// Host set-up: metric and state computed on the host (the functions the
// set-up tests compare with the reference) and uploaded.
static int init_torus_host(kgpu_ctx *c, const kgpu_torus_params *tp, const kgpu_rad_params *rp, double eradatm) {
  const kgpu_config &k = c->cfg;
  Grid &G = c->G;
  int r;
  std::vector<double> g(G.nmet * 20), Gi(G.nmet * 20), kr(G.nmet * 64);
  std::vector<double> gb[3], Gb[3];
  for (int d = 0; d < 3; d++) {
    gb[d].resize(G.nfmet[d] * 20);
    Gb[d].resize(G.nfmet[d] * 20);
  }
  if ((r = kgpu_mks2_metric_tables(tp->spin, tp->r0, tp->h0, k.nx, k.ny, k.nz, k.ng, k.axisym_metric,
                                   c->hxb[0].data(), c->hxb[1].data(), c->hxb[2].data(), g.data(), Gi.data(),
                                   kr.data(), gb[0].data(), gb[1].data(), gb[2].data(), Gb[0].data(), Gb[1].data(),
                                   Gb[2].data())))
    return r;
  if ((r = kgpu_upload_metric(c, g.data(), Gi.data(), kr.data(), gb[0].data(), gb[1].data(), gb[2].data(),
                              Gb[0].data(), Gb[1].data(), Gb[2].data())))
    return r;
  std::vector<double> u(G.ncell * G.nv), p(G.ncell * G.nv);
  r = rp ? kgpu_fm_radtorus_state(tp, rp, eradatm, &k, c->hxb[0].data(), c->hxb[1].data(), c->hxb[2].data(),
                                  g.data(), Gi.data(), u.data(), p.data())
         : kgpu_fm_torus_state(tp, &k, c->hxb[0].data(), c->hxb[1].data(), c->hxb[2].data(), g.data(), Gi.data(),
                               u.data(), p.data());
  if (r) return r;
  return kgpu_upload_state(c, u.data(), p.data());
}

// Device set-up: metric tables and state computed by kernels straight into
// the context's arrays; nothing but the grid faces and the floor table
// (one value per x index) crosses from the host.
static int init_torus_device(kgpu_ctx *c, const kgpu_torus_params *tp, const kgpu_rad_params *rp, double eradatm) {
  Grid &G = c->G;
  int r = setup_mks2_metric_device(G, tp->spin, tp->r0, tp->h0, c->stream);
  if (r < 0) {
    set_err("setup_mks2_metric_device", cudaGetLastError());
    return r;
  }
  c->launches += r;
  c->have_metric = true;
  c->metric_gen++;
  TorusRadConsts rad{0, 0., 0., 0., 0., 0.};
  if (rp) rad = TorusRadConsts{1, rp->sigma, rp->kb, rp->mu, rp->mp, eradatm};
  // c->stage holds ncell * nv doubles: A_phi and the field maximum fit
  r = setup_fm_torus_device(G, *tp, rad, c->stage, c->stream);
  if (r < 0) {
    set_err("setup_fm_torus_device", cudaGetLastError());
    return r;
  }
  c->launches += r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

static int init_torus(kgpu_ctx *c, const kgpu_torus_params *tp, const kgpu_rad_params *rp, double eradatm,
                      int wavespeed_limiter, bool on_device) {
  if (!c || !tp) return KGPU_EINVAL;
  const kgpu_config &k = c->cfg;
  if (k.nz < 2 || k.ny < 2 || k.nv != (rp ? NVR : 9)) return KGPU_EINVAL;
  int r;
  if ((r = torus_grid(c, tp))) return r;
  if ((r = torus_floor(c, tp))) return r;
  if (rp && (r = kgpu_set_radiation(c, rp, wavespeed_limiter))) return r;
  if ((r = on_device ? init_torus_device(c, tp, rp, eradatm) : init_torus_host(c, tp, rp, eradatm))) return r;
  if ((r = launch_bc(c))) return r;
  CK(cudaStreamSynchronize(c->stream));
  return kgpu_begin_run(c);
}

extern "C" int kgpu_init_fm_torus(kgpu_ctx *c, const kgpu_torus_params *tp) {
  return init_torus(c, tp, nullptr, 0., 0, true);
}
extern "C" int kgpu_init_fm_torus_host(kgpu_ctx *c, const kgpu_torus_params *tp) {
  return init_torus(c, tp, nullptr, 0., 0, false);
}

// The radiative torus: the same set-up with the torus pressure shared by gas
// and radiation in thermal equilibrium, a faint radiation field at rest in
// the atmosphere (eradatm times its gas energy), radiation switched on.
extern "C" int kgpu_init_fm_radtorus(kgpu_ctx *c, const kgpu_torus_params *tp, const kgpu_rad_params *rp,
                                     double eradatm, int wavespeed_limiter) {
  if (!rp) return KGPU_EINVAL;
  return init_torus(c, tp, rp, eradatm, wavespeed_limiter, true);
}
extern "C" int kgpu_init_fm_radtorus_host(kgpu_ctx *c, const kgpu_torus_params *tp, const kgpu_rad_params *rp,
                                          double eradatm, int wavespeed_limiter) {
  if (!rp) return KGPU_EINVAL;
  return init_torus(c, tp, rp, eradatm, wavespeed_limiter, false);
}

// ---------------------------------------------------------------------------
// scalar diagnostics (calc_scalars, postproc.c:996-1105) on the device
// ---------------------------------------------------------------------------
// ISCO radius of a Kerr hole in Boyer-Lindquist r (Bardeen, Press and
// Teukolsky 1972, eq. 2.21), in the operation order of r_ISCO_BL
// (metric.c:3838-3844)
static double isco_bl(double ac) {
  double Z1 = 1. + pow(1. - ac * ac, 1. / 3.) * (pow(1. + ac, 1. / 3.) + pow(1. - ac, 1. / 3.));
  double Z2 = pow(3. * ac * ac + Z1 * Z1, 1. / 2.);
  return (3. + Z2 - pow((3. - Z1) * (3. + Z1 + 2. * Z2), 1. / 2.));
}

// first centre whose x1 exceeds the radius (the loops of calc_mdot,
// calc_Bflux, calc_resmri, calc_meantemp, calc_scalars), NX when none does
static int radial_index(const kgpu_ctx *c, double radius) {
  const int nx = c->cfg.nx, ng = c->cfg.ng;
  const std::vector<double> &xb = c->hxb[0];
  int ix;
  for (ix = 0; ix < nx; ix++)
    if (.5 * (xb[ix + ng] + xb[ix + 1 + ng]) > radius) break;
  return ix;
}

static int diag_prepare(kgpu_ctx *c, const kgpu_scalars_params *sp, DiagIdx &I, DiagConsts &K) {
  if (!c || !sp) return KGPU_EINVAL;
  if (!c->have_grid || !c->have_metric) return KGPU_ESTATE;
  if (!(sp->mass > 0.) || !(fabs(sp->spin) < 1.)) return KGPU_EINVAL;
  if (c->cfg.ny < 4) return KGPU_EINVAL;   // the local luminosity reads theta index 3
  if (!c->diag_work) {
    void *p;
    int r;
    if ((r = dalloc(c, &p, DIAG_WORK * sizeof(double)))) return r;
    c->diag_work = (double *)p;
    if ((r = dalloc(c, &p, NSCALARS * sizeof(double)))) return r;
    c->diag_out = (double *)p;
  }
  const double rhorizon = 1. + sqrt(1 - sp->spin * sp->spin);   // r_horizon_BL, metric.c:3831-3834
  const int nx = c->cfg.nx, ng = c->cfg.ng;
  const double x1last = .5 * (c->hxb[0][nx - 1 + ng] + c->hxb[0][nx + ng]);
  I.ix_mdot = radial_index(c, rhorizon);
  I.ix_mri = radial_index(c, x1last / 2.);
  I.ix_temp = radial_index(c, 15.);
  I.ix_lum = radial_index(c, 5.e3);
  // units (ko.h:4-26, choices.h:340): G, c, the mass in cm
  const double GGG = (6.674e-8 / (1.)), CCC = (2.998e10 / (1.)), MASSCM = (sp->mass * 147700.);
  const double rho1 = (1. / GGG * CCC * CCC / MASSCM / MASSCM), vel1 = (1. * CCC), len1 = (1. * MASSCM);
  K.mdotscale = rho1 * vel1 * len1 * len1;
  const double etaNT = 1. - sqrt(1. - 2. / 3. / isco_bl(sp->spin));   // metric.c:4069
  K.mdotedd = 1.09649 * 2.23e18 * sp->mass * (0.057 / etaNT);          // calc_mdotEdd, postproc.c:2151-2162
  kgpu_rad_params rp;
  int r = kgpu_rad_default_params(&rp, sp->mass, c->cfg.gamma, 6.4e22, 0.34);
  if (r) return r;
  K.kb = rp.kb;
  K.mu = rp.mu;
  K.mp = rp.mp;
  K.bhdisk = sp->bhdisk ? 1 : 0;
  K.rad = c->G.rad ? 1 : 0;
  return 0;
}

extern "C" int kgpu_calc_scalars_device(kgpu_ctx *c, const kgpu_scalars_params *sp, double t, double *scalars_dev) {
  (void)t;   // the scalars of this problem class do not depend on the time
  DiagIdx I;
  DiagConsts K;
  int r = diag_prepare(c, sp, I, K);
  if (r) return r;
  if (!scalars_dev) return KGPU_EINVAL;
  r = diag_scalars_enqueue(c->G, I, K, c->diag_work, scalars_dev, c->stream);
  if (r < 0) return r;
  c->launches += r;
  return 0;
}

// ---------------------------------------------------------------------------
// time averages (save_avg, fileop.c:10-70; p2avg, p2u.c:313-541)
// ---------------------------------------------------------------------------
static int avg_count(const kgpu_ctx *c) { return c->G.nv + navg_vars(c->G.nv, c->G.rad != 0); }

static int avg_prepare(kgpu_ctx *c, double mass) {
  int r = ready(c);
  if (r) return r;
  if (!c->avg_ready) {
    if (!(mass > 0.)) return KGPU_EINVAL;
    if (c->G.rad) {
      c->avg_units = kgpu_rad_device_params(c->rp);
    } else {
      kgpu_rad_params u;
      if ((r = kgpu_rad_default_params(&u, mass, c->G.gamma, 0., 0.))) return r;
      c->avg_units = kgpu_rad_device_params(u);
    }
    void *p;
    if ((r = dalloc(c, &p, (size_t)avg_count(c) * c->G.ncell * sizeof(double)))) return r;
    c->pavg = (double *)p;
    if ((r = dalloc(c, &p, 2 * sizeof(double)))) return r;
    c->avgtime = (double *)p;
    CK(cudaMemsetAsync(c->pavg, 0, (size_t)avg_count(c) * c->G.ncell * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->avgtime, 0, 2 * sizeof(double), c->stream));
    c->avg_ready = true;
  }
  return 0;
}

extern "C" int kgpu_avg_count(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  return avg_count(c);
}

extern "C" int kgpu_set_avg(kgpu_ctx *c, int on, double mass) {
  if (!c || (on != 0 && on != 1)) return KGPU_EINVAL;
  int r = avg_prepare(c, mass);
  if (r) return r;
  if (c->avg_on != (on != 0)) drop_graph(c);
  c->avg_on = on != 0;
  return 0;
}

extern "C" int kgpu_save_avg(kgpu_ctx *c, double dt) {
  if (!c) return KGPU_EINVAL;
  if (!c->avg_ready) return KGPU_ESTATE;
  // the time step of this call in the spare device slot (avgtime[1])
  k_fill<<<1, 1, 0, c->stream>>>(c->avgtime + 1, 1, dt);
  CKL("k_fill");
  int r = enqueue_avg(c, c->avgtime + 1);
  if (r) return r;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_reset_avg(kgpu_ctx *c) {
  if (!c) return KGPU_EINVAL;
  if (!c->avg_ready) return KGPU_ESTATE;
  CK(cudaMemsetAsync(c->pavg, 0, (size_t)avg_count(c) * c->G.ncell * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->avgtime, 0, sizeof(double), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_download_avg(kgpu_ctx *c, double *pavg, double *avgtime) {
  if (!c || !pavg) return KGPU_EINVAL;
  if (!c->avg_ready) return KGPU_ESTATE;
  const int nav = avg_count(c);
  const long n = c->G.ncell;
  // KORAL's layout [cell][quantity], transposed on the device in slabs of
  // cells so that the staging stays small
  const long slab = n < (1L << 18) ? n : (1L << 18);
  DevBuf tmp;
  CK(cudaMalloc(&tmp.p, (size_t)nav * slab * sizeof(double)));
  for (long c0 = 0; c0 < n; c0 += slab) {
    const long m = n - c0 < slab ? n - c0 : slab;
    k_soa_slab_to_aos<<<nblocks(m * nav, 256), 256, 0, c->stream>>>(c->pavg, n, c0, m, nav, (double *)tmp.p);
    CKL("k_soa_slab_to_aos");
    CK(cudaMemcpyAsync(pavg + (size_t)c0 * nav, tmp.p, (size_t)nav * m * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
  }
  if (avgtime) CK(cudaMemcpyAsync(avgtime, c->avgtime, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int kgpu_calc_scalars(kgpu_ctx *c, const kgpu_scalars_params *sp, double t, double *scalars) {
  (void)t;
  if (!scalars) return KGPU_EINVAL;
  DiagIdx I;
  DiagConsts K;
  int r = diag_prepare(c, sp, I, K);
  if (r) return r;
  r = diag_scalars_enqueue(c->G, I, K, c->diag_work, c->diag_out, c->stream);
  if (r < 0) return r;
  c->launches += r;
  CK(cudaMemcpyAsync(scalars, c->diag_out, NSCALARS * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// Metric tables back in KORAL's layout (the inverse of kgpu_upload_metric).
static int download_met(kgpu_ctx *c, const double *src, double *g, double *Gi, long npts) {
  std::vector<double> h(npts * 40);
  CK(cudaMemcpyAsync(h.data(), src, npts * 40 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (long i = 0; i < npts; i++)
    for (int k = 0; k < 20; k++) {
      g[i * 20 + k] = h[k * npts + i];
      Gi[i * 20 + k] = h[(20 + k) * npts + i];
    }
  return 0;
}

extern "C" int kgpu_download_metric(kgpu_ctx *c, double *g, double *Gi, double *gKr, double *gbx, double *gby,
                                    double *gbz, double *Gbx, double *Gby, double *Gbz) {
  if (!c || !g || !Gi || !gKr || !gbx || !gby || !gbz || !Gbx || !Gby || !Gbz) return KGPU_EINVAL;
  if (!c->have_metric) return KGPU_ESTATE;
  Grid &G = c->G;
  int r;
  if ((r = download_met(c, G.met_c, g, Gi, G.nmet))) return r;
  double *gb[3] = {gbx, gby, gbz}, *Gb[3] = {Gbx, Gby, Gbz};
  for (int d = 0; d < 3; d++)
    if ((r = download_met(c, G.met_f[d], gb[d], Gb[d], G.nfmet[d]))) return r;
  std::vector<double> h(G.nmet * 64);
  CK(cudaMemcpyAsync(h.data(), G.gkr, G.nmet * 64 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (long i = 0; i < G.nmet; i++)
    for (int k = 0; k < 64; k++) gKr[i * 64 + k] = h[k * G.nmet + i];
  return 0;
}

// ---------------------------------------------------------------------------
// inspection of intermediate arrays (KORAL layout)
// ---------------------------------------------------------------------------
extern "C" int kgpu_download_flux(kgpu_ctx *c, int d, double *out) {
  if (!c || !out || d < 0 || d > 2) return KGPU_EINVAL;
  Grid &G = c->G;
  const long nf = G.nface[d];
  std::vector<double> h(nf * G.nv);
  CK(cudaMemcpyAsync(h.data(), G.flb[d], nf * G.nv * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (long f = 0; f < nf; f++)
    for (int iv = 0; iv < G.nv; iv++) out[f * G.nv + iv] = h[iv * nf + f];
  return 0;
}

extern "C" int kgpu_download_emf(kgpu_ctx *c, double *out) {
  if (!c || !out) return KGPU_EINVAL;
  Grid &G = c->G;
  const long ne = (long)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
  std::vector<double> h(3 * ne);
  CK(cudaMemcpyAsync(h.data(), G.emf, 3 * ne * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (long e = 0; e < ne; e++)
    for (int k = 0; k < 3; k++) out[e * 3 + k] = h[k * ne + e];
  return 0;
}
