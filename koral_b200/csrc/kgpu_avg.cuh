// Time averages on the device (save_avg, fileop.c:10-70, of the quantities
// p2avg computes, p2u.c:313-541).  Internal to the library; the public
// entry points are kgpu_set_avg, kgpu_save_avg, kgpu_download_avg and
// kgpu_reset_avg.
#pragma once

#include <cuda_runtime.h>

#include "kgpu_rad.cuh"

namespace kgpu {

// NAVGVARS (choices.h:260-265): the averaged quantities after the NV
// primitives
constexpr int navg_vars(int nv, bool rad) { return rad ? 153 + 3 * nv : 112 + 3 * nv; }

// Slots of the averaged quantities (mnemonics.h:170-199) for nv variables
struct AvgSlots {
  int nv;
  __host__ __device__ int bsq() const { return nv + 0; }
  __host__ __device__ int ucon(int i) const { return nv + 1 + i; }
  __host__ __device__ int ucov(int i) const { return nv + 5 + i; }
  __host__ __device__ int bcon(int i) const { return nv + 9 + i; }
  __host__ __device__ int bcov(int i) const { return nv + 13 + i; }
  __host__ __device__ int rhoucon(int i) const { return nv + 17 + i; }
  __host__ __device__ int rhoucov(int i) const { return nv + 21 + i; }
  __host__ __device__ int uuucon(int i) const { return nv + 25 + i; }
  __host__ __device__ int uucov(int i) const { return nv + 29 + i; }
  __host__ __device__ int bsqucon(int i) const { return nv + 33 + i; }
  __host__ __device__ int bsqucov(int i) const { return nv + 37 + i; }
  __host__ __device__ int rhouconucov(int i, int j) const { return nv + 41 + i * 4 + j; }
  __host__ __device__ int uuuconucov(int i, int j) const { return nv + 57 + i * 4 + j; }
  __host__ __device__ int bsquconucov(int i, int j) const { return nv + 73 + i * 4 + j; }
  __host__ __device__ int bconbcov(int i, int j) const { return nv + 89 + i * 4 + j; }
  __host__ __device__ int wucon(int i) const { return nv + 105 + i; }
  __host__ __device__ int fluxxl(int i) const { return nv + 109 + i; }
  __host__ __device__ int fluxyl(int i) const { return nv + 109 + nv + i; }
  __host__ __device__ int fluxzl(int i) const { return nv + 109 + 2 * nv + i; }
  __host__ __device__ int rhourdiff() const { return nv + 109 + 3 * nv; }
  __host__ __device__ int tgas() const { return nv + 110 + 3 * nv; }
  __host__ __device__ int ehat() const { return 4 * nv + 111; }
  __host__ __device__ int rij(int i, int j) const { return 4 * nv + 112 + i * 4 + j; }
  __host__ __device__ int ehatucon(int i) const { return 4 * nv + 128 + i; }
  __host__ __device__ int ehatucov(int i) const { return 4 * nv + 132 + i; }
  __host__ __device__ int urfcon(int i) const { return 4 * nv + 136 + i; }
  __host__ __device__ int urfcov(int i) const { return 4 * nv + 140 + i; }
  __host__ __device__ int ghat(int i) const { return 4 * nv + 144 + i; }
  __host__ __device__ int ghatcompt(int i) const { return 4 * nv + 148 + i; }
  __host__ __device__ int trad() const { return 4 * nv + 152; }
};

// Accumulates avg * dt of every domain cell into pavg ([nav][ncell],
// nav = nv + navg_vars) and dt into *avgtime; R holds the unit constants
// (K_BOLTZ, M_PROTON, MU_GAS, SIGMA_RAD) and, with radiation, the opacity
// law.  dtp is the time step in device memory.  Returns the number of
// kernels launched, or a negative KGPU_* status.
int avg_enqueue(const Grid &G, const RadParams &R, const double *dtp, double *pavg, double *avgtime,
                cudaStream_t st);

}  // namespace kgpu
