// Device set-up of the Kerr torus: the MKS2 metric tables and the
// Fishbone-Moncrief state computed on the GPU straight into a context's
// device arrays (kgpu_setup.cu).  Internal to the library; the public entry
// points are kgpu_init_fm_torus and kgpu_init_fm_radtorus.
#pragma once

#include <cuda_runtime.h>

#include "../../include/koral_b200.h"
#include "kgpu_physics.cuh"

namespace kgpu {

// radiation constants of the radiative torus (on = 0: the 9-variable torus)
struct TorusRadConsts {
  int on;
  double sigma, kb, mu, mp;   // SIGMA_RAD, K_BOLTZ, MU_GAS, M_PROTON in code units
  double eradatm;             // atmosphere radiation energy / gas energy (< 0: LTE everywhere)
};

// Fills G.met_c, G.met_f[0..2] and G.gkr from the grid faces G.xb on stream
// st (no synchronisation).  Returns the number of kernels launched, or a
// negative KGPU_* status.
int setup_mks2_metric_device(const Grid &G, double a, double r0, double h0, cudaStream_t st);

// Fills G.p and G.u (domain cells; ghosts zero) with the torus state, from
// the device metric; scratch holds ncell + 1 doubles.  Returns the number of
// kernels launched, or a negative KGPU_* status.
int setup_fm_torus_device(const Grid &G, const kgpu_torus_params &tp, const TorusRadConsts &rad, double *scratch,
                          cudaStream_t st);

}  // namespace kgpu
