// Scalar diagnostics of the black-hole disk on the device (calc_scalars,
// postproc.c:996-1105): reductions over the domain and over radial shells
// written to device memory by kernels on the context's stream, so that an
// output step needs no copy of the state and can sit inside a captured
// graph.  Internal to the library; the public entry points are
// kgpu_calc_scalars and kgpu_calc_scalars_device.
#pragma once

#include <cuda_runtime.h>

#include "kgpu_physics.cuh"

namespace kgpu {

constexpr int NSCALARS = 13;            // NSCALARS, choices.h:256-257
constexpr int DIAG_MASS_BLOCKS = 592;   // 4 blocks per SM of a B200 for the domain sum
constexpr int DIAG_WORK = DIAG_MASS_BLOCKS + 16;

// radial indices of the reference's searches (the first centre whose
// coordinate x1 exceeds the radius; NX when none does)
struct DiagIdx {
  int ix_mdot;   // rhorizonBL: accretion rate and magnetic flux
  int ix_mri;    // half the coordinate of the last centre: MRI resolution
  int ix_temp;   // 15: mean temperature
  int ix_lum;    // 5e3: local luminosity
};

struct DiagConsts {
  double mdotscale;   // rhoGU2CGS(1) velGU2CGS(1) lenGU2CGS(1)^2
  double mdotedd;     // calc_mdotEdd
  double kb, mu, mp;  // K_BOLTZ, MU_GAS, M_PROTON in code units
  int bhdisk;         // BHDISK_PROBLEMTYPE: MRI resolution and mean temperature computed
  int rad;            // radiation carried: R^r_t in the local luminosity
};

// Launches the reductions and the assembly; out receives NSCALARS doubles
// (device memory), work DIAG_WORK doubles.  Returns the number of kernels
// launched, or a negative KGPU_* status.
int diag_scalars_enqueue(const Grid &G, const DiagIdx &ix, const DiagConsts &k, double *work, double *out,
                         cudaStream_t st);

}  // namespace kgpu
