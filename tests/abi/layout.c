/* Sizes and field offsets of the public structs of koral_b200.h, as a C
 * compiler lays them out; tests/test_abi.py compares them with the Python
 * ctypes mirrors in koral_b200/__init__.py. */
#include <stddef.h>
#include <stdio.h>

#include "koral_b200.h"

#define FIELD(T, f) printf("%s.%s %zu\n", #T, #f, offsetof(T, f))

int main(void)
{
  printf("kgpu_config %zu\n", sizeof(kgpu_config));
  FIELD(kgpu_config, bc);
  FIELD(kgpu_config, gamma);
  FIELD(kgpu_config, u2pconv);
  printf("kgpu_torus_params %zu\n", sizeof(kgpu_torus_params));
  printf("kgpu_rad_params %zu\n", sizeof(kgpu_rad_params));
  printf("kgpu_rad_solver_opts %zu\n", sizeof(kgpu_rad_solver_opts));
  FIELD(kgpu_rad_solver_opts, skip);
  FIELD(kgpu_rad_solver_opts, hard);
  printf("kgpu_tuning %zu\n", sizeof(kgpu_tuning));
  FIELD(kgpu_tuning, implicit);
  printf("kgpu_scalars_params %zu\n", sizeof(kgpu_scalars_params));
  FIELD(kgpu_scalars_params, bhdisk);
  return 0;
}
