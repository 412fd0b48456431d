// The library's double-double powers (koral_b200/csrc/kgpu_math.cuh)
// compiled for the host, beside the host C library's pow and log, behind one
// C entry point for the tests: kind 0 x^2, 1 x^4, 2 x^-3.5, 3 x^y with 4y
// an integer (else pow), 4 log(x) of the C library, 5 pow(x, y) of the C
// library.
#include <math.h>

#include "../../koral_b200/csrc/kgpu_math.cuh"

extern "C" void host_powers(long n, int kind, double y, const double *x, double *out) {
  for (long i = 0; i < n; i++) {
    const double v = x[i];
    double r;
    switch (kind) {
      case 0: r = kgpu::pw2(v); break;
      case 1: r = kgpu::pw4(v); break;
      case 2: r = kgpu::pw_m3p5(v); break;
      case 3: r = kgpu::pw_any(v, y); break;
      case 4: r = log(v); break;
      default: r = pow(v, y); break;
    }
    out[i] = r;
  }
}
