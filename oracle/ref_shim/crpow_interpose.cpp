// Test infrastructure: a second build of the reference oracle in which the C
// library's pow is replaced, for the exponents 0.25 and 0.2 and for integer
// exponents 2..64, by the correctly rounded powers of
// m2c_b200/csrc/crpow.cuh and m2c_b200/csrc/physics.cuh (the ones the GPU
// uses: the exact Riemann solver's rarefaction step control,
// ExactRiemannSolverBase.cpp:1298, 1305, 1348-1349, and the van Albada
// limiter and its exponent's setup, Reconstructor.h:107-108,
// Reconstructor.cpp:109). Every other pow call goes to the C library.
// Linked with -Bsymbolic, so the reference objects of this build call this
// definition. Comparing the GPU with this build separates the one known
// source of difference (the C library's rounding of these powers) from
// everything else.
#include <dlfcn.h>

#include "../../m2c_b200/csrc/crpow.cuh"

extern "C" double pow(double x, double y) {
  if (y == 0.25 && x >= 0.0) return m2c::cr_pow_quarter(x);
  if (y == 0.2 && x >= 0.0) return m2c::cr_pow_fifth(x);
  if (y >= 2.0 && y <= 64.0 && y == (double)(int)y) return m2c::cr_pow_int(x, (int)y);
  static double (*libm_pow)(double, double) = (double (*)(double, double))dlsym(RTLD_NEXT, "pow");
  return libm_pow(x, y);
}
