// Test infrastructure: a second build of the reference oracle in which the C
// library's pow is replaced, for the exponents 0.25 and 0.2 only, by the
// correctly rounded roots of m2c_b200/csrc/crpow.cuh (the ones the GPU's
// exact Riemann solver uses in its rarefaction step control,
// ExactRiemannSolverBase.cpp:1298, 1305, 1348-1349). Every other pow call
// goes to the C library. Linked with -Bsymbolic, so the reference objects of
// this build call this definition. Comparing the GPU with this build
// separates the one known source of difference (the C library's rounding of
// these two powers) from everything else.
#include <dlfcn.h>

#include "../../m2c_b200/csrc/crpow.cuh"

extern "C" double pow(double x, double y) {
  if (y == 0.25 && x >= 0.0) return m2c::cr_pow_quarter(x);
  if (y == 0.2 && x >= 0.0) return m2c::cr_pow_fifth(x);
  static double (*libm_pow)(double, double) = (double (*)(double, double))dlsym(RTLD_NEXT, "pow");
  return libm_pow(x, y);
}
