// Stand-in for boost cubic_b_spline, used only so that reference files
// outside the hot path compile for the CPU oracle. Any use aborts.
#ifndef M2C_ORACLE_BOOST_SPLINE_SHIM_H
#define M2C_ORACLE_BOOST_SPLINE_SHIM_H
#include <cstdio>
#include <cstdlib>
namespace boost {
namespace math {
template <class T>
class cubic_b_spline {
 public:
  template <class It>
  cubic_b_spline(It, It, T, T) {
    fprintf(stderr, "boost shim: cubic_b_spline is not available in the oracle build\n");
    abort();
  }
  T operator()(T) const { abort(); }
  T prime(T) const { abort(); }
};
}  // namespace math
}  // namespace boost
#endif
