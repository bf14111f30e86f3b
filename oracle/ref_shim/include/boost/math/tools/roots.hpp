// Stand-in for boost/math/tools/roots.hpp, used only so that reference files
// outside the hot path (ionization, JWL, ANEOS EOS) compile for the CPU
// oracle. The hot path's Riemann solver is compiled with WITHOUT_BOOST and
// never reaches this; any call aborts.
#ifndef M2C_ORACLE_BOOST_ROOTS_SHIM_H
#define M2C_ORACLE_BOOST_ROOTS_SHIM_H
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <utility>
namespace boost {
typedef std::uintmax_t uintmax_t;
namespace math {
namespace tools {
template <class F, class T, class Tol>
std::pair<T, T> toms748_solve(F, const T&, const T&, const T&, const T&, Tol, boost::uintmax_t&) {
  fprintf(stderr, "boost shim: toms748_solve is not available in the oracle build\n");
  abort();
}
template <class F, class T, class Tol>
std::pair<T, T> toms748_solve(F, const T&, const T&, Tol, boost::uintmax_t&) {
  fprintf(stderr, "boost shim: toms748_solve is not available in the oracle build\n");
  abort();
}
}  // namespace tools
}  // namespace math
}  // namespace boost
#endif
