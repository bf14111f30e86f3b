// Test harness: the library's exact Riemann solver (m2c_b200/csrc/riemann.cuh)
// compiled for the host with g++ (no FMA contraction). Two builds of the
// rarefaction step control's pow(x, 0.25) / pow(x, 0.2), chosen per call of
// host_riemann:
//   libm = 1: the host C library's pow, as the reference calls it, so the
//             solver can be compared with the reference's own bit for bit;
//   libm = 0: the correctly rounded roots of crpow.cuh, which the GPU uses,
//             so the GPU can be compared with this build bit for bit.
// Either way every call also evaluates the other one and counts, per
// problem, the calls where the two differ (the C library's pow is not
// correctly rounded there). Not part of the library.
#include <cmath>
#include <vector>

#include "../../m2c_b200/csrc/crpow.cuh"

static int g_libm = 1;
static int g_misrounded = 0;

static double host_pow_quarter(double x) {
  const double a = std::pow(x, 0.25), b = m2c::cr_pow_quarter(x);
  if (a != b) g_misrounded++;
  return g_libm ? a : b;
}

static double host_pow_fifth(double x) {
  const double a = std::pow(x, 0.2), b = m2c::cr_pow_fifth(x);
  if (a != b) g_misrounded++;
  return g_libm ? a : b;
}

#define M2C_RIEMANN_POW_QUARTER(x) host_pow_quarter(x)
#define M2C_RIEMANN_POW_FIFTH(x) host_pow_fifth(x)
#include "../../include/m2c_gpu.h"
#include "../../m2c_b200/csrc/riemann.cuh"

using namespace m2c;

extern "C" int host_riemann(const m2cg_scheme* s, const m2cg_material* mats, int nmat, int n, const double* dir,
                            const double* VL, const int* idl, const double* VR, const int* idr, double* Vs, int* id,
                            double* Vsm, double* Vsp, int* err, int* retried, int libm, int* misrounded) {
  g_libm = libm;
  std::vector<Eos<double>> eos(nmat);
  for (int m = 0; m < nmat; m++) {
    MatParams p;
    p.kind = mats[m].eos;
    p.gam = mats[m].gamma;
    p.pc = mats[m].p_c;
    p.b = mats[m].b;
    p.q = mats[m].q;
    p.rhomin = mats[m].rhomin;
    p.pmin = mats[m].pmin;
    p.rhomax = mats[m].rhomax;
    p.pmax = mats[m].pmax;
    p.failsafe_density = mats[m].failsafe_density;
    eos[m] = make_eos<double>(p);
  }
  RiemannParams P;
  P.maxIts_main = s->riem_maxits_main;
  P.maxIts_bracket = s->riem_maxits_bracket;
  P.maxIts_shock = s->riem_maxits_shock;
  P.numSteps_rarefaction = s->riem_nsteps_rarefaction;
  P.tol_main = s->riem_tol_main;
  P.tol_shock = s->riem_tol_shock;
  P.tol_rarefaction = s->riem_tol_rarefaction;
  P.min_pressure = s->riem_min_pressure;
  P.failure_threshold = s->riem_failure_threshold;
  P.pressure_at_failure = s->riem_pressure_at_failure;
  P.warm_delta = s->riem_warm_delta;
  P.warm_gate = s->riem_warm_gate;
  const int cap = 512;  // the device solver's path capacity (riemann_batch.h)
  std::vector<double> scratch(2 * 3 * cap);
  RiemannSolver rs;
  rs.P = P;
  rs.eos = eos.data();
  rs.path1.pt = scratch.data();
  rs.path1.cap = cap;
  rs.path3.pt = scratch.data() + 3 * cap;
  rs.path3.cap = cap;
  for (int q = 0; q < n; q++) {
    bool bad = false;
    int mid = 0;
    g_misrounded = 0;
    int r = rs.solve(dir + 3 * q, VL + 5 * q, idl[q], VR + 5 * q, idr[q], Vs + 5 * q, mid, Vsm + 5 * q, Vsp + 5 * q,
                     NAN, bad);
    id[q] = mid;
    err[q] = r | (bad ? 4 : 0);
    retried[q] = rs.retried ? 1 : 0;
    if (misrounded) misrounded[q] = g_misrounded;
  }
  return 0;
}

// One-sided (wall) problems, RiemannSolver::solve_wall, with the same pow
// selection; Vs is zeroed first (the solver leaves it untouched where the
// state at the wall is undefined, id = -1).
extern "C" int host_riemann_wall(const m2cg_scheme* s, const m2cg_material* mats, int nmat, int n, const double* dir,
                                 const double* Vm, const int* idm, const double* uwall, double* Vs, int* id,
                                 double* Vsm, int* err, int libm, int* misrounded) {
  g_libm = libm;
  std::vector<Eos<double>> eos(nmat);
  for (int m = 0; m < nmat; m++) {
    MatParams p;
    p.kind = mats[m].eos;
    p.gam = mats[m].gamma;
    p.pc = mats[m].p_c;
    p.b = mats[m].b;
    p.q = mats[m].q;
    p.rhomin = mats[m].rhomin;
    p.pmin = mats[m].pmin;
    p.rhomax = mats[m].rhomax;
    p.pmax = mats[m].pmax;
    p.failsafe_density = mats[m].failsafe_density;
    eos[m] = make_eos<double>(p);
  }
  RiemannParams P;
  P.maxIts_main = s->riem_maxits_main;
  P.maxIts_bracket = s->riem_maxits_bracket;
  P.maxIts_shock = s->riem_maxits_shock;
  P.numSteps_rarefaction = s->riem_nsteps_rarefaction;
  P.tol_main = s->riem_tol_main;
  P.tol_shock = s->riem_tol_shock;
  P.tol_rarefaction = s->riem_tol_rarefaction;
  P.min_pressure = s->riem_min_pressure;
  P.failure_threshold = s->riem_failure_threshold;
  P.pressure_at_failure = s->riem_pressure_at_failure;
  P.warm_delta = s->riem_warm_delta;
  P.warm_gate = s->riem_warm_gate;
  const int cap = 512;
  std::vector<double> scratch(3 * cap);
  RiemannSolver rs;
  rs.P = P;
  rs.eos = eos.data();
  rs.path1.pt = scratch.data();
  rs.path1.cap = cap;
  rs.path3.pt = nullptr;
  rs.path3.cap = 0;
  for (int q = 0; q < n; q++) {
    bool bad = false;
    int mid = 0;
    g_misrounded = 0;
    for (int c = 0; c < 5; c++) Vs[5 * q + c] = 0.0;
    const int r = rs.solve_wall(dir + 3 * q, Vm + 5 * q, idm[q], uwall + 3 * q, Vs + 5 * q, mid, Vsm + 5 * q, bad);
    id[q] = mid;
    err[q] = r | (bad ? 4 : 0);
    if (misrounded) misrounded[q] = g_misrounded;
  }
  return 0;
}
