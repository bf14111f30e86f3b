// Two-material exact Riemann solver (FP64), one problem per thread.
//
// Restates the two-sided path of ExactRiemannSolverBase (ExactRiemannSolverBase.cpp),
// the Boost-free build of the reference (WITHOUT_BOOST):
//   ComputeRiemannSolution        59-342   (safeguarded secant on p*, "main loop")
//   FinalizeSolution              347-514  (state at xi = 0, star states)
//   FindInitialInterval           631-795  (bracketing search)
//   FindInitialFeasiblePoints     959-1059
//   ...ByAcousticTheory           1064-1114 (Kamm 2015, Eqs. 20-22)
//   ComputeRhoUStar               1169-1580 (adaptive RKF45 rarefaction from the
//                                            cached integration path; Hugoniot root)
//   Rarefaction_OneStepRK4        1729-1852 (Cash-Karp/Fehlberg step in pressure)
//   HugoniotEquation              ExactRiemannSolverBase.h:58-75
// and the retry the reference makes when the adaptive solve cannot bracket
// the root or does not converge, ExactRiemannSolverNonAdaptive:
//   ComputeRiemannSolution        2199-2470 (same main loop, no retry)
//   ComputeRhoUStar               2476-2845 (rarefaction by classical RK4 steps
//                                            in pressure; same Hugoniot root)
//   Rarefaction_OneStepRK4        2850-2945
// The step sequence, branch structure and floating-point expressions follow
// the reference so that, compiled without FMA contraction, results agree
// with it to round-off. The step-size control's pow(x, 0.25) and pow(x, 0.2)
// are the correctly rounded ones (crpow.cuh) on the host and the device
// alike, so a GPU solve is bit-identical to the host build of this file; the
// reference's C-library pow rounds the other way on about 6e-4 of these
// calls, and only the problems that meet such a call can differ from the
// reference (a step one ulp longer changes the integrated rarefaction in its
// last bits; measured on seeded problems: about 1.2% of them, largest
// relative difference ~6e-12). A host build can select the C library's pow
// instead (M2C_RIEMANN_POW_QUARTER / M2C_RIEMANN_POW_FIFTH) to reproduce the
// reference bit for bit.
//
// The two integration-path caches of the reference (std::vector members
// integrationPath1/3, ExactRiemannSolverBase.h:28-29) live in a per-problem
// scratch region of global memory with a fixed capacity; running out of it
// is reported (RIEM_PATH_OVERFLOW), never silently ignored.
#pragma once
#include <float.h>

#include "crpow.cuh"
#include "physics.cuh"

#ifndef M2C_RIEMANN_POW_QUARTER
#define M2C_RIEMANN_POW_QUARTER(x) cr_pow_quarter(x)
#endif
#ifndef M2C_RIEMANN_POW_FIFTH
#define M2C_RIEMANN_POW_FIFTH(x) cr_pow_fifth(x)
#endif

namespace m2c {

struct RiemannParams {
  int maxIts_main, maxIts_bracket, maxIts_shock, numSteps_rarefaction;
  double tol_main, tol_shock, tol_rarefaction, min_pressure, failure_threshold, pressure_at_failure;
  double warm_delta;  // half-width of the warm-start bracket, relative to the proposed star pressure
  double warm_gate;   // proposals within this shifted log distance of the acoustic estimate are ignored
};

// result flags
enum {
  RIEM_OK = 0,
  RIEM_FAILED = 1,           // not solved (the non-adaptive retry included)
  RIEM_PATH_OVERFLOW = 2,    // integration-path scratch exhausted
  RIEM_RETRY = 0x100,        // internal: the adaptive solve hands over to the non-adaptive one
};

// Integration path: points (p, rho, u) with decreasing pressure.
struct RPath {
  double* pt;   // [cap][3]
  int n, cap;
  bool overflow;
  M2C_HD double P(int j) const { return pt[3 * j]; }
  M2C_HD double R(int j) const { return pt[3 * j + 1]; }
  M2C_HD double U(int j) const { return pt[3 * j + 2]; }
  M2C_HD void push(double p, double r, double u) {
    if (n >= cap) { overflow = true; return; }
    pt[3 * n] = p; pt[3 * n + 1] = r; pt[3 * n + 2] = u;
    n++;
  }
};

template <typename T> M2C_HD void swap_(T& a, T& b) { T t = a; a = b; b = t; }

struct RiemannSolver {
  RiemannParams P;
  const Eos<double>* eos;  // material table indexed by id
  RPath path1, path3;
  int iterations;          // outer secant iterations of the main loop
  double warm = NAN;       // proposed star pressure of the current solve (NaN: none)
  mutable int evaluations; // star-state evaluations at a trial pressure (bracketing + main loop)
  bool nonadaptive = false; // ExactRiemannSolverNonAdaptive's ComputeRhoUStar in place of the adaptive one
  bool retried = false;     // the last solve went through the non-adaptive retry

  // ExactRiemannSolverNonAdaptive::Rarefaction_OneStepRK4 (2850-2945): one
  // classical RK4 step of d(rho)/dp = 1/c^2, du/dp = -+1/(rho c).
  M2C_HD bool rk4_step(int wave, int id, double rho_0, double u_0, double p_0, double dp, double& rho, double& u,
                       double& p, double& xi) const {
    const Eos<double>& e = eos[id];
    dp = -dp;
    double e_0 = e.energy(rho_0, p_0);
    double c_0_square = e.c2(rho_0, e_0);
    if (rho_0 <= 0 || c_0_square < 0) return false;
    double c_0 = sqrt(c_0_square);
    double rho_1 = rho_0 + 0.5 * dp / c_0_square;
    double p_1 = p_0 + 0.5 * dp;
    double e_1 = e.energy(rho_1, p_1);
    double c_1_square = e.c2(rho_1, e_1);
    if (rho_1 <= 0 || c_1_square < 0) return false;
    double c_1 = sqrt(c_1_square);
    double rho_2 = rho_0 + 0.5 * dp / c_1_square;
    double p_2 = p_1;
    double e_2 = e.energy(rho_2, p_2);
    double c_2_square = e.c2(rho_2, e_2);
    if (rho_2 <= 0 || c_2_square < 0) return false;
    double c_2 = sqrt(c_2_square);
    double rho_3 = rho_0 + dp / c_2_square;
    double p_3 = p_0 + dp;
    double e_3 = e.energy(rho_3, p_3);
    double c_3_square = e.c2(rho_3, e_3);
    if (rho_3 <= 0 || c_3_square < 0) return false;
    double c_3 = sqrt(c_3_square);
    double drho = 1.0 / 6.0 * dp * (1. / c_0_square + 2.0 * (1. / c_1_square + 1. / c_2_square) + 1. / c_3_square);
    double du = 1.0 / 6.0 * dp *
                (1. / c_0 / rho_0 + 2.0 * (1. / c_1 / rho_1 + 1. / c_2 / rho_2) + 1. / c_3 / rho_3);
    if (isnan(du)) return false;
    rho = rho_0 + drho;
    p = p_0 + dp;
    u = (wave == 1) ? u_0 - du : u_0 + du;
    double ee = e.energy(rho, p);
    double c = e.c2(rho, ee);
    if (rho <= 0 || c < 0) return false;
    c = sqrt(c);
    xi = (wave == 1) ? u - c : u + c;
    return true;
  }

  // Rarefaction branch of ExactRiemannSolverNonAdaptive::ComputeRhoUStar
  // (2487-2633): steps in pressure of at most (p - ps)/numSteps, grown by at
  // most 4x per step, from the deepest cached path point above ps.
  M2C_HD bool rarefaction_nonadaptive(int wave, RPath& path, double rho, double u, double p, double ps, int id,
                                      double& rhos, double& us, bool* trans_rare, double* Vrare_x0) const {
    const Eos<double>& e = eos[id];
    double rhos_0 = rho, us_0 = u, ps_0 = p, xi_0;
    double rhos_1 = rho, us_1 = u, ps_1 = p, xi_1 = 0.0;
    double dp_target = (p - ps) / P.numSteps_rarefaction;
    double ee = e.energy(rho, p);
    double dpdrho = e.dpdrho(rho, ee);
    double drho_op1 = (p - ps) / dpdrho / P.numSteps_rarefaction;
    double drho_op2 = rho / (2.5 * P.numSteps_rarefaction);
    double drho_target = smin(drho_op1, drho_op2);
    double dp = smin(dp_target, drho_target * dpdrho);
    double pressure_endpoint_tol = P.tol_rarefaction * smax(1.0, fabs(p));
    double c = e.c2(rho, ee);
    if (rho <= 0 || c < 0) return false;
    c = sqrt(c);
    int index0 = 0;
    if (path.n > 1) {
      for (int j = path.n - 1; j >= 0; j--) {
        if (path.P(j) > ps) {
          index0 = j;
          break;
        }
      }
      ps_0 = path.P(index0);
      rhos_0 = path.R(index0);
      us_0 = path.U(index0);
      dp = smin((p - ps) / P.numSteps_rarefaction, ps_0 - ps);
    }
    double xi = (wave == 1) ? u - c : u + c;
    xi_0 = xi;
    const int moreSteps = 5;
    for (int i = 0; i < P.numSteps_rarefaction * moreSteps; i++) {
      if (fabs(ps_1 - ps) <= pressure_endpoint_tol) {
        rhos = rhos_1;
        us = us_1;
        return !e.bad(rhos, ps);
      }
      bool ok = rk4_step(wave, id, rhos_0, us_0, ps_0, dp, rhos_1, us_1, ps_1, xi_1);
      if (!ok) {
        dp = dp / 2.0;
        if (dp == 0.0) break;
        continue;
      }
      if (ps_1 - ps < -pressure_endpoint_tol) {
        dp = ps_0 - ps;
        continue;
      }
      if (ps_1 < path.P(path.n - 1)) path.push(ps_1, rhos_1, us_1);
      if (trans_rare && Vrare_x0 && xi_0 * xi_1 <= 0) {  // transonic rarefaction
        *trans_rare = true;
        double w0 = fabs(xi_1), w1 = fabs(xi_0);
        double ww = w0 + w1;
        w0 /= ww;
        w1 /= ww;
        Vrare_x0[0] = w0 * rhos_0 + w1 * rhos_1;
        Vrare_x0[1] = w0 * us_0 + w1 * us_1;
        Vrare_x0[2] = w0 * ps_0 + w1 * ps_1;
      }
      dp = smin(smin(dp_target, ps_1 - ps), 4.0 * dp);
      rhos_0 = rhos_1;
      us_0 = us_1;
      ps_0 = ps_1;
      xi_0 = xi_1;
    }
    return false;  // did not reach ps (both of the reference's outcomes fail)
  }

  // Rarefaction_OneStepRK4 (ExactRiemannSolverBase.cpp:1729-1852)
  M2C_HD bool rk_step(int wave, int id, double rho_0, double u_0, double p_0, double dp, double& rho, double& u,
                      double& p, double& xi, double& uErr, double& rhoErr) const {
    const Eos<double>& e = eos[id];
    dp = -dp;
    double e_0 = e.energy(rho_0, p_0);
    double c_0_square = e.c2(rho_0, e_0);
    if (rho_0 <= 0 || c_0_square < 0) return false;
    double c_0 = sqrt(c_0_square);
    double rho_1 = rho_0 + 0.2 * dp / c_0_square;
    double p_1 = p_0 + 0.2 * dp;
    double e_1 = e.energy(rho_1, p_1);
    double c_1_square = e.c2(rho_1, e_1);
    if (rho_1 <= 0 || c_1_square < 0) return false;
    double rho_2 = rho_0 + 3. / 40. * dp / c_0_square + 9. / 40. * dp / c_1_square;
    double p_2 = p_1 + 3. / 10. * dp;
    double e_2 = e.energy(rho_2, p_2);
    double c_2_square = e.c2(rho_2, e_2);
    if (rho_2 <= 0 || c_2_square < 0) return false;
    double c_2 = sqrt(c_2_square);
    double rho_3 = rho_0 + 3. / 10. * dp / c_0_square - 9. / 10. * dp / c_1_square + 6. / 5. * dp / c_2_square;
    double p_3 = p_0 + 3. / 5. * dp;
    double e_3 = e.energy(rho_3, p_3);
    double c_3_square = e.c2(rho_3, e_3);
    if (rho_3 <= 0 || c_3_square < 0) return false;
    double c_3 = sqrt(c_3_square);
    double rho_4 = rho_0 - 11. / 54. * dp / c_0_square + 2.5 * dp / c_1_square - 70. / 27. * dp / c_2_square +
                   35. / 27. * dp / c_3_square;
    double p_4 = p_0 + dp;
    double e_4 = e.energy(rho_4, p_4);
    double c_4_square = e.c2(rho_4, e_4);
    if (rho_4 <= 0 || c_4_square < 0) return false;
    double c_4 = sqrt(c_4_square);
    double rho_5 = rho_0 + 1631. / 55296. * dp / c_0_square + 175. / 512. * dp / c_1_square +
                   575. / 13824. * dp / c_2_square + 44275. / 110592. * dp / c_3_square +
                   253. / 4096. * dp / c_4_square;
    double p_5 = p_0 + 7. / 8. * dp;
    double e_5 = e.energy(rho_5, p_5);
    double c_5_square = e.c2(rho_5, e_5);
    if (rho_5 <= 0 || c_5_square < 0) return false;
    double c_5 = sqrt(c_5_square);
    double drho = (37. / 378. / c_0_square + 250. / 621. / c_2_square + 125. / 594. / c_3_square +
                   512. / 1771. / c_5_square) * dp;
    double drho_err = (2825. / 27648. / c_0_square + 18575. / 48384. / c_2_square + 13525. / 55296. / c_3_square +
                       277. / 14336. / c_4_square + 0.25 / c_5_square) * dp;
    double du = (37. / 378. / c_0 / rho_0 + 250. / 621. / c_2 / rho_2 + 125. / 594. / c_3 / rho_3 +
                 512. / 1771. / c_5 / rho_5) * dp;
    double du_err = (2825. / 27648. / c_0 / rho_0 + 18575. / 48384. / c_2 / rho_2 + 13525. / 55296. / c_3 / rho_3 +
                     277. / 14336. / c_4 / rho_4 + 0.25 / c_5 / rho_5) * dp;
    if (isnan(du) || isnan(du_err)) return false;
    rhoErr = fabs(drho_err - drho);
    uErr = fabs(du_err - du);
    rho = rho_0 + drho;
    p = p_0 + dp;
    u = (wave == 1) ? u_0 - du : u_0 + du;
    double ee = e.energy(rho, p);
    double c = e.c2(rho, ee);
    if (rho <= 0 || c < 0) return false;
    c = sqrt(c);
    xi = (wave == 1) ? u - c : u + c;
    return true;
  }

  // HugoniotEquation (ExactRiemannSolverBase.h:58-75)
  struct Hugo {
    const Eos<double>* e;
    double p, ps, e0, pavg, one_over_rho;
    M2C_HD double operator()(double rhos) const {
      double es = e->energy(rhos, ps);
      return es - e0 + pavg * (1.0 / rhos - one_over_rho);
    }
  };

  // ComputeRhoUStar (ExactRiemannSolverBase.cpp:1169-1580). Returns success.
  M2C_HD_OUTLINE bool rho_u_star(int wave, RPath& path, double rho, double u, double p, double ps, int id, double rhos0,
                         double rhos1, double& rhos, double& us, bool* trans_rare, double* Vrare_x0) const {
    const Eos<double>& e = eos[id];
    if (wave == 1) evaluations++;
    rhos = rho;
    us = u;
    if (p > ps && nonadaptive) return rarefaction_nonadaptive(wave, path, rho, u, p, ps, id, rhos, us, trans_rare,
                                                              Vrare_x0);
    if (p > ps) {  // rarefaction: numerical integration
      double rhos_0 = rho, us_0 = u, ps_0 = p, xi_0;
      double rhos_1 = rho, us_1 = u, ps_1 = p, xi_1 = 0.0;
      double dp = (p - ps) / P.numSteps_rarefaction;
      double dp_min_adaption = dp / 2.5;
      double pressure_endpoint_tol = P.tol_rarefaction * smax(1.0, fabs(p));
      double ee = e.energy(rho, p);
      double c = e.c2(rho, ee);
      if (rho <= 0 || c < 0) return false;
      c = sqrt(c);
      int index0 = 0;
      if (path.n > 1) {
        for (int j = path.n - 1; j >= 0; j--) {
          if (path.P(j) > ps) {
            index0 = j;
            break;
          }
        }
        ps_0 = path.P(index0);
        rhos_0 = path.R(index0);
        us_0 = path.U(index0);
        dp_min_adaption = (ps_0 - ps) / P.numSteps_rarefaction / 2.5;
        if (index0 != path.n - 1)
          dp = ps_0 - ps;
        else
          dp = smin(path.P(index0 - 1) - path.P(index0), ps_0 - ps);
      }
      double xi = (wave == 1) ? u - c : u + c;
      xi_0 = xi;
      bool done = false;
      double uErr = 0., rhoErr = 0.;
      const int moreSteps = 3;
      for (int i = 0; i < P.numSteps_rarefaction * moreSteps; i++) {
        if (fabs(ps_1 - ps) <= pressure_endpoint_tol) {
          rhos = rhos_1;
          us = us_1;
          if (e.bad(rhos, ps)) return false;
          done = true;
          break;
        }
        bool ok = rk_step(wave, id, rhos_0, us_0, ps_0, dp, rhos_1, us_1, ps_1, xi_1, uErr, rhoErr);
        if (!ok) {
          dp = dp / 2.0;
          continue;
        }
        if (ps_1 - ps < -pressure_endpoint_tol) {
          dp = ps_0 - ps;
          continue;
        }
        const double tiny = 1.e-30;
        double errBar = smax(1.0e-8, smin(1.0e-5, 100.0 * P.tol_rarefaction));
        double uErrScaled = uErr / c + tiny;
        double rhoErrScaled = rhoErr / rho + tiny;
        if (isnan(rhoErrScaled) || isnan(uErrScaled)) return false;  // the reference aborts here
        double dpTemp = dp;
        const double safety = 0.9;
        if (rhoErrScaled >= errBar && dp > dp_min_adaption) {
          dpTemp = safety * dp * M2C_RIEMANN_POW_QUARTER(fabs(errBar / rhoErrScaled));
          dpTemp = smax(smax(dpTemp, 0.2 * dp), dp_min_adaption);
          dp = smin(dpTemp, ps_0 - ps);
          continue;
        }
        if (uErrScaled >= errBar && dp > dp_min_adaption) {
          dpTemp = safety * dp * M2C_RIEMANN_POW_QUARTER(fabs(errBar / uErrScaled));
          dpTemp = smax(smax(dpTemp, 0.2 * dp), dp_min_adaption);
          dp = smin(dpTemp, ps_0 - ps);
          continue;
        }
        if (ps_1 < path.P(path.n - 1)) path.push(ps_1, rhos_1, us_1);
        if (trans_rare && Vrare_x0 && xi_0 * xi_1 <= 0) {  // transonic rarefaction
          *trans_rare = true;
          double w0 = fabs(xi_1), w1 = fabs(xi_0);
          double ww = w0 + w1;
          w0 /= ww;
          w1 /= ww;
          Vrare_x0[0] = w0 * rhos_0 + w1 * rhos_1;
          Vrare_x0[1] = w0 * us_0 + w1 * us_1;
          Vrare_x0[2] = w0 * ps_0 + w1 * ps_1;
        }
        double dpTemp_rho = safety * dp * M2C_RIEMANN_POW_FIFTH(fabs(errBar / rhoErrScaled));
        double dpTemp_u = safety * dp * M2C_RIEMANN_POW_FIFTH(fabs(errBar / uErrScaled));
        dpTemp = smin(dpTemp_rho, dpTemp_u);
        dpTemp = smin(dpTemp, 10 * dp);
        dpTemp = smax(dpTemp, dp_min_adaption);
        dp = smin(dpTemp, ps_1 - ps);
        rhos_0 = rhos_1;
        us_0 = us_1;
        ps_0 = ps_1;
        xi_0 = xi_1;
      }
      if (!done) return false;
    } else {  // shock: root of the Hugoniot equation in rhos
      Hugo hugo;
      hugo.e = &e;
      hugo.p = p;
      hugo.ps = ps;
      hugo.e0 = e.energy(rho, p);
      hugo.pavg = 0.5 * (p + ps);
      hugo.one_over_rho = 1.0 / rho;
      double f0, f1;
      double drho = smax(fabs(rhos0 - rhos1), 0.001 * rhos0);
      bool found_rhos0 = false, found_rhos1 = false;
      if (smin(rhos0, rhos1) >= rho) {
        f0 = hugo(rhos0);
        f1 = hugo(rhos1);
        if (f0 * f1 <= 0) {
          if (rhos0 > rhos1) {
            swap_(rhos0, rhos1);
            swap_(f0, f1);
          }
          found_rhos0 = found_rhos1 = true;
        } else {
          rhos0 = rhos1;
          f0 = f1;
        }
      } else {
        if (rhos1 > rhos0) {
          rhos0 = rhos1;
          f0 = hugo(rhos0);
        }
        if (rhos0 < rho) {
          rhos0 = rho;
          f0 = hugo(rhos0);
          found_rhos0 = true;
        } else {
          f0 = hugo(rhos0);
        }
      }
      if (!found_rhos0 || !found_rhos1) {
        int i = 0;
        double factor = 1.5;
        double tmp, ftmp;
        rhos1 = rhos0;
        f1 = f0;
        while (!found_rhos0) {
          if (++i >= P.maxIts_shock) return false;
          tmp = rhos1;
          ftmp = f1;
          rhos1 = rhos0;
          f1 = f0;
          rhos0 = rhos1 - factor * drho;
          if (rhos0 <= rho) {
            rhos0 = rho;
            found_rhos0 = true;
          }
          f0 = hugo(rhos0);
          if (f0 * f1 <= 0) {
            found_rhos0 = found_rhos1 = true;
          } else {
            rhos1 = tmp;
            f1 = ftmp;
            tmp = rhos0;
            ftmp = f0;
            rhos0 = rhos1;
            f0 = f1;
            rhos1 = rhos0 + factor * drho;
            f1 = hugo(rhos1);
            if (f0 * f1 <= 0) {
              found_rhos0 = found_rhos1 = true;
            } else {
              rhos0 = tmp;
              f0 = ftmp;
              drho = rhos1 - rhos0;
            }
          }
        }
        if (!found_rhos1) {
          i = 0;
          double factor2 = 2.5;
          while (!found_rhos1) {
            if (++i >= P.maxIts_shock) return false;
            rhos0 = rhos1;
            f0 = f1;
            rhos1 = rhos0 + factor2 * drho;
            f1 = hugo(rhos1);
            if (f0 * f1 <= 0)
              found_rhos1 = true;
            else
              drho = rhos1 - rhos0;
          }
        }
      }
      double sol_first, sol_second;
      double loc_tol_shock = P.tol_shock * smin(rhos0, rhos1);
      if (f0 == 0.0) {
        sol_first = sol_second = rhos0;
      } else if (f1 == 0.0) {
        sol_first = sol_second = rhos1;
      } else {  // secant with bisection safeguard (the WITHOUT_BOOST branch)
        double rhos2 = rhos1;
        double f2 = f1;
        int it;
        sol_first = sol_second = rhos2;
        for (it = 0; it < P.maxIts_shock; it++) {
          drho = rhos1 - rhos0;
          rhos2 = rhos2 - f2 * (rhos1 - rhos0) / (f1 - f0);
          if (rhos2 >= rhos1 || rhos2 <= rhos0) rhos2 = 0.5 * (rhos0 + rhos1);
          f2 = hugo(rhos2);
          if (f2 == 0.0) {
            sol_first = sol_second = rhos2;
            break;
          }
          if (f2 * f0 < 0) {
            rhos1 = rhos2;
            f1 = f2;
          } else {
            rhos0 = rhos2;
            f0 = f2;
          }
          if (rhos1 - rhos0 < loc_tol_shock) {
            sol_first = rhos0;
            sol_second = rhos1;
            break;
          }
        }
        if (it == P.maxIts_shock) return false;
      }
      rhos = 0.5 * (sol_first + sol_second);
      double du = -(ps - p) * (1.0 / rhos - 1.0 / rho);
      if (du < 0) return false;
      if (e.bad(rhos, ps)) return false;
      us = (wave == 1) ? u - sqrt(du) : u + sqrt(du);
    }
    return true;
  }

  // FindInitialFeasiblePointsByAcousticTheory (1064-1114): returns 0, 1 or 2.
  M2C_HD int acoustic_points(double rhol, double ul, double pl, double cl, int idl, double rhor, double ur, double pr,
                             double cr, int idr, double& p0, double& rhol0, double& rhor0, double& ul0, double& ur0,
                             double& p1, double& rhol1, double& rhor1, double& ul1, double& ur1) {
    int found = 0;
    double Cl = rhol * cl;
    double Cr = rhor * cr;
    p0 = (Cr * pl + Cl * pr + Cl * Cr * (ul - ur)) / (Cl + Cr);
    if (!rho_u_star(1, path1, rhol, ul, pl, p0, idl, rhol, (p0 > pl) ? rhol * 1.1 : rhol * 0.9, rhol0, ul0, nullptr,
                    nullptr))
      return found;
    if (!rho_u_star(3, path3, rhor, ur, pr, p0, idr, rhor, (p0 > pr) ? rhor * 1.1 : rhor * 0.9, rhor0, ur0, nullptr,
                    nullptr))
      return found;
    found = 1;
    double Clbar = (ul0 == ul) ? Cl : fabs(p0 - pl) / fabs(ul0 - ul);
    double Crbar = (ur0 == ur) ? Cr : fabs(p0 - pr) / fabs(ur0 - ur);
    p1 = (Crbar * pl + Clbar * pr + Clbar * Crbar * (ul - ur)) / (Clbar + Crbar);
    double tmp = smax(fabs(p0), fabs(p1));
    if (fabs(p1 - p0) / tmp < 1.0e-8) p1 = p0 + 1.0e-8 * tmp;
    if (!rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol, rhol0, rhol1, ul1, nullptr, nullptr)) return found;
    if (!rho_u_star(3, path3, rhor, ur, pr, p1, idr, rhor, rhor0, rhor1, ur1, nullptr, nullptr)) return found;
    found = 2;
    return found;
  }

  // FindInitialFeasiblePoints (959-1059)
  M2C_HD bool feasible_points(double rhol, double ul, double pl, double cl, int idl, double rhor, double ur, double pr,
                              double cr, int idr, double& p0, double& rhol0, double& rhor0, double& ul0, double& ur0,
                              double& p1, double& rhol1, double& rhor1, double& ul1, double& ur1) {
    bool success = true;
    int found = 0;
    // the acoustic (linearised) estimate the reference starts from
    const double Cl0 = rhol * cl, Cr0 = rhor * cr;
    const double pac = (Cr0 * pl + Cl0 * pr + Cl0 * Cr0 * (ul - ur)) / (Cl0 + Cr0);
    bool use_warm =
        isfinite(warm) && warm != 0.0 && P.warm_delta > 0.0 && !(fabs(warm - pac) <= P.warm_delta * fabs(pac));
    if (use_warm && P.warm_gate > 0.0) {
      // near-acoustic problem: the acoustic estimate starts as close as the
      // proposal would (distance measured with pressures shifted by the
      // smaller stiffness, the scale of the stopping test)
      const double sh = fmin(fabs(eos[idl].pstiff), fabs(eos[idr].pstiff));
      const double qa = pac + sh, qw = warm + sh;
      if (qa > 0.0 && qw > 0.0 && fabs(log(qw / qa)) <= P.warm_gate) use_warm = false;
    }
    if (use_warm) {
      // warm start: a proposal departing from the acoustic estimate by more
      // than the bracket width supplies the two points warm -+ d |warm| in
      // place of the acoustic estimates (p0 < p1, also for a negative
      // proposal on a stiffened gas), when both are feasible;
      // FindInitialInterval then expands them as it would expand the
      // acoustic pair
      const double half = P.warm_delta * fabs(warm);
      p0 = warm - half;
      p1 = warm + half;
      if (rho_u_star(1, path1, rhol, ul, pl, p0, idl, rhol, (p0 > pl) ? rhol * 1.1 : rhol * 0.9, rhol0, ul0, nullptr,
                     nullptr) &&
          rho_u_star(3, path3, rhor, ur, pr, p0, idr, rhor, (p0 > pr) ? rhor * 1.1 : rhor * 0.9, rhor0, ur0, nullptr,
                     nullptr) &&
          rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol, rhol0, rhol1, ul1, nullptr, nullptr) &&
          rho_u_star(3, path3, rhor, ur, pr, p1, idr, rhor, rhor0, rhor1, ur1, nullptr, nullptr))
        return true;
    }
    found = acoustic_points(rhol, ul, pl, cl, idl, rhor, ur, pr, cr, idr, p0, rhol0, rhor0, ul0, ur0, p1, rhol1,
                            rhor1, ul1, ur1);
    if (found == 2) return true;
    if (found != 1) {
      double dp = (pl != pr) ? fabs(pl - pr) : 0.5 * pl;
      for (int i = 0; i < P.maxIts_bracket; i++) {
        p0 = smin(pl, pr) + 0.01 * (i + 1) * (i + 1) * smin(dp, smin(fabs(pl), fabs(pr)));
        if (p0 < P.min_pressure) p0 = P.pressure_at_failure;
        success = rho_u_star(1, path1, rhol, ul, pl, p0, idl, rhol, (p0 > pl) ? rhol * 1.1 : rhol * 0.9, rhol0, ul0,
                             nullptr, nullptr);
        success = success && rho_u_star(3, path3, rhor, ur, pr, p0, idr, rhor, (p0 > pr) ? rhor * 1.1 : rhor * 0.9,
                                        rhor0, ur0, nullptr, nullptr);
        if (success) break;
      }
      if (!success) {
        for (int i = 0; i < P.maxIts_bracket; i++) {
          p0 = smin(pl, pr) - 0.01 * (i + 1) * (i + 1) * smin(dp, smin(fabs(pl), fabs(pr)));
          if (p0 < P.min_pressure || i == (int)(P.maxIts_bracket / 2)) p0 = P.pressure_at_failure;
          success = rho_u_star(1, path1, rhol, ul, pl, p0, idl, rhol, (p0 > pl) ? rhol * 1.1 : rhol * 0.9, rhol0,
                               ul0, nullptr, nullptr);
          success = success && rho_u_star(3, path3, rhor, ur, pr, p0, idr, rhor,
                                          (p0 > pr) ? rhor * 1.1 : rhor * 0.9, rhor0, ur0, nullptr, nullptr);
          if (success) break;
        }
      }
      if (!success) return false;
    }
    // p1
    {
      double dp = smin(fabs(p0 - pl), fabs(p0 - pr));
      for (int i = 0; i < P.maxIts_bracket; i++) {
        p1 = p0 + 0.01 * (i + 1) * (i + 1) * dp;
        success = rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol, rhol0, rhol1, ul1, nullptr, nullptr);
        success = success && rho_u_star(3, path3, rhor, ur, pr, p1, idr, rhor, rhor0, rhor1, ur1, nullptr, nullptr);
        if (success) break;
      }
      if (!success)
        for (int i = 0; i < P.maxIts_bracket; i++) {
          p1 = p0 - 0.01 * (i + 1) * (i + 1) * dp;
          if (p1 < P.min_pressure) p1 = P.pressure_at_failure * 1000.0;
          success = rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol, rhol0, rhol1, ul1, nullptr, nullptr);
          success = success && rho_u_star(3, path3, rhor, ur, pr, p1, idr, rhor, rhor0, rhor1, ur1, nullptr, nullptr);
          if (success) break;
        }
      if (!success) return false;
    }
    if (p0 > p1) {
      swap_(p0, p1);
      swap_(rhol0, rhol1);
      swap_(rhor0, rhor1);
      swap_(ul0, ul1);
      swap_(ur0, ur1);
    }
    return true;
  }

  // FindInitialInterval (631-795)
  M2C_HD bool initial_interval(double rhol, double ul, double pl, double cl, int idl, double rhor, double ur,
                               double pr, double cr, int idr, double& p0, double& rhol0, double& rhor0, double& ul0,
                               double& ur0, double& p1, double& rhol1, double& rhor1, double& ul1, double& ur1) {
    bool success = feasible_points(rhol, ul, pl, cl, idl, rhor, ur, pr, cr, idr, p0, rhol0, rhor0, ul0, ur0, p1,
                                   rhol1, rhor1, ul1, ur1);
    if (!success) {
      p0 = p1 = P.pressure_at_failure;
      return false;
    }
    double p2 = 0, rhol2 = 0, rhor2 = 0, ul2 = 0, ur2 = 0;
    double f0, f1;
    int i;
    double fmin, p_fmin, rhol_fmin, rhor_fmin, ul_fmin, ur_fmin;
    if (fabs(ul0 - ur0) < fabs(ul1 - ur1)) {
      fmin = fabs(ul0 - ur0);
      p_fmin = p0; rhol_fmin = rhol0; rhor_fmin = rhor0; ul_fmin = ul0; ur_fmin = ur0;
    } else {
      fmin = fabs(ul1 - ur1);
      p_fmin = p1; rhol_fmin = rhol1; rhor_fmin = rhor1; ul_fmin = ul1; ur_fmin = ur1;
    }
    for (i = 0; i < P.maxIts_bracket; i++) {
      f0 = ul0 - ur0;
      f1 = ul1 - ur1;
      if (f0 * f1 <= 0.0) return true;
      if (fabs(f0 - f1) > 1e-9) {
        p2 = p1 - f1 * (p1 - p0) / (f1 - f0);
        if (p2 < p0)
          p2 -= 0.1 * (p1 - p0);
        else
          p2 += 0.1 * (p1 - p0);
      } else {
        p2 = 1.1 * p1;
      }
      if (p2 < P.min_pressure || i == int(P.maxIts_bracket / 2)) p2 = 1.0e-8;
      success = rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, nullptr, nullptr);
      success = success && rho_u_star(3, path3, rhor, ur, pr, p2, idr, rhor0, rhor1, rhor2, ur2, nullptr, nullptr);
      if (!success) {
        for (int j = 0; j < P.maxIts_bracket / 2; j++) {
          if (p2 < p0)
            p2 = p0 - 0.5 * (p0 - p2);
          else
            p2 = p1 + 0.5 * (p2 - p1);
          success = rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, nullptr, nullptr);
          success = success && rho_u_star(3, path3, rhor, ur, pr, p2, idr, rhor0, rhor1, rhor2, ur2, nullptr, nullptr);
          if (success) break;
        }
      }
      if (!success) break;
      if (fabs(ul2 - ur2) < fmin) {
        fmin = fabs(ul2 - ur2);
        p_fmin = p2; rhol_fmin = rhol2; rhor_fmin = rhor2; ul_fmin = ul2; ur_fmin = ur2;
      }
      if (p2 < p0) {
        p1 = p0; rhol1 = rhol0; rhor1 = rhor0; ul1 = ul0; ur1 = ur0;
        p0 = p2; rhol0 = rhol2; rhor0 = rhor2; ul0 = ul2; ur0 = ur2;
      } else {
        p0 = p1; rhol0 = rhol1; rhor0 = rhor1; ul0 = ul1; ur0 = ur1;
        p1 = p2; rhol1 = rhol2; rhor1 = rhor2; ul1 = ul2; ur1 = ur2;
      }
    }
    if (!success || i == P.maxIts_bracket) {
      if (fmin < P.failure_threshold * fabs(ul - ur)) {
        p0 = p1 = p_fmin;
        rhol0 = rhol1 = rhol_fmin;
        rhor0 = rhor1 = rhor_fmin;
        ul0 = ul1 = ul_fmin;
        ur0 = ur1 = ur_fmin;
      } else {
        p2 = P.pressure_at_failure;
        success = rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, nullptr, nullptr);
        success = success && rho_u_star(3, path3, rhor, ur, pr, p2, idr, rhor0, rhor1, rhor2, ur2, nullptr, nullptr);
        if (success) {
          p0 = p1 = p2;
          rhol0 = rhol1 = rhol2;
          rhor0 = rhor1 = rhor2;
          ul0 = ul1 = ul2;
          ur0 = ur1 = ur2;
        } else {
          p0 = p1 = p_fmin;
          rhol0 = rhol1 = rhol_fmin;
          rhor0 = rhor1 = rhor_fmin;
          ul0 = ul1 = ul_fmin;
          ur0 = ur1 = ur_fmin;
        }
      }
      return false;
    }
    return true;
  }

  // FinalizeSolution (347-514)
  M2C_HD void finalize(const double* dir, const double* Vm, const double* Vp, double rhol, double ul, double pl,
                       int idl, double rhor, double ur, double pr, int idr, double rhol2, double rhor2, double u2,
                       double p2, bool trans_rare, const double* Vrare_x0, double* Vs, int& id, double* Vsm,
                       double* Vsp, bool& bad) const {
    double utanl[3] = {Vm[1] - ul * dir[0], Vm[2] - ul * dir[1], Vm[3] - ul * dir[2]};
    double utanr[3] = {Vp[1] - ur * dir[0], Vp[2] - ur * dir[1], Vp[3] - ur * dir[2]};
    id = (u2 >= 0) ? idl : idr;
    Vs[0] = Vs[1] = Vs[2] = Vs[3] = Vs[4] = 0.0;
    if (trans_rare) {
      Vs[0] = Vrare_x0[0];
      Vs[1] = Vrare_x0[1] * dir[0];
      Vs[2] = Vrare_x0[1] * dir[1];
      Vs[3] = Vrare_x0[1] * dir[2];
      Vs[4] = Vrare_x0[2];
    } else if (u2 >= 0) {
      bool is_star_state = false;
      if (pl >= p2) {
        double el2 = eos[idl].energy(rhol2, p2);
        double cl2 = eos[idl].c2(rhol2, el2);
        if (rhol2 <= 0 || cl2 < 0) { bad = true; cl2 = 0; }  // the reference aborts
        else cl2 = sqrt(cl2);
        if (u2 - cl2 <= 0) is_star_state = true;
      } else {
        double us = (rhol2 * u2 - rhol * ul) / (rhol2 - rhol);
        if (us <= 0) is_star_state = true;
      }
      if (is_star_state) {
        Vs[0] = rhol2; Vs[1] = u2 * dir[0]; Vs[2] = u2 * dir[1]; Vs[3] = u2 * dir[2]; Vs[4] = p2;
      } else {
        Vs[0] = rhol; Vs[1] = ul * dir[0]; Vs[2] = ul * dir[1]; Vs[3] = ul * dir[2]; Vs[4] = pl;
      }
    } else {
      bool is_star_state = false;
      if (pr >= p2) {
        double er2 = eos[idr].energy(rhor2, p2);
        double cr2 = eos[idr].c2(rhor2, er2);
        if (rhor2 <= 0 || cr2 < 0) { bad = true; cr2 = 0; }
        else cr2 = sqrt(cr2);
        if (u2 - cr2 >= 0) is_star_state = true;
      } else {
        double us = (rhor2 * u2 - rhor * ur) / (rhor2 - rhor);
        if (us >= 0) is_star_state = true;
      }
      if (is_star_state) {
        Vs[0] = rhor2; Vs[1] = u2 * dir[0]; Vs[2] = u2 * dir[1]; Vs[3] = u2 * dir[2]; Vs[4] = p2;
      } else {
        Vs[0] = rhor; Vs[1] = ur * dir[0]; Vs[2] = ur * dir[1]; Vs[3] = ur * dir[2]; Vs[4] = pr;
      }
    }
    if (u2 > 0) {
      for (int i = 1; i <= 3; i++) Vs[i] += utanl[i - 1];
    } else if (u2 < 0) {
      for (int i = 1; i <= 3; i++) Vs[i] += utanr[i - 1];
    } else {
      for (int i = 1; i <= 3; i++) Vs[i] += 0.5 * (utanl[i - 1] + utanr[i - 1]);
    }
    Vsm[0] = rhol2;
    Vsm[1] = utanl[0] + u2 * dir[0];
    Vsm[2] = utanl[1] + u2 * dir[1];
    Vsm[3] = utanl[2] + u2 * dir[2];
    Vsm[4] = p2;
    Vsp[0] = rhor2;
    Vsp[1] = utanr[0] + u2 * dir[0];
    Vsp[2] = utanr[1] + u2 * dir[1];
    Vsp[3] = utanr[2] + u2 * dir[2];
    Vsp[4] = p2;
  }

  // ComputeRiemannSolution (59-342).
  // Warm start (no counterpart in the reference): a finite non-zero warm_p
  // supplies the two starting points of the bracket search (see
  // feasible_points); the bracket expansion, the safeguarded secant loop and
  // its stopping test are the reference's, so a warm-started solve converges
  // to the same root within tol_main.
  // Returns RIEM_OK or RIEM_FAILED (| RIEM_PATH_OVERFLOW); *bad_state set if a
  // state the reference aborts on was met.
  M2C_HD int solve(const double* dir, const double* Vm, int idl, const double* Vp, int idr, double* Vs, int& id,
                   double* Vsm, double* Vsp, double warm_p, bool& bad_state) {
    bad_state = false;
    iterations = 0;
    evaluations = 0;
    nonadaptive = false;
    retried = false;
    warm = warm_p;
    int r = 0, overflow = 0;
    // one loop, so that the solver body is inlined once
    for (int pass = 0; pass < 2; pass++) {
      r = attempt(dir, Vm, idl, Vp, idr, Vs, id, Vsm, Vsp, bad_state);
      overflow |= r & RIEM_PATH_OVERFLOW;
      if (!(r & RIEM_RETRY)) break;
      // ExactRiemannSolverBase.cpp:173-188 and 327-330: a fresh
      // ExactRiemannSolverNonAdaptive (empty integration paths, acoustic
      // starting points) solves the problem again and its result is returned
      nonadaptive = true;
      retried = true;
      warm = NAN;
    }
    nonadaptive = false;
    return r | overflow;
  }

  // One solve by the adaptive (nonadaptive = false) or the non-adaptive
  // solver: ComputeRiemannSolution (59-342) / (2199-2470).
  M2C_HD int attempt(const double* dir, const double* Vm, int idl, const double* Vp, int idr, double* Vs, int& id,
                     double* Vsm, double* Vsp, bool& bad_state) {
    double rhol = Vm[0];
    double ul = Vm[1] * dir[0] + Vm[2] * dir[1] + Vm[3] * dir[2];
    double pl = Vm[4];
    double rhor = Vp[0];
    double ur = Vp[1] * dir[0] + Vp[2] * dir[1] + Vp[3] * dir[2];
    double pr = Vp[4];
    path1.n = path3.n = 0;
    path1.overflow = path3.overflow = false;
    path1.push(pl, rhol, ul);
    path3.push(pr, rhor, ur);
    double el = eos[idl].energy(rhol, pl);
    double cl = eos[idl].c2(rhol, el);
    if (rhol <= 0 || cl < 0) { bad_state = true; return RIEM_FAILED; }
    cl = sqrt(cl);
    double er = eos[idr].energy(rhor, pr);
    double cr = eos[idr].c2(rhor, er);
    if (rhor <= 0 || cr < 0) { bad_state = true; return RIEM_FAILED; }
    cr = sqrt(cr);
    double p0 = DBL_MIN, ul0 = 0.0, ur0 = 0.0, rhol0 = DBL_MIN, rhor0 = DBL_MIN;
    double p1 = DBL_MIN, ul1 = 0.0, ur1 = 0.0, rhol1 = DBL_MIN, rhor1 = DBL_MIN;
    double p2 = DBL_MIN, ul2 = 0.0, ur2 = 0.0, rhol2 = DBL_MIN, rhor2 = DBL_MIN;
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    bool success = true;
    bool trans_rare = false;
    double Vrare_x0[3] = {0, 0, 0};
    if (ul == ur && pl == pr) {  // trivial case
      finalize(dir, Vm, Vp, rhol, ul, pl, idl, rhor, ur, pr, idr, rhol, rhor, ul, pl, trans_rare, Vrare_x0, Vs, id, Vsm,
               Vsp, bad_state);
      return RIEM_OK;
    }
    success = initial_interval(rhol, ul, pl, cl, idl, rhor, ur, pr, cr, idr, p0, rhol0, rhor0, ul0, ur0, p1, rhol1,
                               rhor1, ul1, ur1);
    if (!success) {
      // a best-effort answer at p1 (173-188, 2302-2335); the adaptive solver
      // then hands over to the non-adaptive one, which returns it as failed
      success = rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol0, rhol0 * 1.1, rhol2, ul2, &trans_rare, Vrare_x0);
      success = success && rho_u_star(3, path3, rhor, ur, pr, p1, idr, rhor0, rhol0 * 1.1, rhor2, ur2, &trans_rare,
                                      Vrare_x0);
      if (success) {
        finalize(dir, Vm, Vp, rhol, ul, pl, idl, rhor, ur, pr, idr, rhol2, rhor2, 0.5 * (ul2 + ur2), p1, trans_rare,
                 Vrare_x0, Vs, id, Vsm, Vsp, bad_state);
      } else {  // the initial states as the solution
        for (int i = 0; i < 5; i++) {
          Vsm[i] = Vm[i];
          Vsp[i] = Vp[i];
        }
        const double u_avg = 0.5 * (ul + ur);
        id = u_avg >= 0 ? idl : idr;
        for (int i = 0; i < 5; i++) Vs[i] = u_avg >= 0 ? Vm[i] : Vp[i];
      }
      return (nonadaptive ? RIEM_FAILED : RIEM_RETRY) | ((path1.overflow || path3.overflow) ? RIEM_PATH_OVERFLOW : 0);
    }
    f0 = ul0 - ur0;
    f1 = ul1 - ur1;
    double denom = 0;
    int iter = 0;
    double err_p = 1.0, err_u = 1.0;
    p2 = p1;
    f2 = f1;
    for (iter = 0; iter < P.maxIts_main; iter++) {
      denom = f1 - f0;
      if (denom == 0) {
        p2 = 0.5 * (p0 + p1);
      } else {
        p2 = p2 - f2 * (p1 - p0) / denom;
        if (p2 <= p0 || p2 >= p1) p2 = 0.5 * (p0 + p1);
      }
    try_again:
      success = rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, &trans_rare, Vrare_x0);
      if (!success) {
        p2 = 0.5 * (p2 + p0);
        iter++;
        if (iter < P.maxIts_main)
          goto try_again;
        else
          break;
      }
      success = rho_u_star(3, path3, rhor, ur, pr, p2, idr, rhor0, rhor1, rhor2, ur2, &trans_rare, Vrare_x0);
      if (!success) {
        p2 = 0.5 * (p2 + p1);
        iter++;
        if (iter < P.maxIts_main)
          goto try_again;
        else
          break;
      }
      f2 = ul2 - ur2;
      if (f0 * f2 < 0.0) {
        p1 = p2; f1 = f2; rhol1 = rhol2; rhor1 = rhor2;
      } else {
        p0 = p2; f0 = f2; rhol0 = rhol2; rhor0 = rhor2;
      }
      err_p = fabs(p1 - p0) / smax(fabs(pl + 0.5 * rhol * ul * ul), fabs(pr + 0.5 * rhor * ur * ur));
      err_u = fabs(f2) / smax(cl, cr);
      if ((err_p < P.tol_main && err_u < P.tol_main) || (err_p < P.tol_main * 1e-3) || (err_u < P.tol_main * 1e-3))
        break;
      trans_rare = false;
    }
    iterations += iter + 1;
    double u2 = 0.5 * (ul2 + ur2);
    finalize(dir, Vm, Vp, rhol, ul, pl, idl, rhor, ur, pr, idr, rhol2, rhor2, u2, p2, trans_rare, Vrare_x0, Vs, id,
             Vsm, Vsp, bad_state);
    int flags = (path1.overflow || path3.overflow) ? RIEM_PATH_OVERFLOW : 0;
    if (iter == P.maxIts_main) return (nonadaptive ? RIEM_FAILED : RIEM_RETRY) | flags;
    return RIEM_OK | flags;
  }

  // ---- one-sided (wall) problem: the fluid state on the minus side of a
  // wall moving with normal velocity ustar (ExactRiemannSolverBase.cpp:
  // 1931-2195 and its helpers). Only the 1-wave exists; its star velocity is
  // the wall's.

  // ComputeOneSidedRarefaction (1586-1728): integrate the 1-wave rarefaction
  // in pressure from (rho, u, p) until its velocity reaches us > u. The step
  // is sized by the velocity gained per step (target (us - u) / numSteps).
  M2C_HD bool wall_rarefaction(double rho, double u, double p, double c, int id, double us, double& rhos, double& ps,
                               bool* trans_rare, double* Vrare_x0) const {
    const Eos<double>& e = eos[id];
    rhos = rho;
    ps = p;
    const double du_goal = (us - u) / P.numSteps_rarefaction;
    const double du_cap = du_goal * 1.25;
    const double dp_lin = fabs(du_goal * c * rho);
    const double dp_rel = (fabs(p) + 1.0e-6) / (P.numSteps_rarefaction * 2.5);
    double dp = smin(dp_lin, dp_rel);
    double r0 = rho, v0 = u, q0 = p, x0 = u - c;  // start of the step
    double r1 = rho, v1 = u, q1 = p, x1;          // end of the step
    const double utol = P.tol_rarefaction * smax(us - u, smax(fabs(us), fabs(u)));
    double errU = 0, errR = 0;
    for (int i = 0; i < P.numSteps_rarefaction * 5; i++) {
      if (!rk_step(1, id, r0, v0, q0, dp, r1, v1, q1, x1, errU, errR)) {
        dp /= 2.0;
        continue;
      }
      const double dv = v1 - v0;
      if (dv > du_cap) {
        dp = dp / dv * du_goal;
        continue;
      }
      if (v1 - us > utol) {  // overshot the wall velocity
        if (dv != 0)
          dp = dp / dv * (us - v0);
        else
          dp /= 2.0;
        continue;
      }
      if (trans_rare && Vrare_x0 && x0 * x1 <= 0) {  // the fan crosses xi = 0
        *trans_rare = true;
        double w0 = fabs(x1), w1 = fabs(x0);
        const double ww = w0 + w1;
        w0 /= ww;
        w1 /= ww;
        Vrare_x0[0] = w0 * r0 + w1 * r1;
        Vrare_x0[1] = w0 * v0 + w1 * v1;
        Vrare_x0[2] = w0 * q0 + w1 * q1;
      }
      if (fabs(us - v1) <= utol) {
        rhos = r1;
        ps = q1;
        return !e.bad(rhos, ps);
      }
      dp = smin(dp / dv * smin(du_goal, us - v1), dp * 5.0);
      r0 = r1;
      v0 = v1;
      q0 = q1;
      x0 = x1;
    }
    return false;  // did not reach us (the reference fails either way)
  }

  // FindInitialFeasiblePointsOneSidedByAcousticTheory (1119-1168): 0, 1 or 2
  // points on the 1-wave curve, from the acoustic impedance.
  M2C_HD int wall_acoustic_points(double rhol, double ul, double pl, double cl, int idl, double ustar, double& p0,
                                  double& rhol0, double& ul0, double& p1, double& rhol1, double& ul1) {
    const double Cl = rhol * cl;
    p0 = pl + Cl * (ul - ustar);
    bool ok = rho_u_star(1, path1, rhol, ul, pl, p0, idl, rhol, (p0 > pl) ? rhol * 1.1 : rhol * 0.9, rhol0, ul0,
                         nullptr, nullptr);
    if (!ok) {
      p0 = 1.5 * pl;
      ok = rho_u_star(1, path1, rhol, ul, pl, p0, idl, rhol, (p0 > pl) ? rhol * 1.1 : rhol * 0.9, rhol0, ul0,
                      nullptr, nullptr);
      if (!ok) return 0;
    }
    const double Clbar = (ul0 == ul) ? Cl : fabs(p0 - pl) / fabs(ul0 - ul);
    p1 = pl + Clbar * (ul - ustar);
    const double big = smax(fabs(p0), fabs(p1));
    if (fabs(p1 - p0) / big < 1.0e-8) p1 = p0 + 1.0e-8 * big;
    if (!rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol, rhol0, rhol1, ul1, nullptr, nullptr)) return 1;
    return 2;
  }

  // FindInitialFeasiblePointsOneSided (2946-3016): the acoustic points, else
  // a search at growing distances from pl.
  M2C_HD bool wall_feasible_points(double rhol, double ul, double pl, double cl, int idl, double ustar, double& p0,
                                   double& rhol0, double& ul0, double& p1, double& rhol1, double& ul1) {
    const int found = wall_acoustic_points(rhol, ul, pl, cl, idl, ustar, p0, rhol0, ul0, p1, rhol1, ul1);
    if (found == 2) return true;
    bool ok = true;
    if (found == 0) {
      const double step = ul > ustar ? 0.5 * pl : -0.5 * pl;
      for (int i = 0; i < P.maxIts_bracket; i++) {
        p0 = pl + 0.01 * (i + 1) * (i + 1) * step;
        if (p0 < P.min_pressure) p0 = P.pressure_at_failure;
        ok = rho_u_star(1, path1, rhol, ul, pl, p0, idl, rhol, (p0 > pl) ? rhol * 1.1 : rhol * 0.9, rhol0, ul0,
                        nullptr, nullptr);
        if (ok) break;
      }
      if (!ok) return false;
    }
    const double step = p0 - pl;
    for (int i = 0; i < P.maxIts_bracket; i++) {
      p1 = p0 + 0.01 * (i + 1) * (i + 1) * step;
      ok = rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol, rhol0, rhol1, ul1, nullptr, nullptr);
      if (ok) break;
    }
    if (!ok) return false;
    if (p0 > p1) {
      swap_(p0, p1);
      swap_(rhol0, rhol1);
      swap_(ul0, ul1);
    }
    return true;
  }

  // FindInitialIntervalOneSided (800-958): from two feasible points, secant
  // steps pushed 10% outward until ul(p) - ustar changes sign. On failure the
  // point with the smallest |ul - ustar| (or pressure_at_failure, when that
  // residual is not small) is returned as p0 = p1, and false.
  M2C_HD bool wall_interval(double rhol, double ul, double pl, double cl, int idl, double ustar, double& p0,
                            double& rhol0, double& ul0, double& p1, double& rhol1, double& ul1) {
    if (!wall_feasible_points(rhol, ul, pl, cl, idl, ustar, p0, rhol0, ul0, p1, rhol1, ul1)) {
      p0 = p1 = P.pressure_at_failure;
      return false;
    }
    double p2, rhol2, ul2, f0, f1;
    double best, p_best, rho_best, u_best;  // smallest |f| met (failsafe answer)
    if (fabs(ul0 - ustar) < fabs(ul1 - ustar)) {
      best = fabs(ul0 - ustar); p_best = p0; rho_best = rhol0; u_best = ul0;
    } else {
      best = fabs(ul1 - ustar); p_best = p1; rho_best = rhol1; u_best = ul1;
    }
    bool ok = true;
    int i;
    for (i = 0; i < P.maxIts_bracket; i++) {
      f0 = ul0 - ustar;
      f1 = ul1 - ustar;
      if (f0 * f1 <= 0.0) return true;
      if (fabs(f0 - f1) > 1e-9) {
        p2 = p1 - f1 * (p1 - p0) / (f1 - f0);
        if (p2 < p0)
          p2 -= 0.1 * (p1 - p0);
        else
          p2 += 0.1 * (p1 - p0);
      } else {
        p2 = 1.1 * p1;
      }
      if (p2 < pl || i == int(P.maxIts_bracket / 2)) p2 = pl;
      ok = rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, nullptr, nullptr);
      if (!ok) {  // step back towards [p0, p1]
        for (int j = 0; j < P.maxIts_bracket / 2; j++) {
          if (p2 < p0)
            p2 = p0 - 0.5 * (p0 - p2);
          else
            p2 = p1 + 0.5 * (p2 - p1);
          if (p2 < pl) p2 = pl;
          ok = rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, nullptr, nullptr);
          if (ok) break;
        }
      }
      if (!ok) break;
      if (fabs(ul2 - ustar) < best) {
        best = fabs(ul2 - ustar); p_best = p2; rho_best = rhol2; u_best = ul2;
      }
      if (p2 < p0) {
        p1 = p0; rhol1 = rhol0; ul1 = ul0;
        p0 = p2; rhol0 = rhol2; ul0 = ul2;
      } else {
        p0 = p1; rhol0 = rhol1; ul0 = ul1;
        p1 = p2; rhol1 = rhol2; ul1 = ul2;
      }
    }
    (void)i;
    if (best < P.failure_threshold * fabs(ul - ustar)) {
      p0 = p1 = p_best; rhol0 = rhol1 = rho_best; ul0 = ul1 = u_best;
    } else {  // the problem may have no solution: the prescribed pressure
      p2 = P.pressure_at_failure;
      if (rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, nullptr, nullptr)) {
        p0 = p1 = p2; rhol0 = rhol1 = rhol2; ul0 = ul1 = ul2;
      } else {
        p0 = p1 = p_best; rhol0 = rhol1 = rho_best; ul0 = ul1 = u_best;
      }
    }
    return false;
  }

  // FinalizeOneSidedSolution (519-630): the state at xi = 0 (id = -1 where
  // the wall moves away, ustar < 0, and the point lies beyond the fluid) and
  // the star state Vsm with the tangential velocity of Vm.
  M2C_HD void wall_finalize(const double* dir, const double* Vm, double rhol, double ul, double pl, int idl,
                            double rhol2, double u2, double p2, bool trans_rare, const double* Vrare_x0, double* Vs,
                            int& id, double* Vsm, bool& bad) const {
    const double utanl[3] = {Vm[1] - ul * dir[0], Vm[2] - ul * dir[1], Vm[3] - ul * dir[2]};
    id = u2 >= 0 ? idl : -1;
    if (id != -1) {
      Vs[0] = Vs[1] = Vs[2] = Vs[3] = Vs[4] = 0.0;
      if (trans_rare) {
        Vs[0] = Vrare_x0[0];
        Vs[1] = Vrare_x0[1] * dir[0];
        Vs[2] = Vrare_x0[1] * dir[1];
        Vs[3] = Vrare_x0[1] * dir[2];
        Vs[4] = Vrare_x0[2];
      } else {
        bool star = false;
        if (pl >= p2) {  // rarefaction: is the tail left of xi = 0?
          double el2 = eos[idl].energy(rhol2, p2);
          double cl2 = eos[idl].c2(rhol2, el2);
          if (rhol2 <= 0 || cl2 < 0) { bad = true; cl2 = 0; }  // the reference aborts
          else cl2 = sqrt(cl2);
          if (u2 - cl2 <= 0) star = true;
        } else {  // shock: its speed
          const double sh = (rhol2 * u2 - rhol * ul) / (rhol2 - rhol);
          if (sh <= 0) star = true;
        }
        if (star) {
          Vs[0] = rhol2; Vs[1] = u2 * dir[0]; Vs[2] = u2 * dir[1]; Vs[3] = u2 * dir[2]; Vs[4] = p2;
        } else {
          Vs[0] = rhol; Vs[1] = ul * dir[0]; Vs[2] = ul * dir[1]; Vs[3] = ul * dir[2]; Vs[4] = pl;
        }
      }
      for (int i = 1; i <= 3; i++) Vs[i] += utanl[i - 1];
    }
    Vsm[0] = rhol2;
    Vsm[1] = utanl[0] + u2 * dir[0];
    Vsm[2] = utanl[1] + u2 * dir[1];
    Vsm[3] = utanl[2] + u2 * dir[2];
    Vsm[4] = p2;
  }

  // The input state with its normal velocity replaced by the wall's: the
  // answer of a solve that failed (2022-2040, 2082-2100).
  M2C_HD static void wall_fallback(const double* dir, const double* Vm, double ul, double ustar, int idl, double* Vs,
                                   int& id, double* Vsm) {
    const double utanl[3] = {Vm[1] - ul * dir[0], Vm[2] - ul * dir[1], Vm[3] - ul * dir[2]};
    Vsm[0] = Vm[0];
    Vsm[1] = utanl[0] + ustar * dir[0];
    Vsm[2] = utanl[1] + ustar * dir[1];
    Vsm[3] = utanl[2] + ustar * dir[2];
    Vsm[4] = Vm[4];
    if (ustar >= 0) {
      id = idl;
      for (int i = 0; i < 5; i++) Vs[i] = Vsm[i];
    } else {
      id = -1;
    }
  }

  // ComputeOneSidedRiemannSolution (1931-2195): Vm (id idl) against a wall
  // whose velocity is Ustar, dir the unit normal pointing from the fluid to
  // the wall. Trivial when the normal velocities agree, a rarefaction when
  // the fluid moves away from the wall, else a shock whose pressure is found
  // by the safeguarded secant method. Returns RIEM_OK or RIEM_FAILED
  // (| RIEM_PATH_OVERFLOW); bad_state is set where the reference aborts.
  M2C_HD int solve_wall(const double* dir, const double* Vm, int idl, const double* Ustar, double* Vs, int& id,
                        double* Vsm, bool& bad_state) {
    bad_state = false;
    iterations = 0;
    evaluations = 0;
    const double rhol = Vm[0];
    const double ul = Vm[1] * dir[0] + Vm[2] * dir[1] + Vm[3] * dir[2];
    const double pl = Vm[4];
    const double ustar = Ustar[0] * dir[0] + Ustar[1] * dir[1] + Ustar[2] * dir[2];
    const Eos<double>& e = eos[idl];
    const double el = e.energy(rhol, pl);
    double cl = e.c2(rhol, el);
    if (rhol <= 0 || cl < 0) {  // the reference aborts here
      bad_state = true;
      wall_fallback(dir, Vm, ul, ustar, idl, Vs, id, Vsm);
      return RIEM_FAILED;
    }
    cl = sqrt(cl);
    path1.n = 0;
    path1.overflow = false;
    path1.push(pl, rhol, ul);
    double p0 = DBL_MIN, ul0 = 0.0, rhol0 = DBL_MIN;
    double p1 = DBL_MIN, ul1 = 0.0, rhol1 = DBL_MIN;
    double p2 = DBL_MIN, ul2 = 0.0, rhol2 = DBL_MIN;
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    bool trans_rare = false;
    double Vrare_x0[3] = {0.0, 0.0, 0.0};
    auto flags = [&]() { return path1.overflow ? RIEM_PATH_OVERFLOW : 0; };
    if (fabs(ul - ustar) < 1.0e-20) {
      wall_finalize(dir, Vm, rhol, ul, pl, idl, rhol, ul, pl, trans_rare, Vrare_x0, Vs, id, Vsm, bad_state);
      return RIEM_OK;
    }
    if (ul < ustar) {  // rarefaction
      if (!wall_rarefaction(rhol, ul, pl, cl, idl, ustar, rhol2, p2, &trans_rare, Vrare_x0)) {
        wall_fallback(dir, Vm, ul, ustar, idl, Vs, id, Vsm);
        return RIEM_FAILED | flags();
      }
      wall_finalize(dir, Vm, rhol, ul, pl, idl, rhol2, ustar, p2, trans_rare, Vrare_x0, Vs, id, Vsm, bad_state);
      return RIEM_OK | flags();
    }
    // shock
    if (!wall_interval(rhol, ul, pl, cl, idl, ustar, p0, rhol0, ul0, p1, rhol1, ul1)) {
      if (!rho_u_star(1, path1, rhol, ul, pl, p1, idl, rhol0, rhol0 * 1.1, rhol2, ul2, &trans_rare, Vrare_x0)) {
        wall_fallback(dir, Vm, ul, ustar, idl, Vs, id, Vsm);
        return RIEM_FAILED | flags();
      }
      wall_finalize(dir, Vm, rhol, ul, pl, idl, rhol2, ustar, p1, trans_rare, Vrare_x0, Vs, id, Vsm, bad_state);
      return RIEM_FAILED | flags();
    }
    f0 = ul0 - ustar;
    f1 = ul1 - ustar;
    double denom = 0;
    int iter = 0;
    double err_p = 1.0, err_u = 1.0;
    p2 = p1;
    f2 = f1;
    for (iter = 0; iter < P.maxIts_main; iter++) {
      denom = f1 - f0;
      if (denom == 0) {
        p2 = 0.5 * (p0 + p1);
      } else {
        p2 = p2 - f2 * (p1 - p0) / denom;
        if (p2 <= p0 || p2 >= p1) p2 = 0.5 * (p0 + p1);
      }
    retry_wall:
      if (!rho_u_star(1, path1, rhol, ul, pl, p2, idl, rhol0, rhol1, rhol2, ul2, &trans_rare, Vrare_x0)) {
        p2 = 0.5 * (p2 + p0);
        iter++;
        if (iter < P.maxIts_main)
          goto retry_wall;
        else
          break;
      }
      f2 = ul2 - ustar;
      if (f0 * f2 < 0.0) {
        p1 = p2; f1 = f2; rhol1 = rhol2;
      } else {
        p0 = p2; f0 = f2; rhol0 = rhol2;
      }
      err_p = fabs(p1 - p0) / fabs(pl + 0.5 * rhol * ul * ul);
      err_u = fabs(f2) / cl;
      if ((err_p < P.tol_main && err_u < P.tol_main) || (err_p < P.tol_main * 1e-3) || (err_u < P.tol_main * 1e-3))
        break;
      trans_rare = false;
    }
    iterations = iter + 1;
    wall_finalize(dir, Vm, rhol, ul, pl, idl, rhol2, ustar, p2, trans_rare, Vrare_x0, Vs, id, Vsm, bad_state);
    if (iter == P.maxIts_main) return RIEM_FAILED | flags();
    return RIEM_OK | flags();
  }
};

}  // namespace m2c
