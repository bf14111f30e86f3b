// Point-wise physics of the M2C finite-volume step: equations of state,
// primitive/conservative conversion, state checks and clipping, slope
// limiters, and the HLLC / generalized-Roe / local Lax-Friedrichs fluxes.
//
// Every function is templated on the arithmetic type T (double for the FP64
// path, float for the reconstruction/flux half of the mixed path) and keeps
// the reference's operation order, so that the FP64 path, compiled without
// FMA contraction, reproduces the reference bit for bit:
//   EOS          VarFcnSG.h:64-68, VarFcnNASG.h:55-60, VarFcnBase.h:170-295
//   limiters     Reconstructor.h:95-110
//   HLLC         FluxFcnHLLC.h:47-245 (Toro ch.10 with Hu et al. 2009 wave speeds)
//   Roe          FluxFcnGenRoe.h:56-221 (generalized Roe, Harten entropy fix)
//   LLF          FluxFcnLLF.h:47-185
//   flux F,G,H   FluxFcnBase.h:83-123
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define M2C_HD __host__ __device__ __forceinline__
// Large helpers called from many sites (the Riemann solver's star-state
// evaluation): one out-of-line copy keeps the kernel's code within the
// instruction cache.
#define M2C_HD_OUTLINE __host__ __device__ __noinline__
#else
#define M2C_HD inline
#define M2C_HD_OUTLINE inline
#endif

namespace m2c {

enum { EOS_SG = 0, EOS_NASG = 1 };
enum { FLUX_ROE = 0, FLUX_LLF = 1, FLUX_HLLC = 2 };
enum { LIM_NONE = 0, LIM_GENMINMOD = 1, LIM_VANALBADA = 2 };

// Error codes recorded by kernels (first one wins).
enum {
  ERR_NONE = 0,
  ERR_STATE = 3,      // CheckState failure (SpaceOperator.cpp:3321-3330, 624-631)
  ERR_SOUND = 9,      // c^2 < 0 in a flux or the CFL sweep (FluxFcnHLLC.h:118-130)
  ERR_HLLC = 10,      // NaN S* in HLLC (FluxFcnHLLC.h:235-241)
  ERR_RIEMANN = 4,
  ERR_ITER_CAP = 6,
  ERR_UNSUPPORTED = 8,  // a path the library does not implement was reached (state update)
  ERR_MATERIAL_ID = 11  // an uploaded material ID beyond the materials (or inactive where not allowed)
};

// std::min / std::max semantics (not fmin/fmax): min(a,b) = (b<a)?b:a.
template <typename T> M2C_HD T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T> M2C_HD T smax(T a, T b) { return (a < b) ? b : a; }

template <typename T> M2C_HD bool finite_(T x) { return isfinite(x); }

// Component d of a 3-vector / of the velocity part of a state, by selects
// (no dynamically indexed local arrays).
template <typename T> M2C_HD T pick3(int d, T a, T b, T c) { return d == 0 ? a : (d == 1 ? b : c); }
template <typename T> M2C_HD T vnorm(int d, const T* V) { return pick3(d, V[1], V[2], V[3]); }

// Material parameters in arithmetic type T.
template <typename T>
struct Eos {
  int kind;
  T gam, gam1, invgam1;
  T pstiff;     // SG: Pstiff; NASG: pc
  T gam_ps;     // gam*Pstiff (SG) or gam*pc (NASG), precomputed as the reference does
  T b, q;       // NASG
  T rhomin, pmin, rhomax, pmax;

  // p(rho, e)
  M2C_HD T pressure(T rho, T e) const {
    if (kind == EOS_SG) return gam1 * rho * e - gam_ps;
    return gam1 * (e - q) / (T(1) / rho - b) - gam_ps;
  }
  // e(rho, p)
  M2C_HD T energy(T rho, T p) const {
    if (kind == EOS_SG) return (p + gam_ps) / (gam1 * rho);
    return invgam1 * (p + gam_ps) * (T(1) / rho - b) + q;
  }
  M2C_HD T dpdrho(T rho, T e) const {
    if (kind == EOS_SG) return gam1 * e;
    T V = T(1) / rho;
    return gam1 * V * V * (e - q) / ((V - b) * (V - b));
  }
  M2C_HD T big_gamma(T rho, T e) const {
    if (kind == EOS_SG) return gam1;
    return gam1 / (T(1) - b * rho);
  }
  // VarFcnBase::ComputeSoundSpeedSquare: recomputes p from (rho, e).
  M2C_HD T c2(T rho, T e) const { return dpdrho(rho, e) + pressure(rho, e) / rho * big_gamma(rho, e); }
  // true = violates hyperbolicity (VarFcnSG::CheckState / VarFcnNASG::CheckState)
  M2C_HD bool bad(T rho, T p) const {
    if (!finite_(rho) || !finite_(p)) return true;
    return rho <= T(0) || p + pstiff <= T(0);
  }
  M2C_HD bool bad(const T* V) const {
    if (!finite_(V[0]) || !finite_(V[1]) || !finite_(V[2]) || !finite_(V[3]) || !finite_(V[4])) return true;
    return bad(V[0], V[4]);
  }
  // VarFcnBase::ClipDensityAndPressure (without the U update); returns clipped?
  M2C_HD bool clip(T* V) const {
    bool c = false;
    if (V[0] < rhomin) { V[0] = rhomin; c = true; }
    if (V[4] < pmin) { V[4] = pmin; c = true; }
    if (V[0] > rhomax) { V[0] = rhomax; c = true; }
    if (V[4] > pmax) { V[4] = pmax; c = true; }
    return c;
  }
  // Would clip() change V? (used where the reference reverts instead)
  M2C_HD bool needs_clip(const T* V) const {
    return V[0] < rhomin || V[4] < pmin || V[0] > rhomax || V[4] > pmax;
  }
  // H = e + |u|^2/2 + p/rho (VarFcnBase::ComputeTotalEnthalpyPerUnitMass)
  M2C_HD T enthalpy(const T* V) const {
    T e = energy(V[0], V[4]);
    return e + T(0.5) * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]) + V[4] / V[0];
  }
  M2C_HD void c2p(const T* U, T* V) const {
    V[0] = U[0];
    T inv = T(1) / U[0];
    V[1] = U[1] * inv;
    V[2] = U[2] * inv;
    V[3] = U[3] * inv;
    T e = (U[4] - T(0.5) * V[0] * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3])) * inv;
    V[4] = pressure(V[0], e);
  }
  M2C_HD void p2c(const T* V, T* U) const {
    U[0] = V[0];
    U[1] = V[0] * V[1];
    U[2] = V[0] * V[2];
    U[3] = V[0] * V[3];
    T e = energy(V[0], V[4]);
    U[4] = V[0] * (e + T(0.5) * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]));
  }
};

// Material parameters as set up by VarFcnSG/VarFcnNASG constructors
// (VarFcnSG.h:115-144, VarFcnNASG.h:92-113) from double inputs.
struct MatParams {
  int kind;
  double gam, pc, b, q;
  double rhomin, pmin, rhomax, pmax, failsafe_density;
};

template <typename T>
M2C_HD Eos<T> make_eos(const MatParams& m) {
  Eos<T> e;
  e.kind = m.kind;
  double gam1 = m.gam - 1.0;
  e.gam = T(m.gam);
  e.gam1 = T(gam1);
  e.invgam1 = T(1.0 / gam1);
  e.pstiff = T(m.pc);
  e.gam_ps = T(m.gam * m.pc);
  e.b = T(m.b);
  e.q = T(m.q);
  // Clip bounds: out-of-range doubles (e.g. -DBL_MAX) become -inf in float,
  // which keeps "no clipping" semantics.
  e.rhomin = T(m.rhomin);
  e.pmin = T(m.pmin);
  e.rhomax = T(m.rhomax);
  e.pmax = T(m.pmax);
  return e;
}

// ---------------------------------------------------------------------------
// Slope limiters (Reconstructor.h:95-110).
// ---------------------------------------------------------------------------
template <typename T>
M2C_HD T lim_genminmod(T A, T B, T alpha, T dq0, T dq1) {
  if (dq0 < T(0) && dq1 < T(0)) return smax(alpha * dq0, smax(B / (A + T(1)) * (dq0 + dq1), alpha * dq1));
  if (dq0 > T(0) && dq1 > T(0)) return smin(alpha * dq0, smin(B / (A + T(1)) * (dq0 + dq1), alpha * dq1));
  return T(0);
}

// x^k, correctly rounded, for an integer k >= 1 (the van Albada limiter's
// exponent and the setup of that exponent, Reconstructor.h:107-108,
// Reconstructor.cpp:109). x^2 is the correctly rounded square; a higher
// power is carried as a double-double product (each step an exact fma
// product plus the low part's cross terms, relative error below k 2^-104)
// and rounded once, so it is the correctly rounded value except within
// ~k 2^-104 of a rounding midpoint. The reference takes these powers from
// the C library's pow, which rounds the other way on about 1e-3 of
// arguments (x^2 included); with these the host build, the oracle's
// correctly rounded build and the GPU agree bit for bit.
M2C_HD double cr_pow_int(double x, int k) {
  if (k <= 1) return k == 1 ? x : 1.0;
  if (k == 2) return x * x;
  double h = x, l = 0.0;
  for (int i = 1; i < k; i++) {
    const double p = h * x;
    const double e = fma(h, x, -p) + l * x;  // exact low part of h x, plus l x
    h = p + e;                                // renormalise (|e| << |p|)
    l = e - (h - p);
  }
  return h;
}

// x^k in the compute type: FP64 correctly rounded (cr_pow_int), FP32 by
// repeated multiplication (the mixed path's flux half).
template <typename T>
M2C_HD T ipow(T x, int k) {
  if constexpr (sizeof(T) == 8) {
    return cr_pow_int(x, k);
  } else {
    T r = x;
    for (int i = 1; i < k; i++) r = r * x;
    return r;
  }
}

template <typename T>
M2C_HD T lim_vanalbada(T A, T B, int k, T dq0, T dq1) {
  if (dq0 * dq1 <= T(0)) return T(0);
  if (fabs(dq0 * dq1) < T(1e-16)) return T(0);
  T p0 = ipow(dq0, k), p1 = ipow(dq1, k);
  return B * (dq1 * p0 + dq0 * p1) / (p0 + A * p1);
}

// Generalized minmod with its coefficient C = B/(A+1) precomputed (the
// reference evaluates B/(A+1.0) per call, Reconstructor.h:95-101; the value
// is the same double).
template <typename T>
M2C_HD T lim_genminmod_c(T C, T alpha, T dq0, T dq1) {
  if (dq0 < T(0) && dq1 < T(0)) return smax(alpha * dq0, smax(C * (dq0 + dq1), alpha * dq1));
  if (dq0 > T(0) && dq1 > T(0)) return smin(alpha * dq0, smin(C * (dq0 + dq1), alpha * dq1));
  return T(0);
}

// Slope with limiter; for the generalized minmod B carries C = B/(A+1).
template <typename T>
M2C_HD T limited_slope_c(int limiter, T A, T B, int k, T alpha, T dql, T dqr) {
  if (limiter == LIM_GENMINMOD) return lim_genminmod_c(B, alpha, dql, dqr);
  if (limiter == LIM_VANALBADA) return lim_vanalbada(A, B, k, dql, dqr);
  return T(0.5) * (dql + dqr);
}

template <typename T>
M2C_HD T limited_slope(int limiter, T A, T B, int k, T alpha, T dql, T dqr) {
  if (limiter == LIM_GENMINMOD) return lim_genminmod(A, B, alpha, dql, dqr);
  if (limiter == LIM_VANALBADA) return lim_vanalbada(A, B, k, dql, dqr);
  return T(0.5) * (dql + dqr);
}

// ---------------------------------------------------------------------------
// Characteristic variables for reconstruction (FluxFcnBase.h:309-500): the
// eigenvectors of the flux Jacobian in direction d at the cell state V0.
// ---------------------------------------------------------------------------
template <typename T>
struct CharBasis {
  T e0, c0, dpdrho0, Gamma0, kin0, un0, alpha0, beta0;
  T n[3];
  bool ok;  // c0^2 >= 0 (the reference aborts otherwise)
};

template <typename T>
M2C_HD void char_basis(const Eos<T>& eos, int d, const T* V0, CharBasis<T>& b) {
  b.e0 = eos.energy(V0[0], V0[4]);
  T c2 = eos.c2(V0[0], b.e0);
  b.ok = !(c2 < T(0));
  b.c0 = b.ok ? sqrt(c2) : T(0);
  b.dpdrho0 = eos.dpdrho(V0[0], b.e0);
  b.Gamma0 = eos.big_gamma(V0[0], b.e0);
  b.kin0 = T(0.5) * (V0[1] * V0[1] + V0[2] * V0[2] + V0[3] * V0[3]);
  b.un0 = V0[d + 1];
  b.n[0] = d == 0 ? T(1) : T(0);
  b.n[1] = d == 1 ? T(1) : T(0);
  b.n[2] = d == 2 ? T(1) : T(0);
  b.alpha0 = V0[0] * b.Gamma0 / (V0[4] * b.Gamma0 + V0[0] * b.dpdrho0);
  b.beta0 = (b.e0 - b.kin0 + V0[4] / V0[0]) * b.alpha0;
}

// dW = R0^{-1} x (the conservative-space left eigenvectors)
template <typename T>
M2C_HD void char_rinv(const CharBasis<T>& b, const T* V0, const T* x, T* dW) {
  T R[5][5];
  R[0][0] = T(0.5) * (T(1) - b.beta0 + b.un0 / b.c0);
  for (int i = 0; i < 3; i++) R[0][1 + i] = T(-0.5) * (b.alpha0 * V0[1 + i] + b.n[i] / b.c0);
  R[0][4] = b.alpha0 / T(2);
  for (int i = 0; i < 3; i++) R[1 + i][0] = -V0[1 + i] + (b.beta0 + b.un0) * b.n[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      R[1 + i][1 + j] = (i == j ? T(1) : T(0)) + b.alpha0 * b.n[i] * V0[1 + j] - b.n[i] * b.n[j];
  for (int i = 0; i < 3; i++) R[1 + i][4] = -b.alpha0 * b.n[i];
  R[4][0] = T(0.5) * (T(1) - b.beta0 - b.un0 / b.c0);
  for (int i = 0; i < 3; i++) R[4][1 + i] = T(-0.5) * (b.alpha0 * V0[1 + i] - b.n[i] / b.c0);
  R[4][4] = b.alpha0 / T(2);
  for (int i = 0; i < 5; i++) {
    T acc = T(0);
    for (int j = 0; j < 5; j++) acc += R[i][j] * x[j];
    dW[i] = acc;
  }
}

// R0 dW (the conservative-space right eigenvectors)
template <typename T>
M2C_HD void char_r(const CharBasis<T>& b, const T* V0, const T* dW, T* y) {
  const T H0 = b.e0 + b.kin0 + V0[4] / V0[0];
  T R[5][5];
  R[0][0] = T(1);
  for (int i = 0; i < 3; i++) R[0][1 + i] = b.n[i];
  R[0][4] = T(1);
  for (int i = 0; i < 3; i++) R[1 + i][0] = V0[1 + i] - b.c0 * b.n[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) R[1 + i][1 + j] = (i == j ? T(1) : T(0)) + V0[1 + i] * b.n[j] - b.n[i] * b.n[j];
  for (int i = 0; i < 3; i++) R[1 + i][4] = V0[1 + i] + b.c0 * b.n[i];
  R[4][0] = H0 - b.un0 * b.c0;
  const T param = b.e0 + b.kin0 - b.dpdrho0 / b.Gamma0 - b.un0;
  for (int i = 0; i < 3; i++) R[4][1 + i] = V0[1 + i] + param * b.n[i];
  R[4][4] = H0 + b.un0 * b.c0;
  for (int i = 0; i < 5; i++) {
    T acc = T(0);
    for (int j = 0; j < 5; j++) acc += R[i][j] * dW[j];
    y[i] = acc;
  }
}

// PrimitiveToPrimitiveCharacteristic: dW = R0^{-1} Q0 dV
template <typename T>
M2C_HD void prim_to_char(const CharBasis<T>& b, const T* V0, const T* dV, T* dW) {
  const T Q51 = b.e0 + b.kin0 - b.dpdrho0 / b.Gamma0;
  T t[5];
  t[0] = dV[0];
  t[1] = V0[1] * dV[0] + V0[0] * dV[1];
  t[2] = V0[2] * dV[0] + V0[0] * dV[2];
  t[3] = V0[3] * dV[0] + V0[0] * dV[3];
  t[4] = Q51 * dV[0] + V0[0] * V0[1] * dV[1] + V0[0] * V0[2] * dV[2] + V0[0] * V0[3] * dV[3] + T(1) / b.Gamma0 * dV[4];
  char_rinv(b, V0, t, dW);
}

// PrimitiveCharacteristicToPrimitive: dV = Qbar^{-1} R0 dW
template <typename T>
M2C_HD void char_to_prim(const CharBasis<T>& b, const T* V0, const T* dW, T* dV) {
  T t[5];
  char_r(b, V0, dW, t);
  dV[0] = t[0];
  dV[1] = -V0[1] / V0[0] * t[0] + t[1] / V0[0];
  dV[2] = -V0[2] / V0[0] * t[0] + t[2] / V0[0];
  dV[3] = -V0[3] / V0[0] * t[0] + t[3] / V0[0];
  dV[4] = ((-b.e0 + b.kin0) * b.Gamma0 + b.dpdrho0) * t[0] -
          b.Gamma0 * (V0[1] * t[1] + V0[2] * t[2] + V0[3] * t[3] - t[4]);
}

// ---------------------------------------------------------------------------
// Physical flux in direction d (0 x / F, 1 y / G, 2 z / H).
// ---------------------------------------------------------------------------
template <typename T>
M2C_HD void phys_flux(const Eos<T>& eos, int d, const T* V, T* F) {
  T H = eos.enthalpy(V);
  T vn = vnorm(d, V);
  T rvn = V[0] * vn;
  F[0] = rvn;
  F[1] = d == 0 ? rvn * V[1] + V[4] : rvn * V[1];
  F[2] = d == 1 ? rvn * V[2] + V[4] : rvn * V[2];
  F[3] = d == 2 ? rvn * V[3] + V[4] : rvn * V[3];
  F[4] = rvn * H;
}

template <typename T>
M2C_HD T roe_avg(T w1, T f1, T w2, T f2) { return (w1 * f1 + w2 * f2) / (w1 + w2); }

// Roe-averaged generalized sound speed (Hu, Adams, Iaccarino 2009), shared by
// HLLC (FluxFcnHLLC.h:58-110) and generalized Roe (FluxFcnGenRoe.h:68-118).
template <typename T>
struct RoeHat {
  T rho_hat, sm, sp, em, ep, e_hat, dpdrho_hat, Gamma_hat, c_hat, c_hat2;
};

template <typename T>
M2C_HD void roe_hat(const Eos<T>& eos, int d, const T* Vm, const T* Vp, RoeHat<T>& h) {
  const T eps = T(1e-10);
  h.rho_hat = sqrt(Vm[0] * Vp[0]);
  h.sm = sqrt(Vm[0]);
  h.sp = sqrt(Vp[0]);
  T drho = Vp[0] - Vm[0];
  T dp = Vp[4] - Vm[4];
  T dvel = vnorm(d, Vp) - vnorm(d, Vm);
  T diff = dvel / (h.sm + h.sp);
  T p_over_rho_hat = roe_avg(h.sm, Vm[4] / Vm[0], h.sp, Vp[4] / Vp[0]) + T(0.5) * diff * diff;
  h.em = eos.energy(Vm[0], Vm[4]);
  h.ep = eos.energy(Vp[0], Vp[4]);
  T de = h.ep - h.em;
  h.e_hat = roe_avg(h.sm, h.em, h.sp, h.ep);
  T w_rho = drho * drho / (h.rho_hat * h.rho_hat);
  T w_e = de * de / (h.e_hat * h.e_hat);
  T den = w_rho + w_e + eps;
  T dpdrho_avg = roe_avg(h.sm, eos.dpdrho(Vm[0], h.em), h.sp, eos.dpdrho(Vp[0], h.ep));
  T Gamma_avg = roe_avg(h.sm, eos.big_gamma(Vm[0], h.em), h.sp, eos.big_gamma(Vp[0], h.ep));
  T t1 = (w_e + eps) * dpdrho_avg;
  T t2 = (dp - Gamma_avg * h.rho_hat * de) * drho / (h.rho_hat * h.rho_hat);
  h.dpdrho_hat = (t1 + t2) / den;
  T g1 = (w_rho + eps) * Gamma_avg;
  T g2 = (dp - dpdrho_avg * drho) * de / (h.rho_hat * h.e_hat * h.e_hat);
  h.Gamma_hat = (g1 + g2) / den;
  h.c_hat2 = h.dpdrho_hat + h.Gamma_hat * p_over_rho_hat;
  if (h.c_hat2 <= T(0)) {  // artificial state lost hyperbolicity: c_hat = eps
    h.c_hat = eps;
    h.c_hat2 = h.c_hat * h.c_hat;
  } else {
    h.c_hat = sqrt(h.c_hat2);
  }
}

// HLLC star-region flux F* for one side (FluxFcnHLLC.h:159-195).
template <typename T>
M2C_HD void hllc_fstar(const Eos<T>& eos, int d, const T* V, T S, T Sstar, T* F) {
  T velo = vnorm(d, V);
  T rhostar = V[0] * (S - velo) / (S - Sstar);
  T U[5];
  eos.p2c(V, U);
  T Us[5];
  Us[0] = T(1);
  Us[1] = d == 0 ? Sstar : V[1];
  Us[2] = d == 1 ? Sstar : V[2];
  Us[3] = d == 2 ? Sstar : V[3];
  Us[4] = U[4] / V[0] + (Sstar - velo) * (Sstar + V[4] / (V[0] * (S - velo)));
  for (int i = 0; i < 5; i++) Us[i] = Us[i] * rhostar;
  phys_flux(eos, d, V, F);
  for (int i = 0; i < 5; i++) F[i] = F[i] + S * (Us[i] - U[i]);
}

// Returns an error code (ERR_NONE on success).
template <typename T>
M2C_HD int flux_hllc(const Eos<T>& eos, int d, const T* Vm, const T* Vp, T* F) {
  RoeHat<T> h;
  roe_hat(eos, d, Vm, Vp, h);
  T cm = eos.c2(Vm[0], h.em);
  if (cm < T(0)) return ERR_SOUND;
  cm = sqrt(cm);
  T cp = eos.c2(Vp[0], h.ep);
  if (cp < T(0)) return ERR_SOUND;
  cp = sqrt(cp);
  T vm = vnorm(d, Vm), vp = vnorm(d, Vp);
  T u_hat = roe_avg(h.sm, vm, h.sp, vp);
  T Sm = smin(vm - cm, u_hat - h.c_hat);
  T Sp = smax(vp + cp, u_hat + h.c_hat);
  if (T(0) <= Sm) {
    phys_flux(eos, d, Vm, F);
  } else if (T(0) >= Sp) {
    phys_flux(eos, d, Vp, F);
  } else {
    T Sstar = (Vp[4] - Vm[4] + Vm[0] * vm * (Sm - vm) - Vp[0] * vp * (Sp - vp)) /
              (Vm[0] * (Sm - vm) - Vp[0] * (Sp - vp));
    if (Sstar >= T(0))
      hllc_fstar(eos, d, Vm, Sm, Sstar, F);
    else if (Sstar <= T(0))
      hllc_fstar(eos, d, Vp, Sp, Sstar, F);
    else
      return ERR_HLLC;
  }
  return ERR_NONE;
}

// Generalized Roe flux with Harten's entropy fix (FluxFcnGenRoe.h:64-221).
// The dissipation sum runs over eigenvectors in the outer loop; for every
// flux component the terms are still subtracted in eigenvector order 1..5,
// as the reference's inner loop does.
template <typename T>
M2C_HD int flux_roe(const Eos<T>& eos, int d, const T* Vm, const T* Vp, T delta, T* F) {
  RoeHat<T> h;
  T sm0 = sqrt(Vm[0]), sp0 = sqrt(Vp[0]);
  T vel[3];
  vel[0] = roe_avg(sm0, Vm[1], sp0, Vp[1]);
  vel[1] = roe_avg(sm0, Vm[2], sp0, Vp[2]);
  vel[2] = roe_avg(sm0, Vm[3], sp0, Vp[3]);
  T H = roe_avg(sm0, eos.enthalpy(Vm), sp0, eos.enthalpy(Vp));
  roe_hat(eos, d, Vm, Vp, h);
  const T c = h.c_hat, c2 = h.c_hat2, rho = h.rho_hat;
  const T drho = Vp[0] - Vm[0], dp = Vp[4] - Vm[4];
  const T du = Vp[1] - Vm[1], dv = Vp[2] - Vm[2], dw = Vp[3] - Vm[3];
  const T un = pick3(d, vel[0], vel[1], vel[2]), dn = pick3(d, du, dv, dw);
  const T vel2 = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
  const T r2e = h.e_hat + T(0.5) * vel2 - h.dpdrho_hat / h.Gamma_hat;
  T lam[5];
  lam[0] = un - c;
  lam[1] = lam[2] = lam[3] = un;
  lam[4] = un + c;
  // Harten's entropy fix: tol = delta * max(lam[0], |lam[1..4]|)
  T tol = lam[0];
  for (int i = 1; i < 5; i++)
    if (fabs(lam[i]) > tol) tol = fabs(lam[i]);
  tol = tol * delta;
  for (int i = 0; i < 5; i++)
    if (fabs(lam[i]) < tol) lam[i] = (lam[i] * lam[i] + tol * tol) / (T(2) * tol);
  T fm[5];
  phys_flux(eos, d, Vm, fm);
  phys_flux(eos, d, Vp, F);
  for (int i = 0; i < 5; i++) F[i] = T(0.5) * (fm[i] + F[i]);
  for (int p = 0; p < 5; p++) {
    // eigenvector p and its wave strength (FluxFcnBase.h:155-245, FluxFcnGenRoe.h:125-163)
    T a, r[5];
    if (p == 0 || p == 4) {
      a = p == 0 ? (dp - rho * c * dn) / (T(2) * c2) : (dp + rho * c * dn) / (T(2) * c2);
      T unc = p == 0 ? un - c : un + c;
      r[0] = T(1);
      r[1] = d == 0 ? unc : vel[0];
      r[2] = d == 1 ? unc : vel[1];
      r[3] = d == 2 ? unc : vel[2];
      r[4] = p == 0 ? H - un * c : H + un * c;
    } else {
      int comp = p - 1;  // the middle vectors carry u, v, w in turn
      if (comp == d) {   // entropy wave
        a = -dp / c2 + drho;
        r[0] = T(1);
        r[1] = vel[0]; r[2] = vel[1]; r[3] = vel[2];
        r[4] = r2e;
      } else {           // shear wave
        a = rho * pick3(comp, du, dv, dw);
        r[0] = T(0);
        r[1] = comp == 0 ? T(1) : T(0);
        r[2] = comp == 1 ? T(1) : T(0);
        r[3] = comp == 2 ? T(1) : T(0);
        r[4] = pick3(comp, vel[0], vel[1], vel[2]);
      }
    }
    T coef = T(0.5) * fabs(lam[p]) * a;
    for (int i = 0; i < 5; i++) F[i] = F[i] - coef * r[i];
  }
  return ERR_NONE;
}

// Rusanov / LLF flux; also the material-interface variant with two EOS
// (FluxFcnLLF.h:47-111, 119-185).
template <typename T>
M2C_HD int flux_llf2(const Eos<T>& em, const Eos<T>& ep, int d, const T* Vm, const T* Vp, T* F) {
  T e_m = em.energy(Vm[0], Vm[4]);
  T e_p = ep.energy(Vp[0], Vp[4]);
  T c_m = em.c2(Vm[0], e_m);
  if (c_m < T(0)) return ERR_SOUND;
  c_m = sqrt(c_m);
  T c_p = ep.c2(Vp[0], e_p);
  if (c_p < T(0)) return ERR_SOUND;
  c_p = sqrt(c_p);
  T a = smax(fabs(vnorm(d, Vm)) + c_m, fabs(vnorm(d, Vp)) + c_p);
  T fm[5], fp[5], Um[5], Up[5];
  phys_flux(em, d, Vm, fm);
  phys_flux(ep, d, Vp, fp);
  em.p2c(Vm, Um);
  ep.p2c(Vp, Up);
  for (int i = 0; i < 5; i++) F[i] = T(0.5) * ((fm[i] + fp[i]) - a * (Up[i] - Um[i]));
  return ERR_NONE;
}

template <typename T>
M2C_HD int num_flux(int kind, const Eos<T>& eos, int d, const T* Vm, const T* Vp, T delta, T* F) {
  if (kind == FLUX_HLLC) return flux_hllc(eos, d, Vm, Vp, F);
  if (kind == FLUX_ROE) return flux_roe(eos, d, Vm, Vp, delta, F);
  return flux_llf2(eos, eos, d, Vm, Vp, F);
}

}  // namespace m2c
