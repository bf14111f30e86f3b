// Learned warm start for the exact two-material Riemann solve: features of a
// Riemann problem and the layout of a 16 -> 64 -> 64 -> 64 -> 1 tanh MLP that
// proposes log((p* + S) / B): the star pressure shifted by the smaller
// stiffness S = min(pinf_l, pinf_r) (p* + S > 0 for every admissible star
// state, also where p* < 0), relative to the shifted acoustic (linearised)
// estimate B = max(pac + S, 1e-3 (P + S)), so near-acoustic problems map to
// outputs near 0 and problems whose acoustic estimate is negative still get
// a proposal. The shift also measures the proposal's error on the scale of
// the solver's stopping test (a velocity mismatch, dp / (rho c) with
// rho c^2 ~ gamma (p + pinf)). No counterpart in the reference: the
// reference's solver (ExactRiemannSolverBase.cpp:59-342) starts its bracket
// search from acoustic estimates; a proposal from this network replaces
// those two starting points and the solver itself still decides.
#pragma once
#include "physics.cuh"

namespace m2c {

constexpr int MLP_IN = 16;
constexpr int MLP_H = 64;
// parameter blob (FP32 master copy): W1[64][16] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4
constexpr int MLP_OW1 = 0;
constexpr int MLP_OB1 = MLP_OW1 + MLP_H * MLP_IN;
constexpr int MLP_OW2 = MLP_OB1 + MLP_H;
constexpr int MLP_OB2 = MLP_OW2 + MLP_H * MLP_H;
constexpr int MLP_OW3 = MLP_OB2 + MLP_H;
constexpr int MLP_OB3 = MLP_OW3 + MLP_H * MLP_H;
constexpr int MLP_OW4 = MLP_OB3 + MLP_H;
constexpr int MLP_OB4 = MLP_OW4 + MLP_H;
constexpr int MLP_NPARAM = MLP_OB4 + 1;
// normalisation blob: xmean[16] xstd[16] ymean ystd
constexpr int MLP_NNORM = 2 * MLP_IN + 2;

M2C_HD double mlp_asinh(double x) { return log(x + sqrt(x * x + 1.0)); }

// Dimensionless features of the problem (left state VL with material el,
// right state VR with er, unit normal dir); returns false when no proposal
// can be made (non-positive scale, imaginary sound speed). scale[0] receives
// the target's base B and scale[1] the shift S (the proposal is
// B exp(y) - S). Features, with P = max(|pl|, |pr|): log pressures and
// stiffnesses relative to P, the velocity jump in acoustic units, impedance
// and density ratios, the EOS constants, and the acoustic estimate.
M2C_HD bool mlp_features(const Eos<double>& el, const Eos<double>& er, const double* VL, const double* VR,
                         const double* dir, float* x, double* scale) {
  const double rl = VL[0], pl = VL[4], rr = VR[0], pr = VR[4];
  const double ul = VL[1] * dir[0] + VL[2] * dir[1] + VL[3] * dir[2];
  const double ur = VR[1] * dir[0] + VR[2] * dir[1] + VR[3] * dir[2];
  const double P = fabs(pl) > fabs(pr) ? fabs(pl) : fabs(pr);
  if (!(P > 0.0) || !(rl > 0.0) || !(rr > 0.0)) return false;
  const double c2l = el.c2(rl, el.energy(rl, pl)), c2r = er.c2(rr, er.energy(rr, pr));
  if (!(c2l > 0.0) || !(c2r > 0.0)) return false;
  const double cl = sqrt(c2l), cr = sqrt(c2r);
  const double Cl = rl * cl, Cr = rr * cr;
  const double pac = (Cr * pl + Cl * pr + Cl * Cr * (ul - ur)) / (Cl + Cr);
  const double zeta = Cl * Cr / (Cl + Cr);
  const double S = fmin(fabs(el.pstiff), fabs(er.pstiff));
  const double Q = P + S;
  const double B = fmax(pac + S, 1.0e-3 * Q);
  double f[MLP_IN];
  f[0] = mlp_asinh(pl / P * 10.0);
  f[1] = mlp_asinh(pr / P * 10.0);
  f[2] = 0.25 * log(rl * c2l / P);
  f[3] = 0.25 * log(rr * c2r / P);
  f[4] = (ul - ur) / (cl + cr);
  f[5] = mlp_asinh((ul - ur) * zeta / P);
  f[6] = 0.25 * log(Cl / Cr);
  f[7] = 0.25 * log(rl / rr);
  f[8] = (el.gam - 1.0) / 3.0;
  f[9] = (er.gam - 1.0) / 3.0;
  f[10] = 0.25 * log1p(fabs(el.pstiff) / P);
  f[11] = 0.25 * log1p(fabs(er.pstiff) / P);
  f[12] = mlp_asinh(pac / P);
  f[13] = log(B / Q);
  f[14] = 0.25 * log(cl / cr);
  f[15] = 0.25 * log(Q / P);
  for (int i = 0; i < MLP_IN; i++) x[i] = (float)f[i];
  scale[0] = B;
  scale[1] = S;
  return isfinite(B) && B > 0.0;
}

}  // namespace m2c
