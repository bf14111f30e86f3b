// Device helpers on the level set shared by the level-set kernels and the
// interface Riemann pre-pass: phi at a cell or a face ghost with the level
// set's boundary rule, and the Riemann direction at a material interface face
// from the gradient of phi (SpaceOperator::GetNormalForBimaterialRiemann,
// SpaceOperator.cpp:2966-3193).
#pragma once
#include "levelset.h"
#include "physics.cuh"

namespace m2c {

// device: phi with the boundary rule
__device__ __forceinline__ long long loff(const Grid3& g, int i, int j, int k) {
  return (long long)k * g.plane + (long long)j * g.px + i;
}

// phi at (i,j,k) where at most one index is one cell outside (face ghost),
// or any index outside on a periodic axis.
__device__ inline double phi_at(const Grid3& g, const LsGeom& geo, const double* phi, int i, int j, int k) {
  int c[3] = {i, j, k};
  const int n[3] = {g.nx, g.ny, g.nz};
  int gaxis = -1, gside = 0;
  for (int a = 0; a < 3; a++) {
    if (c[a] >= 0 && c[a] < n[a]) continue;
    if (g.bc[2 * a] == BC_PERIODIC) {
      c[a] = c[a] < 0 ? c[a] + n[a] : c[a] - n[a];
      continue;
    }
    gaxis = a;
    gside = c[a] < 0 ? 0 : 1;
  }
  if (gaxis < 0) return phi[loff(g, c[0], c[1], c[2])];
  // face ghost: LevelSetOperator::ApplyBoundaryConditions
  const int a = gaxis, nA = n[a];
  const int bc = geo.bc[2 * a + gside];
  int im[3] = {c[0], c[1], c[2]};
  im[a] = gside == 0 ? 0 : nA - 1;
  const double image = phi[loff(g, im[0], im[1], im[2])];
  if (bc == M2CG_LSBC_LINEAR_EXTRAPOLATION || bc == M2CG_LSBC_NON_NEGATIVE) {
    double val = image;
    const double* X = geo.xg[a];
    if (nA >= 2) {  // LevelSetOperator.cpp:957 (i+2<NX at i=-1) and 967 (i-2>=0 at i=NX)
      int i1 = gside == 0 ? 0 : nA - 1, i2 = gside == 0 ? 1 : nA - 2;
      int p1[3] = {im[0], im[1], im[2]}, p2[3] = {im[0], im[1], im[2]};
      p1[a] = i1;
      p2[a] = i2;
      const double r = X[(gside == 0 ? -1 : nA) + 1], r1 = X[i1 + 1], r2 = X[i2 + 1];
      const double f1 = phi[loff(g, p1[0], p1[1], p1[2])], f2 = phi[loff(g, p2[0], p2[1], p2[2])];
      val = f1 + (f2 - f1) / (r2 - r1) * (r - r1);
    }
    if (bc == M2CG_LSBC_NON_NEGATIVE) {
      const double d2wall = 0.5 * fabs(X[im[a] + 1] - X[(gside == 0 ? -1 : nA) + 1]);
      val = smax(-d2wall, val);
    }
    return val;
  }
  return image;  // ZERO_NEUMANN
}


// SpaceOperator::CentralDifferenceLocal (SpaceOperator.h:218-223)
__device__ __forceinline__ double central_diff_local(double p0, double p1, double p2, double x0, double x1, double x2) {
  const double c0 = -(x2 - x1) / ((x1 - x0) * (x2 - x0));
  const double c1 = 1.0 / (x1 - x0) - 1.0 / (x2 - x1);
  const double c2 = (x1 - x0) / ((x2 - x0) * (x2 - x1));
  return c0 * p0 + c1 * p1 + c2 * p2;
}

// Gradient of phi at the low face (direction d) of interior cell (i, j, k),
// normalised (CalculateGradientAtCellInterface, SpaceOperator.cpp:3052-3193):
// one-sided along d, central across, interpolated to the face.
__device__ inline void face_grad_phi(const Grid3& g, const LsGeom& geo, const double* phi, int i, int j, int k, int d,
                                     double* dir) {
  auto P = [&](int a, int b, int c) { return phi_at(g, geo, phi, a, b, c); };
  auto X = [&](int axis, int c) { return geo.xg[axis][c + 1]; };
  const int c[3] = {i, j, k};
  // the two transverse axes in the reference's order
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  int m[3] = {i, j, k};
  m[d] -= 1;  // the low neighbour
  dir[d] = (P(i, j, k) - P(m[0], m[1], m[2])) / (X(d, c[d]) - X(d, c[d] - 1));
  double tr[2];
  for (int q = 0; q < 2; q++) {
    const int t = q == 0 ? t1 : t2;
    int a0[3] = {m[0], m[1], m[2]}, a1[3] = {m[0], m[1], m[2]}, b0[3] = {i, j, k}, b1[3] = {i, j, k};
    a0[t] -= 1; a1[t] += 1; b0[t] -= 1; b1[t] += 1;
    const double x0 = X(t, c[t] - 1), x1 = X(t, c[t]), x2 = X(t, c[t] + 1);
    const double dv1 = central_diff_local(P(a0[0], a0[1], a0[2]), P(m[0], m[1], m[2]), P(a1[0], a1[1], a1[2]), x0, x1, x2);
    const double dv2 = central_diff_local(P(b0[0], b0[1], b0[2]), P(i, j, k), P(b1[0], b1[1], b1[2]), x0, x1, x2);
    const double w = d == 0 ? g.dx[i] : (d == 1 ? g.dy[j] : g.dz[k]);
    const double xmh = X(d, c[d]) - 0.5 * w;
    const double dxx = X(d, c[d]) - X(d, c[d] - 1);
    const double k1 = (X(d, c[d]) - xmh) / dxx;
    const double k2 = (xmh - X(d, c[d] - 1)) / dxx;
    tr[q] = k1 * dv1 + k2 * dv2;
  }
  dir[t1] = tr[0];
  dir[t2] = tr[1];
  const double nrm = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  if (nrm != 0.0) {
    const double inv = 1.0 / nrm;  // Vec3D::operator/= (Vector3D.h:190-199)
    dir[0] *= inv; dir[1] *= inv; dir[2] *= inv;
  }
}

// Riemann direction at the low face d of cell (i, j, k) (myid: this cell's
// material, nbid: the low neighbour's): mode 0 LEVEL_SET, 1 MESH, 2 AVERAGE.
__device__ inline void riemann_direction(int mode, const Grid3& g, const LsGeom& geo, const double* phi, int i, int j,
                                         int k, int d, int myid, int nbid, double* dir) {
  dir[0] = dir[1] = dir[2] = 0.0;
  if (mode == 1) {
    dir[d] = 1.0;
    return;
  }
  // CalculateGradPhiAtCellInterface, one level set (SpaceOperator.cpp:2988-3046)
  face_grad_phi(g, geo, phi, i, j, k, d, dir);
  if (nbid == 0) { dir[0] *= -1.0; dir[1] *= -1.0; dir[2] *= -1.0; }
  if (sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]) == 0.0) dir[d] = 1.0;
  if (dir[d] < 0.0) dir[d] *= -1.0;
  (void)myid;
  if (mode == 2) {
    dir[d] += 1.0;
    const double inv = 1.0 / sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    dir[0] *= inv; dir[1] *= inv; dir[2] *= inv;
  }
}

}  // namespace m2c
