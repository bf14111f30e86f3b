// Third-order one-sided finite-difference coefficients of the level-set
// gradient (GradientCalculatorFD3.cpp:300-470): the 4x4 Taylor system
// sum_k c_k d_k^m = delta_{m,1}, m = 0..3, for four stencil offsets d_k,
// solved by Gaussian elimination with partial pivoting. Host and device run
// the same operation sequence (device code is compiled without FMA
// contraction), so coefficients agree bit for bit wherever they are built.
#pragma once
#include "physics.cuh"

namespace m2c {

M2C_HD void taylor4(double d0, double d1, double d2, double d3, double* c) {
  double m[4][5] = {{1.0, 1.0, 1.0, 1.0, 0.0},
                    {d0, d1, d2, d3, 1.0},
                    {d0 * d0, d1 * d1, d2 * d2, d3 * d3, 0.0},
                    {d0 * d0 * d0, d1 * d1 * d1, d2 * d2 * d2, d3 * d3 * d3, 0.0}};
  for (int col = 0; col < 4; col++) {
    int p = col;
    for (int r = col + 1; r < 4; r++)
      if (fabs(m[r][col]) > fabs(m[p][col])) p = r;
    if (p != col)
      for (int q = 0; q <= 4; q++) {
        const double t = m[col][q];
        m[col][q] = m[p][q];
        m[p][q] = t;
      }
    for (int r = col + 1; r < 4; r++) {
      const double f = m[r][col] / m[col][col];
      for (int q = col; q <= 4; q++) m[r][q] -= f * m[col][q];
    }
  }
  for (int i = 3; i >= 0; i--) {
    double s = m[i][4];
    for (int q = i + 1; q < 4; q++) s -= m[i][q] * c[q];
    c[i] = s / m[i][i];
  }
}

M2C_HD double fd4(const double* cf, double p0, double p1, double p2, double p3) {
  return cf[0] * p0 + cf[1] * p1 + cf[2] * p2 + cf[3] * p3;
}

}  // namespace m2c
