// Level-set transport on the GPU (FP64, compiled with -fmad=false).
//
// Residual (LevelSetOperator::ComputeResidualFDM_FullDomain, LevelSetOperator.cpp:1066-1140):
//   R = -( (u>=0 ? a*u : b*u) + (v>=0 ? c*v : d*v) + (w>=0 ? e*w : f*w) )
// with a/b (c/d, e/f) the left/right-biased four-point third-order
// derivatives of GradientCalculatorFD3 (GradientCalculatorFD3.cpp:54-172),
// replaced by first-order one-sided differences where the stencil would
// leave the one-cell ghost layer. The FD3 coefficients come from the same
// 4x4 Taylor system (GradientCalculatorFD3.cpp:455-470), solved here on the
// host by Gaussian elimination with partial pivoting.
//
// The reference's right-biased y coefficients switch to first order on the
// condition i < NY-1 (GradientCalculatorFD3.cpp:413) rather than j < NY-1:
// where i >= NY-1 the y derivative is the first-order difference written
// in coefficient form. That behaviour is reproduced (cr1y).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "levelset.h"

namespace m2c {

// --------------------------------------------------------------------------
// host: geometry and coefficients
// --------------------------------------------------------------------------
static void taylor4(double d0, double d1, double d2, double d3, double* c) {
  // A = [1;d;d^2;d^3] columns, b = (0,1,0,0): Gaussian elimination, partial pivoting
  double m[4][5] = {{1.0, 1.0, 1.0, 1.0, 0.0},
                    {d0, d1, d2, d3, 1.0},
                    {d0 * d0, d1 * d1, d2 * d2, d3 * d3, 0.0},
                    {d0 * d0 * d0, d1 * d1 * d1, d2 * d2 * d2, d3 * d3 * d3, 0.0}};
  for (int col = 0; col < 4; col++) {
    int p = col;
    for (int r = col + 1; r < 4; r++)
      if (std::fabs(m[r][col]) > std::fabs(m[p][col])) p = r;
    if (p != col)
      for (int q = 0; q <= 4; q++) std::swap(m[col][q], m[p][q]);
    for (int r = col + 1; r < 4; r++) {
      double f = m[r][col] / m[col][col];
      for (int q = col; q <= 4; q++) m[r][q] -= f * m[col][q];
    }
  }
  for (int i = 3; i >= 0; i--) {
    double s = m[i][4];
    for (int q = i + 1; q < 4; q++) s -= m[i][q] * c[q];
    c[i] = s / m[i][i];
  }
}

m2cg_status levelset_geom_create(cudaStream_t s, const Grid3& g, const m2cg_levelset& ls, const double* const* xc,
                                 const double* const* dx, LsGeom* out) {
  memset(out, 0, sizeof *out);
  const int nn[3] = {g.nx, g.ny, g.nz};
  // cell-centre coordinates with one ghost per side, as
  // SpaceOperator::PopulateGhostBoundaryCoordinates (SpaceOperator.cpp:218-300):
  // x_{-1} = x_0 - dx_0, x_n = x_{n-1} + dx_{n-1}
  std::vector<double> xg[3], cl[3], cr[3], cr1y;
  for (int a = 0; a < 3; a++) {
    const int n = nn[a];
    xg[a].assign(n + 2, 0.0);
    for (int i = 0; i < n; i++) xg[a][i + 1] = xc[a][i];
    xg[a][0] = xc[a][0] - dx[a][0];
    xg[a][n + 1] = xc[a][n - 1] + dx[a][n - 1];
    double L = 0.0;
    for (int i = 0; i < n; i++) L += dx[a][i];
    const bool per = g.bc[2 * a] == BC_PERIODIC;
    cl[a].assign(4 * n, 0.0);
    cr[a].assign(4 * n, 0.0);
    // coordinate of index i in [-2, n+1]; the reference never uses the
    // second ghost layer (its coordinates are left at 0) unless periodic here
    auto X = [&](int i) {
      if (i >= -1 && i <= n && !(per && (i < 0 || i >= n))) return xg[a][i + 1];
      if (per) return i < 0 ? xc[a][i + n] - L : xc[a][i - n] + L;
      return 0.0;
    };
    for (int i = 0; i < n; i++) {
      double xi = X(i);
      if (i > 0 || per) {
        taylor4(X(i - 2) - xi, X(i - 1) - xi, 0.0, X(i + 1) - xi, &cl[a][4 * i]);
      } else {
        double d = xi - X(i - 1);
        cl[a][4 * i + 1] = -1.0 / d;
        cl[a][4 * i + 2] = 1.0 / d;
      }
      if (i < n - 1 || per) {
        taylor4(X(i - 1) - xi, 0.0, X(i + 1) - xi, X(i + 2) - xi, &cr[a][4 * i]);
      } else {
        double d = X(i + 1) - xi;
        cr[a][4 * i + 1] = -1.0 / d;
        cr[a][4 * i + 2] = 1.0 / d;
      }
    }
  }
  cr1y.assign(4 * nn[1], 0.0);
  for (int j = 0; j < nn[1]; j++) {
    double d = xg[1][j + 2] - xg[1][j + 1];
    cr1y[4 * j + 1] = -1.0 / d;
    cr1y[4 * j + 2] = 1.0 / d;
  }
  size_t total = 0;
  for (int a = 0; a < 3; a++) total += xg[a].size() + cl[a].size() + cr[a].size();
  total += cr1y.size();
  if (cudaMalloc((void**)&out->base, total * 8) != cudaSuccess) return M2CG_ERR_NOMEM;
  double* p = out->base;
  auto put = [&](const std::vector<double>& v) {
    cudaMemcpyAsync(p, v.data(), v.size() * 8, cudaMemcpyHostToDevice, s);
    double* r = p;
    p += v.size();
    return (const double*)r;
  };
  for (int a = 0; a < 3; a++) {
    out->xg[a] = put(xg[a]);
    out->cl[a] = put(cl[a]);
    out->cr[a] = put(cr[a]);
  }
  out->cr1y = put(cr1y);
  for (int q = 0; q < 6; q++) out->bc[q] = ls.bc[q];
  cudaStreamSynchronize(s);
  return M2CG_OK;
}

void levelset_geom_destroy(LsGeom* geo) {
  cudaFree(geo->base);
  geo->base = nullptr;
}

// --------------------------------------------------------------------------
// device: phi with the boundary rule
// --------------------------------------------------------------------------
__device__ __forceinline__ long long loff(const Grid3& g, int i, int j, int k) {
  return (long long)k * g.plane + (long long)j * g.px + i;
}

// phi at (i,j,k) where at most one index is one cell outside (face ghost),
// or any index outside on a periodic axis.
__device__ double phi_at(const Grid3& g, const LsGeom& geo, const double* phi, int i, int j, int k) {
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

__device__ __forceinline__ double fd4(const double* cf, double p0, double p1, double p2, double p3) {
  return cf[0] * p0 + cf[1] * p1 + cf[2] * p2 + cf[3] * p3;
}

// -(u . grad phi) with upwind-biased FD3 at cell (i,j,k)
__device__ double ls_residual(const Grid3& g, const LsGeom& geo, const double* phi, int i, int j, int k, double u,
                              double v, double w) {
  const int n[3] = {g.nx, g.ny, g.nz};
  const double pc = phi[loff(g, i, j, k)];
  double lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    const int c = a == 0 ? i : (a == 1 ? j : k);
    const bool per = g.bc[2 * a] == BC_PERIODIC;
    auto P = [&](int dc) {
      return phi_at(g, geo, phi, i + (a == 0 ? dc : 0), j + (a == 1 ? dc : 0), k + (a == 2 ? dc : 0));
    };
    const double* X = geo.xg[a];  // X[c+1] = coordinate of index c
    // left-biased (a, c, e)
    if (c - 2 >= -1 || per) {
      lo[a] = fd4(geo.cl[a] + 4 * c, P(-2), P(-1), pc, P(1));
    } else {
      lo[a] = (pc - P(-1)) / (X[c + 1] - X[c]);
    }
    // right-biased (b, d, f)
    if (c + 2 <= n[a] || per) {
      const double* cf = geo.cr[a] + 4 * c;
      if (a == 1 && !per && !(i < g.ny - 1)) cf = geo.cr1y + 4 * c;
      hi[a] = fd4(cf, P(-1), pc, P(1), P(2));
    } else {
      hi[a] = (P(1) - pc) / (X[c + 2] - X[c + 1]);
    }
  }
  double r = (u >= 0 ? lo[0] * u : hi[0] * u) + (v >= 0 ? lo[1] * v : hi[1] * v) + (w >= 0 ? lo[2] * w : hi[2] * w);
  return r * -1.0;
}

struct LsStageArgs {
  Grid3 g;
  LsGeom geo;
  const double* Vn[5];
  const double* Us[5];
  int stage;
  const double* clock;
  double a_prev, a_un, bdt_coef;
  const double* in;
  const double* phin;
  double* out;
};

__global__ void k_ls_stage(LsStageArgs a) {
  const Grid3& g = a.g;
  const long long n = (long long)g.nx * g.ny * g.nz;
  const double dt = a.clock[1];
  const double bdt = a.bdt_coef * dt;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx), j = (int)((q / g.nx) % g.ny), k = (int)(q / ((long long)g.nx * g.ny));
    const long long off = loff(g, i, j, k);
    double u, v, w;
    if (a.stage == 1) {
      u = a.Vn[1][off]; v = a.Vn[2][off]; w = a.Vn[3][off];
    } else {  // velocity of C2P(U_s) (VarFcnBase::ConservativeToPrimitive)
      const double inv = 1.0 / a.Us[0][off];
      u = a.Us[1][off] * inv; v = a.Us[2][off] * inv; w = a.Us[3][off] * inv;
    }
    const double R = ls_residual(g, a.geo, a.in, i, j, k, u, v, w);
    double base;
    if (a.stage == 1)
      base = a.phin[off];
    else
      base = a.a_prev * a.in[off] + a.a_un * a.phin[off];
    a.out[off] = base + bdt * R;
  }
}

static int grid1d(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

m2cg_status levelset_stage(cudaStream_t s, const Grid3& g, const SchemeK& sk, const LsGeom& geo, const StageArgs& a,
                           const double* in, const double* phin, double* out) {
  (void)sk;
  LsStageArgs la;
  memset(&la, 0, sizeof la);
  la.g = g;
  la.geo = geo;
  for (int c = 0; c < 5; c++) {
    la.Vn[c] = a.Vn[c];
    la.Us[c] = a.Us[c];
  }
  la.stage = a.stage;
  la.clock = a.clock;
  la.a_prev = a.a_prev;
  la.a_un = a.a_un;
  la.bdt_coef = a.bdt_coef;
  la.in = in;
  la.phin = phin;
  la.out = out;
  k_ls_stage<<<grid1d((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(la);
  return cudaGetLastError() == cudaSuccess ? M2CG_OK : M2CG_ERR_CUDA;
}

// --------------------------------------------------------------------------
// pack / unpack
// --------------------------------------------------------------------------
__global__ void k_ls_unpack(Grid3 g, const double* aos, double* phi) {
  long long n = (long long)g.nx * g.ny * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx), j = (int)((q / g.nx) % g.ny), k = (int)(q / ((long long)g.nx * g.ny));
    phi[loff(g, i, j, k)] = aos[((long long)(k + 1) * (g.ny + 2) + (j + 1)) * (g.nx + 2) + (i + 1)];
  }
}

__global__ void k_ls_pack(Grid3 g, LsGeom geo, const double* phi, double* aos) {
  const int gx = g.nx + 2, gy = g.ny + 2, gz = g.nz + 2;
  long long n = (long long)gx * gy * gz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % gx) - 1, j = (int)((q / gx) % gy) - 1, k = (int)(q / ((long long)gx * gy)) - 1;
    const int nout = (i < 0 || i >= g.nx) + (j < 0 || j >= g.ny) + (k < 0 || k >= g.nz);
    aos[q] = nout <= 1 ? phi_at(g, geo, phi, i, j, k) : 0.0;
  }
}

void levelset_unpack(cudaStream_t s, const Grid3& g, const double* aos, double* phi) {
  k_ls_unpack<<<grid1d((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(g, aos, phi);
}

void levelset_pack(cudaStream_t s, const Grid3& g, const LsGeom& geo, const double* phi, double* aos) {
  k_ls_pack<<<grid1d((long long)(g.nx + 2) * (g.ny + 2) * (g.nz + 2)), 256, 0, s>>>(g, geo, phi, aos);
}

m2cg_status reinit_alloc(long long ncell, double** buf) {
  (void)ncell;
  *buf = nullptr;
  return M2CG_OK;
}

m2cg_status levelset_reinitialize(cudaStream_t s, const Grid3& g, const LsGeom& geo, const m2cg_levelset& ls,
                                  double* phi, double* buf, DevError* err) {
  (void)s; (void)g; (void)geo; (void)ls; (void)phi; (void)buf; (void)err;
  return M2CG_ERR_UNSUPPORTED;
}

}  // namespace m2c
