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

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "fd3.cuh"
#include "levelset.h"
#include "ls_device.cuh"

namespace m2c {

// --------------------------------------------------------------------------
// host: geometry and coefficients
// --------------------------------------------------------------------------
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
  // finite-volume solver: widths with ghosts and the level set's limiter
  // coefficients (Reconstructor::Setup, Reconstructor.cpp:53-121)
  std::vector<double> wg[3], fA[3], fB[3], fK[3];
  for (int a = 0; a < 3; a++) {
    const int n = nn[a];
    const bool per = g.bc[2 * a] == BC_PERIODIC;
    wg[a].assign(n + 2, 0.0);
    for (int i = 0; i < n; i++) wg[a][i + 1] = dx[a][i];
    wg[a][0] = dx[a][0];
    wg[a][n + 1] = dx[a][n - 1];
    fA[a].assign(n, 0.0);
    fB[a].assign(n, 0.0);
    fK[a].assign(n, 0.0);
    for (int i = 0; i < n; i++) {
      const double dm = i > 0 ? dx[a][i - 1] : (per ? dx[a][n - 1] : dx[a][0]);
      const double dp = i < n - 1 ? dx[a][i + 1] : (per ? dx[a][0] : dx[a][n - 1]);
      fA[a][i] = (dm + dx[a][i]) / (dx[a][i] + dp);
      fB[a][i] = 2.0 * dx[a][i] / (dx[a][i] + dp);
      if (ls.solver == M2CG_LS_FINITE_VOLUME && ls.limiter == M2CG_LIM_VANALBADA) {
        int k;
        for (k = 2; k < 1000; k++) {
          const double rhs = 2.0 / (1.0 + m2c::cr_pow_int((k - 1.0) / k, k - 1) / k) * std::min(fA[a][i], 1.0);
          if (fB[a][i] <= rhs) break;
        }
        if (k >= 999) return M2CG_ERR_ARG;
        fK[a][i] = k;
      }
    }
  }
  size_t total = 0;
  for (int a = 0; a < 3; a++)
    total += xg[a].size() + cl[a].size() + cr[a].size() + wg[a].size() + fA[a].size() + fB[a].size() + fK[a].size();
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
  for (int a = 0; a < 3; a++) {
    out->wg[a] = put(wg[a]);
    out->fA[a] = put(fA[a]);
    out->fB[a] = put(fB[a]);
    out->fK[a] = put(fK[a]);
  }
  out->solver = ls.solver;
  out->flux = ls.flux;
  out->rec_linear = ls.rec_type == 1;
  out->limiter = ls.limiter;
  out->delta = ls.delta;
  out->alpha = ls.minmod_coeff;
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
// -(u . grad phi) with upwind-biased FD3 at cell (i,j,k)
__device__ double ls_residual(const Grid3& g, const LsGeom& geo, const double* phi, int i, int j, int k, double u,
                              double v, double w) {
  const int n[3] = {g.nx, g.ny, g.nz};
  const long long off = loff(g, i, j, k);
  const long long stride[3] = {1, g.px, g.plane};
  const double pc = phi[off];
  const double vel[3] = {u, v, w};
  double term[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int c = a == 0 ? i : (a == 1 ? j : k);
    const bool per = g.bc[2 * a] == BC_PERIODIC;
    // neighbours inside the domain are read directly, the rest by the ghost rule
    auto P = [&](int dc) {
      if (c + dc >= 0 && c + dc < n[a]) return phi[off + dc * stride[a]];
      return phi_at(g, geo, phi, i + (a == 0 ? dc : 0), j + (a == 1 ? dc : 0), k + (a == 2 ? dc : 0));
    };
    const double* X = geo.xg[a];  // X[c+1] = coordinate of index c
    // only the upwind-biased derivative is used: left-biased where the
    // velocity is >= 0 (a, c, e), right-biased otherwise (b, d, f)
    double der;
    if (vel[a] >= 0) {
      if (c - 2 >= -1 || per)
        der = fd4(geo.cl[a] + 4 * c, P(-2), P(-1), pc, P(1));
      else
        der = (pc - P(-1)) / (X[c + 1] - X[c]);
    } else {
      if (c + 2 <= n[a] || per) {
        const double* cf = geo.cr[a] + 4 * c;
        if (a == 1 && !per && !(i < g.ny - 1)) cf = geo.cr1y + 4 * c;
        der = fd4(cf, P(-1), pc, P(1), P(2));
      } else {
        der = (P(1) - pc) / (X[c + 2] - X[c + 1]);
      }
    }
    term[a] = der * vel[a];
  }
  double r = term[0] + term[1] + term[2];
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

// Thread (x, y) of CTA (bx, by, bz) owns cells (32 bx + x, 8 by + y, k),
// k = bz, bz + gridDim.z, ...
__global__ void __launch_bounds__(256) k_ls_stage(LsStageArgs a) {
  const Grid3& g = a.g;
  const double dt = a.clock[1];
  const double bdt = a.bdt_coef * dt;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  for (int k = blockIdx.z; k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    double u, v, w;
    if (a.stage == 1) {
      u = a.Vn[1][off]; v = a.Vn[2][off]; w = a.Vn[3][off];
    } else {  // velocity of C2P(U_s) (VarFcnBase::ConservativeToPrimitive)
      const double inv = 1.0 / a.Us[0][off];
      u = a.Us[1][off] * inv; v = a.Us[2][off] * inv; w = a.Us[3][off] * inv;
    }
    double R;
    if (i >= 2 && i < g.nx - 2 && j >= 2 && j < g.ny - 2 && k >= 2 && k < g.nz - 2) {
      // interior: every stencil point is a cell of the domain (the same
      // arithmetic as ls_residual, without its boundary rules)
      const double* ph = a.in + off;
      const long long sy = g.px, sz = g.plane;
      const double pc = ph[0];
      const double tx = u >= 0 ? fd4(a.geo.cl[0] + 4 * i, ph[-2], ph[-1], pc, ph[1]) * u
                               : fd4(a.geo.cr[0] + 4 * i, ph[-1], pc, ph[1], ph[2]) * u;
      // the right-biased y derivative takes its first-order coefficients where
      // i >= ny - 1 (the reference's index test, see ls_residual)
      const double* cry = (g.bc[2] != BC_PERIODIC && !(i < g.ny - 1)) ? a.geo.cr1y : a.geo.cr[1];
      const double ty = v >= 0 ? fd4(a.geo.cl[1] + 4 * j, ph[-2 * sy], ph[-sy], pc, ph[sy]) * v
                               : fd4(cry + 4 * j, ph[-sy], pc, ph[sy], ph[2 * sy]) * v;
      const double tz = w >= 0 ? fd4(a.geo.cl[2] + 4 * k, ph[-2 * sz], ph[-sz], pc, ph[sz]) * w
                               : fd4(a.geo.cr[2] + 4 * k, ph[-sz], pc, ph[sz], ph[2 * sz]) * w;
      R = (tx + ty + tz) * -1.0;
    } else {
      R = ls_residual(g, a.geo, a.in, i, j, k, u, v, w);
    }
    double base;
    if (a.stage == 1)
      base = a.phin[off];
    else
      base = a.a_prev * a.in[off] + a.a_un * a.phin[off];
    a.out[off] = base + bdt * R;
  }
}

// --------------------------------------------------------------------------
// Finite-volume residual (LevelSetOperator::ComputeResidualFVM, 1237-1297):
// MUSCL face values of phi (Reconstructor::Reconstruct, 1 dof) and of the
// normal velocity (Reconstructor::ReconstructIn1D, Reconstructor.cpp:908-1122),
// the level set's flux at every face (ComputeLocalAdvectionFlux, 1516-1550)
// divided by the width of the face's right cell, and phi (u_x + v_y + w_z)
// with the limited velocity slopes (AddSourceTerm, 1552-1570). A cell's sum
// is taken in the order the reference's face loop (1342-1419) reaches it:
// + its low x, y, z faces, then - its high x, y, z faces.
// --------------------------------------------------------------------------

// Velocity component c (1..3) of the stage at cell (i,j,k), interior or one
// cell outside (a face ghost: SpaceOperator::ApplyBoundaryConditions).
__device__ double ls_vel(const LsStageArgs& a, int i, int j, int k, int c) {
  const Grid3& g = a.g;
  int x[3] = {i, j, k};
  const int n[3] = {g.nx, g.ny, g.nz};
  int gaxis = -1, gside = 0;
  for (int d = 0; d < 3; d++) {
    if (x[d] >= 0 && x[d] < n[d]) continue;
    if (g.bc[2 * d] == BC_PERIODIC) {
      x[d] = x[d] < 0 ? x[d] + n[d] : x[d] - n[d];
      continue;
    }
    gaxis = d;
    gside = x[d] < 0 ? 0 : 1;
    x[d] = x[d] < 0 ? 0 : n[d] - 1;
  }
  if (gaxis >= 0) {
    const int bc = g.bc[2 * gaxis + gside];
    if (bc == BC_INLET) return g.inlet[c];
    if (bc == BC_OUTLET) return g.outlet[c];
  }
  const long long off = loff(g, x[0], x[1], x[2]);
  double u;
  if (a.stage == 1) {
    u = a.Vn[c][off];
  } else {
    const double inv = 1.0 / a.Us[0][off];
    u = a.Us[c][off] * inv;
  }
  if (gaxis >= 0) {
    const int bc = g.bc[2 * gaxis + gside];
    if (bc == BC_STICKWALL || c == gaxis + 1) u = -u;
  }
  return u;
}

// Limited slope of a scalar along axis d at axis index c
// (Reconstructor.cpp:964-997 and 580-611 for one dof).
__device__ __forceinline__ double ls_slope(const LsGeom& geo, int d, int c, double qm, double q0, double qp) {
  if (!geo.rec_linear) return 0.0;
  const double dq0 = q0 - qm, dq1 = qp - q0;
  if (geo.limiter == LIM_GENMINMOD) return lim_genminmod(geo.fA[d][c], geo.fB[d][c], geo.alpha, dq0, dq1);
  if (geo.limiter == LIM_VANALBADA) {
    const int kay = (int)round(geo.fK[d][c]);
    return lim_vanalbada(geo.fA[d][c], geo.fB[d][c], kay, dq0, dq1);
  }
  return 0.5 * (dq0 + dq1);
}

__device__ __forceinline__ void step(int d, int* x, int s) { x[d] += s; }

// Face value of phi (vel = false) or of the axis-d velocity (vel = true) of
// cell x on its low (hi = 0) or high (hi = 1) side along d. x may be one
// cell outside along d: the ghost-layer rules of the two reconstructions
// (Reconstructor.cpp:815-875 for phi, 1040-1108 for the velocity, where the
// wall branches write the ghost's other side, so the side a face uses keeps
// its initial zero).
__device__ double ls_face_value(const LsStageArgs& a, int d, const int* x, int hi, bool vel) {
  const Grid3& g = a.g;
  const LsGeom& geo = a.geo;
  const int n = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
  int c[3] = {x[0], x[1], x[2]};
  if (c[d] < 0 || c[d] >= n) {
    if (g.bc[2 * d] == BC_PERIODIC) {
      c[d] = c[d] < 0 ? c[d] + n : c[d] - n;
    } else {
      const int bc = g.bc[2 * d + (c[d] < 0 ? 0 : 1)];
      const bool dirichlet = bc == BC_INLET || bc == BC_OUTLET;
      if (vel) return dirichlet ? ls_vel(a, c[0], c[1], c[2], d + 1) : 0.0;
      if (dirichlet || !geo.rec_linear) return phi_at(g, geo, a.in, c[0], c[1], c[2]);
      // wall: the image's face value on the ghost's own side (vr[ghost] =
      // vl[image] below, vl[ghost] = vr[image] above)
      hi = c[d] < 0 ? 0 : 1;
      c[d] = c[d] < 0 ? 0 : n - 1;
    }
  }
  int m[3] = {c[0], c[1], c[2]}, p[3] = {c[0], c[1], c[2]};
  step(d, m, -1);
  step(d, p, 1);
  double q0, qm, qp;
  if (vel) {
    q0 = ls_vel(a, c[0], c[1], c[2], d + 1);
    qm = ls_vel(a, m[0], m[1], m[2], d + 1);
    qp = ls_vel(a, p[0], p[1], p[2], d + 1);
  } else {
    q0 = a.in[loff(g, c[0], c[1], c[2])];
    qm = phi_at(g, geo, a.in, m[0], m[1], m[2]);
    qp = phi_at(g, geo, a.in, p[0], p[1], p[2]);
  }
  const double sigma = ls_slope(geo, d, c[d], qm, q0, qp);
  return hi ? q0 + 0.5 * sigma : q0 - 0.5 * sigma;
}

// LevelSetOperator::ComputeLocalAdvectionFlux (1516-1550)
__device__ __forceinline__ double ls_local_flux(const LsGeom& geo, double phim, double phip, double um, double up) {
  if (geo.flux == M2CG_LSFLUX_UPWIND) {
    const double vmid = 0.5 * (um + up);
    if (vmid > 0) return phim * um;
    if (vmid < 0) return phip * up;
    return 0.5 * (phim * um + phip * up);
  }
  if (geo.flux == M2CG_LSFLUX_LLF) return 0.5 * (phim * um + phip * up) - 0.5 * smax(fabs(um), fabs(up)) * (phip - phim);
  double lam = fabs(0.5 * (um + up));
  const double tol = smax(fabs(um), fabs(up)) * geo.delta;
  if (lam < tol) lam = (lam * lam + tol * tol) / (2 * tol);
  return 0.5 * (phim * um + phip * up) - 0.5 * lam * (phip - phim);
}

// Flux through the low face (along d) of cell r, divided by r's width.
__device__ double ls_face_flux(const LsStageArgs& a, int d, const int* r) {
  int l[3] = {r[0], r[1], r[2]};
  step(d, l, -1);
  const double phim = ls_face_value(a, d, l, 1, false), phip = ls_face_value(a, d, r, 0, false);
  const double um = ls_face_value(a, d, l, 1, true), up = ls_face_value(a, d, r, 0, true);
  return ls_local_flux(a.geo, phim, phip, um, up) / a.geo.wg[d][r[d] + 1];
}

__global__ void k_ls_fvm_stage(LsStageArgs a) {
  const Grid3& g = a.g;
  const long long n = (long long)g.nx * g.ny * g.nz;
  const double dt = a.clock[1];
  const double bdt = a.bdt_coef * dt;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx), j = (int)((q / g.nx) % g.ny), k = (int)(q / ((long long)g.nx * g.ny));
    const long long off = loff(g, i, j, k);
    const int x[3] = {i, j, k};
    double R = 0.0;
    for (int d = 0; d < 3; d++) R += ls_face_flux(a, d, x);
    for (int d = 0; d < 3; d++) {
      int r[3] = {i, j, k};
      step(d, r, 1);
      R -= ls_face_flux(a, d, r);
    }
    // source term with the limited velocity slopes (slope = sigma / width)
    double div[3];
    for (int d = 0; d < 3; d++) {
      int m[3] = {i, j, k}, p[3] = {i, j, k};
      step(d, m, -1);
      step(d, p, 1);
      const double sigma = ls_slope(a.geo, d, x[d], ls_vel(a, m[0], m[1], m[2], d + 1),
                                    ls_vel(a, i, j, k, d + 1), ls_vel(a, p[0], p[1], p[2], d + 1));
      div[d] = sigma / a.geo.wg[d][x[d] + 1];
    }
    R += a.in[off] * (div[0] + div[1] + div[2]);
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
  if (geo.solver == M2CG_LS_FINITE_VOLUME)
    k_ls_fvm_stage<<<grid1d((long long)g.nx * g.ny * g.nz), 256, 0, s>>>(la);
  else
    k_ls_stage<<<dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz < 65535 ? g.nz : 65535), dim3(32, 8), 0, s>>>(la);
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

// --------------------------------------------------------------------------
// Reinitialisation (LevelSetReinitializer::ReinitializeFullDomain,
// LevelSetReinitializer.cpp:74-171) with every first-layer treatment: FIXED,
// CONSTRAINED1/2 (CR-1/2: the first layer reset once from |grad phi| and a
// curvature-selected correction set, 643-865) and ITERATIVE_CONSTRAINED1/2
// (HCR-1/2: the first layer left free and pulled back after every
// iteration, 1357-1450). The FIXED sequence:
//   tag the first layer (a face neighbour with phi*phi_nb <= 0, 297-428),
//   smoothed sign S = phi / sqrt(phi^2 + min(dx,dy,dz)^2) (594-615),
//   pseudo-time SSP-RK3 of R = -dt S (|grad phi|_Godunov - 1) with the first
//   layer held fixed (953-1033), stopping when the max residual or the max
//   relative change drops below the tolerance; on failure the CFL number is
//   divided by 1.5 and the iteration restarts from the saved phi (154-169).
// --------------------------------------------------------------------------
// first-layer treatments (LevelSetReinitializationData::FirstLayerTreatment)
enum { FL_FIXED = 0, FL_CR1 = 1, FL_CR2 = 2, FL_HCR1 = 3, FL_HCR2 = 4 };

struct ReinitBuf {
  double* phi1;
  double* phi2;
  double* sign;
  double* phibk;
  double* fc;               // [n] first-layer corrections (treatments other than FIXED)
  double* nrm[3];           // [n] unit normals (CR-1/2)
  uint8_t* tag;
  unsigned long long* red;  // [0] max residual bits, [1] max rel. change bits, [2] first-layer count,
                            // [3] converged on the residual (this iteration), [4] attempt finished,
                            // [5] iterations of the attempt, [6] last max rel. change bits
};

static int reinit_arrays(int first_layer) { return first_layer == FL_FIXED ? 4 : 8; }

static ReinitBuf carve(double* base, long long n, int first_layer) {
  ReinitBuf b;
  const int na = reinit_arrays(first_layer);
  b.phi1 = base;
  b.phi2 = base + n;
  b.sign = base + 2 * n;
  b.phibk = base + 3 * n;
  b.fc = na > 4 ? base + 4 * n : nullptr;
  for (int a = 0; a < 3; a++) b.nrm[a] = na > 4 ? base + (5 + a) * n : nullptr;
  b.red = (unsigned long long*)(base + na * n);
  b.tag = (uint8_t*)(base + na * n + 8);
  return b;
}

m2cg_status reinit_alloc(long long ncell, int first_layer, double** buf) {
  size_t bytes = (size_t)(reinit_arrays(first_layer) * ncell + 8) * 8 + (size_t)ncell + 64;
  if (cudaMalloc((void**)buf, bytes) != cudaSuccess) return M2CG_ERR_NOMEM;
  return M2CG_OK;
}

__global__ void k_reinit_prep(Grid3 g, LsGeom geo, const double* phi, ReinitBuf b) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  unsigned long long tagged = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx), j = (int)((q / g.nx) % g.ny), k = (int)(q / ((long long)g.nx * g.ny));
    const long long off = loff(g, i, j, k);
    const double p = phi[off];
    const bool t = p * phi_at(g, geo, phi, i - 1, j, k) <= 0 || p * phi_at(g, geo, phi, i + 1, j, k) <= 0 ||
                   p * phi_at(g, geo, phi, i, j - 1, k) <= 0 || p * phi_at(g, geo, phi, i, j + 1, k) <= 0 ||
                   p * phi_at(g, geo, phi, i, j, k - 1) <= 0 || p * phi_at(g, geo, phi, i, j, k + 1) <= 0;
    b.tag[off] = t ? 1 : 0;
    tagged += t;
    const double f = smin(g.dx[i], smin(g.dy[j], g.dz[k]));  // eps = 1
    b.sign[off] = p / sqrt(p * p + f * f);
    b.phibk[off] = p;
  }
  if (tagged) atomicAdd(&b.red[2], tagged);
}

// pseudo-time residual at an untagged interior cell (LevelSetReinitializer.cpp:985-1012)
__device__ __forceinline__ double reinit_local(const Grid3& g, const LsGeom& geo, const double* phi, int i, int j,
                                               int k, double& local_res) {
  const long long off = loff(g, i, j, k);
  const double p = phi[off];
  const double* X = geo.xg[0];
  const double* Y = geo.xg[1];
  const double* Z = geo.xg[2];
  // neighbours inside the domain are read directly, the rest by the ghost rule
  const double pxm = i > 0 ? phi[off - 1] : phi_at(g, geo, phi, i - 1, j, k);
  const double pxp = i < g.nx - 1 ? phi[off + 1] : phi_at(g, geo, phi, i + 1, j, k);
  const double pym = j > 0 ? phi[off - g.px] : phi_at(g, geo, phi, i, j - 1, k);
  const double pyp = j < g.ny - 1 ? phi[off + g.px] : phi_at(g, geo, phi, i, j + 1, k);
  const double pzm = k > 0 ? phi[off - g.plane] : phi_at(g, geo, phi, i, j, k - 1);
  const double pzp = k < g.nz - 1 ? phi[off + g.plane] : phi_at(g, geo, phi, i, j, k + 1);
  const double a = (p - pxm) / (X[i + 1] - X[i]);
  const double b = (pxp - p) / (X[i + 2] - X[i + 1]);
  const double c = (p - pym) / (Y[j + 1] - Y[j]);
  const double d = (pyp - p) / (Y[j + 2] - Y[j + 1]);
  const double e = (p - pzm) / (Z[k + 1] - Z[k]);
  const double f = (pzp - p) / (Z[k + 2] - Z[k + 1]);
  const double ap = smax(a, 0.0), am = smin(a, 0.0);
  const double bp = smax(b, 0.0), bm = smin(b, 0.0);
  const double cp = smax(c, 0.0), cm = smin(c, 0.0);
  const double dp = smax(d, 0.0), dm = smin(d, 0.0);
  const double ep = smax(e, 0.0), em = smin(e, 0.0);
  const double fp = smax(f, 0.0), fm = smin(f, 0.0);
  if (p >= 0)
    local_res = sqrt(smax(ap * ap, bm * bm) + smax(cp * cp, dm * dm) + smax(ep * ep, fm * fm)) - 1.0;
  else
    local_res = sqrt(smax(am * am, bp * bp) + smax(cm * cm, dp * dp) + smax(em * em, fp * fp)) - 1.0;
  return local_res;
}

// One RK3 stage of the pseudo-time iteration:
//   stage 1: out = in + R(in)                     (in = phi, out = phi1)
//   stage 2: out = 0.25*in + 0.75*phi + 0.25*R(in)  (in = phi1, out = phi2)
//   stage 3: phi = 1/3*phi + 2/3*in + 2/3*R(in)     (in = phi2, out = phi)
// Thread (x, y) of CTA (bx, by, bz) owns cell (32 bx + x, 8 by + y, bz): no
// index division, rows of 32 consecutive cells per warp. Six CTAs per SM (40
// registers, a few spills) rather than four (64): the stage waits on loads,
// and the extra resident warps made it about 13 % faster at 384^3.
__global__ void __launch_bounds__(256, 6) k_reinit_stage(Grid3 g, LsGeom geo, ReinitBuf b, int stage, double cfl,
                                                      double tol, const double* in, double* phi, double* out,
                                                      int fix_first) {
  if (b.red[4] || (stage > 1 && b.red[3])) return;  // attempt finished, or converged on the residual in stage 1
  double maxres = 0.0, maxrel = 0.0;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    double R = 0.0;
    const bool tagged = b.tag[off] != 0;
    if (!tagged || !fix_first) {  // the first layer is held fixed except under HCR-1/2 (967-985)
      const double dx = smin(g.dx[i], smin(g.dy[j], g.dz[k]));
      const double dt = cfl * dx;
      double lr;
      reinit_local(g, geo, in, i, j, k, lr);
      if (fabs(lr) <= 1.0)
        R = -dt * b.sign[off] * lr;
      else
        R = -dt * b.sign[off] * lr / fabs(lr);
      if (!tagged) maxres = smax(maxres, fabs(lr));  // the max residual leaves out the first layer
    }
    if (stage == 1) {
      out[off] = in[off] + R;
    } else if (stage == 2) {
      double t = 0.25 * in[off] + 0.75 * phi[off];
      out[off] = t + 0.25 * R;
    } else {
      const double old = phi[off];
      double t = 1.0 / 3.0 * old + 2.0 / 3.0 * in[off];
      const double nw = t + 2.0 / 3.0 * R;
      phi[off] = nw;
      if (tagged && !fix_first) {
        out[off] = old;  // HCR: the first layer's change is measured after its correction
      } else {
        double le = fabs(nw - old);
        if (nw != 0) le /= fabs(nw);
        maxrel = smax(maxrel, le);
      }
    }
  }
  // maxima over the CTA (warp shuffles, then its 8 warps), one atomic per CTA:
  // per-warp atomics on one address serialised at L2 and bounded the kernel
  for (int o = 16; o > 0; o >>= 1) {
    maxres = smax(maxres, __shfl_xor_sync(0xffffffffu, maxres, o));
    maxrel = smax(maxrel, __shfl_xor_sync(0xffffffffu, maxrel, o));
  }
  __shared__ double wres[8], wrel[8];
  if (threadIdx.x == 0) {
    wres[threadIdx.y] = maxres;
    wrel[threadIdx.y] = maxrel;
  }
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int w = 1; w < 8; w++) {
      maxres = smax(maxres, wres[w]);
      maxrel = smax(maxrel, wrel[w]);
    }
    if (stage == 1 && maxres > 0) atomicMax(&b.red[0], (unsigned long long)__double_as_longlong(maxres));
    if (stage == 3 && maxrel > 0) atomicMax(&b.red[1], (unsigned long long)__double_as_longlong(maxrel));
  }
  (void)tol;
}

__global__ void k_reinit_check(ReinitBuf b, double tol) {
  if (b.red[4]) return;
  const double r = __longlong_as_double((long long)b.red[0]);
  b.red[3] = (r < tol) ? 1ull : 0ull;
}

// Start of an attempt: nothing to do without a first layer.
__global__ void k_reinit_begin(ReinitBuf b) {
  b.red[4] = b.red[2] == 0 ? 1ull : 0ull;
  b.red[5] = 0;
  b.red[0] = b.red[1] = b.red[3] = 0;
}

// End of a pseudo-time iteration (LevelSetReinitializer.cpp:~220-260): count
// it, stop the attempt once the residual (checked before the update) or the
// largest relative change of phi is below the tolerance, and clear the
// reductions for the next iteration.
__global__ void k_reinit_end(ReinitBuf b, double tol) {
  if (b.red[4]) return;
  b.red[5] += 1;
  if (b.red[3]) {
    b.red[4] = 1;
  } else {
    b.red[6] = b.red[1];
    if (__longlong_as_double((long long)b.red[1]) < tol) b.red[4] = 1;
  }
  b.red[0] = b.red[1] = b.red[3] = 0;
}

// ---- first-layer treatments (LevelSetReinitializer.cpp:297-428, 643-952, 1129-1241, 1357-1450) ----

// LevelSetReinitializer::CentralDifferenceLocal (LevelSetReinitializer.h:123-128)
__device__ __forceinline__ double central_local(double p0, double p1, double p2, double x0, double x1, double x2) {
  const double c0 = -(x2 - x1) / ((x1 - x0) * (x2 - x0));
  const double c1 = 1.0 / (x1 - x0) - 1.0 / (x2 - x1);
  const double c2 = (x1 - x0) / ((x2 - x0) * (x2 - x1));
  return c0 * p0 + c1 * p1 + c2 * p2;
}

// Tag of node c (interior: the tag array; face ghost: the reference tags its
// ghost layer with the same test, TagFirstLayerNodes 309-372, where the
// unpopulated edge ghosts it reaches read as zero).
__device__ double fl_tag(const Grid3& g, const LsGeom& geo, const double* phi0, const ReinitBuf& b, int i, int j,
                         int k) {
  const int c[3] = {i, j, k}, n[3] = {g.nx, g.ny, g.nz};
  int out = 0;
  for (int a = 0; a < 3; a++) out += (c[a] < 0 || c[a] >= n[a]) && g.bc[2 * a] != BC_PERIODIC;
  if (out == 0) return b.tag[loff(g, (i + g.nx) % g.nx, (j + g.ny) % g.ny, (k + g.nz) % g.nz)];
  if (out > 1) return 0.0;
  const double p = phi_at(g, geo, phi0, i, j, k);
  for (int q = 0; q < 6; q++) {
    int d[3] = {i, j, k};
    d[q >> 1] += (q & 1) ? 1 : -1;
    int dout = 0, beyond = 0;
    for (int a = 0; a < 3; a++) {
      const bool o = (d[a] < 0 || d[a] >= n[a]) && g.bc[2 * a] != BC_PERIODIC;
      dout += o;
      beyond += d[a] < -1 || d[a] > n[a];
    }
    if (beyond) continue;                      // outside the ghosted range
    const double pn = dout > 1 ? 0.0 : phi_at(g, geo, phi0, d[0], d[1], d[2]);
    if (p * pn <= 0) return 1.0;
  }
  return 0.0;
}

// DifferentiateInFirstLayer (899-951): one-sided, central or zero derivative
// at a first-layer node from the tagged neighbours.
__device__ double fl_diff(double x0, double x1, double x2, double tag0, double tag2, double phi0, double phi1,
                          double phi2, double phi00, double phi3, double eps) {
  bool u0 = tag0 != 0, u2 = tag2 != 0;
  if (!u0 && !u2) return 0.0;
  const double dphi0 = phi1 - phi0, dphi1 = phi2 - phi1;
  const bool condB = dphi0 * dphi1 < 0 || phi0 * phi00 < 0 || phi2 * phi3 < 0;
  if (condB) {
    if (u0 && (phi0 * phi2 < 0) && fabs(dphi0 + eps) < fabs(dphi1)) u0 = false;
    if (u2 && (phi0 * phi2 < 0) && fabs(dphi1 + eps) < fabs(dphi0)) u2 = false;
  }
  if (!u0 && !u2) return 0.0;
  if (u0) return u2 ? central_local(phi0, phi1, phi2, x0, x1, x2) : (phi1 - phi0) / (x1 - x0);
  return (phi2 - phi1) / (x2 - x1);
}

// CR-1/2 step 1 (ReinitializeFirstLayerNodes 660-706): phi = phig / |grad phig|
// at every first-layer node, its unit normal kept. phig (b.phi2) is the level
// set at the start of the reinitialisation.
__global__ void k_fl_rescale(Grid3 g, LsGeom geo, ReinitBuf b, double* phi) {
  const double* pg = b.phi2;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    if (!b.tag[off]) continue;
    const double* X = geo.xg[0];
    const double* Y = geo.xg[1];
    const double* Z = geo.xg[2];
    auto P = [&](int a, int bb, int c) { return phi_at(g, geo, pg, a, bb, c); };
    auto Tg = [&](int a, int bb, int c) { return fl_tag(g, geo, pg, b, a, bb, c); };
    double gr[3];
    gr[0] = fl_diff(X[i], X[i + 1], X[i + 2], Tg(i - 1, j, k), Tg(i + 1, j, k), P(i - 1, j, k), pg[off],
                    P(i + 1, j, k), i - 2 >= -1 ? P(i - 2, j, k) : P(i - 1, j, k),
                    i + 2 <= g.nx ? P(i + 2, j, k) : P(i + 1, j, k), 1.0e-3 * g.dx[i]);
    // (the reference reads j+2 in both branches of its y test; beyond the
    // ghost layer that is the ghost here)
    gr[1] = fl_diff(Y[j], Y[j + 1], Y[j + 2], Tg(i, j - 1, k), Tg(i, j + 1, k), P(i, j - 1, k), pg[off],
                    P(i, j + 1, k), j - 2 >= -1 ? P(i, j - 2, k) : P(i, j - 1, k),
                    P(i, j + 2 <= g.ny ? j + 2 : g.ny, k), 1.0e-3 * g.dy[j]);
    gr[2] = fl_diff(Z[k], Z[k + 1], Z[k + 2], Tg(i, j, k - 1), Tg(i, j, k + 1), P(i, j, k - 1), pg[off],
                    P(i, j, k + 1), k - 2 >= -1 ? P(i, j, k - 2) : P(i, j, k - 1),
                    k + 2 <= g.nz ? P(i, j, k + 2) : P(i, j, k + 1), 1.0e-3 * g.dz[k]);
    const double nrm = sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
    for (int a = 0; a < 3; a++) b.nrm[a][off] = gr[a] / nrm;
    phi[off] = nrm == 0 ? pg[off] : pg[off] / nrm;
  }
}

// CR-1/2: unit normal of phi beyond the first layer
// (ComputeNormalDirectionBeyondFirstLayer 1209-1230); the domain's ghost
// layer still holds the values of the level set before the rescaling.
__global__ void k_fl_normal(Grid3 g, LsGeom geo, ReinitBuf b, const double* phi) {
  const double* pg = b.phi2;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    if (b.tag[off]) continue;
    auto P = [&](int a, int bb, int c) {
      const bool in = a >= 0 && a < g.nx && bb >= 0 && bb < g.ny && c >= 0 && c < g.nz;
      return in ? phi[loff(g, a, bb, c)] : phi_at(g, geo, pg, a, bb, c);
    };
    const double* X = geo.xg[0];
    const double* Y = geo.xg[1];
    const double* Z = geo.xg[2];
    double v[3];
    v[0] = central_local(P(i - 1, j, k), phi[off], P(i + 1, j, k), X[i], X[i + 1], X[i + 2]);
    v[1] = central_local(P(i, j - 1, k), phi[off], P(i, j + 1, k), Y[j], Y[j + 1], Y[j + 2]);
    v[2] = central_local(P(i, j, k - 1), phi[off], P(i, j, k + 1), Z[k], Z[k + 1], Z[k + 2]);
    const double m = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (m != 0.0) {
      const double inv = 1.0 / m;  // Vec3D::operator/=
      for (int a = 0; a < 3; a++) v[a] *= inv;
    }
    for (int a = 0; a < 3; a++) b.nrm[a][off] = v[a];
  }
}

// The opposite-side neighbours S of a first-layer node (TagFirstLayerNodes
// 376-414, from the level set at the start: phig * phig_nb < 0).
__device__ __forceinline__ int fl_set(const Grid3& g, const LsGeom& geo, const double* pg, int i, int j, int k,
                                      double* nb) {
  const double p = pg[loff(g, i, j, k)];
  int s = 0;
  for (int q = 0; q < 6; q++) {
    int d[3] = {i, j, k};
    d[q >> 1] += (q & 1) ? 1 : -1;
    nb[q] = phi_at(g, geo, pg, d[0], d[1], d[2]);
    if (p * nb[q] < 0) s |= 1 << q;
  }
  return s;
}

// CR-1/2 steps 2-3 (721-841): curvature of the normal field selects the
// correction set; its nodes get the averaged ratio of the rescaled to the
// original level set of their opposite-side neighbours. Writes the new value
// (or DBL_MAX: unchanged) into fc; k_fl_apply copies it.
__global__ void k_fl_correct(Grid3 g, LsGeom geo, ReinitBuf b, const double* phi, int mode) {
  const double* pg = b.phi2;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    if (!b.tag[off]) continue;
    const double* X = geo.xg[0];
    const double* Y = geo.xg[1];
    const double* Z = geo.xg[2];
    const int c[3] = {i, j, k}, n[3] = {g.nx, g.ny, g.nz};
    const double* xs[3] = {X, Y, Z};
    double curv = 0.0;
    for (int a = 0; a < 3; a++) {
      int lo[3] = {i, j, k}, hi[3] = {i, j, k};
      lo[a]--; hi[a]++;
      const double* N = b.nrm[a];
      const double* x = xs[a];
      const bool hl = c[a] - 1 >= 0, hh = c[a] + 1 < n[a];
      double ca;
      if (hl && hh)
        ca = central_local(N[loff(g, lo[0], lo[1], lo[2])], N[off], N[loff(g, hi[0], hi[1], hi[2])], x[c[a]],
                           x[c[a] + 1], x[c[a] + 2]);
      else if (hl)
        ca = (N[off] - N[loff(g, lo[0], lo[1], lo[2])]) / (x[c[a] + 1] - x[c[a]]);
      else if (hh)
        ca = (N[loff(g, hi[0], hi[1], hi[2])] - N[off]) / (x[c[a] + 2] - x[c[a] + 1]);
      else
        ca = 0.0;
      curv = a == 0 ? ca : curv + ca;
    }
    const double p0 = pg[off];
    if (!(curv * p0 < 0 || (curv == 0.0 && p0 < 0))) {
      b.fc[off] = DBL_MAX;
      continue;
    }
    double nbg[6];
    const int sset = fl_set(g, geo, pg, i, j, k, nbg);
    auto Pc = [&](int q) {  // the rescaled level set at neighbour q (ghosts: not rescaled)
      int d[3] = {i, j, k};
      d[q >> 1] += (q & 1) ? 1 : -1;
      const bool in = d[0] >= 0 && d[0] < g.nx && d[1] >= 0 && d[1] < g.ny && d[2] >= 0 && d[2] < g.nz;
      return in ? phi[loff(g, d[0], d[1], d[2])] : phi_at(g, geo, pg, d[0], d[1], d[2]);
    };
    double f = 0.0;
    if (mode == FL_CR1) {
      double sum = 0.0;
      int ns = 0;
      for (int q = 0; q < 6; q++)
        if (sset & (1 << q)) { sum += Pc(q) / nbg[q]; ns++; }
      f = ns != 0 ? p0 * sum / (double)ns : 0.0;
    } else {
      double s1 = 0.0, s2 = 0.0;
      for (int q = 0; q < 6; q++)
        if (sset & (1 << q)) { s1 += Pc(q); s2 += nbg[q]; }
      f = s2 != 0 ? p0 * s1 / s2 : 0.0;
    }
    b.fc[off] = f;
  }
}

__global__ void k_fl_apply(Grid3 g, ReinitBuf b, double* phi) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    if (b.tag[off] && b.fc[off] != DBL_MAX) phi[off] = b.fc[off];
  }
}

// HCR-1/2 (ApplyCorrectionToFirstLayerNodes 1357-1450), after every
// iteration: a first-layer node all of whose opposite-side neighbours are
// still on the other side is pulled towards the value the original ratios
// give: F = (sum r_a phi_a / |S| - phi) (HCR-1) or (r0 sum phi_a - phi)
// (HCR-2), over max(dx,dy,dz); then phi += dt beta F (beta 1/2), with the
// relative change of these nodes joining the iteration's maximum.
__global__ void k_hcr_force(Grid3 g, LsGeom geo, ReinitBuf b, const double* phi, int mode) {
  if (b.red[4] || b.red[3]) return;
  const double* pg = b.phibk;  // the level set at the start (HCR has no rescaling step)
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    if (!b.tag[off]) continue;
    double nbg[6];
    const int sset = fl_set(g, geo, pg, i, j, k, nbg);
    const double p = phi[off], p0g = pg[off];
    double cur[6];
    bool in_c = true;
    int ns = 0;
    double sumg = 0.0;
    for (int q = 0; q < 6; q++) {
      int d[3] = {i, j, k};
      d[q >> 1] += (q & 1) ? 1 : -1;
      cur[q] = phi_at(g, geo, phi, d[0], d[1], d[2]);
      if (sset & (1 << q)) {
        ns++;
        sumg += nbg[q];
        if (p * cur[q] >= 0) in_c = false;
      }
    }
    double f = 0.0;
    if (in_c) {
      if (mode == FL_HCR1) {
        double sum = 0.0;
        for (int q = 0; q < 6; q++)
          if (sset & (1 << q)) sum += (p0g / nbg[q]) * cur[q];
        f = ns != 0 ? sum / (double)ns - p : 0.0 - p;
      } else {
        const double r0 = sumg != 0 ? p0g / sumg : 0.0;
        double sum = 0.0;
        for (int q = 0; q < 6; q++)
          if (sset & (1 << q)) sum += cur[q];
        f = r0 * sum - p;
      }
      f /= smax(g.dx[i], smax(g.dy[j], g.dz[k]));
    }
    b.fc[off] = f;
  }
}

__global__ void __launch_bounds__(256) k_hcr_apply(Grid3 g, ReinitBuf b, double* phi, double cfl) {
  if (b.red[4] || b.red[3]) return;
  double maxrel = 0.0;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  for (int k = blockIdx.z; i < g.nx && j < g.ny && k < g.nz; k += gridDim.z) {
    const long long off = loff(g, i, j, k);
    if (!b.tag[off]) continue;
    const double dt = cfl * smin(g.dx[i], smin(g.dy[j], g.dz[k]));
    const double nw = phi[off] + dt * 0.5 * b.fc[off];
    phi[off] = nw;
    const double old = b.phi1[off];  // the value at the start of the iteration (kept by stage 3)
    double le = fabs(nw - old);
    if (nw != 0) le /= fabs(nw);
    maxrel = smax(maxrel, le);
  }
  for (int o = 16; o > 0; o >>= 1) maxrel = smax(maxrel, __shfl_xor_sync(0xffffffffu, maxrel, o));
  __shared__ double wrel[8];
  if (threadIdx.x == 0) wrel[threadIdx.y] = maxrel;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int w = 1; w < 8; w++) maxrel = smax(maxrel, wrel[w]);
    if (maxrel > 0) atomicMax(&b.red[1], (unsigned long long)__double_as_longlong(maxrel));
  }
}

static double bits_to_double(unsigned long long u) {
  double d;
  memcpy(&d, &u, 8);
  return d;
}

m2cg_status levelset_reinitialize(cudaStream_t s, const Grid3& g, const LsGeom& geo, const m2cg_levelset& ls,
                                  double* phi, double* buf, DevError* err, double* cfl_state, int* iterations) {
  (void)err;
  const long long n = g.plane * g.nz;
  const int fl = ls.reinit_first_layer;
  ReinitBuf b = carve(buf, n, fl);
  const long long ni = (long long)g.nx * g.ny * g.nz;
  const int grid = grid1d(ni);
  // each CTA walks a column of planes (k = bz, bz + 64, ...)
  const dim3 grid3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz < 64 ? g.nz : 64), block3(32, 8);
  cudaMemsetAsync(b.red, 0, 8 * sizeof(unsigned long long), s);
  k_reinit_prep<<<grid, 256, 0, s>>>(g, geo, phi, b);
  if (fl == FL_CR1 || fl == FL_CR2) {
    // ReinitializeFullDomain step 2 (86-92): rescale and correct the first
    // layer once (phig = the level set at the start, kept in phi2), then the
    // retry backup is the corrected level set (96)
    cudaMemcpyAsync(b.phi2, phi, n * 8, cudaMemcpyDeviceToDevice, s);
    k_fl_rescale<<<grid3, block3, 0, s>>>(g, geo, b, phi);
    k_fl_normal<<<grid3, block3, 0, s>>>(g, geo, b, phi);
    k_fl_correct<<<grid3, block3, 0, s>>>(g, geo, b, phi, fl);
    k_fl_apply<<<grid3, block3, 0, s>>>(g, b, phi);
    cudaMemcpyAsync(b.phibk, phi, n * 8, cudaMemcpyDeviceToDevice, s);
  }
  const int fix_first = fl == FL_HCR1 || fl == FL_HCR2 ? 0 : 1;
  const double tol = ls.reinit_tol;
  const int maxIts = ls.reinit_maxits;
  // Each attempt queues all its iterations at once; the iterations after
  // convergence find the attempt finished on the device and return at once,
  // so one read-back per attempt (not per iteration) decides on a retry.
  for (;;) {
    const double cfl = *cfl_state;
    k_reinit_begin<<<1, 1, 0, s>>>(b);
    for (int iter = 0; iter < maxIts; iter++) {
      k_reinit_stage<<<grid3, block3, 0, s>>>(g, geo, b, 1, cfl, tol, phi, phi, b.phi1, fix_first);
      k_reinit_check<<<1, 1, 0, s>>>(b, tol);
      k_reinit_stage<<<grid3, block3, 0, s>>>(g, geo, b, 2, cfl, tol, b.phi1, phi, b.phi2, fix_first);
      k_reinit_stage<<<grid3, block3, 0, s>>>(g, geo, b, 3, cfl, tol, b.phi2, phi, b.phi1, fix_first);
      if (!fix_first) {  // HCR-1/2 after every iteration (142, 1357-1450)
        k_hcr_force<<<grid3, block3, 0, s>>>(g, geo, b, phi, fl);
        k_hcr_apply<<<grid3, block3, 0, s>>>(g, b, phi, cfl);
      }
      k_reinit_end<<<1, 1, 0, s>>>(b, tol);
    }
    unsigned long long hred[8];
    cudaMemcpyAsync(hred, b.red, sizeof hred, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return M2CG_ERR_CUDA;
    if (iterations) *iterations += (int)hred[5];
    if (hred[4]) return M2CG_OK;  // converged (or no interface)
    const double dphi_max = bits_to_double(hred[6]);
    if (dphi_max < 0.02) return M2CG_OK;
    if (cfl < 0.02) return M2CG_ERR_REINIT;
    *cfl_state = cfl / 1.5;
    cudaMemcpyAsync(phi, b.phibk, n * 8, cudaMemcpyDeviceToDevice, s);
  }
}

}  // namespace m2c
