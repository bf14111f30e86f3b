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

// --------------------------------------------------------------------------
// Reinitialisation (LevelSetReinitializer::ReinitializeFullDomain,
// LevelSetReinitializer.cpp:74-171) with the FIXED first-layer treatment:
//   tag the first layer (a face neighbour with phi*phi_nb <= 0, 297-428),
//   smoothed sign S = phi / sqrt(phi^2 + min(dx,dy,dz)^2) (594-615),
//   pseudo-time SSP-RK3 of R = -dt S (|grad phi|_Godunov - 1) with the first
//   layer held fixed (953-1033), stopping when the max residual or the max
//   relative change drops below the tolerance; on failure the CFL number is
//   divided by 1.5 and the iteration restarts from the saved phi (154-169).
// --------------------------------------------------------------------------
struct ReinitBuf {
  double* phi1;
  double* phi2;
  double* sign;
  double* phibk;
  uint8_t* tag;
  unsigned long long* red;  // [0] max residual bits, [1] max rel. change bits, [2] first-layer count, [3] done flag
};

static ReinitBuf carve(double* base, long long n) {
  ReinitBuf b;
  b.phi1 = base;
  b.phi2 = base + n;
  b.sign = base + 2 * n;
  b.phibk = base + 3 * n;
  b.red = (unsigned long long*)(base + 4 * n);
  b.tag = (uint8_t*)(base + 4 * n + 8);
  return b;
}

m2cg_status reinit_alloc(long long ncell, double** buf) {
  size_t bytes = (size_t)(4 * ncell + 8) * 8 + (size_t)ncell + 64;
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
  const double p = phi[loff(g, i, j, k)];
  const double* X = geo.xg[0];
  const double* Y = geo.xg[1];
  const double* Z = geo.xg[2];
  const double a = (p - phi_at(g, geo, phi, i - 1, j, k)) / (X[i + 1] - X[i]);
  const double b = (phi_at(g, geo, phi, i + 1, j, k) - p) / (X[i + 2] - X[i + 1]);
  const double c = (p - phi_at(g, geo, phi, i, j - 1, k)) / (Y[j + 1] - Y[j]);
  const double d = (phi_at(g, geo, phi, i, j + 1, k) - p) / (Y[j + 2] - Y[j + 1]);
  const double e = (p - phi_at(g, geo, phi, i, j, k - 1)) / (Z[k + 1] - Z[k]);
  const double f = (phi_at(g, geo, phi, i, j, k + 1) - p) / (Z[k + 2] - Z[k + 1]);
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
__global__ void k_reinit_stage(Grid3 g, LsGeom geo, ReinitBuf b, int stage, double cfl, double tol, const double* in,
                               double* phi, double* out) {
  if (stage > 1 && b.red[3]) return;  // converged on the residual in stage 1
  const long long n = (long long)g.nx * g.ny * g.nz;
  double maxres = 0.0, maxrel = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx), j = (int)((q / g.nx) % g.ny), k = (int)(q / ((long long)g.nx * g.ny));
    const long long off = loff(g, i, j, k);
    double R = 0.0;
    if (!b.tag[off]) {
      const double dx = smin(g.dx[i], smin(g.dy[j], g.dz[k]));
      const double dt = cfl * dx;
      double lr;
      reinit_local(g, geo, in, i, j, k, lr);
      if (fabs(lr) <= 1.0)
        R = -dt * b.sign[off] * lr;
      else
        R = -dt * b.sign[off] * lr / fabs(lr);
      maxres = smax(maxres, fabs(lr));
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
      double le = fabs(nw - old);
      if (nw != 0) le /= fabs(nw);
      maxrel = smax(maxrel, le);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    maxres = smax(maxres, __shfl_xor_sync(0xffffffffu, maxres, o));
    maxrel = smax(maxrel, __shfl_xor_sync(0xffffffffu, maxrel, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (stage == 1 && maxres > 0) atomicMax(&b.red[0], (unsigned long long)__double_as_longlong(maxres));
    if (stage == 3 && maxrel > 0) atomicMax(&b.red[1], (unsigned long long)__double_as_longlong(maxrel));
  }
  (void)tol;
}

__global__ void k_reinit_check(ReinitBuf b, double tol) {
  const double r = __longlong_as_double((long long)b.red[0]);
  b.red[3] = (r < tol) ? 1ull : 0ull;
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
  ReinitBuf b = carve(buf, n);
  const long long ni = (long long)g.nx * g.ny * g.nz;
  const int grid = grid1d(ni);
  cudaMemsetAsync(b.red, 0, 4 * sizeof(unsigned long long), s);
  k_reinit_prep<<<grid, 256, 0, s>>>(g, geo, phi, b);
  unsigned long long hred[4];
  cudaMemcpyAsync(hred, b.red, sizeof hred, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return M2CG_ERR_CUDA;
  if (hred[2] == 0) return M2CG_OK;  // no interface: nothing to do
  const double tol = ls.reinit_tol;
  const int maxIts = ls.reinit_maxits;
  int total = 0;
  for (;;) {
    const double cfl = *cfl_state;
    int iter;
    double dphi_max = 0.0;
    for (iter = 0; iter < maxIts; iter++) {
      cudaMemsetAsync(b.red, 0, 2 * sizeof(unsigned long long), s);
      cudaMemsetAsync(b.red + 3, 0, sizeof(unsigned long long), s);
      k_reinit_stage<<<grid, 256, 0, s>>>(g, geo, b, 1, cfl, tol, phi, phi, b.phi1);
      k_reinit_check<<<1, 1, 0, s>>>(b, tol);
      k_reinit_stage<<<grid, 256, 0, s>>>(g, geo, b, 2, cfl, tol, b.phi1, phi, b.phi2);
      k_reinit_stage<<<grid, 256, 0, s>>>(g, geo, b, 3, cfl, tol, b.phi2, phi, phi);
      cudaMemcpyAsync(hred, b.red, sizeof hred, cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) return M2CG_ERR_CUDA;
      total++;
      if (hred[3]) break;  // residual below the tolerance (checked before updating phi)
      dphi_max = bits_to_double(hred[1]);
      if (dphi_max < tol) break;
    }
    if (iterations) *iterations += total;
    if (iter < maxIts) return M2CG_OK;
    if (dphi_max < 0.02) return M2CG_OK;
    if (cfl < 0.02) return M2CG_ERR_REINIT;
    *cfl_state = cfl / 1.5;
    cudaMemcpyAsync(phi, b.phibk, n * 8, cudaMemcpyDeviceToDevice, s);
  }
}

}  // namespace m2c
