// Viscous fluxes of constant-viscosity materials (see viscous.h).
//
// Per face between the left cell L and the right cell R along axis d
// (ViscosityOperator::AddDiffusionFluxes, ViscosityOperator.cpp:200-408):
//   - the face velocity: linear interpolation cl(L) v(L) + cr(R) v(R) with
//     x_half = x_R - dx_R / 2, cl = (x_R - x_half) / (x_R - x_L),
//     cr = (x_half - x_L) / (x_R - x_L) (InterpolatorLinear::
//     CalculateInterpolationCoefficients, Interpolator.cpp:145-185);
//   - the normal derivative (v(R) - v(L)) / (x_R - x_L)
//     (GradientCalculatorCentral::CentralDifferencingAtCellInterfaces);
//   - each tangential derivative: the central three-point derivative at the
//     cells L and R (one-sided at the first / last cell of that axis where the
//     cell is a ghost in another axis), interpolated to the face as above
//     (CalculateFirstDerivativeAtNodes, CalculateCoefficients);
//   - the stress of ViscoFcnConstant (ViscoFcn.h) and the flux
//     (0, tau_d., u . tau_d.), times the face area of the right cell.
// Where L and R hold different materials each side takes its own material's
// flux, except on z faces, where the reference evaluates the left side with
// the right cell's material too (ViscosityOperator.cpp:384). Ghost velocities
// follow the boundary rules of SpaceOperator::ApplyBoundaryConditions and
// ghost material IDs are their image cells' (MultiPhaseOperator::
// UpdateMaterialIDAtGhostNodes). The arithmetic follows the reference's
// operation order and is compiled without FMA contraction.
#include "viscous.h"

#include <cstring>
#include <vector>

namespace m2c {

struct ViscDev {
  Grid3 g;
  const double* xg[3];  // coordinates incl. one ghost per side (index c + 1)
  const double* wg[3];  // widths incl. one ghost per side
  double mu[MAXMAT];    // ViscoFcnConstant dyna (0 and bulk 0: NONE)
  double bulk[MAXMAT];
  int viscous, heat;    // which fluxes are formed
  // heat diffusion: HeatDiffusionFcnConstant diffusivity and the EOS's
  // temperature law (VarFcnSG.h:70-78, VarFcnNASG.h:61)
  double kappa[MAXMAT];
  double invcv[MAXMAT], T0[MAXMAT], e0[MAXMAT], invcp[MAXMAT], h0[MAXMAT];
  int use_cp[MAXMAT];
  Eos<double> eos[MAXMAT];
  int nmat;
};

struct Viscous {
  ViscDev d;
  double* base = nullptr;  // coordinates and widths
  double* fr = nullptr;    // [3 axes][4][nf] (one allocation)
  double* fl = nullptr;
  double* fh = nullptr;    // heat flux per face [3 axes][nf]
  long long stride = 0;    // faces per component block (the largest axis' face count)
};

namespace {

__device__ __forceinline__ long long voff(const Grid3& g, int i, int j, int k) {
  return (long long)k * g.plane + (long long)j * g.px + i;
}

// Velocity of cell (i, j, k), interior or a face ghost (at most one index
// out of range), from the stage input.
template <typename T>
__device__ void node_vel(const ViscDev& d, const T* const* P, int i, int j, int k, double* v) {
  const Grid3& g = d.g;
  int ix[3] = {i, j, k};
  const int n[3] = {g.nx, g.ny, g.nz};
  int axis = -1, side = 0;
  for (int a = 0; a < 3; a++) {
    if (ix[a] < 0) { axis = a; side = 0; }
    else if (ix[a] >= n[a]) { axis = a; side = 1; }
  }
  if (axis < 0) {
    const long long o = voff(g, i, j, k);
    for (int c = 0; c < 3; c++) v[c] = double(P[1 + c][o]);
    return;
  }
  const int bc = g.bc[2 * axis + side];
  if (bc == BC_INLET || bc == BC_OUTLET) {
    const double* st = bc == BC_INLET ? g.inlet : g.outlet;
    for (int c = 0; c < 3; c++) v[c] = st[1 + c];
    return;
  }
  if (bc == BC_PERIODIC) ix[axis] = side ? ix[axis] - n[axis] : ix[axis] + n[axis];
  else ix[axis] = side ? n[axis] - 1 : 0;
  const long long o = voff(g, ix[0], ix[1], ix[2]);
  for (int c = 0; c < 3; c++) v[c] = double(P[1 + c][o]);
  if (bc == BC_STICKWALL) {
    v[0] = -v[0]; v[1] = -v[1]; v[2] = -v[2];
  } else if (bc != BC_PERIODIC) {  // SYMMETRY / SLIPWALL: the normal velocity flips
    v[axis] = -v[axis];
  }
}

// Density and pressure of cell (i, j, k), interior or a face ghost (the
// boundary rules keep the image's density and pressure except at INLET /
// OUTLET ghosts).
template <typename T>
__device__ void node_rho_p(const ViscDev& d, const T* const* P, int i, int j, int k, double& rho, double& p) {
  const Grid3& g = d.g;
  int ix[3] = {i, j, k};
  const int n[3] = {g.nx, g.ny, g.nz};
  int axis = -1, side = 0;
  for (int a = 0; a < 3; a++) {
    if (ix[a] < 0) { axis = a; side = 0; }
    else if (ix[a] >= n[a]) { axis = a; side = 1; }
  }
  if (axis >= 0) {
    const int bc = g.bc[2 * axis + side];
    if (bc == BC_INLET || bc == BC_OUTLET) {
      const double* st = bc == BC_INLET ? g.inlet : g.outlet;
      rho = st[0];
      p = st[4];
      return;
    }
    if (bc == BC_PERIODIC) ix[axis] = side ? ix[axis] - n[axis] : ix[axis] + n[axis];
    else ix[axis] = side ? n[axis] - 1 : 0;
  }
  const long long o = voff(g, ix[0], ix[1], ix[2]);
  rho = double(P[0][o]);
  p = double(P[4][o]);
}

// HeatDiffusionOperator::AddDiffusionFluxes step 1: the temperature of a cell
// from its EOS (GetInternalEnergyPerUnitMass, then GetTemperature).
__device__ __forceinline__ double temperature(const ViscDev& d, int id, double rho, double p) {
  const Eos<double>& e = d.eos[id];
  const double en = e.energy(rho, p);
  if (e.kind != EOS_SG) return d.invcv[id] * (en - e.q - e.pstiff * (1.0 / rho - e.b));
  if (d.use_cp[id]) {
    const double pp = e.pressure(rho, en);
    return d.T0[id] + d.invcp[id] * (en + pp / rho - d.h0[id]);
  }
  return d.T0[id] + d.invcv[id] * (en - d.e0[id]);
}

__device__ __forceinline__ uint8_t node_id(const Grid3& g, const uint8_t* id, int i, int j, int k) {
  if (!id) return 0;
  const int n[3] = {g.nx, g.ny, g.nz};
  int ix[3] = {i, j, k};
  for (int a = 0; a < 3; a++) {
    const bool per = g.bc[2 * a] == BC_PERIODIC;
    if (ix[a] < 0) ix[a] = per ? ix[a] + n[a] : 0;
    else if (ix[a] >= n[a]) ix[a] = per ? ix[a] - n[a] : n[a] - 1;
  }
  return id[voff(g, ix[0], ix[1], ix[2])];
}

// Derivative of the velocity along axis t at cell c (interior along t; a
// ghost in at most one other axis, ghost_other) (GradientCalculatorCentral.cpp:
// 54-185 and its coefficients, 226-366).
template <typename T>
__device__ void node_deriv(const ViscDev& d, const T* const* P, const int* c, int t, bool ghost_other, double* out) {
  const int n[3] = {d.g.nx, d.g.ny, d.g.nz};
  const double* x = d.xg[t] + 1;  // x[-1 .. n]
  const int it = c[t];
  int cm[3] = {c[0], c[1], c[2]}, cp[3] = {c[0], c[1], c[2]};
  cm[t] = it - 1;
  cp[t] = it + 1;
  // CalculateCoefficients zeroes the coefficients of every node that
  // SpaceVariable3D::OutsidePhysicalDomainAndUnpopulated reports
  // (SpaceVariable.h:150-158). Its x test reads (i < 0 || j >= NX), so a node
  // with j >= NX that is a ghost in y or z counts as an unpopulated edge too
  // (the top y-ghost row when NY >= NX): its derivative is zero.
  const int cnt = int(c[0] < 0 || c[1] >= n[0]) + int(c[1] < 0 || c[1] >= n[1]) + int(c[2] < 0 || c[2] >= n[2]);
  const bool zero = cnt > 1;
  double v0[3], vm[3], vp[3];
  node_vel(d, P, c[0], c[1], c[2], v0);
  if (it == 0 && ghost_other) {
    const double coeff = zero ? 0.0 : 1.0 / (x[it + 1] - x[it]);
    const double cm1 = zero ? 0.0 : -coeff;
    node_vel(d, P, cp[0], cp[1], cp[2], vp);
    for (int q = 0; q < 3; q++) out[q] = cm1 * v0[q] + coeff * vp[q];
  } else if (it == n[t] - 1 && ghost_other) {
    const double coeff = zero ? 0.0 : 1.0 / (x[it] - x[it - 1]);
    const double cm1 = zero ? 0.0 : -coeff;
    node_vel(d, P, cm[0], cm[1], cm[2], vm);
    for (int q = 0; q < 3; q++) out[q] = cm1 * vm[q] + coeff * v0[q];
  } else {
    const double dx0 = x[it] - x[it - 1];
    const double dx1 = x[it + 1] - x[it];
    const double dx2 = dx0 + dx1;
    const double c0 = zero ? 0.0 : -dx1 / (dx0 * dx2);
    const double c1 = zero ? 0.0 : 1.0 / dx0 - 1.0 / dx1;
    const double c2 = zero ? 0.0 : dx0 / (dx1 * dx2);
    node_vel(d, P, cm[0], cm[1], cm[2], vm);
    node_vel(d, P, cp[0], cp[1], cp[2], vp);
    for (int q = 0; q < 3; q++) out[q] = c0 * vm[q] + c1 * v0[q] + c2 * vp[q];
  }
}

// ViscoFcnConstant's flux across a face of axis d (EvaluateViscousFluxFunction_F/G/H).
__device__ __forceinline__ void visc_flux(double mu, double bulk, int d, const double* dx_, const double* dy_,
                                          const double* dz_, const double* v3, double* f) {
  if (mu == 0.0 && bulk == 0.0) {  // ViscosityModelData::NONE
    f[0] = f[1] = f[2] = f[3] = 0.0;
    return;
  }
  const double div = dx_[0] + dy_[1] + dz_[2];
  double t0, t1, t2;
  if (d == 0) {
    t0 = bulk * div + mu * (2.0 * dx_[0] - 2.0 / 3.0 * div);  // tau_xx
    t1 = mu * (dx_[1] + dy_[0]);                              // tau_xy
    t2 = mu * (dx_[2] + dz_[0]);                              // tau_xz
  } else if (d == 1) {
    t0 = mu * (dx_[1] + dy_[0]);                              // tau_xy
    t1 = bulk * div + mu * (2.0 * dy_[1] - 2.0 / 3.0 * div);  // tau_yy
    t2 = mu * (dy_[2] + dz_[1]);                              // tau_yz
  } else {
    t0 = mu * (dx_[2] + dz_[0]);                              // tau_xz
    t1 = mu * (dy_[2] + dz_[1]);                              // tau_yz
    t2 = bulk * div + mu * (2.0 * dz_[2] - 2.0 / 3.0 * div);  // tau_zz
  }
  f[0] = t0;
  f[1] = t1;
  f[2] = t2;
  f[3] = v3[0] * t0 + v3[1] * t1 + v3[2] * t2;
}

// One thread per cell (i, j, k) of [0, nx] x [0, ny] x [0, nz]: the faces of
// the three axes whose right cell it is.
template <typename T>
__global__ void k_visc_faces(ViscDev d, StageArgs a, double* fr, double* fl, double* fh, long long S) {
  const Grid3& g = d.g;
  const T* P[5];
  for (int c = 0; c < 5; c++) P[c] = static_cast<const T*>(a.Pin[c]);
  const long long total = (long long)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % (g.nx + 1));
    const long long r = q / (g.nx + 1);
    const int j = (int)(r % (g.ny + 1)), k = (int)(r / (g.ny + 1));
    const int n[3] = {g.nx, g.ny, g.nz};
    const int cR[3] = {i, j, k};
    for (int ax = 0; ax < 3; ax++) {
      // faces of axis ax exist for the right cells with the other two indices interior
      bool ok = true;
      for (int b = 0; b < 3; b++)
        if (b != ax && cR[b] >= n[b]) ok = false;
      if (!ok) continue;
      int cL[3] = {i, j, k};
      cL[ax] -= 1;
      const double* x = d.xg[ax] + 1;
      const double* w = d.wg[ax] + 1;
      const int iR = cR[ax];
      const double dd = x[iR] - x[iR - 1];
      // area of the right cell (ViscosityOperator.cpp:278-386, HeatDiffusionOperator.cpp:
      // 157-181): widths of its two other axes (a ghost has its boundary cell's)
      const int b1 = ax == 0 ? 1 : 0, b2 = ax == 2 ? 1 : 2;
      const double area = (d.wg[b1] + 1)[cR[b1]] * (d.wg[b2] + 1)[cR[b2]];
      const uint8_t idR = node_id(g, a.id, cR[0], cR[1], cR[2]);
      const uint8_t idL = node_id(g, a.id, cL[0], cL[1], cL[2]);
      long long fidx;
      if (ax == 0) fidx = ((long long)k * g.ny + j) * (g.nx + 1) + i;
      else if (ax == 1) fidx = ((long long)k * (g.ny + 1) + j) * g.nx + i;
      else fidx = ((long long)k * g.ny + j) * g.nx + i;
      if (d.viscous) {
        // interpolation coefficients of the face (Interpolator.cpp:165-176)
        const double xh = x[iR] - 0.5 * w[iR];
        const double cl = (x[iR] - xh) / dd, cr = (xh - x[iR - 1]) / dd;
        double vL[3], vR[3];
        node_vel(d, P, cL[0], cL[1], cL[2], vL);
        node_vel(d, P, cR[0], cR[1], cR[2], vR);
        double v3[3], D[3][3];  // D[t] = d(u, v, w)/d(axis t) at the face
        for (int c = 0; c < 3; c++) v3[c] = cl * vL[c] + cr * vR[c];
        for (int c = 0; c < 3; c++) D[ax][c] = (vR[c] - vL[c]) / dd;
        // a cell is a ghost in another axis than t where it is a ghost of ax (L at the
        // low boundary, R at the high one)
        const bool gL = cL[ax] < 0, gR = cR[ax] >= n[ax];
        for (int t = 0; t < 3; t++) {
          if (t == ax) continue;
          double dl[3], dr[3];
          node_deriv(d, P, cL, t, gL, dl);
          node_deriv(d, P, cR, t, gR, dr);
          for (int c = 0; c < 3; c++) D[t][c] = cl * dl[c] + cr * dr[c];
        }
        double FR[4], FL[4];
        visc_flux(d.mu[idR], d.bulk[idR], ax, D[0], D[1], D[2], v3, FR);
        for (int c = 0; c < 4; c++) FR[c] = FR[c] * area;
        if (idL == idR || ax == 2) {
          for (int c = 0; c < 4; c++) FL[c] = FR[c];
        } else {
          visc_flux(d.mu[idL], d.bulk[idL], ax, D[0], D[1], D[2], v3, FL);
          for (int c = 0; c < 4; c++) FL[c] = area * FL[c];
        }
        for (int c = 0; c < 4; c++) {
          fr[(ax * 4 + c) * S + fidx] = FR[c];
          fl[(ax * 4 + c) * S + fidx] = FL[c];
        }
      }
      if (d.heat) {
        // HeatDiffusionOperator::AddDiffusionFluxes (HeatDiffusionOperator.cpp:96-185):
        // the harmonic mean of the two diffusivities times the central
        // temperature difference across the face. Its y and z faces reuse the
        // denominator of the cell's own x face; where the cell has no x face
        // (the y-ghost row, the z-ghost plane) the denominator is the one the
        // traversal computed last: the x face of cell (nx, ny - 1, k) resp.
        // (nx, ny - 1, nz - 1).
        double rL, pL, rR, pR;
        node_rho_p(d, P, cL[0], cL[1], cL[2], rL, pL);
        node_rho_p(d, P, cR[0], cR[1], cR[2], rR, pR);
        const double dT = (temperature(d, idR, rR, pR) - temperature(d, idL, rL, pL)) / dd;
        const double myk = d.kappa[idR], neighk = d.kappa[idL];
        double denom;
        if (ax == 0) {
          denom = myk + neighk;
        } else if (cR[1] < n[1] && cR[2] < n[2]) {
          denom = myk + d.kappa[node_id(g, a.id, i - 1, j, k)];
        } else {
          const int kk = ax == 1 ? k : n[2] - 1;
          denom = d.kappa[node_id(g, a.id, n[0], n[1] - 1, kk)] + d.kappa[node_id(g, a.id, n[0] - 1, n[1] - 1, kk)];
        }
        double f = (denom == 0) ? 0.0 : 2.0 * myk * neighk / denom * dT;
        f = f * area;
        fh[ax * S + fidx] = f;
      }
    }
  }
}

}  // namespace

m2cg_status viscous_create(cudaStream_t s, const Grid3& g, const Eos<double>* eos, const m2cg_material* mats,
                           int nmat, const double* const* xc, const double* const* dx, Viscous** out) {
  *out = nullptr;
  bool viscous = false, heat = false;
  for (int m = 0; m < nmat; m++) {
    viscous = viscous || mats[m].mu != 0.0 || mats[m].mu_bulk != 0.0;
    heat = heat || mats[m].heat_diffusivity != 0.0;
  }
  if (!viscous && !heat) return M2CG_OK;
  Viscous* v = new Viscous;
  memset(&v->d, 0, sizeof v->d);
  v->d.g = g;
  v->d.nmat = nmat;
  v->d.viscous = viscous ? 1 : 0;
  v->d.heat = heat ? 1 : 0;
  for (int m = 0; m < nmat && m < MAXMAT; m++) {
    v->d.mu[m] = mats[m].mu;
    v->d.bulk[m] = mats[m].mu_bulk;
    // VarFcnSG / VarFcnNASG constructors (VarFcnSG.h:130-142): 1/cv and 1/cp
    // read as 0 where cv, cp are 0; cp is used where cp > 0 and cv <= 0
    v->d.kappa[m] = mats[m].heat_diffusivity;
    v->d.invcv[m] = mats[m].cv == 0.0 ? 0.0 : 1.0 / mats[m].cv;
    v->d.invcp[m] = mats[m].cp == 0.0 ? 0.0 : 1.0 / mats[m].cp;
    v->d.T0[m] = mats[m].T0;
    v->d.e0[m] = mats[m].e0;
    v->d.h0[m] = mats[m].h0;
    v->d.use_cp[m] = (mats[m].cp > 0.0 && mats[m].cv <= 0.0) ? 1 : 0;
    v->d.eos[m] = eos[m];
  }
  const int n[3] = {g.nx, g.ny, g.nz};
  // coordinates and widths with one ghost per side (SpaceOperator::
  // PopulateGhostBoundaryCoordinates: x_{-1} = x_0 - dx_0, a ghost's width is
  // its boundary cell's)
  std::vector<double> host;
  size_t offs[3][2];
  for (int a = 0; a < 3; a++) {
    offs[a][0] = host.size();
    host.push_back(xc[a][0] - dx[a][0]);
    for (int i = 0; i < n[a]; i++) host.push_back(xc[a][i]);
    host.push_back(xc[a][n[a] - 1] + dx[a][n[a] - 1]);
    offs[a][1] = host.size();
    host.push_back(dx[a][0]);
    for (int i = 0; i < n[a]; i++) host.push_back(dx[a][i]);
    host.push_back(dx[a][n[a] - 1]);
  }
  const long long nf[3] = {(long long)(g.nx + 1) * g.ny * g.nz, (long long)g.nx * (g.ny + 1) * g.nz,
                           (long long)g.nx * g.ny * (g.nz + 1)};
  long long big = nf[0];
  if (nf[1] > big) big = nf[1];
  if (nf[2] > big) big = nf[2];
  v->stride = big;
  bool ok = cudaMalloc((void**)&v->base, host.size() * sizeof(double)) == cudaSuccess;
  if (viscous) {
    ok = ok && cudaMalloc((void**)&v->fr, 3 * 4 * big * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&v->fl, 3 * 4 * big * sizeof(double)) == cudaSuccess;
  }
  if (heat) ok = ok && cudaMalloc((void**)&v->fh, 3 * big * sizeof(double)) == cudaSuccess;
  if (!ok) {
    viscous_destroy(v);
    return M2CG_ERR_NOMEM;
  }
  cudaMemcpyAsync(v->base, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  for (int a = 0; a < 3; a++) {
    v->d.xg[a] = v->base + offs[a][0];
    v->d.wg[a] = v->base + offs[a][1];
  }
  *out = v;
  return cudaGetLastError() == cudaSuccess ? M2CG_OK : M2CG_ERR_CUDA;
}

bool viscous_has_viscosity(const Viscous* v) { return v && v->d.viscous; }

void viscous_destroy(Viscous* v) {
  if (!v) return;
  cudaFree(v->base);
  cudaFree(v->fr);
  cudaFree(v->fl);
  cudaFree(v->fh);
  delete v;
}

m2cg_status viscous_faces(Viscous* v, cudaStream_t s, StageArgs& a, bool mixed) {
  const Grid3& g = v->d.g;
  const long long total = (long long)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (mixed)
    k_visc_faces<float><<<(int)blocks, 256, 0, s>>>(v->d, a, v->fr, v->fl, v->fh, v->stride);
  else
    k_visc_faces<double><<<(int)blocks, 256, 0, s>>>(v->d, a, v->fr, v->fl, v->fh, v->stride);
  if (cudaGetLastError() != cudaSuccess) return M2CG_ERR_CUDA;
  // viscous: axis ax's block starts at ax * 4 * stride, component c of face f
  // at + c * stride + f; heat: axis ax's face f at ax * stride + f
  for (int ax = 0; ax < 3; ax++) {
    a.visc.fr[ax] = v->fr ? v->fr + ax * 4 * v->stride : nullptr;
    a.visc.fl[ax] = v->fl ? v->fl + ax * 4 * v->stride : nullptr;
    a.visc.fh[ax] = v->fh ? v->fh + ax * v->stride : nullptr;
    a.visc.nf[ax] = v->stride;
  }
  return M2CG_OK;
}

}  // namespace m2c
