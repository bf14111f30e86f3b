// One fused Runge-Kutta stage of the finite-volume step on a structured box:
//   load state (C2P + clip on the fly) -> MUSCL slopes + face states with the
//   reference's revert rules -> numerical fluxes on every face once ->
//   per-cell residual in the reference's summation order -> RK update ->
//   (last stage) primitive output + CFL reduction.
//
// Replaces, per stage, SpaceOperator::ComputeResidual (SpaceOperator.cpp:3351-3409)
// = Reconstructor::Reconstruct (Reconstructor.cpp:332-904) +
//   SpaceOperator::CheckReconstructedStates (SpaceOperator.cpp:3198-3347) +
//   the face loop of SpaceOperator::ComputeAdvectionFluxes (2423-2815),
// and the RK arithmetic of TimeIntegratorRK2/RK3::AdvanceOneTimeStep
// (TimeIntegrator.cpp:291-428, 496-690) with ConservativeToPrimitive,
// ClipDensityAndPressure and ApplyBoundaryConditions (SpaceOperator.cpp:553-649, 1667-1745).
//
// Layout in HBM: structure-of-arrays FP64, interior cells only
// (index (k*ny + j)*px + i, row pitch px); ghost values are never stored:
// they are rebuilt from interior cells by the boundary rule when loaded.
//
// Work decomposition: a CTA owns a 32 x TY column of cells and marches along
// z through a chunk of planes, keeping a ring of 3 primitive planes
// (with a 2-cell x/y halo) in shared memory. Each plane step:
//   (1) load plane m+2 (ghost rules applied on the fly),
//   (2) slopes + revert mask for every cell of plane m+1 (x -1..32, y -1..TY),
//   (3) x/y face fluxes of plane m and the z face m+1/2 (one flux per face),
//   (4) residual + RK update of plane m; the z face m-1/2 is carried in
//       registers from the previous step.
// Face states follow Reconstructor.cpp: slope-limited primitive values, the
// first face (in the order l,r,b,t,k,f) failing CheckState reverted to the
// cell value, every face needing clipping reverted to the cell value, and
// a remaining CheckState failure reported as an error.
#pragma once
#include "physics.cuh"

namespace m2c {

constexpr int MAXMAT = 4;
constexpr int TX = 32;

enum { BC_NONE = 0, BC_INLET = 1, BC_OUTLET = 2, BC_SLIPWALL = 3, BC_STICKWALL = 4, BC_SYMMETRY = 5,
       BC_PERIODIC = 100 };

struct DevError {
  int code;
  int cell;   // linear interior index of the first failing cell (or -1)
  int where;  // stage * 16 + site
  int pad;
};

struct Grid3 {
  int nx, ny, nz;
  long long px, plane;  // row pitch, plane size (elements)
  int bc[6];
  double inlet[5], outlet[5];
  const double* dx;     // per axis cell widths (interior, length n)
  const double* dy;
  const double* dz;
  const double* lA[3];  // limiter coefficient A per axis index
  const double* lB[3];  // limiter coefficient B per axis index
  const int* lK[3];     // van Albada exponent per axis index
};

struct SchemeK {
  int flux, limiter, rec_linear, slope_zero_at_interface;
  double alpha, delta;
  int nmat;
  Eos<double> ed[MAXMAT];  // per-material EOS, FP64 (built on the host)
  Eos<float> ef[MAXMAT];   // the same in FP32 for the mixed path's flux half
};

struct StageArgs {
  Grid3 g;
  SchemeK s;
  const double* Vn[5];   // V^n (primitive) - step state
  const double* Us[5];   // flux source of stages >= 2 (conserved, raw)
  double* Uo[5];         // stage output (conserved) for non-final stages
  double* Vo[5];         // final-stage output (primitive)
  const uint8_t* id;     // material id per cell (nullptr: all 0)
  int stage;             // 1-based
  int final_stage;
  double a_prev, a_un;   // U_new = a_prev*U_s + a_un*U^n (stages >= 2)
  double bdt_coef;       // U_new += (bdt_coef*dt)*R; 1.0 for stage 1
  const double* clock;   // device clock: [0] t, [1] dt
  const int* us_clipped; // non-zero: U_s := P2C(clip(C2P(U_s))) everywhere (TimeIntegrator.cpp:542-545)
  int* clipped_out;      // set if any cell of this stage's output was clipped
  unsigned long long* dtmin_bits;  // final stage: min dx/(|u|+c) as ordered bits
  DevError* err;
  int zchunk;
  double* Ro[5];         // if set: write the residual R only (no RK update)
};

__device__ __forceinline__ void report(DevError* e, int code, int cell, int where) {
  if (atomicCAS(&e->code, 0, code) == 0) {
    e->cell = cell;
    e->where = where;
  }
}

template <typename T, int TY>
struct StageSmem {
  static constexpr int RX = TX + 4, RY = TY + 4;   // loaded region: x -2..TX+1, y -2..TY+1
  static constexpr int MX = TX + 2, MY = TY + 2;   // mask region: x -1..TX, y -1..TY
  T v[3][5][RY][RX];
  T sig[2][3][5][MY][MX];
  T fx[5][TY][TX + 1];
  T fy[5][TY + 1][TX];
  uint8_t mask[2][MY][MX];
  uint8_t real[3][RY][RX];  // 1 = real (interior or periodic image), 0 = ghost / unused
  uint8_t ids[3][RY][RX];
  double red[TY * TX / 32];
};

// Resolve a possibly-outside index along one axis. Returns the interior index
// to read; sets ghost side (-1 none, 0 low, 1 high) or far (outside by > 1).
__device__ __forceinline__ int resolve_axis(int c, int n, int bclo, int bchi, int& side, bool& far) {
  side = -1;
  if (c >= 0 && c < n) return c;
  int bc = c < 0 ? bclo : bchi;
  if (bc == BC_PERIODIC) return ((c % n) + n) % n;
  if (c == -1) { side = 0; return 0; }
  if (c == n) { side = 1; return n - 1; }
  far = true;
  return c < 0 ? 0 : n - 1;
}

template <typename T> struct EosPick;
template <> struct EosPick<double> {
  __device__ static const Eos<double>& get(const SchemeK& s, int id) { return s.ed[id < s.nmat ? id : 0]; }
};
template <> struct EosPick<float> {
  __device__ static const Eos<float>& get(const SchemeK& s, int id) { return s.ef[id < s.nmat ? id : 0]; }
};
template <typename T>
__device__ __forceinline__ Eos<T> eos_of(const SchemeK& s, int id) {
  return EosPick<T>::get(s, id);
}

// Load one primitive state (FP64 on the way in, rounded to T for the flux
// half) at global (i,j,k), applying ghost rules. Returns 1 if the cell is
// real, 0 if it is a ghost/unused cell. For stage >= 2 the state comes from
// U_s by C2P + clip (SpaceOperator::ConservativeToPrimitive + ClipDensityAndPressure).
template <typename T>
__device__ int load_cell(const StageArgs& a, int i, int j, int k, T* out, uint8_t& idout) {
  const Grid3& g = a.g;
  int sx, sy, sz;
  bool far = false;
  int ii = resolve_axis(i, g.nx, g.bc[0], g.bc[1], sx, far);
  int jj = resolve_axis(j, g.ny, g.bc[2], g.bc[3], sy, far);
  int kk = resolve_axis(k, g.nz, g.bc[4], g.bc[5], sz, far);
  int nghost = (sx >= 0) + (sy >= 0) + (sz >= 0);
  long long off = (long long)kk * g.plane + (long long)jj * g.px + ii;
  uint8_t id = a.id ? a.id[off] : 0;
  idout = id;
  double V[5];
  if (a.stage == 1) {
    for (int p = 0; p < 5; p++) V[p] = a.Vn[p][off];
  } else {
    double U[5];
    for (int p = 0; p < 5; p++) U[p] = a.Us[p][off];
    Eos<double> e = eos_of<double>(a.s, id);
    e.c2p(U, V);
    e.clip(V);
  }
  int real = (nghost == 0 && !far) ? 1 : 0;
  if (nghost == 1 && !far) {
    int axis = sx >= 0 ? 0 : sy >= 0 ? 1 : 2;
    int side = sx >= 0 ? sx : sy >= 0 ? sy : sz;
    int bc = g.bc[2 * axis + side];
    if (bc == BC_INLET) {
      for (int p = 0; p < 5; p++) V[p] = g.inlet[p];
    } else if (bc == BC_OUTLET) {
      for (int p = 0; p < 5; p++) V[p] = g.outlet[p];
    } else if (bc == BC_STICKWALL) {
      V[1] = -V[1]; V[2] = -V[2]; V[3] = -V[3];
    } else {  // SYMMETRY / SLIPWALL
      V[axis + 1] = -V[axis + 1];
    }
  }
  for (int p = 0; p < 5; p++) out[p] = T(V[p]);
  return real;
}

// Reconstructed face states of one real cell and the revert mask
// (bit 0 l, 1 r, 2 b, 3 t, 4 k, 5 f). Returns ERR_NONE or ERR_STATE.
template <typename T>
__device__ __forceinline__ int cell_faces(const Eos<T>& e, const T* v, const T* sx, const T* sy, const T* sz,
                                          uint8_t& mask) {
  T f[6][5];
  for (int p = 0; p < 5; p++) {
    T hx = T(0.5) * sx[p], hy = T(0.5) * sy[p], hz = T(0.5) * sz[p];
    f[0][p] = v[p] - hx; f[1][p] = v[p] + hx;
    f[2][p] = v[p] - hy; f[3][p] = v[p] + hy;
    f[4][p] = v[p] - hz; f[5][p] = v[p] + hz;
  }
  uint8_t m = 0;
  // Reconstructor.cpp:719-775: only the first non-physical face is reverted.
  for (int q = 0; q < 6; q++)
    if (e.bad(f[q])) { m |= uint8_t(1u << q); break; }
  // SpaceOperator.cpp:3240-3273: faces needing clipping revert to the cell value.
  for (int q = 0; q < 6; q++)
    if (!(m & (1u << q)) && e.needs_clip(f[q])) m |= uint8_t(1u << q);
  mask = m;
  // SpaceOperator.cpp:3275-3277: any face still non-physical is fatal.
  for (int q = 0; q < 6; q++)
    if (!(m & (1u << q)) && e.bad(f[q])) return ERR_STATE;
  return ERR_NONE;
}

// Final face value of a real cell: side 0 = minus face (v - s/2), 1 = plus face.
template <typename T>
__device__ __forceinline__ void face_value(const T* v, const T* s, bool reverted, int side, T* out) {
  if (reverted) {
    for (int p = 0; p < 5; p++) out[p] = v[p];
  } else if (side == 0) {
    for (int p = 0; p < 5; p++) out[p] = v[p] - T(0.5) * s[p];
  } else {
    for (int p = 0; p < 5; p++) out[p] = v[p] + T(0.5) * s[p];
  }
}

// Boundary face state built from the interior neighbour's face state
// (Reconstructor.cpp:822-875) followed by the clip check of
// CheckReconstructedStates on the ghost's inward face (3279-3318).
template <typename T>
__device__ __forceinline__ void ghost_face(int bc, int axis, const T* inner_face, const T* ghost_cell,
                                           const Eos<T>& e, T* out) {
  if (bc == BC_INLET || bc == BC_OUTLET) {
    for (int p = 0; p < 5; p++) out[p] = ghost_cell[p];
  } else {
    for (int p = 0; p < 5; p++) out[p] = inner_face[p];
    if (bc == BC_STICKWALL) {
      out[1] = -out[1]; out[2] = -out[2]; out[3] = -out[3];
    } else {
      out[axis + 1] = -out[axis + 1];
    }
  }
  if (e.needs_clip(out))
    for (int p = 0; p < 5; p++) out[p] = ghost_cell[p];
}

template <typename T, int TY>
__global__ void __launch_bounds__(TX * TY, 1) stage_kernel(const StageArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  typedef StageSmem<T, TY> S;
  S& sm = *reinterpret_cast<S*>(smem_raw);
  const Grid3& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int NT = TX * TY;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int kb = blockIdx.z * a.zchunk;
  const int ke = min(kb + a.zchunk, g.nz);
  if (kb >= ke) return;
  const bool zper = g.bc[4] == BC_PERIODIC;
  const double dt = a.clock[1];
  const double bdt = a.bdt_coef * dt;
  const bool us_clip = (a.stage > 1) && a.us_clipped && *a.us_clipped;
  const T alpha = T(a.s.alpha), delta = T(a.s.delta);
  const int where = a.stage * 16;

  auto slot3 = [](int p) { return ((p % 3) + 3) % 3; };
  auto plane_is_ghost = [&](int p) { return !zper && (p < 0 || p >= g.nz); };

  // (1) load plane p into the ring
  auto load_plane = [&](int p) {
    int s = slot3(p);
    for (int q = tid; q < S::RY * S::RX; q += NT) {
      int ly = q / S::RX, lx = q % S::RX;
      T v[5];
      uint8_t id;
      int real = load_cell<T>(a, i0 + lx - 2, j0 + ly - 2, p, v, id);
      for (int c = 0; c < 5; c++) sm.v[s][c][ly][lx] = v[c];
      sm.real[s][ly][lx] = (uint8_t)real;
      sm.ids[s][ly][lx] = id;
    }
  };

  // (2) slopes + mask for plane p (needs planes p-1, p, p+1 in the ring)
  auto mask_plane = [&](int p) {
    int sm1 = slot3(p - 1), s0 = slot3(p), sp1 = slot3(p + 1), ms = p & 1;
    for (int q = tid; q < S::MY * S::MX; q += NT) {
      int my = q / S::MX, mx = q % S::MX;
      int ly = my + 1, lx = mx + 1;  // position in the loaded region
      if (!sm.real[s0][ly][lx]) { sm.mask[ms][my][mx] = 0; continue; }
      int gi = i0 + mx - 1, gj = j0 + my - 1;
      uint8_t id = sm.ids[s0][ly][lx];
      Eos<T> e = eos_of<T>(a.s, id);
      T v[5], sx[5], sy[5], sz[5];
      int ia = ((gi % g.nx) + g.nx) % g.nx, ja = ((gj % g.ny) + g.ny) % g.ny, ka = ((p % g.nz) + g.nz) % g.nz;
      T Ax = T(g.lA[0][ia]), Bx = T(g.lB[0][ia]), Ay = T(g.lA[1][ja]), By = T(g.lB[1][ja]);
      T Az = T(g.lA[2][ka]), Bz = T(g.lB[2][ka]);
      int Kx = g.lK[0][ia], Ky = g.lK[1][ja], Kz = g.lK[2][ka];
      bool zx = false, zy = false, zz = false;
      if (a.s.slope_zero_at_interface && a.id) {
        zx = id != sm.ids[s0][ly][lx - 1] || id != sm.ids[s0][ly][lx + 1];
        zy = id != sm.ids[s0][ly - 1][lx] || id != sm.ids[s0][ly + 1][lx];
        zz = id != sm.ids[sm1][ly][lx] || id != sm.ids[sp1][ly][lx];
      }
      for (int c = 0; c < 5; c++) {
        T vc = sm.v[s0][c][ly][lx];
        v[c] = vc;
        if (a.s.rec_linear) {
          sx[c] = limited_slope(a.s.limiter, Ax, Bx, Kx, alpha, vc - sm.v[s0][c][ly][lx - 1], sm.v[s0][c][ly][lx + 1] - vc);
          sy[c] = limited_slope(a.s.limiter, Ay, By, Ky, alpha, vc - sm.v[s0][c][ly - 1][lx], sm.v[s0][c][ly + 1][lx] - vc);
          sz[c] = limited_slope(a.s.limiter, Az, Bz, Kz, alpha, vc - sm.v[sm1][c][ly][lx], sm.v[sp1][c][ly][lx] - vc);
          if (zx) sx[c] = T(0);
          if (zy) sy[c] = T(0);
          if (zz) sz[c] = T(0);
        } else {
          sx[c] = sy[c] = sz[c] = T(0);
        }
        sm.sig[ms][0][c][my][mx] = sx[c];
        sm.sig[ms][1][c][my][mx] = sy[c];
        sm.sig[ms][2][c][my][mx] = sz[c];
      }
      uint8_t m;
      int err = cell_faces(e, v, sx, sy, sz, m);
      sm.mask[ms][my][mx] = m;
      if (err) report(a.err, err, (int)((long long)p * g.ny * g.nx + (long long)gj * g.nx + gi), where + 1);
    }
  };

  // Face state of a real cell at mask-region position (mx,my) in plane p,
  // direction d, side (0 minus, 1 plus).
  auto cell_face = [&](int p, int mx, int my, int d, int side, T* out) {
    int s0 = slot3(p), ms = p & 1;
    T v[5], s[5];
    for (int c = 0; c < 5; c++) {
      v[c] = sm.v[s0][c][my + 1][mx + 1];
      s[c] = sm.sig[ms][d][c][my][mx];
    }
    bool rev = (sm.mask[ms][my][mx] >> (2 * d + side)) & 1u;
    face_value(v, s, rev, side, out);
  };

  // Flux across the face between mask-region cells L and R (R = L + e_d).
  // pL/pR are the planes of L and R; real flags say whether each is a real cell.
  auto face_flux = [&](int d, int pL, int mxL, int myL, int pR, int mxR, int myR, T* F) {
    bool rL = sm.real[slot3(pL)][myL + 1][mxL + 1], rR = sm.real[slot3(pR)][myR + 1][mxR + 1];
    T VL[5], VR[5];
    uint8_t idL = sm.ids[slot3(pL)][myL + 1][mxL + 1], idR = sm.ids[slot3(pR)][myR + 1][mxR + 1];
    int bcside;
    if (rL) cell_face(pL, mxL, myL, d, 1, VL);
    if (rR) cell_face(pR, mxR, myR, d, 0, VR);
    if (!rL && !rR) {
      for (int c = 0; c < 5; c++) F[c] = T(0);
      return;
    }
    if (!rL) {  // low-side boundary face
      bcside = 2 * d;
      T gc[5];
      for (int c = 0; c < 5; c++) gc[c] = sm.v[slot3(pL)][c][myL + 1][mxL + 1];
      ghost_face(g.bc[bcside], d, VR, gc, eos_of<T>(a.s, idL), VL);
    }
    if (!rR) {  // high-side boundary face
      bcside = 2 * d + 1;
      T gc[5];
      for (int c = 0; c < 5; c++) gc[c] = sm.v[slot3(pR)][c][myR + 1][mxR + 1];
      ghost_face(g.bc[bcside], d, VL, gc, eos_of<T>(a.s, idR), VR);
    }
    // same material (single-material path): flux with the right cell's EOS,
    // as the reference's face loop does (myid = id of the right cell).
    uint8_t idf = rR ? idR : idL;
    int err = num_flux(a.s.flux, eos_of<T>(a.s, idf), d, VL, VR, delta, F);
    if (err) report(a.err, err, -1, where + 2);
  };

  // ---- prologue ----
  T Hprev[5];
  if (!plane_is_ghost(kb - 1)) {
    load_plane(kb - 2);
    load_plane(kb - 1);
    load_plane(kb);
    __syncthreads();
    mask_plane(kb - 1);
    __syncthreads();
    load_plane(kb + 1);
    __syncthreads();
    mask_plane(kb);
    __syncthreads();
  } else {
    load_plane(kb - 1);
    load_plane(kb);
    load_plane(kb + 1);
    __syncthreads();
    mask_plane(kb);
    __syncthreads();
  }
  face_flux(2, kb - 1, tx + 1, ty + 1, kb, tx + 1, ty + 1, Hprev);

  const int gi = i0 + tx, gj = j0 + ty;
  const bool own = gi < g.nx && gj < g.ny;
  double dxi = 0, dyj = 0;
  if (own) { dxi = g.dx[gi]; dyj = g.dy[gj]; }
  double dtmin_local = 1.0e300;
  int clipped_local = 0;

  for (int m = kb; m < ke; m++) {
    __syncthreads();
    load_plane(m + 2);
    __syncthreads();
    if (!plane_is_ghost(m + 1)) mask_plane(m + 1);
    __syncthreads();
    // (3) faces of plane m
    {
      T F[5];
      face_flux(0, m, tx, ty + 1, m, tx + 1, ty + 1, F);
      for (int c = 0; c < 5; c++) sm.fx[c][ty][tx] = F[c];
      if (tid < TY) {
        face_flux(0, m, TX, tid + 1, m, TX + 1, tid + 1, F);
        for (int c = 0; c < 5; c++) sm.fx[c][tid][TX] = F[c];
      }
      face_flux(1, m, tx + 1, ty, m, tx + 1, ty + 1, F);
      for (int c = 0; c < 5; c++) sm.fy[c][ty][tx] = F[c];
      if (tid < TX) {
        face_flux(1, m, tid + 1, TY, m, tid + 1, TY + 1, F);
        for (int c = 0; c < 5; c++) sm.fy[c][TY][tid] = F[c];
      }
    }
    T Hnext[5];
    face_flux(2, m, tx + 1, ty + 1, m + 1, tx + 1, ty + 1, Hnext);
    __syncthreads();
    // (4) residual + RK update
    if (own) {
      double dzk = g.dz[m];
      double ax = dyj * dzk, ay = dxi * dzk, az = dxi * dyj;
      double vol = dxi * dyj * dzk;
      long long off = (long long)m * g.plane + (long long)gj * g.px + gi;
      uint8_t id = a.id ? a.id[off] : 0;
      Eos<double> e = eos_of<double>(a.s, id);
      double Un[5], Unew[5], Vn[5];
      for (int c = 0; c < 5; c++) Vn[c] = a.Vn[c][off];
      e.p2c(Vn, Un);
      if (a.stage == 1) {
        for (int c = 0; c < 5; c++) Unew[c] = Un[c];
      } else {
        double Us[5];
        for (int c = 0; c < 5; c++) Us[c] = a.Us[c][off];
        if (us_clip) {
          double Vs[5];
          e.c2p(Us, Vs);
          e.clip(Vs);
          e.p2c(Vs, Us);
        }
        for (int c = 0; c < 5; c++) Unew[c] = a.a_prev * Us[c] + a.a_un * Un[c];
      }
      for (int c = 0; c < 5; c++) {
        double f = 0.0;
        f = f - double(sm.fx[c][ty][tx]) * ax;
        f = f - double(sm.fy[c][ty][tx]) * ay;
        f = f - double(Hprev[c]) * az;
        f = f + double(sm.fx[c][ty][tx + 1]) * ax;
        f = f + double(sm.fy[c][ty + 1][tx]) * ay;
        f = f + double(Hnext[c]) * az;
        double R = f / (-vol);
        if (a.Ro[0]) a.Ro[c][off] = R;
        Unew[c] = Unew[c] + bdt * R;
      }
      if (!a.Ro[0]) {
      double V[5];
      e.c2p(Unew, V);
      bool clipped = e.clip(V);
      clipped_local |= clipped ? 1 : 0;
      if (e.bad(V)) report(a.err, ERR_STATE, (int)(off), where + 3);
      if (a.final_stage) {
        for (int c = 0; c < 5; c++) a.Vo[c][off] = V[c];
        double ee = e.energy(V[0], V[4]);
        double c2 = e.c2(V[0], ee);
        if (c2 < 0.0) report(a.err, ERR_SOUND, (int)off, where + 4);
        double cs = sqrt(c2);
        double lx = fabs(V[1]) + cs, ly = fabs(V[2]) + cs, lz = fabs(V[3]) + cs;
        double r = smin(dxi / lx, smin(dyj / ly, dzk / lz));
        dtmin_local = smin(dtmin_local, r);
      } else {
        for (int c = 0; c < 5; c++) a.Uo[c][off] = Unew[c];
      }
      }  // !Ro
    }
    for (int c = 0; c < 5; c++) Hprev[c] = Hnext[c];
  }

  if (a.clipped_out && __syncthreads_or(clipped_local)) {
    if (tid == 0) atomicOr(a.clipped_out, 1);
  }
  if (a.final_stage && a.dtmin_bits) {
    double v = dtmin_local;
    for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (tx == 0) sm.red[ty] = v;
    __syncthreads();
    if (tid == 0) {
      double r = sm.red[0];
      for (int q = 1; q < TY; q++) r = smin(r, sm.red[q]);
      if (r < 1.0e300) atomicMin(a.dtmin_bits, (unsigned long long)__double_as_longlong(r));
    }
  }
}

}  // namespace m2c
