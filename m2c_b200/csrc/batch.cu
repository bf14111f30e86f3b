// Batched 1D two-material shock tubes: thousands of independent tubes of
// uneven lengths advanced together, FP64 (compiled with -fmad=false).
//
// Each tube is one reference run on an nx x 1 x 1 grid over [0, 1] with an
// INLET ghost (left state) and an OUTLET ghost (right state), one level set
// phi = 0.5 - x (material 1 where phi < 0), HLLC (or the scheme's flux) with
// MUSCL, the exact two-material Riemann solve at the interface face, RK2/RK3
// with a per-tube CFL time step: TimeIntegratorRK2/RK3::AdvanceOneTimeStep
// (TimeIntegrator.cpp:291-690) + SpaceOperator::ComputeTimeStepSize (2128-2227)
// + MultiPhaseOperator updates (127-332, 824-1027), restricted to one axis.
// On a one-cell-wide grid with symmetry walls the y and z faces contribute
// exact zeros to the reference's residual sum, so only x faces are evaluated.
//
// All tubes live in one concatenated structure-of-arrays state. A step is
//   k_tube_begin   one warp per tube: CFL time step, ID snapshot, interface faces
//   per RK stage:
//     k_tube_riemann  one thread per interface face of every tube: exact Riemann
//     k_tube_stage    persistent CTAs over (tube, chunk of cells_per_block)
//                     work items: slopes + revert chain, face fluxes, residual,
//                     RK update, C2P/clip/check, level-set FD3 stage
//   k_tube_end     one warp per tube: material ID from the phi sign change and
//                  the ordered Riemann-solution update of cells that changed
// and the step sequence is captured once in CUDA graphs and replayed.
// cells_per_block and threads_per_block come from a measured autotuning pass
// over candidate shapes at creation unless the caller fixes them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/m2c_gpu.h"
#include "fd3.cuh"
#include "mlp.cuh"
#include "riemann_batch.h"
#include "stage.cuh"

namespace m2c {

void set_last_error(const char* msg);
cudaError_t mlp_warm_device(const m2cg_mlp* m, cudaStream_t s, const float* X, const int* valid, const double* P,
                            int n, float* y, double* warm, const int* ndev);

constexpr int TUBE_IFACE_CAP = 8;        // interface faces tracked per tube
constexpr int TUBE_RIEMANN_THREADS = 16384; // threads of the Riemann kernel (each owns path scratch)

struct TubeArgs {
  int ntubes;
  long long ncell;
  const long long* off;     // [T+1] first cell of each tube
  const Eos<double>* eos;   // [2T] materials 0 and 1 of each tube
  const double* bcl;        // [T][5] INLET ghost state
  const double* bcr;        // [T][5] OUTLET ghost state
  double* clock;            // [T][2]: t, dt
  double* V[2][5];          // primitive state, ping-pong across steps
  double* U[2][5];          // conserved stage outputs
  double* phi[2];           // phi^n, ping-pong across steps
  double* phis[2];          // stage outputs of phi
  uint8_t* id;              // material id (current)
  uint8_t* idn;             // material id at the start of the step
  int* nif;                 // [T] interface faces this step
  int* iface;               // [T][CAP] tube-local index of the right cell of each interface face
  double* Vsm;              // [T][CAP][5] star states of the current stage
  double* Vsp;
  double* Vmid;
  int* midid;               // [T][CAP]
  double* rsVsm;            // [T][CAP][5] stage-1 star states (RiemannSolutions)
  double* rsVsp;
  uint8_t* rsValid;         // [T][CAP]
  int* clip;                // [T][4] clip flag per stage
  int* terr;                // [T] first error code of each tube
  unsigned long long* cnt;  // [0] Riemann calls, [1] iterations, [2] errors, [3] unresolved, [5] evaluations
  DevError* err;
  // scheme
  int flux, limiter, rec_linear, slope_zero, mp_flux, rk, vak;
  double alpha, delta, cfl, limA, limB, limC;
  RiemannParams P;
  double* scratch;          // Riemann path scratch, one slot per Riemann-kernel thread
  const int2* items;        // (tube, first cell) work items of the stage kernel
  int nitems, cpb;
  const double* warm;       // optional [T][CAP] star-pressure warm starts (NaN = none)
};

struct TubeStage {
  int stage, final_stage, cur;
  double a_prev, a_un, bdt_coef;
};

__device__ __forceinline__ void tube_fail(const TubeArgs& A, int t, int code, int cell, int where) {
  atomicCAS(&A.terr[t], 0, code);
  report(A.err, code, cell, where);
}

// SpaceOperator::ComputeTimeStepSize per tube (dy = dz = 1), the ID snapshot,
// and the ordered list of interface faces (ID differs across the face).
__device__ void tube_begin(const TubeArgs& A, int t, int cur, int lane) {
  // a tube that reported an error stops where it failed (the reference
  // aborts there); the warp decides from one read
  if (__shfl_sync(0xffffffffu, lane == 0 ? A.terr[t] : 0, 0)) return;
  const long long o = A.off[t];
  const int n = (int)(A.off[t + 1] - o);
  const double h = 1.0 / n;
  double best = 1.0e300;
  int nf = 0;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    bool ifc = false;
    if (i < n) {
      const uint8_t me = A.id[o + i];
      A.idn[o + i] = me;
      const Eos<double>& e = A.eos[2 * t + me];
      const double rho = A.V[cur][0][o + i], p = A.V[cur][4][o + i];
      const double c2 = e.c2(rho, e.energy(rho, p));
      if (c2 < 0.0) tube_fail(A, t, ERR_SOUND, (int)(o + i), 5);
      const double c = sqrt(c2);
      const double r = smin(h / (fabs(A.V[cur][1][o + i]) + c),
                            smin(1.0 / (fabs(A.V[cur][2][o + i]) + c), 1.0 / (fabs(A.V[cur][3][o + i]) + c)));
      best = smin(best, r);
      ifc = i > 0 && A.id[o + i - 1] != me;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ifc);
    if (ifc) {
      const int k = nf + __popc(bal & ((1u << lane) - 1));
      if (k < TUBE_IFACE_CAP) A.iface[t * TUBE_IFACE_CAP + k] = i;
    }
    nf += __popc(bal);
  }
  for (int s = 16; s > 0; s >>= 1) best = smin(best, __shfl_xor_sync(0xffffffffu, best, s));
  if (lane == 0) {
    const double dt = A.cfl * best;
    A.clock[2 * t + 1] = dt;
    A.clock[2 * t] = A.clock[2 * t] + dt;
    if (nf > TUBE_IFACE_CAP) {
      tube_fail(A, t, ERR_ITER_CAP, (int)o, 10);
      nf = TUBE_IFACE_CAP;
    }
    A.nif[t] = nf;
    for (int q = 0; q < 4; q++) A.clip[4 * t + q] = 0;
  }
}

__global__ void k_tube_begin(TubeArgs A, int cur) {
  const int lane = threadIdx.x & 31;
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= A.ntubes) return;
  tube_begin(A, t, cur, lane);
}

// Primitive state of a real cell at this stage: V^n (stage 1) or clip(C2P(U_s)).
__device__ __forceinline__ void tube_state(const TubeArgs& A, const TubeStage& S, const Eos<double>& e, long long q,
                                           double* V) {
  if (S.stage == 1) {
    for (int c = 0; c < 5; c++) V[c] = A.V[S.cur][c][q];
  } else {
    double U[5];
    for (int c = 0; c < 5; c++) U[c] = A.U[(S.stage - 2) & 1][c][q];
    e.c2p(U, V);
    e.clip(V);
  }
}

// Exact Riemann problem at every interface face of every tube
// (SpaceOperator.cpp:2499-2523: MESH normal, cell-centred states, star
// states clipped with each side's EOS; stage-1 results kept).
__device__ void tube_riemann(const TubeArgs& A, const TubeStage& S, int t, int k, RiemannSolver& rs) {
  const long long w = (long long)t * TUBE_IFACE_CAP + k;
  const long long o = A.off[t];
  const int i = A.iface[w];
  const uint8_t idL = A.id[o + i - 1], idR = A.id[o + i];
  const Eos<double>* eos = A.eos + 2 * t;
  double VL[5], VR[5];
  tube_state(A, S, eos[idL], o + i - 1, VL);
  tube_state(A, S, eos[idR], o + i, VR);
  const double dir[3] = {1.0, 0.0, 0.0};
  double Vs[5], Vsm[5], Vsp[5];
  int mid = 0;
  bool bad = false;
  rs.eos = eos;
  const double warm = A.warm ? A.warm[w] : NAN;
  const int r = rs.solve(dir, VL, idL, VR, idR, Vs, mid, Vsm, Vsp, warm, bad);
  eos[idL].clip(Vsm);
  eos[idR].clip(Vsp);
  for (int c = 0; c < 5; c++) {
    A.Vsm[w * 5 + c] = Vsm[c];
    A.Vsp[w * 5 + c] = Vsp[c];
    A.Vmid[w * 5 + c] = Vs[c];
  }
  A.midid[w] = mid;
  if (S.stage == 1) {
    for (int c = 0; c < 5; c++) {
      A.rsVsm[w * 5 + c] = Vsm[c];
      A.rsVsp[w * 5 + c] = Vsp[c];
    }
    A.rsValid[w] = (r == RIEM_OK) ? 1 : 0;
  }
  atomicAdd(&A.cnt[0], 1ull);
  atomicAdd(&A.cnt[1], (unsigned long long)rs.iterations);
  atomicAdd(&A.cnt[5], (unsigned long long)rs.evaluations);
  if (r != RIEM_OK) atomicAdd(&A.cnt[2], 1ull);
  if (r & RIEM_PATH_OVERFLOW) tube_fail(A, t, ERR_ITER_CAP, (int)(o + i), 7);
  if (bad) tube_fail(A, t, ERR_STATE, (int)(o + i), 8);
}

__global__ void k_tube_riemann(TubeArgs A, TubeStage S) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  RiemannSolver rs;
  rs.P = A.P;
  rs.path1.pt = A.scratch + tid * 2 * 3 * RIEMANN_PATH_CAP;
  rs.path1.cap = RIEMANN_PATH_CAP;
  rs.path3.pt = rs.path1.pt + 3 * RIEMANN_PATH_CAP;
  rs.path3.cap = RIEMANN_PATH_CAP;
  // one thread per tube (tubes rarely hold more than one interface face)
  for (long long tt = tid; tt < A.ntubes; tt += nth) {
    if (A.terr[tt]) continue;  // failed tubes stop
    for (int k = 0; k < A.nif[tt]; k++) tube_riemann(A, S, (int)tt, k, rs);
  }
}

// Features of every interface problem of this stage (the states the Riemann
// kernel will use), for the learned warm start; slots without an interface
// face are marked invalid.
__global__ void k_tube_features(TubeArgs A, TubeStage S, float* X, double* P, int* valid) {
  const long long total = (long long)A.ntubes * TUBE_IFACE_CAP;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(w / TUBE_IFACE_CAP), k = (int)(w - (long long)t * TUBE_IFACE_CAP);
    int ok = 0;
    if (k < A.nif[t] && !A.terr[t]) {
      const long long o = A.off[t];
      const int i = A.iface[w];
      const uint8_t idL = A.id[o + i - 1], idR = A.id[o + i];
      const Eos<double>* eos = A.eos + 2 * t;
      double VL[5], VR[5];
      tube_state(A, S, eos[idL], o + i - 1, VL);
      tube_state(A, S, eos[idR], o + i, VR);
      const double dir[3] = {1.0, 0.0, 0.0};
      double Pq[2] = {0.0, 0.0};
      ok = mlp_features(eos[idL], eos[idR], VL, VR, dir, X + w * MLP_IN, Pq) ? 1 : 0;
      P[2 * w] = Pq[0];
      P[2 * w + 1] = Pq[1];
    }
    valid[w] = ok;
  }
}

// Shared-memory layout of one work item (cells c0-2 .. c0+cpb+1 loaded).
struct TubeSmem {
  double* v[5];   // [cpb+4] stage primitive states
  double* sg[5];  // [cpb+4] limited slopes
  double* F[5];   // [cpb+1] flux seen by the left cell of each face
  double* F2[5];  // [cpb+1] flux seen by the right cell
  double* ph;     // [cpb+4] phi (stage input)
  uint8_t* ids;   // [cpb+4]
  uint8_t* real;  // [cpb+4]
  uint8_t* mask;  // [cpb+4] revert bits (1 left face, 2 right face)
};

__host__ __device__ inline size_t tube_smem_bytes(int cpb) {
  const size_t m = (size_t)cpb + 4, f = (size_t)cpb + 1;
  return (10 * m + 10 * f + m) * sizeof(double) + 3 * m + 16;
}

__device__ __forceinline__ TubeSmem tube_smem(unsigned char* base, int cpb) {
  TubeSmem s;
  const int m = cpb + 4, f = cpb + 1;
  double* p = reinterpret_cast<double*>(base);
  for (int c = 0; c < 5; c++) { s.v[c] = p; p += m; }
  for (int c = 0; c < 5; c++) { s.sg[c] = p; p += m; }
  for (int c = 0; c < 5; c++) { s.F[c] = p; p += f; }
  for (int c = 0; c < 5; c++) { s.F2[c] = p; p += f; }
  s.ph = p; p += m;
  uint8_t* b = reinterpret_cast<uint8_t*>(p);
  s.ids = b; s.real = b + m; s.mask = b + 2 * m;
  return s;
}

__device__ __forceinline__ double tube_x(int i, int n, double h) {
  // MeshGenerator uniform centres (a + h/2 + i h) with the ghost coordinates
  // of SpaceOperator::PopulateGhostBoundaryCoordinates (x_0 - dx, x_{n-1} + dx).
  if (i < 0) return (0.5 * h + 0 * h) - h;
  if (i >= n) return (0.5 * h + (n - 1) * h) + h;
  return 0.5 * h + i * h;
}

// One work item of a stage: cells c0 .. c0+cpb-1 of tube t (all threads of
// the CTA; barriers inside).
__device__ __forceinline__ void tube_stage_item(const TubeArgs& A, const TubeStage& S, const TubeSmem& sm, int t,
                                                int c0) {
  const int cpb = A.cpb;
  const int NT = blockDim.x, tid = threadIdx.x;
  const int ld = cpb + 4;
  const int where = S.stage * 16;
  const double* const* Us = A.U[(S.stage - 2) & 1];
  double* const* Uo = A.U[(S.stage - 1) & 1];
  const double* phin = A.phi[S.cur];
  const double* phin_stage = S.stage == 1 ? phin : A.phis[(S.stage - 2) & 1];
  double* phout = S.final_stage ? A.phi[1 - S.cur] : A.phis[(S.stage - 1) & 1];
  const long long o = A.off[t];
  const int n = (int)(A.off[t + 1] - o);
  const int ce = min(c0 + cpb, n);
  const Eos<double>* eos = A.eos + 2 * t;
  const double dt = A.clock[2 * t + 1];
  const double bdt = S.bdt_coef * dt;
  const bool us_clip = S.stage > 1 && A.clip[4 * t + S.stage - 2];
  const double h = 1.0 / n;
  __syncthreads();
  // load cells c0-2 .. c0+cpb+1 (ghost rules: INLET/OUTLET states, phi by ZERO_NEUMANN)
  for (int j = tid; j < ld; j += NT) {
    const int i = c0 - 2 + j;
    double V[5];
    uint8_t id = 0, real = 0;
    double ph = 0.0;
    if (i >= 0 && i < n) {
      id = A.id[o + i];
      tube_state(A, S, eos[id], o + i, V);
      ph = phin_stage[o + i];
      real = 1;
    } else if (i == -1 || i == n) {
      const int img = i < 0 ? 0 : n - 1;
      id = A.id[o + img];
      const double* b = i < 0 ? A.bcl + 5 * t : A.bcr + 5 * t;
      for (int c = 0; c < 5; c++) V[c] = b[c];
      ph = phin_stage[o + img];
    } else {
      for (int c = 0; c < 5; c++) V[c] = 0.0;
    }
    for (int c = 0; c < 5; c++) sm.v[c][j] = V[c];
    sm.ids[j] = id;
    sm.real[j] = real;
    sm.ph[j] = ph;
  }
  __syncthreads();
  // slopes and revert chain of real cells c0-1 .. c0+cpb
  for (int j = 1 + tid; j < ld - 1; j += NT) {
    if (!sm.real[j]) { sm.mask[j] = 0; continue; }
    const uint8_t id = sm.ids[j];
    const Eos<double>& e = eos[id];
    const bool zx = A.slope_zero && (id != sm.ids[j - 1] || id != sm.ids[j + 1]);
    double v[5], s[5];
    for (int c = 0; c < 5; c++) {
      const double vc = sm.v[c][j];
      v[c] = vc;
      s[c] = A.rec_linear ? limited_slope_c(A.limiter, A.limA, A.limiter == LIM_GENMINMOD ? A.limC : A.limB, A.vak,
                                            A.alpha, vc - sm.v[c][j - 1], sm.v[c][j + 1] - vc)
                          : 0.0;
      if (zx) s[c] = 0.0;
      sm.sg[c][j] = s[c];
    }
    // Reconstructor.cpp:719-775 and SpaceOperator.cpp:3240-3277, faces l, r
    uint8_t m = 0;
    bool chain = false;
    for (int q = 0; q < 2; q++) {
      double f[5];
      for (int c = 0; c < 5; c++) f[c] = q ? v[c] + 0.5 * s[c] : v[c] - 0.5 * s[c];
      const bool bad = e.bad(f);
      bool rev = false;
      if (!chain && bad) { rev = true; chain = true; }
      if (!rev && e.needs_clip(f)) rev = true;
      if (rev) m |= uint8_t(1u << q);
      else if (bad) tube_fail(A, t, ERR_STATE, (int)(o + c0 - 2 + j), where + 1);
    }
    sm.mask[j] = m;
  }
  __syncthreads();
  // faces c0-1/2 .. ce-1/2 (face f: between cells c0+f-1 and c0+f)
  for (int f = tid; f <= ce - c0; f += NT) {
    const int jL = f + 1, jR = f + 2;
    const bool rL = sm.real[jL], rR = sm.real[jR];
    const uint8_t idL = sm.ids[jL], idR = sm.ids[jR];
    double VL[5], VR[5], F[5], F2[5];
    if (rL) {
      const bool rev = sm.mask[jL] & 2;
      for (int c = 0; c < 5; c++) VL[c] = rev ? sm.v[c][jL] : sm.v[c][jL] + 0.5 * sm.sg[c][jL];
    }
    if (rR) {
      const bool rev = sm.mask[jR] & 1;
      for (int c = 0; c < 5; c++) VR[c] = rev ? sm.v[c][jR] : sm.v[c][jR] - 0.5 * sm.sg[c][jR];
    }
    if (!rL) {  // INLET ghost face (Reconstructor.cpp:822-833 + clip check)
      double gc[5];
      for (int c = 0; c < 5; c++) gc[c] = sm.v[c][jL];
      ghost_face(BC_INLET, 0, VR, gc, eos[idL], VL);
    }
    if (!rR) {  // OUTLET ghost face
      double gc[5];
      for (int c = 0; c < 5; c++) gc[c] = sm.v[c][jR];
      ghost_face(BC_OUTLET, 0, VL, gc, eos[idR], VR);
    }
    int err = ERR_NONE;
    if (rL && rR && idL != idR) {
      // material interface (SpaceOperator.cpp:2486-2542)
      double WL[5], WR[5];
      for (int c = 0; c < 5; c++) { WL[c] = sm.v[c][jL]; WR[c] = sm.v[c][jR]; }
      if (A.mp_flux == 2) {
        err = flux_llf2(eos[idL], eos[idR], 0, WL, WR, F);
        for (int c = 0; c < 5; c++) F2[c] = F[c];
      } else {
        const int gi = c0 + f;  // tube-local index of the right cell
        int k = -1;
        const int nf = A.nif[t];
        for (int q = 0; q < nf; q++)
          if (A.iface[t * TUBE_IFACE_CAP + q] == gi) k = q;
        if (k < 0) {
          tube_fail(A, t, ERR_STATE, (int)(o + gi), where + 5);
          for (int c = 0; c < 5; c++) F[c] = F2[c] = 0.0;
        } else {
          const long long b = ((long long)t * TUBE_IFACE_CAP + k) * 5;
          if (A.mp_flux == 0) {
            double Vm[5];
            for (int c = 0; c < 5; c++) Vm[c] = A.Vmid[b + c];
            phys_flux(eos[A.midid[t * TUBE_IFACE_CAP + k]], 0, Vm, F);
            for (int c = 0; c < 5; c++) F2[c] = F[c];
          } else {
            double Sm[5], Sp[5];
            for (int c = 0; c < 5; c++) { Sm[c] = A.Vsm[b + c]; Sp[c] = A.Vsp[b + c]; }
            err = num_flux(A.flux, eos[idL], 0, WL, Sm, A.delta, F);
            if (!err) err = num_flux(A.flux, eos[idR], 0, Sp, WR, A.delta, F2);
          }
        }
      }
    } else {
      err = num_flux(A.flux, eos[rR ? idR : idL], 0, VL, VR, A.delta, F);
      for (int c = 0; c < 5; c++) F2[c] = F[c];
    }
    if (err) tube_fail(A, t, err, (int)(o + c0 + f), where + 2);
    for (int c = 0; c < 5; c++) { sm.F[c][f] = F[c]; sm.F2[c][f] = F2[c]; }
  }
  __syncthreads();
  // residual, RK update, C2P/clip/check; level-set stage
  for (int i = c0 + tid; i < ce; i += NT) {
    const int f = i - c0, j = f + 2;
    const long long q = o + i;
    const uint8_t id = sm.ids[j];
    const Eos<double>& e = eos[id];
    double Vn[5], Un[5], Unew[5];
    for (int c = 0; c < 5; c++) Vn[c] = A.V[S.cur][c][q];
    e.p2c(Vn, Un);
    double u_ls;
    if (S.stage == 1) {
      for (int c = 0; c < 5; c++) Unew[c] = Un[c];
      u_ls = Vn[1];
    } else {
      double Usv[5];
      for (int c = 0; c < 5; c++) Usv[c] = Us[c][q];
      const double inv = 1.0 / Usv[0];
      u_ls = Usv[1] * inv;
      if (us_clip) {
        double Vs[5];
        e.c2p(Usv, Vs);
        e.clip(Vs);
        e.p2c(Vs, Usv);
      }
      for (int c = 0; c < 5; c++) Unew[c] = S.a_prev * Usv[c] + S.a_un * Un[c];
    }
    // y and z faces of the one-cell-wide grid: SYMMETRY ghosts (the cell
    // with its normal velocity negated), zero transverse slopes (the limiter
    // sees differences of opposite sign or zero), so the face states are
    // the cell's own state against its mirror image
    // (SpaceOperator::ComputeAdvectionFluxes, Reconstructor.cpp:822-875).
    // Their fluxes are not exactly zero in general (the star-state
    // arithmetic rounds), so they are formed and summed as the reference
    // sums them.
    double Vc[5], M[5], G[4][5];
    for (int c = 0; c < 5; c++) Vc[c] = sm.v[c][j];
    for (int dd = 1; dd < 3; dd++) {
      for (int c = 0; c < 5; c++) M[c] = Vc[c];
      M[1 + dd] = -M[1 + dd];
      int e2 = num_flux(A.flux, e, dd, M, Vc, A.delta, G[2 * (dd - 1)]);        // low face: ghost | cell
      if (!e2) e2 = num_flux(A.flux, e, dd, Vc, M, A.delta, G[2 * (dd - 1) + 1]);  // high face: cell | ghost
      if (e2) tube_fail(A, t, e2, (int)q, where + 2);
    }
    // residual in the reference's summation order (SpaceOperator.cpp:3351-3409)
    const double vol = h * 1.0 * 1.0;
    const double ax = 1.0 * 1.0, ay = h * 1.0, az = h * 1.0;
    const double inv_mvol = 1.0 / (-vol);
    for (int c = 0; c < 5; c++) {
      double fs = 0.0;
      fs = fs - sm.F2[c][f] * ax;
      fs = fs - G[0][c] * ay;
      fs = fs - G[2][c] * az;
      fs = fs + sm.F[c][f + 1] * ax;
      fs = fs + G[1][c] * ay;
      fs = fs + G[3][c] * az;
      const double R = fs * inv_mvol;
      Unew[c] = Unew[c] + bdt * R;
    }
    double V[5];
    e.c2p(Unew, V);
    if (e.clip(V)) atomicOr(&A.clip[4 * t + S.stage - 1], 1);
    if (e.bad(V)) tube_fail(A, t, ERR_STATE, (int)q, where + 3);
    if (S.final_stage) {
      for (int c = 0; c < 5; c++) A.V[1 - S.cur][c][q] = V[c];
    } else {
      for (int c = 0; c < 5; c++) Uo[c][q] = Unew[c];
    }
    // level set: -(u dphi/dx) with FD3 (LevelSetOperator.cpp:1066-1140)
    const double xi = tube_x(i, n, h);
    const double pc = sm.ph[j];
    double lo, hi;
    if (i - 2 >= -1) {
      double cf[4];
      taylor4(tube_x(i - 2, n, h) - xi, tube_x(i - 1, n, h) - xi, 0.0, tube_x(i + 1, n, h) - xi, cf);
      lo = fd4(cf, sm.ph[j - 2], sm.ph[j - 1], pc, sm.ph[j + 1]);
    } else {
      lo = (pc - sm.ph[j - 1]) / (xi - tube_x(i - 1, n, h));
    }
    if (i + 2 <= n) {
      double cf[4];
      taylor4(tube_x(i - 1, n, h) - xi, 0.0, tube_x(i + 1, n, h) - xi, tube_x(i + 2, n, h) - xi, cf);
      hi = fd4(cf, sm.ph[j - 1], pc, sm.ph[j + 1], sm.ph[j + 2]);
    } else {
      hi = (sm.ph[j + 1] - pc) / (tube_x(i + 1, n, h) - xi);
    }
    const double rphi = ((u_ls >= 0 ? lo * u_ls : hi * u_ls) + 0.0 + 0.0) * -1.0;
    const double base = S.stage == 1 ? phin[q] : S.a_prev * phin_stage[q] + S.a_un * phin[q];
    phout[q] = base + bdt * rphi;
  }
}

__global__ void k_tube_stage(const __grid_constant__ TubeArgs A, const TubeStage S) {
  extern __shared__ __align__(16) unsigned char tube_smem_raw[];
  const TubeSmem sm = tube_smem(tube_smem_raw, A.cpb);
  __shared__ int failed;
  for (int item = blockIdx.x; item < A.nitems; item += gridDim.x) {
    const int2 it = A.items[item];
    __syncthreads();
    if (threadIdx.x == 0) failed = A.terr[it.x];
    __syncthreads();
    if (failed) continue;  // the CTA skips a failed tube's chunk together
    tube_stage_item(A, S, sm, it.x, it.y);
  }
}

// Star state stored on the low (side 0) or high (side 1) face of tube cell i.
__device__ __forceinline__ bool tube_stored(const TubeArgs& A, int t, long long o, int n, int i, int side, double* Sv,
                                            int& sid) {
  const int ci = side ? i + 1 : i;  // right cell of the face
  if (ci <= 0 || ci >= n) return false;
  if (A.idn[o + ci] == A.idn[o + ci - 1]) return false;
  int k = -1;
  const int nf = A.nif[t];
  for (int q = 0; q < nf; q++)
    if (A.iface[t * TUBE_IFACE_CAP + q] == ci) k = q;
  if (k < 0) return false;
  const long long w = (long long)t * TUBE_IFACE_CAP + k;
  if (!A.rsValid[w]) return false;
  const double* src = side == 0 ? A.rsVsm : A.rsVsp;
  for (int c = 0; c < 5; c++) Sv[c] = src[w * 5 + c];
  sid = side == 0 ? A.idn[o + ci - 1] : A.idn[o + ci];
  return true;
}

// LocalUpdateByRiemannSolutions (MultiPhaseOperator.cpp:916-1027) on one axis.
__device__ int tube_local_update(const TubeArgs& A, double* const* V, int t, long long o, int n, int i, int myid,
                                 double* v, bool upwind) {
  int counter = 0;
  double weight = 0, sum_weight = 0;
  for (int side = 0; side < 2; side++) {
    double Sv[5];
    int sid;
    if (!tube_stored(A, t, o, n, i, side, Sv, sid)) continue;
    if (sid != myid) continue;
    const long long nq = o + (side ? i + 1 : i - 1);
    double nv[5];
    for (int p = 0; p < 5; p++) nv[p] = V[p][nq];
    const double vn = nv[1];
    if (upwind && !(side == 0 ? vn > 0 : vn < 0)) continue;
    const double nrm = sqrt(nv[1] * nv[1] + nv[2] * nv[2] + nv[3] * nv[3]);
    weight = upwind ? (side == 0 ? vn / nrm : -vn / nrm) : 1.0;
    sum_weight += weight;
    if (counter == 0) {
      for (int p = 0; p < 5; p++) v[p] = weight * Sv[p];
    } else {
      for (int p = 0; p < 5; p++) v[p] += weight * Sv[p];
    }
    counter++;
  }
  if (sum_weight > 0.0) {
    const double inv = 1.0 / sum_weight;
    for (int p = 0; p < 5; p++) v[p] *= inv;
  }
  return counter;
}

// Material ID from the sign change of phi and the ordered update of cells
// whose ID changed (MultiPhaseOperator.cpp:127-332, 824-1027); one warp per tube.
__device__ void tube_end(const TubeArgs& A, int t, int cur_new, int lane) {
  if (__shfl_sync(0xffffffffu, lane == 0 ? A.terr[t] : 0, 0)) return;
  const long long o = A.off[t];
  const int n = (int)(A.off[t + 1] - o);
  const double* phnew = A.phi[cur_new];
  const double* phold = A.phi[1 - cur_new];
  for (int i = lane; i < n; i += 32) {
    const double p = phnew[o + i], p0 = phold[o + i];
    if (p * p0 > 0.0) continue;
    A.id[o + i] = p < 0 ? (uint8_t)1 : (uint8_t)0;
  }
  __syncwarp();
  double* const* V = A.V[cur_new];
  int unresolved = 0;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    const bool ch = i < n && A.id[o + i] != A.idn[o + i];
    unsigned bal = __ballot_sync(0xffffffffu, ch);
    if (lane == 0) {
      while (bal) {
        const int b = __ffs(bal) - 1;
        bal &= bal - 1;
        const int ci = i0 + b;
        const int myid = A.id[o + ci];
        double v[5];
        for (int p = 0; p < 5; p++) v[p] = V[p][o + ci];
        int counter = tube_local_update(A, V, t, o, n, ci, myid, v, true);
        if (counter == 0) counter = tube_local_update(A, V, t, o, n, ci, myid, v, false);
        if (counter == 0) {
          unresolved++;
          continue;
        }
        const Eos<double>& e = A.eos[2 * t + myid];
        e.clip(v);
        if (e.bad(v)) tube_fail(A, t, ERR_STATE, (int)(o + ci), 9);
        for (int p = 0; p < 5; p++) V[p][o + ci] = v[p];
      }
    }
    __syncwarp();
  }
  if (lane == 0 && unresolved) atomicAdd(&A.cnt[3], (unsigned long long)unresolved);
}

__global__ void k_tube_end(TubeArgs A, int cur_new) {
  const int lane = threadIdx.x & 31;
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (t >= A.ntubes) return;
  tube_end(A, t, cur_new, lane);
}

// The whole run in one persistent launch: tubes are independent (each has
// its own CFL time step), so a CTA takes the next tube from a work counter
// (tubes ordered longest first) and advances it by nsteps complete steps on
// its own: warp 0 computes the time step and the interface faces, the
// interface Riemann problems are solved by one thread each, every thread
// works on the stage's cell chunks, and warp 0 makes the ID and ordered state
// update; CTA barriers order the phases. No CTA waits on another. A slow
// interface solve delays only its own tube.
__global__ void __launch_bounds__(128) k_tube_run(const __grid_constant__ TubeArgs A, int nsteps, int cur0,
                                                  int* next, const int* order) {
  extern __shared__ __align__(16) unsigned char tube_smem_raw[];
  const TubeSmem sm = tube_smem(tube_smem_raw, A.cpb);
  __shared__ int tube;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  RiemannSolver rs;
  rs.P = A.P;
  if (threadIdx.x < TUBE_IFACE_CAP) {
    rs.path1.pt = A.scratch + ((long long)blockIdx.x * TUBE_IFACE_CAP + threadIdx.x) * 2 * 3 * RIEMANN_PATH_CAP;
    rs.path1.cap = RIEMANN_PATH_CAP;
    rs.path3.pt = rs.path1.pt + 3 * RIEMANN_PATH_CAP;
    rs.path3.cap = RIEMANN_PATH_CAP;
  }
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const int w = atomicAdd(next, 1);
      tube = w < A.ntubes ? order[w] : -1;
    }
    __syncthreads();
    const int t = tube;
    if (t < 0) return;
    const int n = (int)(A.off[t + 1] - A.off[t]);
    int cur = cur0;
    __shared__ int failed;
    for (int step = 0; step < nsteps; step++) {
      __syncthreads();
      if (threadIdx.x == 0) failed = A.terr[t];
      __syncthreads();
      if (failed) break;  // a tube that reported an error stops where it failed
      if (warp == 0) tube_begin(A, t, cur, lane);
      __syncthreads();
      for (int st = 1; st <= A.rk; st++) {
        TubeStage S;
        S.stage = st;
        S.final_stage = st == A.rk;
        S.cur = cur;
        S.a_prev = 0.0; S.a_un = 1.0; S.bdt_coef = 1.0;
        if (st > 1) {
          if (A.rk == 2) { S.a_prev = 0.5; S.a_un = 0.5; S.bdt_coef = 0.5; }
          else if (st == 2) { S.a_prev = 0.25; S.a_un = 0.75; S.bdt_coef = 0.25; }
          else { S.a_prev = 2.0 / 3.0; S.a_un = 1.0 / 3.0; S.bdt_coef = 2.0 / 3.0; }
        }
        if ((int)threadIdx.x < A.nif[t]) tube_riemann(A, S, t, threadIdx.x, rs);
        __syncthreads();
        for (int c0 = 0; c0 < n; c0 += A.cpb) tube_stage_item(A, S, sm, t, c0);
        __syncthreads();
      }
      if (warp == 0) tube_end(A, t, 1 - cur, lane);
      __syncthreads();
      cur = 1 - cur;
    }
  }
}

}  // namespace m2c

using namespace m2c;

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct m2cg_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  m2cg_scheme scheme;
  int ntubes = 0;
  long long ncell = 0;
  TubeArgs A;
  m2cg_batch_tuning tuning;
  int cur = 0;
  long long steps = 0;
  std::vector<char*> allocs;
  int2* items = nullptr;
  int stage_grid = 0;
  int stage_threads = 0;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};  // one step from cur 0, from cur 1, two steps from 0
  // host copies for re-initialisation
  std::vector<double> hV, hphi;
  std::vector<uint8_t> hid;
  long long launches = 0;
  // learned warm start (optional)
  const m2cg_mlp* mlp = nullptr;
  float* fX = nullptr;
  double* fP = nullptr;
  int* fvalid = nullptr;
  float* fy = nullptr;
  double* fwarm = nullptr;
  // one persistent launch per run (use_graph == 2): tubes longest first, the
  // work counter, and the grid
  int* run_order = nullptr;
  int* run_next = nullptr;
  int run_grid = 0;
};

static m2cg_status bfail(m2cg_status st, const char* msg) {
  set_last_error(msg);
  return st;
}

static void rk_coefs(int r, int s, double& a_prev, double& a_un, double& bdt) {
  a_prev = 0.0; a_un = 1.0; bdt = 1.0;
  if (s == 1) return;
  if (r == 2) { a_prev = 0.5; a_un = 0.5; bdt = 0.5; return; }
  if (s == 2) { a_prev = 0.25; a_un = 0.75; bdt = 0.25; return; }
  a_prev = 2.0 / 3.0; a_un = 1.0 / 3.0; bdt = 2.0 / 3.0;
}

static cudaError_t set_items(m2cg_batch* b, int cpb) {
  std::vector<int2> items;
  // longest tubes first so the tail of the persistent loop holds short work
  std::vector<int> order(b->ntubes);
  std::vector<long long> off(b->ntubes + 1);
  for (int t = 0; t < b->ntubes; t++) order[t] = t;
  std::vector<int> len(b->ntubes);
  {
    std::vector<long long> h(b->ntubes + 1);
    cudaMemcpy(h.data(), b->A.off, sizeof(long long) * (b->ntubes + 1), cudaMemcpyDeviceToHost);
    for (int t = 0; t < b->ntubes; t++) len[t] = (int)(h[t + 1] - h[t]);
  }
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return len[x] > len[y]; });
  for (int t : order)
    for (int c = 0; c < len[t]; c += cpb) items.push_back(make_int2(t, c));
  if (b->items) cudaFree(b->items);
  cudaError_t e = cudaMalloc((void**)&b->items, items.size() * sizeof(int2));
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(b->items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice);
  b->A.items = b->items;
  b->A.nitems = (int)items.size();
  b->A.cpb = cpb;
  return e;
}

static cudaError_t configure_stage(m2cg_batch* b, int threads, int cpb) {
  const size_t smem = tube_smem_bytes(cpb);
  cudaError_t e = cudaFuncSetAttribute(k_tube_stage, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tube_stage, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  e = set_items(b, cpb);
  if (e != cudaSuccess) return e;
  b->stage_threads = threads;
  b->stage_grid = std::min(b->A.nitems, per_sm * nsm);
  b->tuning.cells_per_block = cpb;
  b->tuning.threads_per_block = threads;
  return cudaSuccess;
}

// The persistent whole-run kernel's grid for the current cells_per_block:
// resident CTAs of 128 threads, at most one per tube and at most the
// Riemann scratch's CTA slots.
static cudaError_t configure_run(m2cg_batch* b) {
  const size_t smem = tube_smem_bytes(b->A.cpb);
  cudaError_t e = cudaFuncSetAttribute(k_tube_run, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0, nsm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tube_run, 128, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  b->run_grid = std::min(std::min(per_sm * nsm, b->ntubes), TUBE_RIEMANN_THREADS / TUBE_IFACE_CAP);
  return cudaSuccess;
}

// nsteps steps of every tube in one launch of the persistent kernel.
static cudaError_t enqueue_run(m2cg_batch* b, int nsteps) {
  cudaError_t e = cudaMemsetAsync(b->run_next, 0, sizeof(int), b->stream);
  if (e != cudaSuccess) return e;
  k_tube_run<<<b->run_grid, 128, tube_smem_bytes(b->A.cpb), b->stream>>>(b->A, nsteps, b->cur, b->run_next,
                                                                         b->run_order);
  b->cur ^= nsteps & 1;
  return cudaGetLastError();
}

// Queue one step starting from state parity `cur`.
static cudaError_t enqueue_step(m2cg_batch* b, int cur) {
  TubeArgs& A = b->A;
  const int warps_blocks = (b->ntubes * 32 + 255) / 256;
  k_tube_begin<<<warps_blocks, 256, 0, b->stream>>>(A, cur);
  const int r = b->scheme.rk_order;
  const size_t smem = tube_smem_bytes(A.cpb);
  for (int s = 1; s <= r; s++) {
    TubeStage S;
    S.stage = s;
    S.final_stage = s == r;
    S.cur = cur;
    rk_coefs(r, s, S.a_prev, S.a_un, S.bdt_coef);
    if (b->mlp) {
      const int nslot = b->ntubes * TUBE_IFACE_CAP;
      k_tube_features<<<(nslot + 255) / 256, 256, 0, b->stream>>>(A, S, b->fX, b->fP, b->fvalid);
      mlp_warm_device(b->mlp, b->stream, b->fX, b->fvalid, b->fP, nslot, b->fy, b->fwarm, nullptr);
    }
    k_tube_riemann<<<TUBE_RIEMANN_THREADS / 64, 64, 0, b->stream>>>(A, S);
    k_tube_stage<<<b->stage_grid, b->stage_threads, smem, b->stream>>>(A, S);
  }
  k_tube_end<<<warps_blocks, 256, 0, b->stream>>>(A, 1 - cur);
  return cudaGetLastError();
}

static void destroy_graphs(m2cg_batch* b) {
  for (auto& g : b->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

static cudaError_t capture(m2cg_batch* b, int first_cur, int nsteps, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  int cur = first_cur;
  cudaError_t le = cudaSuccess;
  for (int k = 0; k < nsteps; k++) {
    cudaError_t q = enqueue_step(b, cur);
    if (le == cudaSuccess) le = q;
    cur = 1 - cur;
  }
  e = cudaStreamEndCapture(b->stream, &g);
  if (e == cudaSuccess) e = le;
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
  if (g) cudaGraphDestroy(g);
  return e;
}

static cudaError_t build_graphs(m2cg_batch* b) {
  destroy_graphs(b);
  cudaError_t e = capture(b, 0, 1, &b->graph[0]);
  if (e == cudaSuccess) e = capture(b, 1, 1, &b->graph[1]);
  if (e == cudaSuccess) e = capture(b, 0, 2, &b->graph[2]);
  return e;
}

static cudaError_t reset_state(m2cg_batch* b) {
  const long long N = b->ncell;
  cudaError_t e = cudaSuccess;
  for (int c = 0; c < 5 && e == cudaSuccess; c++)
    e = cudaMemcpyAsync(b->A.V[0][c], b->hV.data() + c * N, N * 8, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->A.phi[0], b->hphi.data(), N * 8, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->A.id, b->hid.data(), N, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->A.clock, 0, sizeof(double) * 2 * b->ntubes, b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->A.terr, 0, sizeof(int) * b->ntubes, b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->A.cnt, 0, sizeof(unsigned long long) * 8, b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->A.err, 0, sizeof(DevError), b->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->A.rsValid, 0, (size_t)b->ntubes * TUBE_IFACE_CAP, b->stream);
  b->cur = 0;
  b->steps = 0;
  return e;
}

// Measured choice of (threads_per_block, cells_per_block, launch mode): each
// candidate advances a copy of the initial state by a few steps, the fastest
// wins, and the state is restored afterwards. Modes: 1 = the step sequence as
// kernels per phase (graph-replayed), 2 = one persistent launch per run
// (128 threads). fix_mode 0 tries both.
static cudaError_t autotune(m2cg_batch* b, int fix_threads, int fix_cpb, int fix_mode) {
  const int cand[][3] = {{128, 128, 1}, {128, 256, 1}, {256, 256, 1}, {256, 512, 1}, {128, 512, 1}, {512, 512, 1},
                         {256, 1024, 1}, {512, 1024, 1}, {64, 128, 1}, {256, 128, 1},
                         {128, 256, 2}, {128, 512, 2}, {128, 1024, 2}};
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
  float best = 1e30f;
  int bt = 0, bc = 0, bm = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t err = cudaSuccess;
  for (auto& c : cand) {
    const int mode = c[2];
    if (fix_mode && (fix_mode == 2) != (mode == 2)) continue;
    if (mode == 2 && fix_threads && fix_threads != 128) continue;
    const int th = mode == 2 ? 128 : (fix_threads ? fix_threads : c[0]), cpb = fix_cpb ? fix_cpb : c[1];
    if (tube_smem_bytes(cpb) > (size_t)maxsm) continue;
    if (configure_stage(b, th, cpb) != cudaSuccess || (mode == 2 && configure_run(b) != cudaSuccess)) {
      cudaGetLastError();
      continue;
    }
    err = reset_state(b);
    if (err != cudaSuccess) break;
    if (mode == 2) {
      enqueue_run(b, 1);  // warm-up
      cudaEventRecord(e0, b->stream);
      enqueue_run(b, 2);
    } else {
      int cur = 0;
      enqueue_step(b, cur);  // warm-up
      cur = 1 - cur;
      cudaEventRecord(e0, b->stream);
      for (int k = 0; k < 2; k++) {
        enqueue_step(b, cur);
        cur = 1 - cur;
      }
    }
    cudaEventRecord(e1, b->stream);
    err = cudaEventSynchronize(e1);
    if (err != cudaSuccess) break;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) { best = ms; bt = th; bc = cpb; bm = mode; }
    if (fix_threads && fix_cpb && fix_mode) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return err;
  if (!bt) return cudaErrorInvalidConfiguration;
  err = configure_stage(b, bt, bc);
  if (err == cudaSuccess && bm == 2) err = configure_run(b);
  if (err == cudaSuccess) err = reset_state(b);
  if (bm == 2) b->tuning.use_graph = 2;
  return err;
}

static int van_albada_k() {
  // uniform tube meshes: A = B = 1 (Reconstructor.cpp:103-121)
  for (int k = 2; k < 1000; k++) {
    const double rhs = 2.0 / (1.0 + m2c::cr_pow_int((k - 1.0) / k, k - 1) / k) * std::min(1.0, 1.0);
    if (1.0 <= rhs) return k;
  }
  return -1;
}

extern "C" m2cg_status m2cg_batch_create(const m2cg_scheme* scheme, int ntubes, const int* len,
                                         const m2cg_material* mats, const double* VL, const double* VR,
                                         const m2cg_batch_tuning* tuning, m2cg_batch** out) {
  if (!scheme || ntubes < 1 || !len || !mats || !VL || !VR || !out) return bfail(M2CG_ERR_ARG, "null argument");
  *out = nullptr;
  if (scheme->flux < 0 || scheme->flux > 2) return bfail(M2CG_ERR_UNSUPPORTED, "flux not supported");
  if (scheme->rec_var != M2CG_RECVAR_PRIMITIVE)
    return bfail(M2CG_ERR_UNSUPPORTED, "only primitive-variable reconstruction is implemented");
  if (scheme->rk_order < 1 || scheme->rk_order > 3) return bfail(M2CG_ERR_ARG, "rk_order must be 1, 2 or 3");
  for (int q = 0; q < 2 * ntubes; q++)
    if (mats[q].mu != 0.0 || mats[q].mu_bulk != 0.0 || mats[q].heat_diffusivity != 0.0)
      return bfail(M2CG_ERR_UNSUPPORTED, "viscous or heat-diffusive materials are not implemented for the batched tubes");
  if (scheme->mp_recon != 0 || scheme->mp_phasechange_type != 0)
    return bfail(M2CG_ERR_UNSUPPORTED, "interface recon must be CONSTANT with the Riemann-solution update");
  long long N = 0;
  for (int t = 0; t < ntubes; t++) {
    if (len[t] < 4) return bfail(M2CG_ERR_ARG, "every tube needs at least 4 cells");
    N += len[t];
  }
  if (N > 0x7fffffffLL) return bfail(M2CG_ERR_ARG, "more than 2^31 cells in a batch");
  if (tuning && tuning->use_graph == 2 && tuning->threads_per_block != 0 && tuning->threads_per_block != 128)
    return bfail(M2CG_ERR_ARG, "the persistent launch (use_graph 2) runs 128 threads per block");
  m2cg_batch* b = new m2cg_batch;
  b->scheme = *scheme;
  b->ntubes = ntubes;
  b->ncell = N;
  memset(&b->A, 0, sizeof b->A);
  cudaGetDevice(&b->device);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return bfail(M2CG_ERR_CUDA, "cudaStreamCreate failed (no CUDA device?)");
  }
  bool ok = true;
  auto alloc = [&](size_t bytes) -> char* {
    char* p = nullptr;
    if (cudaMalloc((void**)&p, bytes ? bytes : 16) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    b->allocs.push_back(p);
    return p;
  };
  TubeArgs& A = b->A;
  const int T = ntubes;
  A.ntubes = T;
  A.ncell = N;
  A.off = (const long long*)alloc(sizeof(long long) * (T + 1));
  A.eos = (const Eos<double>*)alloc(sizeof(Eos<double>) * 2 * T);
  A.bcl = (const double*)alloc(sizeof(double) * 5 * T);
  A.bcr = (const double*)alloc(sizeof(double) * 5 * T);
  A.clock = (double*)alloc(sizeof(double) * 2 * T);
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 5; c++) {
      A.V[s][c] = (double*)alloc(N * 8);
      A.U[s][c] = (double*)alloc(N * 8);
    }
  for (int s = 0; s < 2; s++) {
    A.phi[s] = (double*)alloc(N * 8);
    A.phis[s] = (double*)alloc(N * 8);
  }
  A.id = (uint8_t*)alloc(N);
  A.idn = (uint8_t*)alloc(N);
  A.nif = (int*)alloc(sizeof(int) * T);
  A.iface = (int*)alloc(sizeof(int) * T * TUBE_IFACE_CAP);
  A.Vsm = (double*)alloc(sizeof(double) * 5 * T * TUBE_IFACE_CAP);
  A.Vsp = (double*)alloc(sizeof(double) * 5 * T * TUBE_IFACE_CAP);
  A.Vmid = (double*)alloc(sizeof(double) * 5 * T * TUBE_IFACE_CAP);
  A.midid = (int*)alloc(sizeof(int) * T * TUBE_IFACE_CAP);
  A.rsVsm = (double*)alloc(sizeof(double) * 5 * T * TUBE_IFACE_CAP);
  A.rsVsp = (double*)alloc(sizeof(double) * 5 * T * TUBE_IFACE_CAP);
  A.rsValid = (uint8_t*)alloc((size_t)T * TUBE_IFACE_CAP);
  A.clip = (int*)alloc(sizeof(int) * 4 * T);
  A.terr = (int*)alloc(sizeof(int) * T);
  A.cnt = (unsigned long long*)alloc(sizeof(unsigned long long) * 8);
  A.err = (DevError*)alloc(sizeof(DevError));
  A.scratch = (double*)alloc(sizeof(double) * (size_t)TUBE_RIEMANN_THREADS * 2 * 3 * RIEMANN_PATH_CAP);
  if (!ok) {
    m2cg_batch_destroy(b);
    return bfail(M2CG_ERR_NOMEM, "device allocation for the batch failed");
  }
  // scheme parameters
  A.flux = scheme->flux;
  A.limiter = scheme->limiter;
  A.rec_linear = scheme->rec_type == M2CG_REC_LINEAR;
  A.slope_zero = scheme->slope_near_interface == 0;
  A.mp_flux = scheme->mp_flux;
  A.rk = scheme->rk_order;
  A.alpha = scheme->minmod_coeff;
  A.delta = scheme->roe_delta;
  A.cfl = scheme->cfl;
  A.limA = 1.0;
  A.limB = 1.0;
  A.limC = 1.0 / (1.0 + 1.0);
  A.vak = scheme->limiter == M2CG_LIM_VANALBADA ? van_albada_k() : 0;
  A.P = riemann_params(*scheme);
  A.warm = nullptr;
  // tubes: offsets, materials, boundary states, initial state
  std::vector<long long> off(T + 1, 0);
  std::vector<Eos<double>> heos(2 * T);
  for (int t = 0; t < T; t++) {
    off[t + 1] = off[t] + len[t];
    for (int m = 0; m < 2; m++) {
      const m2cg_material& q = mats[2 * t + m];
      MatParams p;
      p.kind = q.eos; p.gam = q.gamma; p.pc = q.p_c; p.b = q.b; p.q = q.q;
      p.rhomin = q.rhomin; p.pmin = q.pmin; p.rhomax = q.rhomax; p.pmax = q.pmax;
      p.failsafe_density = q.failsafe_density;
      heos[2 * t + m] = make_eos<double>(p);
    }
  }
  b->hV.assign(5 * N, 0.0);
  b->hphi.assign(N, 0.0);
  b->hid.assign(N, 0);
  for (int t = 0; t < T; t++) {
    const int n = len[t];
    const double h = (1.0 - 0.0) / n;
    for (int i = 0; i < n; i++) {
      const double x = 0.0 + 0.5 * h + i * h;
      const double ph = 0.5 - x;
      const int m = ph < 0 ? 1 : 0;
      const double* src = m ? VR + 5 * t : VL + 5 * t;
      const long long q = off[t] + i;
      for (int c = 0; c < 5; c++) b->hV[c * N + q] = src[c];
      b->hphi[q] = ph;
      b->hid[q] = (uint8_t)m;
    }
  }
  cudaError_t e = cudaMemcpy((void*)A.off, off.data(), sizeof(long long) * (T + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy((void*)A.eos, heos.data(), sizeof(Eos<double>) * 2 * T, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy((void*)A.bcl, VL, sizeof(double) * 5 * T, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy((void*)A.bcr, VR, sizeof(double) * 5 * T, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    m2cg_batch_destroy(b);
    return bfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  }
  // the persistent kernel's tube order (longest first) and work counter
  {
    std::vector<int> ord(T);
    for (int t = 0; t < T; t++) ord[t] = t;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return len[x] > len[y]; });
    b->run_order = (int*)alloc(sizeof(int) * T);
    b->run_next = (int*)alloc(sizeof(int));
    if (!ok) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaMemcpy(b->run_order, ord.data(), sizeof(int) * T, cudaMemcpyHostToDevice);
  }
  const int fix_t = tuning ? tuning->threads_per_block : 0;
  const int fix_c = tuning ? tuning->cells_per_block : 0;
  // use_graph: 0 kernels per phase launched directly, 1 the same captured in
  // graphs, 2 one persistent launch per run; without a tuning both 1 and 2
  // are measured
  const int mode = tuning ? tuning->use_graph : -1;
  b->tuning.use_graph = mode < 0 ? 1 : mode;
  if (e == cudaSuccess) e = autotune(b, fix_t, fix_c, mode < 0 ? 0 : (mode == 2 ? 2 : 1));
  if (e == cudaSuccess && b->tuning.use_graph == 1) e = build_graphs(b);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof msg, "batch setup failed: %s", cudaGetErrorString(e));
    m2cg_batch_destroy(b);
    return bfail(M2CG_ERR_CUDA, msg);
  }
  *out = b;
  return M2CG_OK;
}

static m2cg_status batch_check(m2cg_batch* b) {
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return bfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  DevError h;
  if (cudaMemcpy(&h, b->A.err, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return bfail(M2CG_ERR_CUDA, "read-back failed");
  if (h.code) {
    char msg[200];
    snprintf(msg, sizeof msg, "device error %d at cell %d (site %d)", h.code, h.cell, h.where);
    set_last_error(msg);
    if (h.code == ERR_ITER_CAP) return M2CG_ERR_ITER_CAP;
    return M2CG_ERR_STATE;
  }
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_batch_run(m2cg_batch* b, int nsteps) {
  if (!b || nsteps < 0) return bfail(M2CG_ERR_ARG, "bad argument");
  int left = nsteps;
  cudaError_t e = cudaSuccess;
  if (b->tuning.use_graph == 2) {
    if (nsteps > 0) e = enqueue_run(b, nsteps);
  } else if (b->tuning.use_graph) {
    if (left > 0 && b->cur == 1) {
      e = cudaGraphLaunch(b->graph[1], b->stream);
      b->cur = 0;
      left--;
    }
    while (e == cudaSuccess && left >= 2) {
      e = cudaGraphLaunch(b->graph[2], b->stream);
      left -= 2;
    }
    if (e == cudaSuccess && left == 1) {
      e = cudaGraphLaunch(b->graph[0], b->stream);
      b->cur = 1;
      left = 0;
    }
  } else {
    for (; left > 0 && e == cudaSuccess; left--) {
      e = enqueue_step(b, b->cur);
      b->cur = 1 - b->cur;
    }
  }
  if (e != cudaSuccess) return bfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  b->steps += nsteps;
  b->launches += b->tuning.use_graph == 2 ? 1 : (long long)nsteps * (2 + (b->mlp ? 5 : 2) * b->scheme.rk_order);
  return batch_check(b);
}

extern "C" m2cg_status m2cg_batch_download(m2cg_batch* b, double* V, int* ID, double* t_per_tube) {
  if (!b) return bfail(M2CG_ERR_ARG, "null argument");
  // a tube's error stops that tube only: the states are still copied (the
  // failed tubes' are not defined) and the status names the error
  const m2cg_status st = batch_check(b);
  if (st == M2CG_ERR_CUDA) return st;
  const long long N = b->ncell;
  if (V) {
    std::vector<double> tmp(N);
    for (int c = 0; c < 5; c++) {
      if (cudaMemcpy(tmp.data(), b->A.V[b->cur][c], N * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return bfail(M2CG_ERR_CUDA, "download failed");
      for (long long q = 0; q < N; q++) V[5 * q + c] = tmp[q];
    }
  }
  if (ID) {
    std::vector<uint8_t> tmp(N);
    if (cudaMemcpy(tmp.data(), b->A.id, N, cudaMemcpyDeviceToHost) != cudaSuccess)
      return bfail(M2CG_ERR_CUDA, "download failed");
    for (long long q = 0; q < N; q++) ID[q] = tmp[q];
  }
  if (t_per_tube) {
    std::vector<double> clk(2 * b->ntubes);
    if (cudaMemcpy(clk.data(), b->A.clock, sizeof(double) * 2 * b->ntubes, cudaMemcpyDeviceToHost) != cudaSuccess)
      return bfail(M2CG_ERR_CUDA, "download failed");
    for (int t = 0; t < b->ntubes; t++) t_per_tube[t] = clk[2 * t];
  }
  return st;
}

extern "C" m2cg_status m2cg_batch_get_tuning(const m2cg_batch* b, m2cg_batch_tuning* t) {
  if (!b || !t) return bfail(M2CG_ERR_ARG, "null argument");
  *t = b->tuning;
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_batch_get_counters(m2cg_batch* b, m2cg_counters* c) {
  if (!b || !c) return bfail(M2CG_ERR_ARG, "null argument");
  unsigned long long h[8];
  if (cudaMemcpy(h, b->A.cnt, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return bfail(M2CG_ERR_CUDA, "read-back failed");
  memset(c, 0, sizeof *c);
  c->steps = b->steps;
  c->cells_updated = b->steps * b->ncell;
  c->riemann_calls = (long long)h[0];
  c->riemann_iterations = (long long)h[1];
  c->riemann_errors = (long long)h[2];
  c->unresolved_cells = (long long)h[3];
  c->kernel_launches = b->launches;
  c->riemann_evaluations = (long long)h[5];
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_batch_tube_errors(m2cg_batch* b, int* codes) {
  if (!b || !codes) return bfail(M2CG_ERR_ARG, "null argument");
  if (cudaMemcpy(codes, b->A.terr, sizeof(int) * b->ntubes, cudaMemcpyDeviceToHost) != cudaSuccess)
    return bfail(M2CG_ERR_CUDA, "read-back failed");
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_batch_time_steps(m2cg_batch* b, int nsteps, float* ms) {
  if (!b || !ms) return bfail(M2CG_ERR_ARG, "null argument");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, b->stream);
  m2cg_status st = M2CG_OK;
  // same launch sequence as m2cg_batch_run, without the per-call error check
  int left = nsteps;
  cudaError_t e = cudaSuccess;
  if (b->tuning.use_graph == 2) {
    if (nsteps > 0) e = enqueue_run(b, nsteps);
  } else if (b->tuning.use_graph) {
    if (left > 0 && b->cur == 1) { e = cudaGraphLaunch(b->graph[1], b->stream); b->cur = 0; left--; }
    while (e == cudaSuccess && left >= 2) { e = cudaGraphLaunch(b->graph[2], b->stream); left -= 2; }
    if (e == cudaSuccess && left == 1) { e = cudaGraphLaunch(b->graph[0], b->stream); b->cur = 1; }
  } else {
    for (; left > 0 && e == cudaSuccess; left--) { e = enqueue_step(b, b->cur); b->cur = 1 - b->cur; }
  }
  cudaEventRecord(e1, b->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e != cudaSuccess) st = bfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  if (!st) cudaEventElapsedTime(ms, e0, e1);  // written even when a tube reports an error below
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->steps += nsteps;
  b->launches += b->tuning.use_graph == 2 ? 1 : (long long)nsteps * (2 + (b->mlp ? 5 : 2) * b->scheme.rk_order);
  if (st) return st;
  return batch_check(b);
}

extern "C" m2cg_status m2cg_batch_set_mlp(m2cg_batch* b, const m2cg_mlp* m) {
  if (!b) return bfail(M2CG_ERR_ARG, "null argument");
  cudaStreamSynchronize(b->stream);
  const size_t nslot = (size_t)b->ntubes * TUBE_IFACE_CAP;
  if (m && !b->fX) {
    if (cudaMalloc((void**)&b->fX, nslot * MLP_IN * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&b->fP, 2 * nslot * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&b->fvalid, nslot * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&b->fy, nslot * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&b->fwarm, nslot * sizeof(double)) != cudaSuccess)
      return bfail(M2CG_ERR_NOMEM, "warm-start buffers: allocation failed");
  }
  b->mlp = m;
  b->A.warm = m ? b->fwarm : nullptr;
  // the network's inference runs over all tubes between phases, which the
  // persistent whole-run kernel does not have: use the graph-replayed steps
  if (m && b->tuning.use_graph == 2) {
    cudaError_t e = configure_stage(b, 128, b->A.cpb);
    if (e != cudaSuccess) return bfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
    b->tuning.use_graph = 1;
  }
  if (b->tuning.use_graph == 1) {
    cudaError_t e = build_graphs(b);
    if (e != cudaSuccess) return bfail(M2CG_ERR_CUDA, cudaGetErrorString(e));
  }
  return M2CG_OK;
}

extern "C" m2cg_status m2cg_batch_destroy(m2cg_batch* b) {
  if (!b) return M2CG_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  destroy_graphs(b);
  cudaFree(b->fX); cudaFree(b->fP); cudaFree(b->fvalid); cudaFree(b->fy); cudaFree(b->fwarm);
  for (char* p : b->allocs) cudaFree(p);
  if (b->items) cudaFree(b->items);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return M2CG_OK;
}
