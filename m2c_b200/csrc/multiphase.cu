// Two-material machinery of the time step on the GPU: one level set,
// material IDs, the exact Riemann problems at material interfaces and the
// post-step state update of cells that changed material.
//
// Per step (TimeIntegratorRK2/RK3::AdvanceOneTimeStep + UpdateSolutionAfterTimeStepping,
// TimeIntegrator.cpp:291-797):
//   begin: Phi_tmp = Phi, IDn = ID; interface faces (ID differs across a
//          face) are collected once, since IDs are fixed during the stages.
//   stage s: exact Riemann problem on every interface face with the stage's
//          cell states (SpaceOperator.cpp:2486-2542, MultiPhase recon CONSTANT);
//          stage 1 keeps its star states as the "riemann_solutions" of the
//          reference (RiemannSolutions.h); level-set RK stage with the stage's
//          velocity (LevelSetOperator::ComputeResidualFDM_FullDomain, 1066-1140);
//          the fused N-S stage kernel consumes the star states.
//   end:   material ID from the sign change of phi
//          (MultiPhaseOperator::UpdateMaterialIDByLevelSet, 127-332), optional
//          reinitialisation, and the state update of cells whose ID changed
//          from the stored star states with upwind weights
//          (UpdateStateVariablesByRiemannSolutions / LocalUpdateByRiemannSolutions,
//          857-1027), processed in the reference's (k, j, i) order because
//          each update reads neighbours already updated in the same pass.
//
// Compiled with -fmad=false (FP64 path).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "levelset.h"
#include "ls_device.cuh"
#include "multiphase.h"
#include "mlp.cuh"
#include "riemann_batch.h"

namespace m2c {
cudaError_t mlp_warm_device(const m2cg_mlp* m, cudaStream_t s, const float* X, const int* valid, const double* P,
                            int n, float* y, double* warm, const int* ndev);

// Threads running Riemann problems at once (each owns an integration-path
// scratch region of 2 x RIEMANN_PATH_CAP x 3 doubles).
constexpr int IFACE_RIEMANN_THREADS = 148 * 4 * 128;
// Resident CTAs of 128 threads per SM the interface Riemann kernel is
// compiled for (register budget 65536 / (128 * M2C_IFACE_MINB) per thread).
// Measured on the 384^3 bubble cluster (mixed, 10 steps): 2 CTAs (255
// registers) 130.7 ms per step, 3 (168) 125.9 ms, 4 (128, with spills to L1)
// 122.2 ms: the solve is latency-bound, so more resident warps win over the
// spill traffic.
#ifndef M2C_IFACE_MINB
#define M2C_IFACE_MINB 4
#endif

struct Multiphase {
  Grid3 g;
  SchemeK sk;
  m2cg_scheme scheme;
  m2cg_levelset ls;
  RiemannParams rp;
  Eos<double>* d_eos = nullptr;  // material table on the device
  long long ncell = 0;           // allocated cells (plane * nz)
  // level set buffers (interior, SoA single component, same indexing as V)
  double* phiN = nullptr;  // phi^n / phi^{n+1}
  double* phiA = nullptr;  // stage 1 output
  double* phiB = nullptr;  // stage 2 output (RK3)
  double* phiT = nullptr;  // phi at the start of the step (Phi_tmp)
  LsGeom lsg;
  uint8_t* idn = nullptr;  // ID at the start of the step
  // interface faces
  int* slot = nullptr;     // per cell: slot of its low faces (valid where flagged)
  int* faces = nullptr;    // [cap_faces][3]: cell offset, slot, direction
  int* counts = nullptr;   // [0] slots, [1] faces, [2] overflow, [3] riemann errors, [4] iterations (low), [5] calls,
                           // [6] evaluations, [7] non-trivial calls, [8 + stage] work counters,
                           // [16...] wave-pattern group sizes
  int* order = nullptr;    // [cap_faces] faces grouped by wave pattern (the solve order of a stage)
  uint8_t* pattern = nullptr;  // [cap_faces] wave pattern of each face at this stage
  long long cap_slots = 0, cap_faces = 0;
  double* Vsm = nullptr;   // [slot][3][5] current stage
  double* Vsp = nullptr;
  double* Vmid = nullptr;
  int* midid = nullptr;    // [slot][3]
  double* rsVsm = nullptr; // stage-1 copies (the reference's riemann_solutions)
  double* rsVsp = nullptr;
  uint8_t* rsValid = nullptr;  // [slot][3]
  double* scratch = nullptr;   // Riemann integration paths
  double* faceV = nullptr;     // LINEAR interface reconstruction: [slot][3][left, right][5] face states
  // changed cells (ordered)
  int* changed = nullptr;      // [ncell] ordered list of linear offsets
  int* blockcnt = nullptr;     // per-block counts for the ordered compaction
  int* nchanged = nullptr;     // [0] changed, [1] unresolved
  int nblocks_scan = 0;
  int iface_blocks = 0;          // resident CTAs of k_iface_riemann (at most IFACE_RIEMANN_THREADS / 128)
  int time_step = 0;
  int stage = 0;
  // host-side counters
  long long riemann_calls = 0, riemann_iterations = 0, riemann_errors = 0, unresolved = 0, reinit_calls = 0;
  long long riemann_evaluations = 0, failsafe_cells = 0, riemann_nontrivial = 0;
  // per-run totals accumulated on the device at the end of every step (no
  // host round trip per step): [0] calls, [1] iterations, [2] errors,
  // [3] evaluations, [4] non-trivial calls, [5] unresolved, [6] failsafe cells
  long long* totals = nullptr;
  // learned warm start (optional): per interface face the network's features,
  // base pressure, validity, output and proposed star pressure
  const m2cg_mlp* mlp = nullptr;
  float* fX = nullptr;
  double* fP = nullptr;
  int* fvalid = nullptr;
  float* fy = nullptr;
  double* fwarm = nullptr;
  uint8_t* mask = nullptr;       // [interior cells] unresolved-list membership, zero between updates
  double failsafe[MAXMAT] = {};  // MaterialModelData::failsafe_density
  double* reinit_buf = nullptr;  // reinitialisation work arrays
  double reinit_cfl = 0.8;       // pseudo-time CFL, reduced on failed attempts
  long long reinit_iterations = 0;
};

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cell_coords(const Grid3& g, long long q, int& i, int& j, int& k) {
  i = (int)(q % g.nx);
  j = (int)((q / g.nx) % g.ny);
  k = (int)(q / ((long long)g.nx * g.ny));
}

__device__ __forceinline__ long long offset_of(const Grid3& g, int i, int j, int k) {
  return (long long)k * g.plane + (long long)j * g.px + i;
}

// Neighbour across the low face in direction d; false if it is a (non-periodic) ghost.
__device__ __forceinline__ bool low_neighbour(const Grid3& g, int i, int j, int k, int d, int& ni, int& nj, int& nk) {
  ni = i; nj = j; nk = k;
  int* c = d == 0 ? &ni : (d == 1 ? &nj : &nk);
  const int n = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
  *c -= 1;
  if (*c < 0) {
    if (g.bc[2 * d] != BC_PERIODIC) return false;
    *c += n;
  }
  return true;
}

// Collect interface faces: every low face whose two cells carry different IDs.
// 2D CTAs of 32 x 8 cells over (i, j), walking a column of planes; slots
// and face entries are taken in arrival order (any order serves: every
// later pass addresses them through slot[] and faces[]).
__global__ void k_detect_iface(Grid3 g, const uint8_t* id, int* slot, int* faces, int* counts, long long cap_slots,
                               long long cap_faces) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  for (int k = blockIdx.z; k < g.nz; k += gridDim.z) {
    const long long q = ((long long)k * g.ny + j) * g.nx + i;
    const long long off = offset_of(g, i, j, k);
    const uint8_t me = id[off];
    int mask = 0;
    for (int d = 0; d < 3; d++) {
      int ni, nj, nk;
      if (!low_neighbour(g, i, j, k, d, ni, nj, nk)) continue;
      if (id[offset_of(g, ni, nj, nk)] != me) mask |= 1 << d;
    }
    if (!mask) continue;
    int s = atomicAdd(&counts[0], 1);
    if (s >= cap_slots) {
      atomicOr(&counts[2], 1);
      continue;
    }
    slot[off] = s;
    for (int d = 0; d < 3; d++) {
      if (!(mask & (1 << d))) continue;
      int f = atomicAdd(&counts[1], 1);
      if (f >= cap_faces) {
        atomicOr(&counts[2], 1);
        continue;
      }
      faces[3 * f] = (int)q;  // linear interior index of the right cell
      faces[3 * f + 1] = s;
      faces[3 * f + 2] = d;
    }
  }
}

// Primitive state of a cell at this stage: V^n (stage 1) or clip(C2P(U_s)).
__device__ __forceinline__ void stage_state(const StageArgs& a, const Eos<double>* eos, long long off, uint8_t id,
                                            double* V) {
  if (a.stage == 1) {
    for (int c = 0; c < 5; c++) V[c] = a.Vn[c][off];
  } else {
    double U[5];
    for (int c = 0; c < 5; c++) U[c] = a.Us[c][off];
    eos[id].c2p(U, V);
    eos[id].clip(V);
  }
}

struct IfaceRiemannArgs {
  StageArgs st;           // the stage's state pointers (Vn, Us, stage)
  const Eos<double>* eos;
  RiemannParams P;
  const int* faces;
  int* counts;
  long long cap_faces;
  double* Vsm;
  double* Vsp;
  double* Vmid;
  int* midid;
  double* rsVsm;          // stage 1: also written here
  double* rsVsp;
  uint8_t* rsValid;
  double* scratch;
  DevError* err;
  const int* order;       // faces grouped by wave pattern
  uint8_t* pattern;       // classification scratch
  int* group_out;         // the same array as order, written by k_iface_group
  int normal_mode;        // MultiPhaseData::riemann_normal
  const double* phi;      // phi^n (the reference's loose coupling uses the step's phi)
  LsGeom geo;
  const double* warm;     // per face: proposed star pressure of the learned warm start, or NULL
  const double* faceV;    // LINEAR reconstruction: the face pass's states, [slot][3][2][5]; NULL: cell states
};

// Left and right states of the interface problem on face f (low face d of
// cell offR, whose slot is s): the cell-centred states of the stage, or
// under LINEAR reconstruction the face states vr[L] and vl[R] that the
// stage kernel's face pass wrote (SpaceOperator.cpp:2503-2506).
__device__ __forceinline__ void iface_states(const IfaceRiemannArgs& a, int s, int d, long long offL, uint8_t idL,
                                             long long offR, uint8_t idR, double* VL, double* VR) {
  if (a.faceV) {
    const double* o = a.faceV + ((long long)s * 3 + d) * 10;
    for (int c = 0; c < 5; c++) {
      VL[c] = o[c];
      VR[c] = o[5 + c];
    }
    return;
  }
  stage_state(a.st, a.eos, offL, idL, VL);
  stage_state(a.st, a.eos, offR, idR, VR);
}

// Groups: 4 wave patterns x IFACE_STRENGTHS rarefaction strengths; sizes in
// counts[IFACE_GROUP0 ...], fill positions in the IFACE_GROUPS entries after.
constexpr int IFACE_STRENGTHS = 8;
constexpr int IFACE_GROUPS = 4 * IFACE_STRENGTHS;
constexpr int IFACE_GROUP0 = 16;

// Wave pattern of each interface problem from the acoustic star-pressure
// estimate (the solver's own first trial point): bit 1 left shock, bit 0
// right shock, refined by the pressure ratio of the stronger rarefaction. Solving the problems grouped by pattern keeps the lanes of a
// warp in the same branches of the star-state evaluation (Hugoniot root or
// rarefaction integration on each side); the results do not depend on the
// order. Counts per pattern go to counts[12..15].
__global__ void k_iface_classify(IfaceRiemannArgs a) {
  const Grid3& g = a.st.g;
  long long nf = a.counts[1];
  if (nf > a.cap_faces) nf = a.cap_faces;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
    const int q = a.faces[3 * f], sl = a.faces[3 * f + 1], d = a.faces[3 * f + 2];
    int i, j, k;
    cell_coords(g, q, i, j, k);
    int ni, nj, nk;
    low_neighbour(g, i, j, k, d, ni, nj, nk);
    const long long offR = offset_of(g, i, j, k), offL = offset_of(g, ni, nj, nk);
    const uint8_t idR = a.st.id[offR], idL = a.st.id[offL];
    double VL[5], VR[5];
    iface_states(a, sl, d, offL, idL, offR, idR, VL, VR);
    const double c2l = a.eos[idL].c2(VL[0], a.eos[idL].energy(VL[0], VL[4]));
    const double c2r = a.eos[idR].c2(VR[0], a.eos[idR].energy(VR[0], VR[4]));
    int pat = 0;
    if (c2l > 0 && c2r > 0 && VL[0] > 0 && VR[0] > 0) {
      const double Cl = VL[0] * sqrt(c2l), Cr = VR[0] * sqrt(c2r);
      const double p0 = (Cr * VL[4] + Cl * VR[4] + Cl * Cr * (VL[1 + d] - VR[1 + d])) / (Cl + Cr);
      // strength of the stronger rarefaction (its pressure ratio, in octaves)
      double r = 1.0;
      if (p0 < VL[4] && p0 > 0) r = fmax(r, VL[4] / p0);
      if (p0 < VR[4] && p0 > 0) r = fmax(r, VR[4] / p0);
      const double lr = log2(r);  // r may be +inf: compare before converting
      const int oct = lr >= IFACE_STRENGTHS - 1 ? IFACE_STRENGTHS - 1 : (lr > 0 ? (int)lr : 0);
      pat = ((p0 > VL[4] ? 2 : 0) | (p0 > VR[4] ? 1 : 0)) * IFACE_STRENGTHS + oct;
    }
    a.pattern[f] = (uint8_t)pat;
    atomicAdd(&a.counts[IFACE_GROUP0 + pat], 1);
  }
}

__global__ void k_iface_group(IfaceRiemannArgs a) {
  long long nf = a.counts[1];
  if (nf > a.cap_faces) nf = a.cap_faces;
  __shared__ int base[IFACE_GROUPS];
  if (threadIdx.x == 0) {
    int o = 0;
    for (int c = 0; c < IFACE_GROUPS; c++) {
      base[c] = o;
      o += a.counts[IFACE_GROUP0 + c];
    }
  }
  __syncthreads();
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
    const int pat = a.pattern[f];
    const int pos = atomicAdd(&a.counts[IFACE_GROUP0 + IFACE_GROUPS + pat], 1);
    a.group_out[base[pat] + pos] = (int)f;
  }
}

// One exact Riemann problem per interface face (SpaceOperator.cpp:2499-2523):
// direction by the riemann_normal rule, cell-centred states (constant
// reconstruction at the interface), star states clipped with each side's EOS,
// stage-1 results kept. The grid holds only resident CTAs and every thread
// takes the next unsolved face from a counter when it finishes one, so a
// thread that met a hard problem is not also handed more, and lanes of a warp
// do not idle while another lane iterates (problems take from one to hundreds
// of star-state evaluations).
__global__ void __launch_bounds__(128, M2C_IFACE_MINB) k_iface_riemann(IfaceRiemannArgs a) {
  const Grid3& g = a.st.g;
  long long nf = a.counts[1];
  if (nf > a.cap_faces) nf = a.cap_faces;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int* next = &a.counts[8 + a.st.stage];  // zeroed at the start of the step
  RiemannSolver rs;
  rs.P = a.P;
  rs.eos = a.eos;
  rs.path1.pt = a.scratch + tid * 2 * 3 * RIEMANN_PATH_CAP;
  rs.path1.cap = RIEMANN_PATH_CAP;
  rs.path3.pt = rs.path1.pt + 3 * RIEMANN_PATH_CAP;
  rs.path3.cap = RIEMANN_PATH_CAP;
  for (long long w = atomicAdd(next, 1); w < nf; w = atomicAdd(next, 1)) {
    const long long f = a.order[w];
    const int q = a.faces[3 * f], s = a.faces[3 * f + 1], d = a.faces[3 * f + 2];
    int i, j, k;
    cell_coords(g, q, i, j, k);
    int ni, nj, nk;
    low_neighbour(g, i, j, k, d, ni, nj, nk);
    const long long offR = offset_of(g, i, j, k), offL = offset_of(g, ni, nj, nk);
    if (a.st.wall.mask && ((a.st.wall.mask[offR] >> d) & 1)) {
      // a face cut by an embedded surface takes the wall branch: no interface
      // problem and no stored Riemann solution there (SpaceOperator.cpp:2438)
      if (a.rsValid) a.rsValid[s * 3 + d] = 0;
      continue;
    }
    const uint8_t idR = a.st.id[offR], idL = a.st.id[offL];
    double VL[5], VR[5];
    iface_states(a, s, d, offL, idL, offR, idR, VL, VR);
    double dir[3];
    riemann_direction(a.normal_mode, g, a.geo, a.phi, i, j, k, d, idR, idL, dir);
    double Vs[5], Vsm[5], Vsp[5];
    int mid = 0;
    bool bad = false;
    int r = rs.solve(dir, VL, idL, VR, idR, Vs, mid, Vsm, Vsp, a.warm ? a.warm[f] : NAN, bad);
    a.eos[idL].clip(Vsm);
    a.eos[idR].clip(Vsp);
    const long long b = ((long long)s * 3 + d) * 5;
    for (int c = 0; c < 5; c++) {
      a.Vsm[b + c] = Vsm[c];
      a.Vsp[b + c] = Vsp[c];
      a.Vmid[b + c] = Vs[c];
    }
    a.midid[s * 3 + d] = mid;
    if (a.rsVsm) {
      for (int c = 0; c < 5; c++) {
        a.rsVsm[b + c] = Vsm[c];
        a.rsVsp[b + c] = Vsp[c];
      }
      a.rsValid[s * 3 + d] = (r == RIEM_OK) ? 1 : 0;
    }
    if (r != RIEM_OK) atomicAdd(&a.counts[3], 1);
    if (r & RIEM_PATH_OVERFLOW) report(a.err, ERR_ITER_CAP, q, 7);
    if (bad) report(a.err, ERR_STATE, q, 8);
    atomicAdd(&a.counts[4], rs.iterations);
    atomicAdd(&a.counts[6], rs.evaluations);
    atomicAdd(&a.counts[5], 1);
    if (rs.evaluations > 0) atomicAdd(&a.counts[7], 1);  // not answered by the trivial branch
  }
}

// Features of the learned warm start for every interface face of the stage:
// the same left/right states and Riemann direction the solve will use.
__global__ void k_iface_features(IfaceRiemannArgs a, float* X, double* P, int* valid) {
  const Grid3& g = a.st.g;
  long long nf = a.counts[1];
  if (nf > a.cap_faces) nf = a.cap_faces;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
    const int q = a.faces[3 * f], sl = a.faces[3 * f + 1], d = a.faces[3 * f + 2];
    int i, j, k;
    cell_coords(g, q, i, j, k);
    int ni, nj, nk;
    low_neighbour(g, i, j, k, d, ni, nj, nk);
    const long long offR = offset_of(g, i, j, k), offL = offset_of(g, ni, nj, nk);
    const uint8_t idR = a.st.id[offR], idL = a.st.id[offL];
    double VL[5], VR[5], dir[3], Pq[2] = {0.0, 0.0};
    iface_states(a, sl, d, offL, idL, offR, idR, VL, VR);
    riemann_direction(a.normal_mode, g, a.geo, a.phi, i, j, k, d, idR, idL, dir);
    valid[f] = mlp_features(a.eos[idL], a.eos[idR], VL, VR, dir, X + f * MLP_IN, Pq) ? 1 : 0;
    P[2 * f] = Pq[0];
    P[2 * f + 1] = Pq[1];
  }
}

// Material ID from the sign change of phi (MultiPhaseOperator.cpp:150-202):
// with one level set and two materials a swept cell becomes the level set's
// material where phi < 0 and material 0 otherwise.
// 2D CTAs of 32 x 8 cells over (i, j), walking a column of planes.
__global__ void k_update_id(Grid3 g, const double* phi, const double* phi0, uint8_t* id, int ls_mat) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  for (int k = blockIdx.z; k < g.nz; k += gridDim.z) {
    const long long off = offset_of(g, i, j, k);
    const double p = phi[off], p0 = phi0[off];
    if (p * p0 > 0.0) continue;
    id[off] = p < 0 ? (uint8_t)ls_mat : (uint8_t)0;
  }
}

// Ordered compaction of cells whose ID changed: per-block counts, then
// exclusive offsets, then in-block ordered writes (linear index order is the
// reference's k, j, i loop order).
__global__ void k_count_changed(Grid3 g, const uint8_t* id, const uint8_t* idn, int* blockcnt, long long per_block) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  long long n = (long long)g.nx * g.ny * g.nz;
  long long b0 = blockIdx.x * per_block, b1 = min(n, b0 + per_block);
  int local = 0;
  for (long long q = b0 + threadIdx.x; q < b1; q += blockDim.x) {
    int i, j, k;
    cell_coords(g, q, i, j, k);
    long long off = offset_of(g, i, j, k);
    local += id[off] != idn[off];
  }
  atomicAdd(&cnt, local);
  __syncthreads();
  if (threadIdx.x == 0) blockcnt[blockIdx.x] = cnt;
}

__global__ void k_scan_blocks(int* blockcnt, int nb, int* total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int s = 0;
    for (int b = 0; b < nb; b++) {
      int c = blockcnt[b];
      blockcnt[b] = s;
      s += c;
    }
    *total = s;
  }
}

__global__ void k_write_changed(Grid3 g, const uint8_t* id, const uint8_t* idn, const int* blockoff, long long per_block,
                                int* list) {
  __shared__ int warp_sums[32];
  long long n = (long long)g.nx * g.ny * g.nz;
  long long b0 = blockIdx.x * per_block, b1 = min(n, b0 + per_block);
  int base = blockoff[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (long long c0 = b0; c0 < b1; c0 += blockDim.x) {
    long long q = c0 + threadIdx.x;
    int flag = 0;
    if (q < b1) {
      int i, j, k;
      cell_coords(g, q, i, j, k);
      long long off = offset_of(g, i, j, k);
      flag = id[off] != idn[off];
    }
    unsigned bal = __ballot_sync(0xffffffffu, flag);
    int wpre = __popc(bal & ((1u << lane) - 1));
    if (lane == 0) warp_sums[warp] = __popc(bal);
    __syncthreads();
    int before = 0, tot = 0;
    for (int w = 0; w < nwarps; w++) {
      if (w < warp) before += warp_sums[w];
      tot += warp_sums[w];
    }
    if (flag) list[base + before + wpre] = (int)q;
    base += tot;
    __syncthreads();
  }
}

struct StateUpdateArgs {
  Grid3 g;
  const Eos<double>* eos;
  double* V[5];
  float* Vf[5];         // FP32 copy of V kept in step (mixed path), or null
  const uint8_t* id;
  const uint8_t* idn;
  const int* slot;
  const double* rsVsm;
  const double* rsVsp;
  const uint8_t* rsValid;
  int* changed;         // ordered changed cells; the unresolved ones are compacted into its head
  int* nchanged;        // [0] changed, [1] unresolved after the first pass, [2] still unresolved, [3] failsafe
  DevError* err;
  int use_rs;           // stage-1 Riemann solutions of this step are available
  int type;             // MultiPhaseData::phasechange_type: 0 RIEMANN_SOLUTION, 1 EXTRAPOLATION
  int upwind;           // MultiPhaseData::phasechange_dir == UPWIND
  int failsafe;         // MultiPhaseData::apply_failsafe_density == On
  LsGeom geo;           // cell-centre coordinates (one ghost per side)
  uint8_t* mask;        // [interior cells] member of the unresolved list (all zero between calls)
  double failsafe_rho[MAXMAT];  // MaterialModelData::failsafe_density
};

// Star state stored on one face of cell (i,j,k): side 0 = its low face
// ("left/bottom/back": Vsm of the slot of this cell), side 1 = its high
// face ("right/top/front": Vsp of the slot of the neighbour above).
__device__ bool stored_state(const StateUpdateArgs& a, int i, int j, int k, int d, int side, double* S, int& sid) {
  const Grid3& g = a.g;
  int ci = i, cj = j, ck = k;
  if (side == 1) {
    int* c = d == 0 ? &ci : (d == 1 ? &cj : &ck);
    const int n = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
    *c += 1;
    if (*c >= n) {
      if (g.bc[2 * d + 1] != BC_PERIODIC) return false;
      *c -= n;
    }
  }
  int ni, nj, nk;
  if (!low_neighbour(g, ci, cj, ck, d, ni, nj, nk)) return false;
  const long long offc = offset_of(g, ci, cj, ck), offn = offset_of(g, ni, nj, nk);
  if (a.idn[offc] == a.idn[offn]) return false;  // not an interface face this step
  const int s = a.slot[offc];
  if (!a.rsValid[s * 3 + d]) return false;       // Riemann solve reported an error: not stored
  const double* src = side == 0 ? a.rsVsm : a.rsVsp;
  for (int c = 0; c < 5; c++) S[c] = src[((long long)s * 3 + d) * 5 + c];
  sid = side == 0 ? a.idn[offn] : a.idn[offc];
  return true;
}

// LocalUpdateByRiemannSolutions (MultiPhaseOperator.cpp:916-1027)
__device__ int local_update(const StateUpdateArgs& a, int i, int j, int k, int myid, double* v, bool upwind) {
  const Grid3& g = a.g;
  int counter = 0;
  double weight = 0, sum_weight = 0;
  // faces in the reference's order: left, right, bottom, top, back, front
  for (int q = 0; q < 6; q++) {
    const int d = q >> 1, side = q & 1;
    double S[5];
    int sid;
    if (!stored_state(a, i, j, k, d, side, S, sid)) continue;
    if (sid != myid) continue;
    // neighbour state on that side (ghost rule applied for boundaries)
    int ni = i, nj = j, nk = k;
    int* c = d == 0 ? &ni : (d == 1 ? &nj : &nk);
    const int n = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
    *c += side ? 1 : -1;
    double nv[5];
    if (*c < 0 || *c >= n) {
      if (g.bc[2 * d + side] == BC_PERIODIC) {
        *c = (*c + n) % n;
      } else {
        continue;  // a boundary face is never an interface face
      }
    }
    const long long off = offset_of(g, ni, nj, nk);
    for (int p = 0; p < 5; p++) nv[p] = a.V[p][off];
    const double vn = nv[d + 1];
    if (upwind && !(side == 0 ? vn > 0 : vn < 0)) continue;
    const double nrm = sqrt(nv[1] * nv[1] + nv[2] * nv[2] + nv[3] * nv[3]);
    weight = upwind ? (side == 0 ? vn / nrm : -vn / nrm) : 1.0;
    sum_weight += weight;
    if (counter == 0) {
      for (int p = 0; p < 5; p++) v[p] = weight * S[p];
    } else {
      for (int p = 0; p < 5; p++) v[p] += weight * S[p];
    }
    counter++;
  }
  if (sum_weight > 0.0) {
    const double inv = 1.0 / sum_weight;  // Vec5D::operator/= (Vector5D.h:172-181)
    for (int p = 0; p < 5; p++) v[p] *= inv;
  }
  return counter;
}

__device__ __forceinline__ void centre(const LsGeom& geo, int i, int j, int k, double* x) {
  x[0] = geo.xg[0][i + 1];
  x[1] = geo.xg[1][j + 1];
  x[2] = geo.xg[2][k + 1];
}

__device__ __forceinline__ bool outside(const Grid3& g, int i, int j, int k) {
  return i < 0 || i >= g.nx || j < 0 || j >= g.ny || k < 0 || k >= g.nz;
}

__device__ __forceinline__ double norm3(const double* a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// max(0, (x0 - x1)/|x0 - x1| . v1/|v1|), the upwind weight of a neighbour at
// x1 with velocity v1 for the cell at x0 (Vec3D::operator/= multiplies by the
// reciprocal). *dist receives |x0 - x1|.
__device__ __forceinline__ double upwind_weight(const double* x0, const double* x1, const double* nv, double* dist) {
  double v1[3] = {nv[1], nv[2], nv[3]};
  const double v1norm = norm3(v1);
  if (v1norm != 0) {
    const double inv = 1.0 / v1norm;
    v1[0] *= inv; v1[1] *= inv; v1[2] *= inv;
  }
  double d[3] = {x0[0] - x1[0], x0[1] - x1[1], x0[2] - x1[2]};
  const double dn = norm3(d);
  *dist = dn;
  const double inv = 1.0 / dn;
  d[0] *= inv; d[1] *= inv; d[2] *= inv;
  const double w = d[0] * v1[0] + d[1] * v1[1] + d[2] * v1[2];
  return w > 0.0 ? w : 0.0;
}

// UpdateStateVariablesByExtrapolation, one cell (MultiPhaseOperator.cpp:1032-1128):
// weighted average of the 26 neighbours that keep the cell's new ID and did
// not change ID themselves; false if no weight.
__device__ bool extrapolate(const StateUpdateArgs& a, int i, int j, int k, int myid, double* v) {
  const Grid3& g = a.g;
  double x0[3];
  centre(a.geo, i, j, k, x0);
  double sum_weight = 0.0, vsum[5] = {0, 0, 0, 0, 0};
  for (int nk = k - 1; nk <= k + 1; nk++)
    for (int nj = j - 1; nj <= j + 1; nj++)
      for (int ni = i - 1; ni <= i + 1; ni++) {
        if (outside(g, ni, nj, nk)) continue;
        const long long off = offset_of(g, ni, nj, nk);
        if (a.id[off] != myid) continue;
        if (a.id[off] != a.idn[off]) continue;
        double x1[3], nv[5];
        centre(a.geo, ni, nj, nk, x1);
        for (int p = 0; p < 5; p++) nv[p] = a.V[p][off];
        double weight;
        if (!a.upwind) {
          double d[3] = {x0[0] - x1[0], x0[1] - x1[1], x0[2] - x1[2]};
          weight = 1.0 / norm3(d);
        } else {
          double dist;
          weight = upwind_weight(x0, x1, nv, &dist);
        }
        if (weight > 0) {
          sum_weight += weight;
          for (int p = 0; p < 5; p++) vsum[p] += weight * nv[p];
        }
      }
  if (sum_weight == 0) return false;
  for (int p = 0; p < 5; p++) v[p] = vsum[p] / sum_weight;  // Vec5D::operator/ divides
  return true;
}

__device__ __forceinline__ void store(const StateUpdateArgs& a, long long off, const double* v) {
  for (int p = 0; p < 5; p++) a.V[p][off] = v[p];
  if (a.Vf[0])
    for (int p = 0; p < 5; p++) a.Vf[p][off] = (float)v[p];
}

// Sequential pass over the changed cells in (k, j, i) order
// (UpdateStateVariablesByRiemannSolutions, MultiPhaseOperator.cpp:857-911, or
// ...ByExtrapolation, 1032-1151), then FixUnresolvedNodes (1156-1400) over
// the cells neither could update, in the same order. Every updated cell is
// clipped and checked (ClipDensityAndPressure after the update,
// TimeIntegrator.cpp:767).
__global__ void k_state_update(StateUpdateArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const Grid3& g = a.g;
  const int n = a.nchanged[0];
  int nun = 0;
  for (int t = 0; t < n; t++) {
    const int q = a.changed[t];
    int i, j, k;
    cell_coords(g, q, i, j, k);
    const long long off = offset_of(g, i, j, k);
    const int myid = a.id[off];
    double v[5];
    for (int p = 0; p < 5; p++) v[p] = a.V[p][off];
    bool done;
    if (a.type == 1) {
      done = extrapolate(a, i, j, k, myid, v);
    } else {
      int counter = a.use_rs ? local_update(a, i, j, k, myid, v, true) : 0;
      if (counter == 0 && a.use_rs) counter = local_update(a, i, j, k, myid, v, false);
      done = counter != 0;
    }
    if (!done) {
      a.changed[nun++] = q;  // unresolved: compacted in order into the head of the list
      a.mask[q] = 1;
      continue;
    }
    a.eos[myid].clip(v);
    if (a.eos[myid].bad(v)) report(a.err, ERR_STATE, q, 9);
    store(a, off, v);
  }
  a.nchanged[1] = nun;
  // FixUnresolvedNodes. `reset` is set once per call, not per cell, as in the
  // reference (1183): from the second cell with an upwind neighbour on, the
  // upwind sum adds to the cell's current state instead of replacing it.
  bool reset = false;
  int still = 0, nfailsafe = 0;
  for (int t = 0; t < nun; t++) {
    const int q = a.changed[t];
    int i, j, k;
    cell_coords(g, q, i, j, k);
    const long long off = offset_of(g, i, j, k);
    const int myid = a.id[off];
    double x0[3];
    centre(a.geo, i, j, k, x0);
    double v[5], vtmp[5] = {0, 0, 0, 0, 0};
    for (int p = 0; p < 5; p++) v[p] = a.V[p][off];
    double sum_weight = 0.0, sum_weight2 = 0.0;
    for (int nk = k - 1; nk <= k + 1; nk++)
      for (int nj = j - 1; nj <= j + 1; nj++)
        for (int ni = i - 1; ni <= i + 1; ni++) {
          if (outside(g, ni, nj, nk)) continue;
          const long long noff = offset_of(g, ni, nj, nk);
          if (a.id[noff] != myid) continue;
          if (ni == i && nj == j && nk == k) continue;
          if (a.mask[((long long)nk * g.ny + nj) * g.nx + ni]) continue;
          double x1[3], nv[5], dist;
          centre(a.geo, ni, nj, nk, x1);
          for (int p = 0; p < 5; p++) nv[p] = a.V[p][noff];
          const double weight = upwind_weight(x0, x1, nv, &dist);
          if (weight > 0) {
            sum_weight += weight;
            if (reset) {
              for (int p = 0; p < 5; p++) v[p] += weight * nv[p];
            } else {
              for (int p = 0; p < 5; p++) v[p] = weight * nv[p];
              reset = true;
            }
          }
          const double w2 = 1.0 / dist;
          for (int p = 0; p < 5; p++) vtmp[p] += w2 * nv[p];
          sum_weight2 += w2;
        }
    bool done = false;
    if (a.upwind && sum_weight > 0) {
      const double inv = 1.0 / sum_weight;  // Vec5D::operator/=
      for (int p = 0; p < 5; p++) v[p] *= inv;
      done = true;
    } else if (sum_weight2 > 0) {
      for (int p = 0; p < 5; p++) v[p] = vtmp[p] / sum_weight2;
      done = true;
    } else {
      // last resort: keep velocity and pressure, take the density from the
      // nearest layer (up to 10) that has valid cells, inverse-distance weighted
      double density = 0.0;
      for (int layer = 1; layer <= 10 && !done; layer++) {
        for (int nk = k - layer; nk <= k + layer; nk++)
          for (int nj = j - layer; nj <= j + layer; nj++)
            for (int ni = i - layer; ni <= i + layer; ni++) {
              if (outside(g, ni, nj, nk)) continue;
              const long long noff = offset_of(g, ni, nj, nk);
              if (a.id[noff] != myid) continue;
              if (ni == i && nj == j && nk == k) continue;
              if (a.mask[((long long)nk * g.ny + nj) * g.nx + ni]) continue;
              double x1[3];
              centre(a.geo, ni, nj, nk, x1);
              double d[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
              const double dist = norm3(d);
              sum_weight += 1.0 / dist;
              density += (1.0 / dist) * a.V[0][noff];
            }
        if (sum_weight > 0) {
          v[0] = density / sum_weight;
          done = true;
        }
      }
      if (!done) {
        if (myid != 0 || a.failsafe) {
          v[0] = a.failsafe_rho[myid];
          nfailsafe++;
          done = true;
        } else {
          still++;  // left for the level-set correction, which is not built: reported by the host
        }
      }
    }
    if (done) {
      a.eos[myid].clip(v);
      if (a.eos[myid].bad(v)) report(a.err, ERR_STATE, q, 9);
      store(a, off, v);
    }
  }
  for (int t = 0; t < nun; t++) a.mask[a.changed[t]] = 0;
  a.nchanged[2] = still;
  a.nchanged[3] = nfailsafe;
}

void set_last_error(const char* msg);

static int grid1d(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace m2c

using namespace m2c;

// ---------------------------------------------------------------------------
// host interface
// ---------------------------------------------------------------------------
m2cg_status multiphase_create(cudaStream_t s, const Grid3& g, const SchemeK& sk, const m2cg_scheme& scheme,
                              const m2cg_material* mats, int nmat, const m2cg_levelset& ls, const double* const* xc,
                              const double* const* dx, Multiphase** out) {
  *out = nullptr;
  if (scheme.mp_recon != 0 && scheme.mp_recon != 1) return M2CG_ERR_ARG;
  if (scheme.mp_phasechange_type != 0 && scheme.mp_phasechange_type != 1) return M2CG_ERR_UNSUPPORTED;
  if (ls.material_id != 1) return M2CG_ERR_UNSUPPORTED;
  if (ls.reinit_first_layer < 0 || ls.reinit_first_layer > 4) return M2CG_ERR_ARG;
  if (ls.solver != M2CG_LS_FINITE_VOLUME && ls.solver != M2CG_LS_FINITE_DIFFERENCE) return M2CG_ERR_ARG;
  if (ls.solver == M2CG_LS_FINITE_VOLUME &&
      (ls.flux < 0 || ls.flux > 2 || ls.rec_type < 0 || ls.rec_type > 1 || ls.limiter < 0 || ls.limiter > 2))
    return M2CG_ERR_ARG;
  Multiphase* mp = new Multiphase;
  mp->g = g;
  mp->sk = sk;
  mp->scheme = scheme;
  mp->ls = ls;
  mp->rp = riemann_params(scheme);
  mp->reinit_cfl = ls.reinit_cfl;
  mp->ncell = g.plane * g.nz;
  for (int m = 0; m < nmat && m < MAXMAT; m++) mp->failsafe[m] = mats[m].failsafe_density;
  const long long n = mp->ncell;
  const long long ninterior = (long long)g.nx * g.ny * g.nz;
  mp->cap_slots = ninterior < 65536 ? ninterior : (ninterior / 8 > 65536 ? ninterior / 8 : 65536);
  mp->cap_faces = 3 * mp->cap_slots;
  bool ok = true;
  auto A = [&](void** p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) ok = false;
  };
  A((void**)&mp->d_eos, sizeof(Eos<double>) * MAXMAT);
  A((void**)&mp->phiN, n * 8);
  A((void**)&mp->phiA, n * 8);
  A((void**)&mp->phiB, n * 8);
  A((void**)&mp->phiT, n * 8);
  A((void**)&mp->idn, n);
  A((void**)&mp->slot, n * 4);
  A((void**)&mp->faces, mp->cap_faces * 3 * 4);
  A((void**)&mp->order, mp->cap_faces * 4);
  A((void**)&mp->pattern, mp->cap_faces);
  A((void**)&mp->counts, (IFACE_GROUP0 + 2 * IFACE_GROUPS) * 4);
  A((void**)&mp->Vsm, mp->cap_slots * 15 * 8);
  A((void**)&mp->Vsp, mp->cap_slots * 15 * 8);
  A((void**)&mp->Vmid, mp->cap_slots * 15 * 8);
  A((void**)&mp->midid, mp->cap_slots * 3 * 4);
  A((void**)&mp->rsVsm, mp->cap_slots * 15 * 8);
  A((void**)&mp->rsVsp, mp->cap_slots * 15 * 8);
  A((void**)&mp->rsValid, mp->cap_slots * 3);
  A((void**)&mp->scratch, (size_t)IFACE_RIEMANN_THREADS * 2 * 3 * RIEMANN_PATH_CAP * 8);
  if (scheme.mp_recon == 1 && scheme.mp_flux != M2CG_MPFLUX_LLF) A((void**)&mp->faceV, (size_t)mp->cap_slots * 3 * 10 * 8);
  A((void**)&mp->changed, ninterior * 4);
  mp->nblocks_scan = 148 * 8;
  {
    int per_sm = 0, dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_iface_riemann, 128, 0) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    const int blocks = per_sm * nsm;
    mp->iface_blocks = blocks < IFACE_RIEMANN_THREADS / 128 ? blocks : IFACE_RIEMANN_THREADS / 128;
  }
  A((void**)&mp->blockcnt, mp->nblocks_scan * 4);
  A((void**)&mp->nchanged, 4 * 4);
  A((void**)&mp->totals, 8 * sizeof(long long));
  A((void**)&mp->mask, ninterior);
  if (!ok) {
    multiphase_destroy(mp);
    return M2CG_ERR_NOMEM;
  }
  cudaMemcpyAsync(mp->d_eos, sk.ed, sizeof(Eos<double>) * MAXMAT, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(mp->counts, 0, 16 * 4, s);
  cudaMemsetAsync(mp->rsValid, 0, mp->cap_slots * 3, s);
  cudaMemsetAsync(mp->mask, 0, ninterior, s);
  cudaMemsetAsync(mp->totals, 0, 8 * sizeof(long long), s);
  if (levelset_geom_create(s, g, ls, xc, dx, &mp->lsg) != M2CG_OK) {
    multiphase_destroy(mp);
    return M2CG_ERR_NOMEM;
  }
  if (ls.reinit_frequency > 0 && reinit_alloc(mp->ncell, ls.reinit_first_layer, &mp->reinit_buf) != M2CG_OK) {
    multiphase_destroy(mp);
    return M2CG_ERR_NOMEM;
  }
  *out = mp;
  return M2CG_OK;
}

void multiphase_destroy(Multiphase* mp) {
  if (!mp) return;
  cudaFree(mp->d_eos);
  cudaFree(mp->phiN); cudaFree(mp->phiA); cudaFree(mp->phiB); cudaFree(mp->phiT);
  cudaFree(mp->idn); cudaFree(mp->slot); cudaFree(mp->faces); cudaFree(mp->counts);
  cudaFree(mp->order); cudaFree(mp->pattern);
  cudaFree(mp->Vsm); cudaFree(mp->Vsp); cudaFree(mp->Vmid); cudaFree(mp->midid);
  cudaFree(mp->rsVsm); cudaFree(mp->rsVsp); cudaFree(mp->rsValid); cudaFree(mp->scratch);
  cudaFree(mp->faceV);
  cudaFree(mp->changed); cudaFree(mp->blockcnt); cudaFree(mp->nchanged); cudaFree(mp->mask);
  cudaFree(mp->totals);
  cudaFree(mp->fX); cudaFree(mp->fP); cudaFree(mp->fvalid); cudaFree(mp->fy); cudaFree(mp->fwarm);
  cudaFree(mp->reinit_buf);
  levelset_geom_destroy(&mp->lsg);
  delete mp;
}

m2cg_status multiphase_upload_phi(Multiphase* mp, cudaStream_t s, const double* phi_host, double* staging,
                                  uint8_t* id) {
  (void)id;
  if (!phi_host) return M2CG_ERR_ARG;
  const Grid3& g = mp->g;
  size_t ng = (size_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
  if (cudaMemcpyAsync(staging, phi_host, ng * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) return M2CG_ERR_CUDA;
  levelset_unpack(s, g, staging, mp->phiN);
  return cudaGetLastError() == cudaSuccess ? M2CG_OK : M2CG_ERR_CUDA;
}

m2cg_status multiphase_download_phi(Multiphase* mp, cudaStream_t s, double* phi_host) {
  const Grid3& g = mp->g;
  size_t ng = (size_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
  double* tmp = nullptr;
  if (cudaMallocAsync((void**)&tmp, ng * 8, s) != cudaSuccess) return M2CG_ERR_NOMEM;
  levelset_pack(s, g, mp->lsg, mp->phiN, tmp);
  cudaMemcpyAsync(phi_host, tmp, ng * 8, cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(tmp, s);
  return cudaGetLastError() == cudaSuccess ? M2CG_OK : M2CG_ERR_CUDA;
}

void multiphase_set_step(Multiphase* mp, int time_step) {
  if (time_step > 0)
    mp->time_step = time_step;
  else
    mp->time_step++;
}

m2cg_status multiphase_begin_step(Multiphase* mp, cudaStream_t s, double* const* Vn, const uint8_t* id) {
  (void)Vn;
  const Grid3& g = mp->g;
  const long long n = mp->ncell;
  cudaMemcpyAsync(mp->phiT, mp->phiN, n * 8, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(mp->idn, id, n, cudaMemcpyDeviceToDevice, s);
  cudaMemsetAsync(mp->counts, 0, 16 * 4, s);
  k_detect_iface<<<dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz < 64 ? g.nz : 64), dim3(32, 8), 0, s>>>(
      g, id, mp->slot, mp->faces, mp->counts,
                                                                        mp->cap_slots, mp->cap_faces);
  mp->stage = 0;
  return cudaGetLastError() == cudaSuccess ? M2CG_OK : M2CG_ERR_CUDA;
}

bool multiphase_face_pass(Multiphase* mp, StageArgs& a) {
  if (!mp->faceV) return false;
  a.iface.slot = mp->slot;
  a.iface.mp_flux = mp->scheme.mp_flux;
  a.iface.mp_recon = mp->scheme.mp_recon;
  a.iface.faces_out = mp->faceV;
  for (int p = 0; p < 5; p++) {
    a.Po[p] = nullptr;
    a.Uo[p] = nullptr;
    a.Vo[p] = nullptr;
    a.Vfo[p] = nullptr;
    a.Ro[p] = nullptr;
  }
  a.final_stage = 0;
  a.clipped_out = nullptr;
  a.dtmin_bits = nullptr;
  return true;
}

m2cg_status multiphase_stage(Multiphase* mp, cudaStream_t s, StageArgs& a) {
  mp->stage = a.stage;
  // exact Riemann problems at the interface faces
  IfaceRiemannArgs ra;
  memset(&ra, 0, sizeof ra);
  ra.st = a;
  ra.eos = mp->d_eos;
  ra.P = mp->rp;
  ra.faces = mp->faces;
  ra.counts = mp->counts;
  ra.cap_faces = mp->cap_faces;
  ra.Vsm = mp->Vsm;
  ra.Vsp = mp->Vsp;
  ra.Vmid = mp->Vmid;
  ra.midid = mp->midid;
  if (a.stage == 1 && !a.Ro[0]) {
    ra.rsVsm = mp->rsVsm;
    ra.rsVsp = mp->rsVsp;
    ra.rsValid = mp->rsValid;
  }
  ra.scratch = mp->scratch;
  ra.err = a.err;
  ra.normal_mode = mp->scheme.mp_riemann_normal;
  ra.phi = mp->phiN;
  ra.geo = mp->lsg;
  ra.order = mp->order;
  ra.pattern = mp->pattern;
  ra.group_out = mp->order;
  ra.faceV = mp->faceV;
  cudaMemsetAsync(mp->counts + IFACE_GROUP0, 0, 2 * IFACE_GROUPS * sizeof(int), s);
  k_iface_classify<<<148 * 8, 256, 0, s>>>(ra);
  k_iface_group<<<148 * 8, 256, 0, s>>>(ra);
  if (mp->mlp) {
    // the network's proposals for this stage's problems, counted on the device
    k_iface_features<<<148 * 8, 256, 0, s>>>(ra, mp->fX, mp->fP, mp->fvalid);
    mlp_warm_device(mp->mlp, s, mp->fX, mp->fvalid, mp->fP, (int)mp->cap_faces, mp->fy, mp->fwarm, &mp->counts[1]);
    ra.warm = mp->fwarm;
  }
  k_iface_riemann<<<mp->iface_blocks, 128, 0, s>>>(ra);
  if (cudaGetLastError() != cudaSuccess) return M2CG_ERR_CUDA;
  a.iface.slot = mp->slot;
  a.iface.Vsm = mp->Vsm;
  a.iface.Vsp = mp->Vsp;
  a.iface.Vmid = mp->Vmid;
  a.iface.midid = mp->midid;
  a.iface.mp_flux = mp->scheme.mp_flux;
  a.iface.mp_recon = mp->scheme.mp_recon;
  if (a.Ro[0]) return M2CG_OK;  // residual only: no level-set stage
  // level-set RK stage with this stage's velocity (loose coupling,
  // TimeIntegrator.cpp:553-558, 608-614, 658-664)
  const int r = mp->scheme.rk_order;
  const double* in = a.stage == 1 ? mp->phiN : (a.stage == 2 ? mp->phiA : mp->phiB);
  double* outp = (a.stage == r) ? mp->phiN : (a.stage == 1 ? mp->phiA : mp->phiB);
  return levelset_stage(s, mp->g, mp->sk, mp->lsg, a, in, mp->phiN, outp);
}

m2cg_status multiphase_end_step(Multiphase* mp, cudaStream_t s, double* const* Vold, double* const* Vnew,
                                float* const* Vfnew, uint8_t* id,
                                const double* clock, DevError* err, m2cg_counters* counters) {
  (void)Vold;
  (void)clock;
  const Grid3& g = mp->g;
  const long long ninterior = (long long)g.nx * g.ny * g.nz;
  // material ID from the sign change of phi
  k_update_id<<<dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz < 64 ? g.nz : 64), dim3(32, 8), 0, s>>>(
      g, mp->phiN, mp->phiT, id, mp->ls.material_id);
  // reinitialisation every `frequency` steps (LevelSetOperator::Reinitialize, 1599-1624)
  if (mp->ls.reinit_frequency > 0 && mp->time_step % mp->ls.reinit_frequency == 0) {
    int its = 0;
    m2cg_status st = levelset_reinitialize(s, g, mp->lsg, mp->ls, mp->phiN, mp->reinit_buf, err, &mp->reinit_cfl, &its);
    if (st) return st;
    mp->reinit_calls++;
    mp->reinit_iterations += its;
  }
  m2cg_status st = multiphase_update_states(mp, s, Vnew, Vfnew, id, err, true, true, nullptr);
  if (st) return st;
  if (counters) counters->kernel_launches += 8 + 3 * mp->scheme.rk_order;
  return M2CG_OK;
}

// End of a step's state update: add the step's counts to the run totals and
// turn the two conditions the host used to check after the step into device
// errors (read by the caller's next error check).
__global__ void k_step_totals(const int* counts, const int* nchanged, long long* totals, DevError* err,
                              int step_counts) {
  if (step_counts) {
    totals[0] += counts[5];
    totals[1] += counts[4];
    totals[2] += counts[3];
    totals[3] += counts[6];
    totals[4] += counts[7];
    if (counts[2]) report(err, ERR_ITER_CAP, -1, 9);  // interface capacity exceeded
  }
  totals[5] += nchanged[1];
  totals[6] += nchanged[3];
  if (nchanged[2]) report(err, ERR_UNSUPPORTED, -1, 10);
}

uint8_t* multiphase_idn(Multiphase* mp) { return mp->idn; }

m2cg_status multiphase_update_states(Multiphase* mp, cudaStream_t s, double* const* V, float* const* Vf, uint8_t* id,
                                     DevError* err, bool use_rs, bool in_step, int* unresolved) {
  const Grid3& g = mp->g;
  const long long ninterior = (long long)g.nx * g.ny * g.nz;
  // ordered list of cells whose ID changed, then the sequential update
  long long per_block = (ninterior + mp->nblocks_scan - 1) / mp->nblocks_scan;
  k_count_changed<<<mp->nblocks_scan, 256, 0, s>>>(g, id, mp->idn, mp->blockcnt, per_block);
  k_scan_blocks<<<1, 1, 0, s>>>(mp->blockcnt, mp->nblocks_scan, mp->nchanged);
  k_write_changed<<<mp->nblocks_scan, 256, 0, s>>>(g, id, mp->idn, mp->blockcnt, per_block, mp->changed);
  StateUpdateArgs ua;
  memset(&ua, 0, sizeof ua);
  ua.g = g;
  ua.eos = mp->d_eos;
  for (int p = 0; p < 5; p++) ua.V[p] = V[p];
  for (int p = 0; p < 5; p++) ua.Vf[p] = Vf ? Vf[p] : nullptr;
  ua.id = id;
  ua.idn = mp->idn;
  ua.slot = mp->slot;
  ua.rsVsm = mp->rsVsm;
  ua.rsVsp = mp->rsVsp;
  ua.rsValid = mp->rsValid;
  ua.changed = mp->changed;
  ua.nchanged = mp->nchanged;
  ua.err = err;
  ua.use_rs = use_rs ? 1 : 0;
  ua.type = mp->scheme.mp_phasechange_type;
  ua.upwind = mp->scheme.mp_phasechange_dir == 1;
  ua.failsafe = mp->scheme.mp_apply_failsafe_density != 0;
  ua.geo = mp->lsg;
  ua.mask = mp->mask;
  for (int m = 0; m < MAXMAT; m++) ua.failsafe_rho[m] = mp->failsafe[m];
  k_state_update<<<1, 32, 0, s>>>(ua);
  // step counters into the device totals; interface-capacity overflow and
  // the unsupported trapped-cell correction become device errors
  // (only a step's own update counts its Riemann solves)
  k_step_totals<<<1, 1, 0, s>>>(mp->counts, mp->nchanged, mp->totals, err, in_step ? 1 : 0);
  if (cudaGetLastError() != cudaSuccess) return M2CG_ERR_CUDA;
  if (in_step) return M2CG_OK;  // no host round trip inside a step
  int hn[4];
  cudaMemcpyAsync(hn, mp->nchanged, sizeof hn, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return M2CG_ERR_CUDA;
  if (unresolved) *unresolved = hn[1];
  return M2CG_OK;
}

m2cg_status multiphase_read_totals(const Multiphase* mp, long long* t7) {
  if (cudaMemcpy(t7, mp->totals, 7 * sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    return M2CG_ERR_CUDA;
  return M2CG_OK;
}

void multiphase_counters(const Multiphase* mp, m2cg_counters* out) {
  long long t[7] = {};
  multiphase_read_totals(mp, t);
  out->riemann_calls = t[0];
  out->riemann_iterations = t[1];
  out->riemann_errors = t[2];
  out->reinit_calls = mp->reinit_calls;
  out->unresolved_cells = t[5];
  out->riemann_evaluations = t[3];
  out->failsafe_cells = t[6];
  out->riemann_nontrivial = t[4];
}

m2cg_status multiphase_set_mlp(Multiphase* mp, const m2cg_mlp* m) {
  if (m && !mp->fX) {
    const size_t n = (size_t)mp->cap_faces;
    if (cudaMalloc((void**)&mp->fX, n * MLP_IN * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&mp->fP, 2 * n * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&mp->fvalid, n * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&mp->fy, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&mp->fwarm, n * sizeof(double)) != cudaSuccess) {
      cudaFree(mp->fX); cudaFree(mp->fP); cudaFree(mp->fvalid); cudaFree(mp->fy); cudaFree(mp->fwarm);
      mp->fX = nullptr; mp->fP = nullptr; mp->fvalid = nullptr; mp->fy = nullptr; mp->fwarm = nullptr;
      return M2CG_ERR_NOMEM;
    }
  }
  mp->mlp = m;
  return M2CG_OK;
}
