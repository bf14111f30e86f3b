// Faces cut by embedded surfaces: host setup and the per-stage one-sided
// Riemann pre-pass (see walls.h). Compiled with -fmad=false: the solves and
// the normal of AVERAGE keep the reference's rounding.
#include "walls.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "riemann_batch.h"

namespace m2c {

struct Walls {
  int nslot = 0;            // cells with at least one cut low face
  int normal_mode = 1;      // EmbeddedBoundaryMethodData::riemann_normal
  RiemannParams P;
  uint8_t* mask = nullptr;  // per cell (context layout): bit d = low face along d is cut
  int* slot = nullptr;      // per cell, where mask != 0
  int* cell = nullptr;      // [slot][3] = (i, j, k)
  double* geo = nullptr;    // [slot][3 faces][12] = nf, uf, nb, ub
  double* Vsm = nullptr;    // [slot][3][5]
  double* Vsp = nullptr;
  unsigned long long* cnt = nullptr;  // [0] solves, [1] failed solves
  int* work = nullptr;                // one-sided problems: (slot * 3 + d) * 2 + side
  int linear = 0;                     // LINEAR reconstruction at the surface
  double* faceV = nullptr;            // LINEAR: the face pass's states, [slot][3][low, high][5]
  int nwork = 0;
  double* scratch = nullptr;          // per thread: one integration path
  int threads = 0;
};

namespace {

struct WallPassArgs {
  StageArgs st;
  RiemannParams P;
  const int* cell;
  const double* geo;
  double* Vsm;
  double* Vsp;
  unsigned long long* cnt;
  const int* work;
  const double* faceV;
  double* scratch;
  int nwork;
  int normal_mode;
};

// Primitive state of a cell at this stage: V^n (stage 1) or clip(C2P(U_s)),
// the states the stage kernel's cells carry.
__device__ __forceinline__ void wall_stage_state(const StageArgs& a, long long off, uint8_t id, double* V) {
  const Eos<double>& e = a.s.ed[id < a.s.nmat ? id : 0];
  if (a.stage == 1) {
    for (int c = 0; c < 5; c++) V[c] = a.Vn[c][off];
  } else {
    double U[5];
    for (int c = 0; c < 5; c++) U[c] = a.Us[c][off];
    e.c2p(U, V);
    e.clip(V);
  }
}

// SpaceOperator::GetNormalForOneSidedRiemann (SpaceOperator.cpp:3505-3530):
// the face normal (MESH), the surface normal turned to point along
// fb * e_d (EMBEDDED_SURFACE), or their normalised sum (AVERAGE).
__device__ __forceinline__ void wall_direction(int mode, int d, int fb, const double* nw, double* dir) {
  if (mode == 1) {  // MESH
    dir[0] = dir[1] = dir[2] = 0.0;
    dir[d] = (double)fb;
    return;
  }
  for (int c = 0; c < 3; c++) dir[c] = nw[c];
  if (dir[d] * (double)fb < 0.0) dir[d] *= -1;
  if (mode == 2) {  // AVERAGE: Vec3D::operator/= multiplies by the reciprocal
    dir[d] += (double)fb;
    double inv = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    inv = 1.0 / inv;
    for (int c = 0; c < 3; c++) dir[c] *= inv;
  }
}

// One thread per one-sided problem (a side of a cut face): the two sides of
// a face are independent solves, so splitting them doubles the resident
// warps that hide the FP64 latency of the rarefaction integration (4 CTAs
// per SM at 128 registers: more resident warps beat the few spills).
__global__ void __launch_bounds__(128, 4) k_wall_riemann(WallPassArgs a) {
  const Grid3& g = a.st.g;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  RiemannSolver rs;
  rs.P = a.P;
  rs.eos = a.st.s.ed;
  rs.path1.pt = a.scratch + tid * 3 * (long long)RIEMANN_PATH_CAP;
  rs.path1.cap = RIEMANN_PATH_CAP;
  rs.path3.pt = nullptr;
  rs.path3.cap = 0;
  unsigned long long solves = 0, failed = 0;
  for (long long w = tid; w < a.nwork; w += (long long)gridDim.x * blockDim.x) {
    const int item = a.work[w];
    const int side = item & 1, sl = (item >> 1) / 3, d = (item >> 1) - 3 * sl;
    const int i = a.cell[3 * sl], j = a.cell[3 * sl + 1], k = a.cell[3 * sl + 2];
    const long long offR = (long long)k * g.plane + (long long)j * g.px + i;
    // side 0: the low cell against the surface seen forward; side 1: the high
    // cell against it seen backward (SpaceOperator.cpp:2440-2479)
    const long long off = side ? offR : offR - (d == 0 ? 1LL : (d == 1 ? g.px : g.plane));
    const uint8_t id = a.st.id[off];
    if (id >= a.st.s.nmat) continue;  // an inactive side gets no flux and no problem
    double V[5];
    if (a.faceV) {  // LINEAR: vr of the low cell, vl of the high cell (SpaceOperator.cpp:2452, 2474)
      const double* fv = a.faceV + (3LL * sl + d) * 10 + 5 * side;
      for (int c = 0; c < 5; c++) V[c] = fv[c];
    } else {
      wall_stage_state(a.st, off, id, V);
    }
    const double* gm = a.geo + (3LL * sl + d) * 12 + 6 * side;
    double dir[3], Vs[5], Vst[5];
    int mid = 0;
    bool bad = false;
    wall_direction(a.normal_mode, d, side ? -1 : 1, gm, dir);
    const int r = rs.solve_wall(dir, V, id, gm + 3, Vs, mid, Vst, bad);
    a.st.s.ed[id < a.st.s.nmat ? id : 0].clip(Vst);
    double* out = (side ? a.Vsp : a.Vsm) + (3LL * sl + d) * 5;
    for (int c = 0; c < 5; c++) out[c] = Vst[c];
    solves += 1;
    failed += (r & RIEM_FAILED) ? 1 : 0;
    const int cellR = (int)(((long long)k * g.ny + j) * g.nx + i);
    if (r & RIEM_PATH_OVERFLOW) report(a.st.err, ERR_ITER_CAP, cellR, 9);
    if (bad) report(a.st.err, ERR_STATE, cellR, 10);
  }
  if (solves) atomicAdd(&a.cnt[0], solves);
  if (failed) atomicAdd(&a.cnt[1], failed);
}

}  // namespace

m2cg_status walls_create(cudaStream_t s, const Grid3& g, size_t nalloc, const m2cg_scheme& scheme, int n,
                         const int* faces, const double* nf, const double* uf, const double* nb, const double* ub,
                         Walls** out, char* msg, size_t msglen) {
  *out = nullptr;
  auto refuse = [&](m2cg_status st, const char* why) {
    snprintf(msg, msglen, "%s", why);
    return st;
  };
  if (n < 1 || !faces || !nf || !uf || !nb || !ub) return refuse(M2CG_ERR_ARG, "no faces or a null array");
  if (scheme.ebm_recon != 0 && scheme.ebm_recon != 1)
    return refuse(M2CG_ERR_ARG, "ebm_recon must be 0 (CONSTANT) or 1 (LINEAR)");
  if (scheme.ebm_riemann_normal < 0 || scheme.ebm_riemann_normal > 2)
    return refuse(M2CG_ERR_ARG, "ebm_riemann_normal must be 0 (EMBEDDED_SURFACE), 1 (MESH) or 2 (AVERAGE)");
  const int nn[3] = {g.nx, g.ny, g.nz};
  // cells with cut low faces, in first-appearance order
  std::vector<int> slot_of;  // per interior cell, -1 = none
  slot_of.assign((size_t)g.nx * g.ny * g.nz, -1);
  std::vector<int> cells;
  std::vector<uint8_t> bits;
  std::vector<double> geo;
  for (int q = 0; q < n; q++) {
    const int d = faces[4 * q], i = faces[4 * q + 1], j = faces[4 * q + 2], k = faces[4 * q + 3];
    if (d < 0 || d > 2) return refuse(M2CG_ERR_ARG, "face axis must be 0, 1 or 2");
    const int ix[3] = {i, j, k};
    for (int a = 0; a < 3; a++)
      if (ix[a] < 0 || ix[a] >= nn[a]) return refuse(M2CG_ERR_ARG, "face cell outside the subdomain");
    if (ix[d] < 1)
      return refuse(M2CG_ERR_UNSUPPORTED, "a cut face must lie inside the subdomain (cell index >= 1 along its axis)");
    for (int c = 0; c < 3; c++)
      if (!std::isfinite(nf[3 * q + c]) || !std::isfinite(uf[3 * q + c]) || !std::isfinite(nb[3 * q + c]) ||
          !std::isfinite(ub[3 * q + c]))
        return refuse(M2CG_ERR_ARG, "non-finite surface normal or velocity");
    const size_t lin = ((size_t)k * g.ny + j) * g.nx + i;
    int sl = slot_of[lin];
    if (sl < 0) {
      sl = (int)cells.size() / 3;
      slot_of[lin] = sl;
      cells.push_back(i);
      cells.push_back(j);
      cells.push_back(k);
      bits.push_back(0);
      geo.resize(geo.size() + 36, 0.0);
    }
    if (bits[sl] & (1 << d)) return refuse(M2CG_ERR_ARG, "a face is listed twice");
    bits[sl] |= (uint8_t)(1 << d);
    double* gm = &geo[((size_t)sl * 3 + d) * 12];
    for (int c = 0; c < 3; c++) {
      gm[c] = nf[3 * q + c];
      gm[3 + c] = uf[3 * q + c];
      gm[6 + c] = nb[3 * q + c];
      gm[9 + c] = ub[3 * q + c];
    }
  }
  Walls* w = new Walls;
  w->nslot = (int)bits.size();
  w->normal_mode = scheme.ebm_riemann_normal;
  w->linear = scheme.ebm_recon == 1 && scheme.rec_type == M2CG_REC_LINEAR;
  w->P = riemann_params(scheme);
  // the one-sided problems, both sides of every cut face
  std::vector<int> work;
  for (int sl = 0; sl < w->nslot; sl++)
    for (int d = 0; d < 3; d++)
      if (bits[sl] & (1 << d)) {
        work.push_back((sl * 3 + d) * 2);
        work.push_back((sl * 3 + d) * 2 + 1);
      }
  w->nwork = (int)work.size();
  // one integration path (12 KiB) per thread, at most 4 resident 128-thread
  // CTAs per SM
  w->threads = (int)std::min<long long>((w->nwork + 127) / 128 * 128, 148LL * 4 * 128);
  bool ok = cudaMalloc((void**)&w->mask, nalloc) == cudaSuccess &&
            cudaMalloc((void**)&w->slot, nalloc * sizeof(int)) == cudaSuccess &&
            cudaMalloc((void**)&w->cell, cells.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc((void**)&w->geo, geo.size() * sizeof(double)) == cudaSuccess &&
            cudaMalloc((void**)&w->Vsm, (size_t)w->nslot * 15 * sizeof(double)) == cudaSuccess &&
            cudaMalloc((void**)&w->Vsp, (size_t)w->nslot * 15 * sizeof(double)) == cudaSuccess &&
            cudaMalloc((void**)&w->cnt, 2 * sizeof(unsigned long long)) == cudaSuccess &&
            cudaMalloc((void**)&w->work, work.size() * sizeof(int)) == cudaSuccess &&
            (!w->linear || cudaMalloc((void**)&w->faceV, (size_t)w->nslot * 30 * sizeof(double)) == cudaSuccess) &&
            cudaMalloc((void**)&w->scratch, (size_t)w->threads * 3 * RIEMANN_PATH_CAP * sizeof(double)) == cudaSuccess;
  if (!ok) {
    walls_destroy(w);
    return refuse(M2CG_ERR_NOMEM, "device allocation for the cut faces failed");
  }
  // per-cell mask and slot in the context's layout
  std::vector<uint8_t> hmask(nalloc, 0);
  std::vector<int> hslot(nalloc, -1);
  for (int sl = 0; sl < w->nslot; sl++) {
    const size_t off = (size_t)cells[3 * sl + 2] * g.plane + (size_t)cells[3 * sl + 1] * g.px + cells[3 * sl];
    hmask[off] = bits[sl];
    hslot[off] = sl;
  }
  cudaError_t e = cudaMemcpyAsync(w->mask, hmask.data(), nalloc, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->slot, hslot.data(), nalloc * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(w->cell, cells.data(), cells.size() * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(w->geo, geo.data(), geo.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->work, work.data(), work.size() * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(w->cnt, 0, 2 * sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host vectors go out of scope
  if (e != cudaSuccess) {
    walls_destroy(w);
    return refuse(M2CG_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = w;
  return M2CG_OK;
}

void walls_destroy(Walls* w) {
  if (!w) return;
  cudaFree(w->mask);
  cudaFree(w->slot);
  cudaFree(w->cell);
  cudaFree(w->geo);
  cudaFree(w->Vsm);
  cudaFree(w->Vsp);
  cudaFree(w->cnt);
  cudaFree(w->work);
  cudaFree(w->faceV);
  cudaFree(w->scratch);
  delete w;
}

m2cg_status walls_stage(Walls* w, cudaStream_t s, StageArgs& a) {
  WallPassArgs p;
  p.st = a;
  p.P = w->P;
  p.cell = w->cell;
  p.geo = w->geo;
  p.Vsm = w->Vsm;
  p.Vsp = w->Vsp;
  p.cnt = w->cnt;
  p.work = w->work;
  p.faceV = w->faceV;
  p.scratch = w->scratch;
  p.nwork = w->nwork;
  p.normal_mode = w->normal_mode;
  k_wall_riemann<<<w->threads / 128, 128, 0, s>>>(p);
  if (cudaGetLastError() != cudaSuccess) return M2CG_ERR_CUDA;
  walls_view(w, a);
  return M2CG_OK;
}

void walls_view(const Walls* w, StageArgs& a) {
  a.wall.mask = w->mask;
  a.wall.slot = w->slot;
  a.wall.Vsm = w->Vsm;
  a.wall.Vsp = w->Vsp;
  a.wall.linear = w->linear;
  a.wall.faces_out = nullptr;
}

bool walls_face_pass(const Walls* w, StageArgs& a) {
  if (!w->linear) return false;
  walls_view(w, a);
  a.wall.faces_out = w->faceV;
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

void walls_counters(Walls* w, cudaStream_t s, long long* solves, long long* failures) {
  unsigned long long h[2] = {0, 0};
  cudaMemcpyAsync(h, w->cnt, sizeof h, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  *solves = (long long)h[0];
  *failures = (long long)h[1];
}

}  // namespace m2c
