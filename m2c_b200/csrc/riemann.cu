// Batched two-material exact Riemann problems on the GPU (FP64, one problem
// per thread) and the m2cg_riemann_batch entry point.
//
// Compiled with -fmad=false: the solver restates
// ExactRiemannSolverBase::ComputeRiemannSolution (ExactRiemannSolverBase.cpp:59-342)
// and keeps its rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/m2c_gpu.h"
#include "riemann_batch.h"

namespace m2c {

__global__ void k_riemann_batch(RiemannBatchArgs a) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.n; q += (long long)gridDim.x * blockDim.x) {
    RiemannSolver rs;
    rs.P = a.P;
    rs.eos = a.eos;
    rs.path1.pt = a.scratch + (q % a.scratch_slots) * 2 * 3 * (long long)a.path_cap;
    rs.path1.cap = a.path_cap;
    rs.path3.pt = rs.path1.pt + 3 * (long long)a.path_cap;
    rs.path3.cap = a.path_cap;
    double Vm[5], Vp[5], dir[3];
    for (int c = 0; c < 5; c++) {
      Vm[c] = a.VL[5 * q + c];
      Vp[c] = a.VR[5 * q + c];
    }
    for (int c = 0; c < 3; c++) dir[c] = a.dir[3 * q + c];
    double Vs[5], Vsm[5], Vsp[5];
    int id = 0;
    bool bad = false;
    const double warm = a.warm ? a.warm[q] : NAN;
    int r = rs.solve(dir, Vm, a.idl[q], Vp, a.idr[q], Vs, id, Vsm, Vsp, warm, bad);
    for (int c = 0; c < 5; c++) {
      a.Vs[5 * q + c] = Vs[c];
      a.Vsm[5 * q + c] = Vsm[c];
      a.Vsp[5 * q + c] = Vsp[c];
    }
    a.id[q] = id;
    if (a.iters) a.iters[q] = rs.iterations;
    if (a.evals) a.evals[q] = rs.evaluations;
    a.err[q] = r | (bad ? 4 : 0);
  }
}

// One-sided (wall) problems: the same thread-to-slot mapping, one path per
// slot (the 1-wave's).
struct RiemannWallArgs {
  long long n;
  RiemannParams P;
  const Eos<double>* eos;
  const double* Vm;     // [n][5]
  const int* idm;
  const double* uwall;  // [n][3]
  const double* dir;    // [n][3]
  double* Vs;           // [n][5] (zero where id = -1)
  double* Vsm;          // [n][5]
  int* id;
  int* iters;           // or nullptr
  int* err;
  double* scratch;      // [slots][path_cap][3]
  int path_cap;
  long long scratch_slots;
};

__global__ void k_riemann_wall(RiemannWallArgs a) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.n; q += (long long)gridDim.x * blockDim.x) {
    RiemannSolver rs;
    rs.P = a.P;
    rs.eos = a.eos;
    rs.path1.pt = a.scratch + (q % a.scratch_slots) * 3 * (long long)a.path_cap;
    rs.path1.cap = a.path_cap;
    rs.path3.pt = nullptr;
    rs.path3.cap = 0;
    double Vm[5], uw[3], dir[3], Vs[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, Vsm[5];
    for (int c = 0; c < 5; c++) Vm[c] = a.Vm[5 * q + c];
    for (int c = 0; c < 3; c++) {
      uw[c] = a.uwall[3 * q + c];
      dir[c] = a.dir[3 * q + c];
    }
    int id = 0;
    bool bad = false;
    const int r = rs.solve_wall(dir, Vm, a.idm[q], uw, Vs, id, Vsm, bad);
    for (int c = 0; c < 5; c++) {
      a.Vs[5 * q + c] = Vs[c];
      a.Vsm[5 * q + c] = Vsm[c];
    }
    a.id[q] = id;
    if (a.iters) a.iters[q] = rs.iterations;
    a.err[q] = r | (bad ? 4 : 0);
  }
}

RiemannParams riemann_params(const m2cg_scheme& s) {
  RiemannParams P;
  P.maxIts_main = s.riem_maxits_main;
  P.maxIts_bracket = s.riem_maxits_bracket;
  P.maxIts_shock = s.riem_maxits_shock;
  P.numSteps_rarefaction = s.riem_nsteps_rarefaction;
  P.tol_main = s.riem_tol_main;
  P.tol_shock = s.riem_tol_shock;
  P.tol_rarefaction = s.riem_tol_rarefaction;
  P.min_pressure = s.riem_min_pressure;
  P.failure_threshold = s.riem_failure_threshold;
  P.pressure_at_failure = s.riem_pressure_at_failure;
  P.warm_delta = s.riem_warm_delta;
  P.warm_gate = s.riem_warm_gate;
  return P;
}

// One thread per path-scratch slot: a.scratch_slots is a multiple of 128, so
// the grid-stride loop maps every problem of a thread to that thread's slot.
cudaError_t launch_riemann_batch(const RiemannBatchArgs& a, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  if (a.scratch_slots <= 0 || a.scratch_slots % 128) return cudaErrorInvalidValue;
  const int block = 128;
  const long long grid = a.scratch_slots / block;
  k_riemann_batch<<<(int)grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

void set_last_error(const char* msg);

}  // namespace m2c

using namespace m2c;

static Eos<double> eos_of_material(const m2cg_material& m) {
  MatParams p;
  p.kind = m.eos; p.gam = m.gamma; p.pc = m.p_c; p.b = m.b; p.q = m.q;
  p.rhomin = m.rhomin; p.pmin = m.pmin; p.rhomax = m.rhomax; p.pmax = m.pmax;
  p.failsafe_density = m.failsafe_density;
  return make_eos<double>(p);
}

// Host arrays in, host arrays out: one device allocation carved into every
// array, one for the path scratch, one stream; the material table heos is
// indexed by idl/idr.
static m2cg_status riemann_host(const m2cg_scheme& scheme, const std::vector<Eos<double>>& heos, int n,
                                const double* VL, const int* idl, const double* VR, const int* idr,
                                const double* dir, const double* warm, double* Vs, int* id, double* Vsm,
                                double* Vsp, int* iters, int* evals, int* err) {
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    set_last_error("m2cg_riemann_batch: cudaStreamCreate failed (no CUDA device?)");
    return M2CG_ERR_CUDA;
  }
  RiemannBatchArgs a;
  memset(&a, 0, sizeof a);
  a.n = n;
  a.P = riemann_params(scheme);
  a.path_cap = RIEMANN_PATH_CAP;
  // one path-scratch slot (24 KiB) per thread, at most 148 x 8 x 128 threads
  const long long max_slots = 148LL * 8 * 128;
  a.scratch_slots = std::min<long long>(((long long)n + 127) / 128 * 128, max_slots);
  // One allocation holds every array, each starting on a 256-byte boundary.
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t nn = (size_t)n;
  const size_t eos_bytes = heos.size() * sizeof(Eos<double>);
  const size_t total = 5 * rup(nn * 40) + rup(nn * 24) + 6 * rup(nn * 4) + (warm ? rup(nn * 8) : 0) +
                       rup(eos_bytes);
  size_t bytes_scratch = (size_t)a.scratch_slots * 2 * 3 * RIEMANN_PATH_CAP * sizeof(double);
  char* buf = nullptr;
  m2cg_status st = M2CG_OK;
  if (cudaMalloc((void**)&buf, total) != cudaSuccess || cudaMalloc((void**)&a.scratch, bytes_scratch) != cudaSuccess) {
    cudaFree(buf);
    cudaStreamDestroy(s);
    set_last_error("m2cg_riemann_batch: device allocation failed");
    return M2CG_ERR_NOMEM;
  }
  char* p = buf;
  auto take = [&](size_t b) { char* r = p; p += rup(b); return r; };
  double* dVL = (double*)take(nn * 40); double* dVR = (double*)take(nn * 40); double* ddir = (double*)take(nn * 24);
  int* didl = (int*)take(nn * 4); int* didr = (int*)take(nn * 4);
  double* dwarm = warm ? (double*)take(nn * 8) : nullptr;
  double* dVs = (double*)take(nn * 40); double* dVsm = (double*)take(nn * 40); double* dVsp = (double*)take(nn * 40);
  int* did = (int*)take(nn * 4); int* diters = (int*)take(nn * 4); int* derr = (int*)take(nn * 4);
  int* devals = (int*)take(nn * 4);
  Eos<double>* deos = (Eos<double>*)take(eos_bytes);
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  if ((size_t)(p - buf) == total) {  // the carve-up stays inside the allocation
    ck(cudaMemcpyAsync(dVL, VL, nn * 40, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(dVR, VR, nn * 40, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(ddir, dir, nn * 24, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(didl, idl, nn * 4, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(didr, idr, nn * 4, cudaMemcpyHostToDevice, s));
    if (warm) ck(cudaMemcpyAsync(dwarm, warm, nn * 8, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(deos, heos.data(), eos_bytes, cudaMemcpyHostToDevice, s));
    a.VL = dVL; a.VR = dVR; a.dir = ddir; a.idl = didl; a.idr = didr; a.warm = dwarm;
    a.Vs = dVs; a.Vsm = dVsm; a.Vsp = dVsp; a.id = did; a.iters = diters; a.evals = devals; a.err = derr; a.eos = deos;
    if (e == cudaSuccess) ck(launch_riemann_batch(a, s));
    if (e == cudaSuccess) {
      ck(cudaMemcpyAsync(Vs, dVs, nn * 40, cudaMemcpyDeviceToHost, s));
      ck(cudaMemcpyAsync(Vsm, dVsm, nn * 40, cudaMemcpyDeviceToHost, s));
      ck(cudaMemcpyAsync(Vsp, dVsp, nn * 40, cudaMemcpyDeviceToHost, s));
      ck(cudaMemcpyAsync(id, did, nn * 4, cudaMemcpyDeviceToHost, s));
      if (iters) ck(cudaMemcpyAsync(iters, diters, nn * 4, cudaMemcpyDeviceToHost, s));
      if (evals) ck(cudaMemcpyAsync(evals, devals, nn * 4, cudaMemcpyDeviceToHost, s));
      ck(cudaMemcpyAsync(err, derr, nn * 4, cudaMemcpyDeviceToHost, s));
    }
    ck(cudaStreamSynchronize(s));
    if (e != cudaSuccess) {
      char msg[200];
      snprintf(msg, sizeof msg, "m2cg_riemann_batch: %s", cudaGetErrorString(e));
      set_last_error(msg);
      st = M2CG_ERR_CUDA;
    }
  } else {
    set_last_error("m2cg_riemann_batch: internal buffer layout error");
    st = M2CG_ERR_ARG;
  }
  cudaFree(buf);
  cudaFree(a.scratch);
  cudaStreamDestroy(s);
  return st;
}

extern "C" m2cg_status m2cg_riemann_batch(const m2cg_scheme* scheme, const m2cg_material* mats, int nmat, int n,
                                          const double* VL, const int* idl, const double* VR, const int* idr,
                                          const double* dir, const double* warm, double* Vs, int* id, double* Vsm,
                                          double* Vsp, int* iters, int* err) {
  if (!scheme || !mats || nmat < 1 || nmat > MAXMAT_RIEMANN || n < 0 || !VL || !idl || !VR || !idr || !dir || !Vs ||
      !id || !Vsm || !Vsp || !err)
    return M2CG_ERR_ARG;
  if (n == 0) return M2CG_OK;
  for (int q = 0; q < n; q++)
    if (idl[q] < 0 || idl[q] >= nmat || idr[q] < 0 || idr[q] >= nmat) return M2CG_ERR_ARG;
  std::vector<Eos<double>> heos(MAXMAT_RIEMANN);
  for (int m = 0; m < nmat; m++) heos[m] = eos_of_material(mats[m]);
  return riemann_host(*scheme, heos, n, VL, idl, VR, idr, dir, warm, Vs, id, Vsm, Vsp, iters, nullptr, err);
}

extern "C" m2cg_status m2cg_riemann_batch_pairs(const m2cg_scheme* scheme, const m2cg_material* mats, int n,
                                                const double* VL, const double* VR, const double* dir,
                                                const double* warm, double* Vs, int* id, double* Vsm, double* Vsp,
                                                int* iters, int* evals, int* err) {
  if (!scheme || !mats || n < 0 || !VL || !VR || !dir || !Vs || !id || !Vsm || !Vsp || !err) return M2CG_ERR_ARG;
  if (n == 0) return M2CG_OK;
  std::vector<Eos<double>> heos(2 * (size_t)n);
  std::vector<int> idl(n), idr(n);
  for (int q = 0; q < n; q++) {
    heos[2 * q] = eos_of_material(mats[2 * q]);
    heos[2 * q + 1] = eos_of_material(mats[2 * q + 1]);
    idl[q] = 2 * q;
    idr[q] = 2 * q + 1;
  }
  m2cg_status st = riemann_host(*scheme, heos, n, VL, idl.data(), VR, idr.data(), dir, warm, Vs, id, Vsm, Vsp, iters,
                                evals, err);
  if (st == M2CG_OK)
    for (int q = 0; q < n; q++) id[q] = id[q] & 1;
  return st;
}

extern "C" m2cg_status m2cg_riemann_wall_batch(const m2cg_scheme* scheme, const m2cg_material* mats, int nmat, int n,
                                               const double* Vm, const int* idm, const double* uwall,
                                               const double* dir, double* Vs, int* id, double* Vsm, int* iters,
                                               int* err) {
  if (!scheme || !mats || nmat < 1 || nmat > MAXMAT_RIEMANN || n < 0 || !Vm || !idm || !uwall || !dir || !Vs || !id ||
      !Vsm || !err) {
    set_last_error("m2cg_riemann_wall_batch: null argument or material count outside 1..4");
    return M2CG_ERR_ARG;
  }
  if (n == 0) return M2CG_OK;
  for (int q = 0; q < n; q++)
    if (idm[q] < 0 || idm[q] >= nmat) {
      set_last_error("m2cg_riemann_wall_batch: material id outside 0..nmat-1");
      return M2CG_ERR_ARG;
    }
  std::vector<Eos<double>> heos(MAXMAT_RIEMANN);
  for (int m = 0; m < nmat; m++) heos[m] = eos_of_material(mats[m]);
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    set_last_error("m2cg_riemann_wall_batch: cudaStreamCreate failed (no CUDA device?)");
    return M2CG_ERR_CUDA;
  }
  RiemannWallArgs a;
  memset(&a, 0, sizeof a);
  a.n = n;
  a.P = riemann_params(*scheme);
  a.path_cap = RIEMANN_PATH_CAP;
  const long long max_slots = 148LL * 8 * 128;
  a.scratch_slots = std::min<long long>(((long long)n + 127) / 128 * 128, max_slots);
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t nn = (size_t)n;
  const size_t eos_bytes = heos.size() * sizeof(Eos<double>);
  const size_t total = 3 * rup(nn * 40) + 2 * rup(nn * 24) + 4 * rup(nn * 4) + rup(eos_bytes);
  const size_t bytes_scratch = (size_t)a.scratch_slots * 3 * RIEMANN_PATH_CAP * sizeof(double);
  char* buf = nullptr;
  if (cudaMalloc((void**)&buf, total) != cudaSuccess || cudaMalloc((void**)&a.scratch, bytes_scratch) != cudaSuccess) {
    cudaFree(buf);
    cudaStreamDestroy(s);
    set_last_error("m2cg_riemann_wall_batch: device allocation failed");
    return M2CG_ERR_NOMEM;
  }
  char* p = buf;
  auto take = [&](size_t b) { char* r = p; p += rup(b); return r; };
  double* dVm = (double*)take(nn * 40);
  double* duw = (double*)take(nn * 24);
  double* ddir = (double*)take(nn * 24);
  int* didm = (int*)take(nn * 4);
  double* dVs = (double*)take(nn * 40);
  double* dVsm = (double*)take(nn * 40);
  int* did = (int*)take(nn * 4);
  int* diters = (int*)take(nn * 4);
  int* derr = (int*)take(nn * 4);
  Eos<double>* deos = (Eos<double>*)take(eos_bytes);
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  ck(cudaMemcpyAsync(dVm, Vm, nn * 40, cudaMemcpyHostToDevice, s));
  ck(cudaMemcpyAsync(duw, uwall, nn * 24, cudaMemcpyHostToDevice, s));
  ck(cudaMemcpyAsync(ddir, dir, nn * 24, cudaMemcpyHostToDevice, s));
  ck(cudaMemcpyAsync(didm, idm, nn * 4, cudaMemcpyHostToDevice, s));
  ck(cudaMemcpyAsync(deos, heos.data(), eos_bytes, cudaMemcpyHostToDevice, s));
  a.eos = deos; a.Vm = dVm; a.idm = didm; a.uwall = duw; a.dir = ddir;
  a.Vs = dVs; a.Vsm = dVsm; a.id = did; a.iters = diters; a.err = derr;
  if (e == cudaSuccess) {
    // one thread per scratch slot (a multiple of 128 threads)
    k_riemann_wall<<<(int)(a.scratch_slots / 128), 128, 0, s>>>(a);
    ck(cudaGetLastError());
  }
  if (e == cudaSuccess) {
    ck(cudaMemcpyAsync(Vs, dVs, nn * 40, cudaMemcpyDeviceToHost, s));
    ck(cudaMemcpyAsync(Vsm, dVsm, nn * 40, cudaMemcpyDeviceToHost, s));
    ck(cudaMemcpyAsync(id, did, nn * 4, cudaMemcpyDeviceToHost, s));
    if (iters) ck(cudaMemcpyAsync(iters, diters, nn * 4, cudaMemcpyDeviceToHost, s));
    ck(cudaMemcpyAsync(err, derr, nn * 4, cudaMemcpyDeviceToHost, s));
  }
  ck(cudaStreamSynchronize(s));
  m2cg_status st = M2CG_OK;
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof msg, "m2cg_riemann_wall_batch: %s", cudaGetErrorString(e));
    set_last_error(msg);
    st = M2CG_ERR_CUDA;
  }
  cudaFree(buf);
  cudaFree(a.scratch);
  cudaStreamDestroy(s);
  return st;
}
