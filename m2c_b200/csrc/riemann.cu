// Batched two-material exact Riemann problems on the GPU (FP64, one problem
// per thread) and the m2cg_riemann_batch entry point.
//
// Compiled with -fmad=false: the solver restates
// ExactRiemannSolverBase::ComputeRiemannSolution (ExactRiemannSolverBase.cpp:59-342)
// and keeps its rounding.
#include <cuda_runtime.h>

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
  return P;
}

cudaError_t launch_riemann_batch(const RiemannBatchArgs& a, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  int block = 128;
  long long grid = (a.n + block - 1) / block;
  if (grid > 148 * 32) grid = 148 * 32;
  k_riemann_batch<<<(int)grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

void set_last_error(const char* msg);

}  // namespace m2c

using namespace m2c;

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
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return M2CG_ERR_CUDA;
  Eos<double> heos[MAXMAT_RIEMANN];
  for (int m = 0; m < nmat; m++) {
    MatParams p;
    p.kind = mats[m].eos; p.gam = mats[m].gamma; p.pc = mats[m].p_c; p.b = mats[m].b; p.q = mats[m].q;
    p.rhomin = mats[m].rhomin; p.pmin = mats[m].pmin; p.rhomax = mats[m].rhomax; p.pmax = mats[m].pmax;
    p.failsafe_density = mats[m].failsafe_density;
    heos[m] = make_eos<double>(p);
  }
  RiemannBatchArgs a;
  memset(&a, 0, sizeof a);
  a.n = n;
  a.P = riemann_params(*scheme);
  a.path_cap = RIEMANN_PATH_CAP;
  a.scratch_slots = n;
  // One allocation holds every array, each starting on a 256-byte boundary.
  auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t nn = (size_t)n;
  const size_t total = 5 * rup(nn * 40) + rup(nn * 24) + 5 * rup(nn * 4) + (warm ? rup(nn * 8) : 0) +
                       rup(sizeof(heos));
  size_t bytes_scratch = nn * 2 * 3 * RIEMANN_PATH_CAP * sizeof(double);
  char* buf = nullptr;
  m2cg_status st = M2CG_OK;
  if (cudaMalloc((void**)&buf, total) != cudaSuccess || cudaMalloc((void**)&a.scratch, bytes_scratch) != cudaSuccess) {
    cudaFree(buf);
    cudaStreamDestroy(s);
    return M2CG_ERR_NOMEM;
  }
  char* p = buf;
  auto take = [&](size_t b) { char* r = p; p += rup(b); return r; };
  double* dVL = (double*)take(nn * 40); double* dVR = (double*)take(nn * 40); double* ddir = (double*)take(nn * 24);
  int* didl = (int*)take(nn * 4); int* didr = (int*)take(nn * 4);
  double* dwarm = warm ? (double*)take(nn * 8) : nullptr;
  double* dVs = (double*)take(nn * 40); double* dVsm = (double*)take(nn * 40); double* dVsp = (double*)take(nn * 40);
  int* did = (int*)take(nn * 4); int* diters = (int*)take(nn * 4); int* derr = (int*)take(nn * 4);
  Eos<double>* deos = (Eos<double>*)take(sizeof(heos));
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  if ((size_t)(p - buf) == total) {  // the carve-up stays inside the allocation
    ck(cudaMemcpyAsync(dVL, VL, nn * 40, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(dVR, VR, nn * 40, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(ddir, dir, nn * 24, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(didl, idl, nn * 4, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(didr, idr, nn * 4, cudaMemcpyHostToDevice, s));
    if (warm) ck(cudaMemcpyAsync(dwarm, warm, nn * 8, cudaMemcpyHostToDevice, s));
    ck(cudaMemcpyAsync(deos, heos, sizeof(heos), cudaMemcpyHostToDevice, s));
    a.VL = dVL; a.VR = dVR; a.dir = ddir; a.idl = didl; a.idr = didr; a.warm = dwarm;
    a.Vs = dVs; a.Vsm = dVsm; a.Vsp = dVsp; a.id = did; a.iters = diters; a.err = derr; a.eos = deos;
    if (e == cudaSuccess) ck(launch_riemann_batch(a, s));
    if (e == cudaSuccess) {
      ck(cudaMemcpyAsync(Vs, dVs, nn * 40, cudaMemcpyDeviceToHost, s));
      ck(cudaMemcpyAsync(Vsm, dVsm, nn * 40, cudaMemcpyDeviceToHost, s));
      ck(cudaMemcpyAsync(Vsp, dVsp, nn * 40, cudaMemcpyDeviceToHost, s));
      ck(cudaMemcpyAsync(id, did, nn * 4, cudaMemcpyDeviceToHost, s));
      if (iters) ck(cudaMemcpyAsync(iters, diters, nn * 4, cudaMemcpyDeviceToHost, s));
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
