// m2cg_riemann_batch_noalloc: the batched exact Riemann solve on buffers the
// caller already holds on the device, for callers that cannot allocate device
// memory (an application whose memory pool owns the whole GPU and forbids
// other allocators, code running inside a captured or replayed launch
// sequence, a host environment with no cudaMalloc binding).
//
// The only memory beyond the caller's inputs and outputs is the integration
// path scratch of the solver, which lives in the file-scope device array
// below. Compiled with -fmad=false, like the allocating entry point, so both
// give the same bits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/m2c_gpu.h"
#include "riemann_batch.h"

namespace m2c {
void set_last_error(const char* msg);
}

using namespace m2c;

namespace {

constexpr long long NOALLOC_SLOT_DOUBLES = 2LL * 3 * RIEMANN_PATH_CAP;  // two waves of [cap][3] points

// Integration paths of M2CG_NOALLOC_MAX_PROBLEMS problems: 24 KiB each,
// 24 MiB in all, held by every device that loads the library until exit.
// Every path is written before it is read within one problem's solve, so
// nothing here needs clearing between calls; the array keeps the last call's
// contents.
static __device__ __align__(256) double g_noalloc_paths[M2CG_NOALLOC_MAX_PROBLEMS * NOALLOC_SLOT_DOUBLES];

struct NoAllocArgs {
  RiemannBatchArgs a;
  Eos<double> eos[MAXMAT_RIEMANN];
  int nmat;
};

// One problem per thread, problem q uses path slot q (n <= the slot count).
// Material ids are checked here because the host cannot read them.
__global__ void k_riemann_batch_noalloc(const __grid_constant__ NoAllocArgs p) {
  __shared__ Eos<double> eos[MAXMAT_RIEMANN];
  if (threadIdx.x < MAXMAT_RIEMANN) eos[threadIdx.x] = p.eos[threadIdx.x];
  __syncthreads();
  const RiemannBatchArgs& a = p.a;
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= a.n) return;
  const int il = a.idl[q], ir = a.idr[q];
  if (il < 0 || il >= p.nmat || ir < 0 || ir >= p.nmat) {
    for (int c = 0; c < 5; c++) a.Vs[5 * q + c] = a.Vsm[5 * q + c] = a.Vsp[5 * q + c] = NAN;
    a.id[q] = -1;
    if (a.iters) a.iters[q] = 0;
    a.err[q] = M2CG_RIEMANN_ERR_MATERIAL_ID;
    return;
  }
  RiemannSolver rs;
  rs.P = a.P;
  rs.eos = eos;
  rs.path1.pt = a.scratch + q * NOALLOC_SLOT_DOUBLES;
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
  const int r = rs.solve(dir, Vm, il, Vp, ir, Vs, id, Vsm, Vsp, warm, bad);
  for (int c = 0; c < 5; c++) {
    a.Vs[5 * q + c] = Vs[c];
    a.Vsm[5 * q + c] = Vsm[c];
    a.Vsp[5 * q + c] = Vsp[c];
  }
  a.id[q] = id;
  if (a.iters) a.iters[q] = rs.iterations;
  a.err[q] = r | (bad ? 4 : 0);
}

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
double* g_paths_on_device[MAX_DEVICES];  // last looked-up device address of g_noalloc_paths, per device

// The host-side name g_noalloc_paths is only a stand-in for the symbol; the
// address a kernel may use is looked up with the device current. Outside a
// stream capture it is looked up again on every call (a table lookup in the
// runtime), so a device reset, after which the module is loaded again and
// the array may sit elsewhere, cannot leave a stale address behind. While
// `stream` is being captured the address of the last call outside a capture
// is used: a capture must follow at least one call on that device since the
// last reset.
m2cg_status paths_address(cudaStream_t stream, double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e));
    return M2CG_ERR_CUDA;
  }
  if (dev < 0 || dev >= MAX_DEVICES) {
    set_last_error("m2cg_riemann_batch_noalloc: device ordinal beyond the supported range");
    return M2CG_ERR_UNSUPPORTED;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
    cudaGetLastError();  // an implicit-capture query error is not this call's failure
    cap = cudaStreamCaptureStatusActive;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (cap == cudaStreamCaptureStatusNone) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_paths);
    if (e != cudaSuccess) {
      char msg[160];
      snprintf(msg, sizeof msg, "m2cg_riemann_batch_noalloc: cudaGetSymbolAddress failed: %s",
               cudaGetErrorString(e));
      set_last_error(msg);
      return M2CG_ERR_CUDA;
    }
    g_paths_on_device[dev] = (double*)ptr;
  } else if (!g_paths_on_device[dev]) {
    set_last_error("m2cg_riemann_batch_noalloc: first call on this device made during a stream capture; "
                   "make one call (n = 0 is enough) before capturing");
    return M2CG_ERR_ARG;
  }
  *out = g_paths_on_device[dev];
  return M2CG_OK;
}

}  // namespace

extern "C" m2cg_status m2cg_riemann_batch_noalloc(const m2cg_scheme* scheme, const m2cg_material* mats, int nmat,
                                                  int n, const double* VL, const int* idl, const double* VR,
                                                  const int* idr, const double* dir, const double* warm, double* Vs,
                                                  int* id, double* Vsm, double* Vsp, int* iters, int* err,
                                                  void* stream) {
  if (!scheme || !mats || nmat < 1 || nmat > MAXMAT_RIEMANN || n < 0 || !VL || !idl || !VR || !idr || !dir ||
      !Vs || !id || !Vsm || !Vsp || !err) {
    set_last_error("m2cg_riemann_batch_noalloc: null pointer or nmat outside [1, 4]");
    return M2CG_ERR_ARG;
  }
  if (n > M2CG_NOALLOC_MAX_PROBLEMS) {
    char msg[160];
    snprintf(msg, sizeof msg, "m2cg_riemann_batch_noalloc: %d problems exceed the maximum of %d per call", n,
             M2CG_NOALLOC_MAX_PROBLEMS);
    set_last_error(msg);
    return M2CG_ERR_ARG;
  }
  double* paths = nullptr;
  m2cg_status st = paths_address((cudaStream_t)stream, &paths);
  if (st != M2CG_OK) return st;
  if (n == 0) return M2CG_OK;
  NoAllocArgs p;
  memset(&p, 0, sizeof p);
  for (int m = 0; m < nmat; m++) {
    MatParams mp;
    mp.kind = mats[m].eos; mp.gam = mats[m].gamma; mp.pc = mats[m].p_c; mp.b = mats[m].b; mp.q = mats[m].q;
    mp.rhomin = mats[m].rhomin; mp.pmin = mats[m].pmin; mp.rhomax = mats[m].rhomax; mp.pmax = mats[m].pmax;
    mp.failsafe_density = mats[m].failsafe_density;
    p.eos[m] = make_eos<double>(mp);
  }
  p.nmat = nmat;
  RiemannBatchArgs& a = p.a;
  a.n = n;
  a.P = riemann_params(*scheme);
  a.VL = VL; a.VR = VR; a.dir = dir; a.idl = idl; a.idr = idr; a.warm = warm;
  a.Vs = Vs; a.Vsm = Vsm; a.Vsp = Vsp; a.id = id; a.iters = iters; a.err = err;
  a.scratch = paths;
  a.path_cap = RIEMANN_PATH_CAP;
  a.scratch_slots = M2CG_NOALLOC_MAX_PROBLEMS;
  const int block = 128;
  k_riemann_batch_noalloc<<<(n + block - 1) / block, block, 0, (cudaStream_t)stream>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e));
    return M2CG_ERR_CUDA;
  }
  return M2CG_OK;
}
